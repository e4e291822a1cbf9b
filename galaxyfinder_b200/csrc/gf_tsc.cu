// TSC mass assignment and TSC-weighted mesh interpolation.
//
// This translation unit is compiled with --fmad=false: every float and
// double operation below is rounded separately, in the order the reference
// evaluates it, so the per-particle stencil weights are bit-identical to
// NewGalFinder/tsc_omp2.c:301-353 (deposit) and :51-94 (interpolation) for
// the same FP64 positions.  The only difference left in the deposited mesh
// is the order in which float atomics sum the contributions of different
// particles to one cell.
#include <limits.h>

#include <algorithm>

#include "gf_tsc_weights.cuh"

namespace gf {

namespace {

__global__ void box_init_kernel(int32_t *__restrict__ boxes, int64_t nint) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nint; i += (int64_t)gridDim.x * blockDim.x)
        boxes[i] = (i & 1) ? INT_MIN : INT_MAX;  // empty ranges: lo > hi
}

// Widens the occupied boxes of the halos of this warp's particles: the lanes
// of one halo reduce their ranges, and one of them updates the halo's box.
// c: stencil cell ranges of the lane's particle; h < 0 for none.
__device__ __forceinline__ void box_update(int32_t *__restrict__ boxes, int h, bool dep, const int (&c)[6]) {
    const unsigned grp = __match_any_sync(0xffffffffu, h);
    if (h < 0) return;
    int ev[6], dp[6];
#pragma unroll
    for (int a = 0; a < 6; a += 2) {
        ev[a] = __reduce_min_sync(grp, c[a]);
        ev[a + 1] = __reduce_max_sync(grp, c[a + 1]);
        dp[a] = __reduce_min_sync(grp, dep ? c[a] : INT_MAX);
        dp[a + 1] = __reduce_max_sync(grp, dep ? c[a + 1] : INT_MIN);
    }
    if ((threadIdx.x & 31) != __ffs(grp) - 1) return;
    int32_t *b = boxes + (int64_t)kMeshBoxInts * h;
#pragma unroll
    for (int a = 0; a < 6; a += 2) {
        // a plain read first: most warps of a large halo widen nothing
        if (dp[a] < __ldcg(b + a)) atomicMin(b + a, dp[a]);
        if (dp[a + 1] > __ldcg(b + a + 1)) atomicMax(b + a + 1, dp[a + 1]);
        if (ev[a] < __ldcg(b + 6 + a)) atomicMin(b + 6 + a, ev[a]);
        if (ev[a + 1] > __ldcg(b + 7 + a)) atomicMax(b + 7 + a, ev[a + 1]);
    }
}

__global__ void tsc_deposit_kernel(int64_t n, const double *__restrict__ x,
                                   const double *__restrict__ y, const double *__restrict__ z,
                                   const double *__restrict__ mass,
                                   const int32_t *__restrict__ type,
                                   const int32_t *__restrict__ hid,
                                   const gf_mesh_desc *__restrict__ mesh,
                                   float *__restrict__ den, float volfold, int *err,
                                   const int32_t *__restrict__ order, int32_t *__restrict__ boxes) {
    // whole warps step together (the box update reduces over the warp)
    for (int64_t t0 = blockIdx.x * (int64_t)blockDim.x; t0 < n; t0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = t0 + threadIdx.x;
        int hb = -1;  // halo whose box this particle widens
        bool dep = false;
        int c[6];
        if (t < n) {
            // with an order (the octree's permutation) a warp deposits spatial
            // neighbours, whose stencils share cache lines of the mesh
            const int64_t p = order ? (int64_t)order[t] : t;
            const int h = hid ? hid[p] : 0;
            const gf_mesh_desc m = mesh[h];
            dep = m.ptype == GF_TYPE_ALL || (type ? type[p] : GF_TYPE_DM) == m.ptype;
            // the stencil of every particle when boxes are wanted (findDen
            // reads there), else of the deposited ones; on-chip meshes none
            if (m.ptype != kMeshOnChip && (dep || boxes)) {
                TscStencil s;
                float xd1, yd1, zd1;
                tsc_cells(x[p], y[p], z[p], m, s, xd1, yd1, zd1);
                if (!tsc_in_mesh(s, m)) {
                    if (dep) atomicOr(err, GF_ERRBIT_RANGE);
                } else {
                    hb = h;
                    c[0] = (int)s.i[0] - 1; c[1] = (int)s.i[0] + 1;
                    c[2] = (int)s.j[0] - 1; c[3] = (int)s.j[0] + 1;
                    c[4] = (int)s.k[0] - 1; c[5] = (int)s.k[0] + 1;
                    if (dep) {
                        tsc_deposit_weights(s, xd1, yd1, zd1, mass[p]);
                        const int64_t mx = 2 * (m.nx / 2 + 1);
                        float *mesh_h = den + m.off;
#pragma unroll
                        for (int cc = 0; cc < 3; cc++) {
#pragma unroll
                            for (int b = 0; b < 3; b++) {
#pragma unroll
                                for (int a = 0; a < 3; a++) {
                                    // volfold is 1 or an exact power of two (see launch_tsc_deposit)
                                    atomicAdd(mesh_h + s.i[a] + mx * (s.j[b] + (int64_t)m.ny * s.k[cc]),
                                              tsc_deposit_value(s, a, b, cc, volfold));
                                }
                            }
                        }
                    }
                }
            }
        }
        if (boxes) box_update(boxes, hb, dep, c);
    }
}

// The occupied boxes alone, before any deposit: the stencil ranges of the
// deposited particles (deposit box) and of every particle (evaluation box) of
// each device-memory mesh, with the same stencils as the deposit.  The
// box-restricted mesh stage zeroes only the deposit boxes from them.
__global__ void mesh_box_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                                const double *__restrict__ z, const int32_t *__restrict__ type,
                                const int32_t *__restrict__ hid, const gf_mesh_desc *__restrict__ mesh,
                                int32_t *__restrict__ boxes) {
    // whole warps step together (the box update reduces over the warp)
    for (int64_t t0 = blockIdx.x * (int64_t)blockDim.x; t0 < n; t0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = t0 + threadIdx.x;
        int hb = -1;
        bool dep = false;
        int c[6] = {0, 0, 0, 0, 0, 0};
        if (p < n) {
            const int h = hid ? hid[p] : 0;
            const gf_mesh_desc m = mesh[h];
            if (m.ptype != kMeshOnChip) {
                TscStencil s;
                float xd1, yd1, zd1;
                tsc_cells(x[p], y[p], z[p], m, s, xd1, yd1, zd1);
                if (tsc_in_mesh(s, m)) {  // particles outside are flagged by the deposit and findDen
                    hb = h;
                    dep = m.ptype == GF_TYPE_ALL || (type ? type[p] : GF_TYPE_DM) == m.ptype;
                    c[0] = (int)s.i[0] - 1; c[1] = (int)s.i[0] + 1;
                    c[2] = (int)s.j[0] - 1; c[3] = (int)s.j[0] + 1;
                    c[4] = (int)s.k[0] - 1; c[5] = (int)s.k[0] + 1;
                }
            }
        }
        box_update(boxes, hb, dep, c);
    }
}

// ---------------------------------------------------------------- tiled deposit
// The deposit through shared-memory tiles.  A block takes kTileChunk
// consecutive particles in octree order (spatial neighbours; the halos'
// particle ranges are the batch's, so a chunk splits into halo segments at
// pstart).  For each segment the block reduces the cell box its stencils
// cover.  When the box holds at most GF_TSC_TILE cells, and at most half as
// many as the segment's 27 stencil cells, the stencils are summed into the
// tile with shared-memory atomics and each nonzero tile cell is then added
// to the mesh with one global atomic; otherwise every stencil cell is a
// global atomic, as in tsc_deposit_kernel.  The weights are the same; the
// float sums run in two levels (tile, then mesh), in no fixed order.  The
// occupied boxes are widened once per segment.
constexpr int kTileThreads = 256;
constexpr int kTileChunk = 2048;

struct BlockBox {
    int v[12];  // deposit box (lo, hi per axis), evaluation box
    int ndep;   // deposited particles
};

__device__ __forceinline__ void block_box_reduce(BlockBox &b, int *scratch /* [8 warps][13] */) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int a = 0; a < 12; a += 2) {
        b.v[a] = __reduce_min_sync(0xffffffffu, b.v[a]);
        b.v[a + 1] = __reduce_max_sync(0xffffffffu, b.v[a + 1]);
    }
    b.ndep = __reduce_add_sync(0xffffffffu, (unsigned)b.ndep);
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 12; a++) scratch[13 * w + a] = b.v[a];
        scratch[13 * w + 12] = b.ndep;
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 12; a++) b.v[a] = scratch[a];
    b.ndep = scratch[12];
    for (int ww = 1; ww < kTileThreads / 32; ww++) {
#pragma unroll
        for (int a = 0; a < 12; a += 2) {
            b.v[a] = min(b.v[a], scratch[13 * ww + a]);
            b.v[a + 1] = max(b.v[a + 1], scratch[13 * ww + a + 1]);
        }
        b.ndep += scratch[13 * ww + 12];
    }
    __syncthreads();  // scratch is reused by the next reduction
}

template <int TILE>
__global__ void __launch_bounds__(kTileThreads)
tsc_tile_deposit_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, const double *__restrict__ mass,
                        const int32_t *__restrict__ type, const int64_t *__restrict__ pstart,
                        const int32_t *__restrict__ order, const int32_t *__restrict__ thalo,
                        const gf_mesh_desc *__restrict__ mesh, float *__restrict__ den, float volfold,
                        int *err, int32_t *__restrict__ boxes) {
    __shared__ float tile[TILE];
    __shared__ int scratch[13 * (kTileThreads / 32)];
    for (int64_t c0 = (int64_t)blockIdx.x * kTileChunk; c0 < n; c0 += (int64_t)gridDim.x * kTileChunk) {
        const int64_t c1 = min(c0 + (int64_t)kTileChunk, n);
        int64_t s0 = c0;
        while (s0 < c1) {
            const int h = thalo[s0];  // octree order keeps each halo's range [pstart[h], pstart[h+1])
            const int64_t s1 = min(c1, pstart[h + 1]);
            const gf_mesh_desc m = mesh[h];
            if (m.ptype == kMeshOnChip) {  // deposited on chip
                s0 = s1;
                continue;
            }
            BlockBox bb;
#pragma unroll
            for (int a = 0; a < 12; a += 2) {
                bb.v[a] = INT_MAX;
                bb.v[a + 1] = INT_MIN;
            }
            bb.ndep = 0;
            for (int64_t t = s0 + threadIdx.x; t < s1; t += kTileThreads) {
                const int64_t p = order[t];
                const bool dep = m.ptype == GF_TYPE_ALL || (type ? type[p] : GF_TYPE_DM) == m.ptype;
                TscStencil s;
                float xd1, yd1, zd1;
                tsc_cells(x[p], y[p], z[p], m, s, xd1, yd1, zd1);
                if (!tsc_in_mesh(s, m)) {
                    if (dep) atomicOr(err, GF_ERRBIT_RANGE);
                    continue;
                }
                const int c[6] = {(int)s.i[0] - 1, (int)s.i[0] + 1, (int)s.j[0] - 1,
                                  (int)s.j[0] + 1, (int)s.k[0] - 1, (int)s.k[0] + 1};
#pragma unroll
                for (int a = 0; a < 6; a += 2) {
                    bb.v[6 + a] = min(bb.v[6 + a], c[a]);
                    bb.v[7 + a] = max(bb.v[7 + a], c[a + 1]);
                    if (dep) {
                        bb.v[a] = min(bb.v[a], c[a]);
                        bb.v[a + 1] = max(bb.v[a + 1], c[a + 1]);
                    }
                }
                bb.ndep += dep;
            }
            block_box_reduce(bb, scratch);
            if (boxes && threadIdx.x == 0) {
                int32_t *bx = boxes + (int64_t)kMeshBoxInts * h;
#pragma unroll
                for (int a = 0; a < 12; a += 2) {
                    if (bb.v[a] < __ldcg(bx + a)) atomicMin(bx + a, bb.v[a]);
                    if (bb.v[a + 1] > __ldcg(bx + a + 1)) atomicMax(bx + a + 1, bb.v[a + 1]);
                }
            }
            if (bb.ndep > 0) {
                const int wx = bb.v[1] - bb.v[0] + 1, wy = bb.v[3] - bb.v[2] + 1, wz = bb.v[5] - bb.v[4] + 1;
                const int64_t vol = (int64_t)wx * wy * wz;
                const bool use_tile = vol <= TILE && 2 * vol <= 27 * (int64_t)bb.ndep;
                const int64_t mx = 2 * (m.nx / 2 + 1);
                float *mesh_h = den + m.off;
                if (use_tile) {
                    for (int e = threadIdx.x; e < (int)vol; e += kTileThreads) tile[e] = 0.f;
                    __syncthreads();
                }
                for (int64_t t = s0 + threadIdx.x; t < s1; t += kTileThreads) {
                    const int64_t p = order[t];
                    if (!(m.ptype == GF_TYPE_ALL || (type ? type[p] : GF_TYPE_DM) == m.ptype)) continue;
                    TscStencil s;
                    float xd1, yd1, zd1;
                    tsc_cells(x[p], y[p], z[p], m, s, xd1, yd1, zd1);
                    if (!tsc_in_mesh(s, m)) continue;
                    tsc_deposit_weights(s, xd1, yd1, zd1, mass[p]);
#pragma unroll
                    for (int cc = 0; cc < 3; cc++) {
#pragma unroll
                        for (int b = 0; b < 3; b++) {
#pragma unroll
                            for (int a = 0; a < 3; a++) {
                                // volfold is 1 or an exact power of two (see launch_tsc_deposit)
                                const float v = tsc_deposit_value(s, a, b, cc, volfold);
                                if (use_tile)
                                    atomicAdd(tile + ((int)s.i[a] - bb.v[0]) +
                                                  wx * (((int)s.j[b] - bb.v[2]) + wy * ((int)s.k[cc] - bb.v[4])),
                                              v);
                                else
                                    atomicAdd(mesh_h + s.i[a] + mx * (s.j[b] + (int64_t)m.ny * s.k[cc]), v);
                            }
                        }
                    }
                }
                if (use_tile) {
                    __syncthreads();
                    for (int e = threadIdx.x; e < (int)vol; e += kTileThreads) {
                        const float v = tile[e];
                        if (v != 0.f) {
                            const int i = bb.v[0] + e % wx;
                            const int j = bb.v[2] + (e / wx) % wy;
                            const int k = bb.v[4] + e / (wx * wy);
                            atomicAdd(mesh_h + i + mx * (j + (int64_t)m.ny * k), v);
                        }
                    }
                    __syncthreads();  // the tile is reused by the next segment
                }
            }
            s0 = s1;
        }
    }
}

__global__ void find_den_kernel(int64_t n, const double *__restrict__ x,
                                const double *__restrict__ y, const double *__restrict__ z,
                                const int32_t *__restrict__ hid,
                                const gf_mesh_desc *__restrict__ mesh,
                                const float *__restrict__ den, float *__restrict__ densph,
                                int *err, const int32_t *__restrict__ order) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = order ? (int64_t)order[t] : t;  // octree order: shared stencil lines
        const gf_mesh_desc m = mesh[hid ? hid[p] : 0];
        if (m.ptype == kMeshOnChip) continue;  // interpolated on chip
        TscStencil s;
        float xd1, yd1, zd1;
        tsc_cells(x[p], y[p], z[p], m, s, xd1, yd1, zd1);
        if (!tsc_in_mesh(s, m)) {
            atomicOr(err, GF_ERRBIT_RANGE);
            densph[p] = 0.f;
            continue;
        }
        tsc_interp_weights(s, xd1, yd1, zd1);
        const int64_t mx = 2 * (m.nx / 2 + 1);
        const float *mesh_h = den + m.off;
        // tsc_omp2.c:96-124: for each z plane, y rows in order 1,2,3, x in
        // order 1,2,3; each term is (den * wxwy) * wz.
        float density = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) {
#pragma unroll
            for (int b = 0; b < 3; b++) {
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const float v = __ldg(mesh_h + s.i[a] + mx * (s.j[b] + (int64_t)m.ny * s.k[c]));
                    density = tsc_interp_add(density, v, s, a, b, c);
                }
            }
        }
        densph[p] = density;
    }
}

__global__ void scale_kernel(float *__restrict__ den, int64_t n, double factor) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        den[p] = (float)(den[p] * factor);  // tsc_omp2.c:497 (float *= double)
}

inline int grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    const int64_t cap = (int64_t)sm_count() * 16;  // 16 resident blocks per SM at most
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

bool is_pow2_double(double v) {
    int e;
    double f = frexp(v, &e);
    return f == 0.5;
}

}  // namespace

double tsc_volfact() {
    // tsc_omp2.c:188, TSC_CELL_SIZE = 0.004 (params.h:92)
    const double r = 0.001 / 0.004;
    return r * r * r;
}

int launch_tsc_deposit(gf_ctx *ctx, int64_t n, const double *x, const double *y,
                       const double *z, const double *mass, const int32_t *type,
                       const int32_t *hid, const gf_mesh_desc *mesh, float *den,
                       double volfact, const int32_t *order, int32_t nhalo, int32_t *boxes) {
    if (boxes) {
        const int64_t nint = (int64_t)kMeshBoxInts * std::max(nhalo, 1);
        box_init_kernel<<<grid_for(nint, 256), 256, 0, ctx->stream>>>(boxes, nint);
        GF_LAUNCH_CHECK();
    }
    if (n <= 0) return GF_OK;
    // A power-of-two volfact commutes with every float rounding, so folding
    // it into the weights gives the same bits as the reference's final
    // den *= volfact pass without a second sweep over the mesh.
    float fold = is_pow2_double(volfact) ? (float)volfact : 1.f;
    const int block = 256;
    tsc_deposit_kernel<<<grid_for(n, block), block, 0, ctx->stream>>>(
        n, x, y, z, mass, type, hid, mesh, den, fold, ctx->d_err, order, boxes);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

int launch_scale(gf_ctx *ctx, float *den, int64_t ncells, double factor) {
    const int block = 256;
    scale_kernel<<<grid_for(ncells, block), block, 0, ctx->stream>>>(den, ncells, factor);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

int launch_find_den(gf_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                    const int32_t *hid, const gf_mesh_desc *mesh, const float *den,
                    float *densph, const int32_t *order) {
    if (n <= 0) return GF_OK;
    const int block = 256;
    find_den_kernel<<<grid_for(n, block), block, 0, ctx->stream>>>(n, x, y, z, hid, mesh, den,
                                                                   densph, ctx->d_err, order);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

bool volfact_folds(double v) { return is_pow2_double(v); }

int launch_mesh_boxes(gf_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                      const int32_t *type, const int32_t *hid, int32_t nhalo, const gf_mesh_desc *mesh,
                      int32_t *boxes) {
    const int64_t nint = (int64_t)kMeshBoxInts * std::max(nhalo, 1);
    box_init_kernel<<<grid_for(nint, 256), 256, 0, ctx->stream>>>(boxes, nint);
    GF_LAUNCH_CHECK();
    if (n <= 0) return GF_OK;
    mesh_box_kernel<<<grid_for(n, 256), 256, 0, ctx->stream>>>(n, x, y, z, type, hid, mesh, boxes);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

int launch_stage_deposit(gf_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                         const double *mass, const int32_t *type, const int32_t *hid, const int64_t *pstart,
                         const int32_t *order, const int32_t *thalo, int32_t nhalo, const gf_mesh_desc *mesh,
                         float *den, double volfact, int32_t *boxes) {
    if (GF_TSC_TILE == 0 || !order || !thalo)
        return launch_tsc_deposit(ctx, n, x, y, z, mass, type, hid, mesh, den, volfact, nullptr, nhalo, boxes);
    if (boxes) {
        const int64_t nint = (int64_t)kMeshBoxInts * std::max(nhalo, 1);
        box_init_kernel<<<grid_for(nint, 256), 256, 0, ctx->stream>>>(boxes, nint);
        GF_LAUNCH_CHECK();
    }
    if (n <= 0) return GF_OK;
    const float fold = is_pow2_double(volfact) ? (float)volfact : 1.f;
    const int64_t chunks = (n + kTileChunk - 1) / kTileChunk;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(chunks, (int64_t)sm_count() * 8));
    tsc_tile_deposit_kernel<(GF_TSC_TILE > 0 ? GF_TSC_TILE : 1024)><<<grid, kTileThreads, 0, ctx->stream>>>(
        n, x, y, z, mass, type, pstart, order, thalo, mesh, den, fold, ctx->d_err, boxes);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

}  // namespace gf
