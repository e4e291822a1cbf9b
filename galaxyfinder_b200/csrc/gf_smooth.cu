// Gaussian smoothing of TSC meshes, the operation of NewGalFinder/gsmooth.c:14-115:
//   forward r2c 3-D FFT -> multiply mode (i,j,k) by
//   exp(-(pi RG)^2 (i^2/nx^2 + j^2/ny^2 + k^2/nz^2)) with signed j,k and
//   i in [0, nx/2] -> c2r -> scale 1/(nx ny nz).
//
// The factor is a product of three real, even, per-axis factors, so the 3-D
// operation equals three independent 1-D circular convolutions (one per axis)
// with the real even kernels h_n = IDFT(G_n).  Each pass below loads a tile of
// pencils along one axis into shared memory once, and
//   * for power-of-two lengths runs a Stockham radix-2 FFT, multiplies the
//     spectrum by G_n/n, and runs the inverse FFT, all in shared memory;
//   * for any other length applies the full n-tap circular convolution with
//     the exact h_n (computed in FP64 on the host), so arbitrary sizes such
//     as the reference's extent/cellsize + 10 meshes are exact too.
// Two real pencils are packed into one complex pencil (real and imaginary
// parts): because G_n is real and even, filtering preserves that split.
// Every pass reads and writes each mesh element once (8 B per element per
// axis); twiddles and filters are generated in FP64 on the host.
#include <math.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <utility>

#include <cooperative_groups.h>

#include "gf_tsc_weights.cuh"

namespace gf {

namespace {

struct SmoothTile {
    int32_t halo;
    int32_t base;   // first pencil: row index (x) or first i (y, z)
    int32_t other;  // k (y axis) or j (z axis); unused for x
    int32_t npen;   // pencils in this tile
};

struct AxisTable {
    int32_t n;
    int32_t logn;     // log2(n) for the FFT path, -1 for the direct path
    int64_t tab_off;  // float offset of this axis' tables
};

struct GroupLaunch {
    const int32_t *halos;      // halos of this (axis, length) group
    const int64_t *tile_start; // prefix of tile counts over the group (ngroup + 1)
    int32_t ngroup;
};

template <int AXIS>
__device__ __forceinline__ SmoothTile decode_group_tile(int64_t b, const GroupLaunch &g,
                                                        const gf_mesh_desc *__restrict__ mesh,
                                                        int pmax) {
    int lo = 0, hi = g.ngroup;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (g.tile_start[mid] <= b) lo = mid; else hi = mid;
    }
    const int64_t local = b - g.tile_start[lo];
    const int h = g.halos[lo];
    const gf_mesh_desc &m = mesh[h];
    SmoothTile t;
    t.halo = h;
    if (AXIS == 0) {
        const int rows = m.ny * m.nz;
        t.base = (int)(local * pmax);
        t.other = 0;
        t.npen = min(pmax, rows - t.base);
    } else {
        const int cx = (m.nx + pmax - 1) / pmax;
        t.other = (int)(local / cx);
        t.base = (int)(local - (int64_t)t.other * cx) * pmax;
        t.npen = min(pmax, m.nx - t.base);
    }
    return t;
}

// Whether a tile's pencils can change the result, from the mesh's occupied
// boxes (kMeshBoxInts ints: deposit box, then evaluation box; lo > hi when
// empty).  The passes run along x, then y, then z.  A pencil whose input is
// all zero filters to zero, so skipping it is exact: along x, the rows
// (y, z) outside the deposit box are zero; after the x pass every x of an
// occupied row is set, so along y the columns (x, z) with z outside the
// deposit box are zero.  Along z every column is set; with trim the pass
// runs only over the columns (x, y) of the evaluation box.
template <int AXIS>
__device__ __forceinline__ bool tile_needed(const SmoothTile &t, const gf_mesh_desc &m,
                                            const int32_t *__restrict__ box, int trim) {
    if (AXIS == 0) {
        const int ylo = box[2], yhi = box[3], zlo = box[4], zhi = box[5];
        const int r0 = t.base, r1 = t.base + t.npen - 1;  // rows r = y + ny z
        const int za = r0 / m.ny, zb = r1 / m.ny;
        for (int zz = max(za, zlo); zz <= min(zb, zhi); zz++) {
            const int ya = zz == za ? r0 - zz * m.ny : 0;
            const int yb = zz == zb ? r1 - zz * m.ny : m.ny - 1;
            if (max(ya, ylo) <= min(yb, yhi)) return true;
        }
        return false;
    }
    if (AXIS == 1) return t.other >= box[4] && t.other <= box[5];
    if (!trim) return box[0] <= box[1];  // all zero when nothing was deposited
    return t.other >= box[8] && t.other <= box[9] && t.base <= box[7] && t.base + t.npen - 1 >= box[6];
}

constexpr int kThreads = 256;

template <int AXIS>
__device__ __forceinline__ int64_t elem_addr(const gf_mesh_desc &m, int64_t mx, const SmoothTile &t,
                                             int p, int s) {
    if (AXIS == 0) return m.off + mx * (int64_t)(t.base + p) + s;
    if (AXIS == 1) return m.off + (t.base + p) + mx * ((int64_t)s + (int64_t)m.ny * t.other);
    return m.off + (t.base + p) + mx * ((int64_t)t.other + (int64_t)m.ny * s);
}

template <int AXIS>
__global__ void __launch_bounds__(kThreads)
smooth_axis_kernel(float *__restrict__ den, const gf_mesh_desc *__restrict__ mesh,
                   GroupLaunch g, const AxisTable *__restrict__ axes,
                   const float *__restrict__ tables, int pmax, const int32_t *__restrict__ boxes,
                   int trim) {
    extern __shared__ float2 smem[];
    const SmoothTile t = decode_group_tile<AXIS>(blockIdx.x, g, mesh, pmax);
    const gf_mesh_desc m = mesh[t.halo];
    // the whole block leaves together (before any barrier)
    if (boxes && !tile_needed<AXIS>(t, m, boxes + (int64_t)kMeshBoxInts * t.halo, trim)) return;
    const AxisTable at = axes[3 * t.halo + AXIS];
    const int n = at.n;
    const int64_t mx = 2 * (m.nx / 2 + 1);
    const int npair = (t.npen + 1) >> 1;
    float2 *bufA = smem;
    float2 *bufB = smem + (size_t)((pmax + 1) >> 1) * n;
    float *fa = reinterpret_cast<float *>(bufA);

    // ---- load: pencil p -> component (p & 1) of complex pencil p >> 1
    const int total = 2 * npair * n;
    for (int e = threadIdx.x; e < total; e += kThreads) {
        int p, s;
        if (AXIS == 0) { p = e / n; s = e - p * n; }
        else { s = e / (2 * npair); p = e - s * (2 * npair); }
        float v = 0.f;
        if (p < t.npen) v = den[elem_addr<AXIS>(m, mx, t, p, s)];
        fa[2 * ((p >> 1) * n + s) + (p & 1)] = v;
    }
    __syncthreads();

    float2 *src = bufA, *dst = bufB;
    if (at.logn >= 0) {
        const float2 *tw = reinterpret_cast<const float2 *>(tables + at.tab_off);  // n/2 twiddles
        const float *filt = tables + at.tab_off + n;                               // n factors
        const int half = n >> 1;
        const int work = npair * half;
        for (int dir = 0; dir < 2; dir++) {
            const float sgn = dir == 0 ? 1.f : -1.f;  // inverse uses conjugate twiddles
            for (int ls = 0; ls < at.logn; ls++) {
                const int smask = (1 << ls) - 1;
                for (int e = threadIdx.x; e < work; e += kThreads) {
                    const int c = e / half;
                    const int tt = e - c * half;
                    const int q = tt & smask;
                    const int p = tt >> ls;
                    const float2 *x = src + c * n;
                    float2 *y = dst + c * n;
                    const float2 a = x[q + (p << ls)];
                    const float2 b = x[q + (p << ls) + half];
                    float2 w = tw[p << ls];
                    w.y *= sgn;
                    const float2 d = make_float2(a.x - b.x, a.y - b.y);
                    y[q + (p << (ls + 1))] = make_float2(a.x + b.x, a.y + b.y);
                    y[q + (p << (ls + 1)) + (1 << ls)] =
                        make_float2(d.x * w.x - d.y * w.y, d.x * w.y + d.y * w.x);
                }
                __syncthreads();
                float2 *tmp = src; src = dst; dst = tmp;
            }
            if (dir == 0) {
                for (int e = threadIdx.x; e < npair * n; e += kThreads) {
                    const int k = e % n;
                    const float g = filt[k];
                    src[e].x *= g;
                    src[e].y *= g;
                }
                __syncthreads();
            }
        }
    } else {
        // direct n-tap circular convolution with the exact periodic kernel
        const float *h = tables + at.tab_off;
        for (int e = threadIdx.x; e < npair * n; e += kThreads) {
            const int c = e / n;
            const int s = e - c * n;
            const float2 *x = src + c * n;
            float ar = 0.f, ai = 0.f;
            int idx = s;
            for (int mm = 0; mm < n; mm++) {
                const float hv = h[mm];
                const float2 v = x[idx];
                ar = fmaf(hv, v.x, ar);
                ai = fmaf(hv, v.y, ai);
                idx = idx == 0 ? n - 1 : idx - 1;
            }
            dst[e] = make_float2(ar, ai);
        }
        __syncthreads();
        src = dst;
    }

    // ---- store
    const float *fs = reinterpret_cast<const float *>(src);
    for (int e = threadIdx.x; e < total; e += kThreads) {
        int p, s;
        if (AXIS == 0) { p = e / n; s = e - p * n; }
        else { s = e / (2 * npair); p = e - s * (2 * npair); }
        if (p < t.npen) den[elem_addr<AXIS>(m, mx, t, p, s)] = fs[2 * ((p >> 1) * n + s) + (p & 1)];
    }
}

// ---------------------------------------------------------------- FFT path
// In-register R-point DFT (R = 2, 4, 8) of a[], forward e^{-2 pi i jk/R} or
// inverse (conjugate) kernel.
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 v) {  // v * (-i) forward, v * (+i) inverse
    return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3) {
    const float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3);
    const float2 t3 = mul_mi<INV>(csub(a1, a3));
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, t3);
    a3 = csub(t1, t3);
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2 (&a)[R]) {
    if (R == 2) {
        const float2 t = a[0];
        a[0] = cadd(t, a[1]);
        a[1] = csub(t, a[1]);
    } else if (R == 4) {
        dft4<INV>(a[0], a[1], a[2], a[3]);
    } else {  // R == 8: two 4-point DFTs (even, odd) and the W8 butterflies
        float2 e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
        float2 o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
        dft4<INV>(e0, e1, e2, e3);
        dft4<INV>(o0, o1, o2, o3);
        const float h = 0.70710678118654752f;
        // W8^1 = (1 - i)/sqrt2 forward, (1 + i)/sqrt2 inverse; W8^2 = -/+ i; W8^3 = (-1 -/+ i)/sqrt2
        o1 = INV ? make_float2(h * (o1.x - o1.y), h * (o1.x + o1.y))
                 : make_float2(h * (o1.x + o1.y), h * (o1.y - o1.x));
        o2 = mul_mi<INV>(o2);
        o3 = INV ? make_float2(-h * (o3.x + o3.y), h * (o3.x - o3.y))
                 : make_float2(h * (o3.y - o3.x), -h * (o3.x + o3.y));
        a[0] = cadd(e0, o0); a[4] = csub(e0, o0);
        a[1] = cadd(e1, o1); a[5] = csub(e1, o1);
        a[2] = cadd(e2, o2); a[6] = csub(e2, o2);
        a[3] = cadd(e3, o3); a[7] = csub(e3, o3);
    }
}

// Shared-memory layout of the FFT tiles: complex element k of pencil c sits
// at c*SN + k + k/8 (one padding slot per 8 elements, pencil stride
// SN = N + N/8 + 1), so the radix-8 strided stores and the 16-pencil
// column loads of the y/z passes spread over all 32 banks.
template <int N>
struct FftLayout {
    static constexpr int SN = N + N / 8 + 1;
    __device__ static __forceinline__ int at(int c, int k) { return c * SN + k + (k >> 3); }
};

// One Stockham radix-R pass over npair complex pencils of length N held in
// shared memory (src -> dst), stride S = product of the radices already done:
//   y[q + S (R p + j)] = w^(p S j) * sum_r x[q + S (p + r M)] e^{-+2 pi i r j/R},
// M = N/(S R), w = e^{-2 pi i/N} (table tw, conjugated for the inverse).  The
// final pass of the forward transform multiplies by the filter.
template <int N, int R, int S, bool INV, bool FILTER>
__device__ __forceinline__ void stockham_pass(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                              int npair, const float2 *__restrict__ tw,
                                              const float *__restrict__ filt) {
    using L = FftLayout<N>;
    constexpr int ITEMS = N / R;  // butterflies per pencil
    // Inputs of a butterfly: k0 + r N/R; N/R is a multiple of 8 for every
    // radix plan, so in the padded layout they are base + r (N/R)(9/8).
    constexpr int IN_STRIDE = N / R + N / (8 * R);
    // Outputs: kb + S j with kb = q + S R p; for S >= 8 the padded stride is
    // S (9/8); for S == 1 (first pass, R == 8) kb = 8p and the outputs are
    // the 8 consecutive padded slots 9p .. 9p + 7.
    constexpr int OUT_STRIDE = S >= 8 ? S + S / 8 : 1;
    static_assert(S >= 8 || R == 8, "the first pass is radix 8");
    // In the last pass (S R == N) p is always 0: every twiddle is w^0 = 1,
    // and multiplying by (1, 0) returns its operand exactly, so it is skipped.
    constexpr bool LAST = S * R == N;
    for (int e = threadIdx.x; e < npair * ITEMS; e += blockDim.x) {
        const int c = e / ITEMS;  // ITEMS is a power of two
        const int t = e - c * ITEMS;
        const int q = LAST ? t : t % S;
        const int p = LAST ? 0 : t / S;
        const int k0 = q + S * p;
        const float2 *x = src + c * L::SN + k0 + (k0 >> 3);
        float2 a[R];
#pragma unroll
        for (int r = 0; r < R; r++) a[r] = x[r * IN_STRIDE];
        dft<R, INV>(a);
        if (!LAST) {
#pragma unroll
            for (int j = 1; j < R; j++) {
                float2 w = tw[(p * S * j) & (N - 1)];
                if (INV) w.y = -w.y;
                a[j] = cmul(a[j], w);
            }
        }
        const int kb = q + S * R * p;
        float2 *y = dst + c * L::SN + kb + (kb >> 3);
#pragma unroll
        for (int j = 0; j < R; j++) {
            float2 v = a[j];
            if (FILTER) {
                const float g = filt[kb + S * j];
                v.x *= g;
                v.y *= g;
            }
            y[j * OUT_STRIDE] = v;
        }
    }
    __syncthreads();
}

// Forward FFT, filter, inverse FFT of every pencil pair; result in b0.
template <int LOGN>
__device__ __forceinline__ void fft_filter_ifft(float2 *b0, float2 *b1, int npair, const float2 *tw,
                                                const float *filt) {
    constexpr int N = 1 << LOGN;
    // radix plan: 8, 8, then 1 (LOGN 6), 2 (7), 4 (8), 8 (9)
    constexpr int R3 = LOGN == 6 ? 1 : LOGN == 7 ? 2 : LOGN == 8 ? 4 : 8;
    static_assert(LOGN >= 6 && LOGN <= 9, "FFT lengths 64..512");
    if (R3 == 1) {
        stockham_pass<N, 8, 1, false, false>(b0, b1, npair, tw, filt);
        stockham_pass<N, 8, 8, false, true>(b1, b0, npair, tw, filt);
        stockham_pass<N, 8, 1, true, false>(b0, b1, npair, tw, filt);
        stockham_pass<N, 8, 8, true, false>(b1, b0, npair, tw, filt);
    } else {
        constexpr int R3v = R3 == 1 ? 2 : R3;
        stockham_pass<N, 8, 1, false, false>(b0, b1, npair, tw, filt);
        stockham_pass<N, 8, 8, false, false>(b1, b0, npair, tw, filt);
        stockham_pass<N, R3v, 64, false, true>(b0, b1, npair, tw, filt);
        stockham_pass<N, 8, 1, true, false>(b1, b0, npair, tw, filt);
        stockham_pass<N, 8, 8, true, false>(b0, b1, npair, tw, filt);
        stockham_pass<N, R3v, 64, true, false>(b1, b0, npair, tw, filt);
    }
}

// ---------------------------------------------------------------- on-chip meshes
// The whole mesh stage of a 64^3 mesh inside one cluster of 8 CTAs: CTA r
// holds z planes [8r, 8r + 8) in shared memory (rows padded to 65 floats, so
// columns along y and x-consecutive lanes are conflict-free), and reaches the
// other planes through distributed shared memory.  Per mesh: zero the slabs,
// deposit the TSC weights (the reference's arithmetic, float atomics into the
// owning CTA's slab), filter along x and y (local planes) and along z (columns
// read from all eight CTAs), then interpolate at every particle.  Each filter
// pass moves tiles of 128 real pencils into a padded buffer and runs the same
// Stockham FFT -> filter -> inverse FFT as the device-memory kernels.  Nothing
// of the mesh touches device memory; a cluster loops over meshes.
namespace oc {
constexpr int kN = kOnChipMesh;                 // 64 cells per axis
constexpr int kCtas = 8;                        // CTAs per cluster
constexpr int kPlanes = kN / kCtas;             // z planes per CTA
constexpr int kRow = kN + 1;                    // padded row stride (floats)
constexpr int kPlane = kN * kRow;               // plane stride (floats)
constexpr int kSlab = kPlanes * kPlane;         // floats per CTA
constexpr int kOcThreads = 512;
constexpr int kTilePencils = 128;               // real pencils per FFT tile
constexpr int kPairs = kTilePencils / 2;
constexpr int kTiles = kPlanes * kN / kTilePencils;  // tiles per pass per CTA (4)
using L = FftLayout<kN>;
constexpr size_t kSmem = (size_t)kSlab * sizeof(float) + 2 * (size_t)kPairs * L::SN * sizeof(float2);
static_assert(kOcThreads == kPairs * (kN / 8), "one radix-8 butterfly per thread and pass");
static_assert(kSmem <= 227 * 1024, "shared memory per CTA");
}  // namespace oc

struct OnChipArgs {
    int32_t nmesh;
    const int32_t *halos;
    int32_t ptype;
    const int64_t *pstart;
    const double *x, *y, *z, *mass;
    const int32_t *type;
    const gf_mesh_desc *mesh;
    const AxisTable *axes;
    const float *tables;
    float volfold;
    float *densph;
    int *err;
};

// One filter pass over the tile of real pencils whose element (p, s) lives
// at address(p, s) in (local or remote) shared memory.
template <class Addr>
__device__ __forceinline__ void onchip_tile(float2 *b0, float2 *b1, const AxisTable &at,
                                            const float *__restrict__ tables, Addr address) {
    using namespace oc;
    float *fa = reinterpret_cast<float *>(b0);
    constexpr int PER = kTilePencils * kN / kOcThreads;  // 16
    float v[PER];
#pragma unroll
    for (int r = 0; r < PER; r++) {
        const int e = threadIdx.x + r * kOcThreads;
        v[r] = *address(e & (kTilePencils - 1), e >> 7);
    }
#pragma unroll
    for (int r = 0; r < PER; r++) {
        const int e = threadIdx.x + r * kOcThreads;
        const int p = e & (kTilePencils - 1), s = e >> 7;
        fa[2 * L::at(p >> 1, s) + (p & 1)] = v[r];
    }
    __syncthreads();
    const float2 *tw = reinterpret_cast<const float2 *>(tables + at.tab_off);
    const float *filt = tables + at.tab_off + 2 * kN;
    fft_filter_ifft<6>(b0, b1, kPairs, tw, filt);
    const float *fs = reinterpret_cast<const float *>(b0);
#pragma unroll
    for (int r = 0; r < PER; r++) {
        const int e = threadIdx.x + r * kOcThreads;
        const int p = e & (kTilePencils - 1), s = e >> 7;
        *address(p, s) = fs[2 * L::at(p >> 1, s) + (p & 1)];
    }
    __syncthreads();
}

__global__ void __cluster_dims__(oc::kCtas, 1, 1) __launch_bounds__(oc::kOcThreads, 1)
mesh_onchip_kernel(OnChipArgs a) {
    using namespace oc;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    extern __shared__ float4 smem_f4[];
    float *slab = reinterpret_cast<float *>(smem_f4);
    float2 *b0 = reinterpret_cast<float2 *>(slab + kSlab);
    float2 *b1 = b0 + kPairs * L::SN;
    // the slab of CTA r of the cluster (distributed shared memory window)
    auto slabs = [&](int r) { return cluster.map_shared_rank(slab, r); };
    const int nclusters = gridDim.x / kCtas;
    for (int mi = blockIdx.x / kCtas; mi < a.nmesh; mi += nclusters) {
        const int h = a.halos[mi];
        const gf_mesh_desc m = a.mesh[h];
        for (int e = threadIdx.x; e < kSlab; e += kOcThreads) slab[e] = 0.f;
        cluster.sync();
        // ---- TSC deposit (tsc_omp2.c:166-506), into the CTA owning each plane
        const int64_t p0 = a.pstart[h], p1 = a.pstart[h + 1];
        for (int64_t p = p0 + rank * kOcThreads + threadIdx.x; p < p1; p += kCtas * kOcThreads) {
            if (a.ptype != GF_TYPE_ALL && (a.type ? a.type[p] : GF_TYPE_DM) != a.ptype) continue;
            TscStencil st;
            float xd1, yd1, zd1;
            tsc_cells(a.x[p], a.y[p], a.z[p], m, st, xd1, yd1, zd1);
            if (!tsc_in_mesh(st, m)) {
                atomicOr(a.err, GF_ERRBIT_RANGE);
                continue;
            }
            tsc_deposit_weights(st, xd1, yd1, zd1, a.mass[p]);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int k = (int)st.k[c];
                float *dst = slabs(k / kPlanes) + (k % kPlanes) * kPlane;
#pragma unroll
                for (int b = 0; b < 3; b++) {
#pragma unroll
                    for (int i = 0; i < 3; i++)
                        atomicAdd(dst + (int)st.j[b] * kRow + (int)st.i[i], tsc_deposit_value(st, i, b, c, a.volfold));
                }
            }
        }
        cluster.sync();
        // ---- filter along x: the CTA's 512 rows (plane, y), 128 per tile
        const AxisTable ax = a.axes[3 * h], ay = a.axes[3 * h + 1], az = a.axes[3 * h + 2];
        for (int t = 0; t < kTiles; t++) {
            onchip_tile(b0, b1, ax, a.tables, [&](int p, int s) {
                const int row = t * kTilePencils + p;
                return slab + (row / kN) * kPlane + (row % kN) * kRow + s;
            });
        }
        // ---- along y: columns (plane, x) of the CTA's planes
        for (int t = 0; t < kTiles; t++) {
            onchip_tile(b0, b1, ay, a.tables, [&](int p, int s) {
                const int col = t * kTilePencils + p;
                return slab + (col / kN) * kPlane + s * kRow + (col % kN);
            });
        }
        cluster.sync();
        // ---- along z: the CTA's share of the 64 x 64 columns, through all slabs
        for (int t = 0; t < kTiles; t++) {
            onchip_tile(b0, b1, az, a.tables, [&](int p, int s) {
                const int col = rank * (kN * kN / kCtas) + t * kTilePencils + p;
                return slabs(s / kPlanes) + (s % kPlanes) * kPlane + (col / kN) * kRow + (col % kN);
            });
        }
        cluster.sync();
        // ---- findDen (tsc_omp2.c:40-163) at every particle of the halo
        for (int64_t p = p0 + rank * kOcThreads + threadIdx.x; p < p1; p += kCtas * kOcThreads) {
            TscStencil st;
            float xd1, yd1, zd1;
            tsc_cells(a.x[p], a.y[p], a.z[p], m, st, xd1, yd1, zd1);
            if (!tsc_in_mesh(st, m)) {
                atomicOr(a.err, GF_ERRBIT_RANGE);
                a.densph[p] = 0.f;
                continue;
            }
            tsc_interp_weights(st, xd1, yd1, zd1);
            float density = 0.f;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int k = (int)st.k[c];
                const float *src = slabs(k / kPlanes) + (k % kPlanes) * kPlane;
#pragma unroll
                for (int b = 0; b < 3; b++) {
#pragma unroll
                    for (int i = 0; i < 3; i++)
                        density = tsc_interp_add(density, src[(int)st.j[b] * kRow + (int)st.i[i]], st, i, b, c);
                }
            }
            a.densph[p] = density;
        }
        cluster.sync();  // before the next mesh clears the slabs
    }
}

int launch_onchip(gf_ctx *ctx, const OnChipArgs &a) {
    if (a.nmesh <= 0) return GF_OK;
    GF_CUDA_TRY(cudaFuncSetAttribute(mesh_onchip_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)oc::kSmem));
    // as many clusters as can be resident at once (each loops over meshes)
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = oc::kCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(oc::kOcThreads);
    cfg.gridDim = dim3(oc::kCtas * 64);
    cfg.dynamicSmemBytes = oc::kSmem;
    cfg.stream = ctx->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, mesh_onchip_kernel, &cfg) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        nclusters = std::max(1, sm_count() / oc::kCtas);
    }
    nclusters = std::min(nclusters, a.nmesh);
    mesh_onchip_kernel<<<nclusters * oc::kCtas, oc::kOcThreads, oc::kSmem, ctx->stream>>>(a);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

constexpr int kPencils = GF_FFT_PENCILS;  // real pencils per FFT tile (2 per complex pencil)

// Real pencils per tile of an FFT axis of 2^LOGN cells: wider tiles for the
// short axes, whose tiles are otherwise small (8 KB at 64 cells).
template <int LOGN>
struct FftTile {
    static constexpr int P = LOGN == 6 ? GF_FFT_PENCILS_64 : LOGN == 7 ? GF_FFT_PENCILS_128 : kPencils;
    static constexpr int NT = (P / 2) * (1 << LOGN) / 8;  // threads per tile
};
static_assert(FftTile<9>::NT <= 1024 && FftTile<6>::NT <= 1024 && FftTile<7>::NT <= 1024, "FFT tile threads");

int fft_tile_pencils(int n) {
    return n == 64 ? FftTile<6>::P : n == 128 ? FftTile<7>::P : kPencils;
}

template <int AXIS, int LOGN>
__global__ void __launch_bounds__(FftTile<LOGN>::NT)
smooth_fft_kernel(float *__restrict__ den, const gf_mesh_desc *__restrict__ mesh, GroupLaunch g,
                  const AxisTable *__restrict__ axes, const float *__restrict__ tables,
                  const int32_t *__restrict__ boxes, int trim) {
    constexpr int N = 1 << LOGN;
    constexpr int P = FftTile<LOGN>::P;
    using L = FftLayout<N>;
    extern __shared__ float2 smem[];
    const SmoothTile t = decode_group_tile<AXIS>(blockIdx.x, g, mesh, P);
    const gf_mesh_desc m = mesh[t.halo];
    // the whole block leaves together (before any barrier)
    if (boxes && !tile_needed<AXIS>(t, m, boxes + (int64_t)kMeshBoxInts * t.halo, trim)) return;
    const AxisTable at = axes[3 * t.halo + AXIS];
    const int64_t mx = 2 * (m.nx / 2 + 1);
    const int npair = (t.npen + 1) >> 1;
    float2 *b0 = smem;
    float2 *b1 = smem + (P / 2) * L::SN;
    float *fa = reinterpret_cast<float *>(b0);
    // element (pencil p, position s) lives at base + p*pstride + s*sstride;
    // within one tile the offsets fit in 32 bits (axes <= 512, mx*ny < 2^21)
    int64_t base;
    int pstride, sstride;
    if (AXIS == 0) { base = m.off + mx * t.base; pstride = (int)mx; sstride = 1; }
    else if (AXIS == 1) { base = m.off + t.base + mx * (int64_t)m.ny * t.other; pstride = 1; sstride = (int)mx; }
    else { base = m.off + t.base + mx * (int64_t)t.other; pstride = 1; sstride = (int)(mx * m.ny); }
    const float *gsrc = den + base;
    const int npen2 = 2 * npair;  // pencils held, the last one zero when npen is odd
    // All of a thread's loads are issued before any is stored to shared
    // memory (a fixed count per thread, unrolled), so each warp keeps them
    // all in flight.
    constexpr int NT = FftTile<LOGN>::NT;  // threads per tile
    if (AXIS == 0) {  // rows: consecutive threads walk along a row
        constexpr int PER = P * N / NT;
        float v[PER];
#pragma unroll
        for (int r = 0; r < PER; r++) {
            const int e = threadIdx.x + r * NT;
            const int p = e >> LOGN, s = e & (N - 1);
            v[r] = p < t.npen ? gsrc[p * pstride + s] : 0.f;
        }
#pragma unroll
        for (int r = 0; r < PER; r++) {
            const int e = threadIdx.x + r * NT;
            const int p = e >> LOGN, s = e & (N - 1);
            fa[2 * L::at(p >> 1, s) + (p & 1)] = v[r];
        }
    } else {  // columns: consecutive threads take consecutive pencils (x), groups of P step along the axis
        constexpr int NG = NT / P;
        constexpr int PER = N / NG;
        const int p = threadIdx.x % P;
        const int w = threadIdx.x / P;
        if (p < npen2) {
            float v[PER];
#pragma unroll
            for (int r = 0; r < PER; r++) v[r] = p < t.npen ? gsrc[p + (w + r * NG) * sstride] : 0.f;
#pragma unroll
            for (int r = 0; r < PER; r++) fa[2 * L::at(p >> 1, w + r * NG) + (p & 1)] = v[r];
        }
    }
    __syncthreads();
    // full twiddle table e^{-2 pi i k/N}, k < N, then N filter factors G/N
    const float2 *tw = reinterpret_cast<const float2 *>(tables + at.tab_off);
    const float *filt = tables + at.tab_off + 2 * N;
    fft_filter_ifft<LOGN>(b0, b1, npair, tw, filt);
    const float *fs = reinterpret_cast<const float *>(b0);
    float *gdst = den + base;
    if (AXIS == 0) {
        for (int e = threadIdx.x; e < npen2 * N; e += blockDim.x) {
            const int p = e >> LOGN, s = e & (N - 1);
            if (p < t.npen) gdst[p * pstride + s] = fs[2 * L::at(p >> 1, s) + (p & 1)];
        }
    } else {
        constexpr int NG = NT / P;
        const int p = threadIdx.x % P;
        if (p < t.npen) {
            for (int s = threadIdx.x / P; s < N; s += NG)
                gdst[p + s * sstride] = fs[2 * L::at(p >> 1, s) + (p & 1)];
        }
    }
}

// ------------------------------------------------- box-restricted passes
// The stage's meshes are read only by findDen, at the cells of the
// evaluation box E (the stencils of every particle); the deposit writes only
// the deposit box D (E contains D).  Each pass then needs only part of the
// mesh, and every cell it reads outside D is a known zero:
//   x: rows (y, z) in D_y x D_z; reads x in D_x (zero elsewhere); writes x in E_x
//   y: columns (x, z) in E_x x D_z; reads y in D_y; writes y in E_y
//   z: columns (x, y) in E_x x E_y; reads z in D_z; writes z in E_z
// so only D has to be zeroed before the deposit, and findDen reads exactly
// the cells the z pass wrote.  The FFT of a pencil whose zeros come from
// registers instead of memory is the same computation, so the values at the
// cells findDen reads equal those of full passes over a zeroed mesh (up to
// the pairing of real pencils into complex ones, a rounding-level change).
// A mesh with no deposited particle gets its evaluation box zeroed instead
// and no pass.  The tile lists are counted on the device from the boxes
// (a CUDA graph replays them for new particle positions).
struct BoxGeom {
    int u0, nu, v0, nv;                // pencil grid: u fastest
    int ustride, vstride, sstride;     // float offsets within the mesh
    int l0, l1, s0, s1;                // read and write ranges along the pencil
};

__device__ __forceinline__ int box_len(int lo, int hi) { return hi >= lo ? hi - lo + 1 : 0; }

template <int AXIS>
__device__ __forceinline__ BoxGeom box_geom(const gf_mesh_desc &m, const int32_t *__restrict__ bx) {
    const int mx = 2 * (m.nx / 2 + 1);
    BoxGeom g;
    if (AXIS == 0) {
        g.u0 = bx[2]; g.nu = box_len(bx[2], bx[3]); g.v0 = bx[4]; g.nv = box_len(bx[4], bx[5]);
        g.ustride = mx; g.vstride = mx * m.ny; g.sstride = 1;
        g.l0 = bx[0]; g.l1 = bx[1]; g.s0 = bx[6]; g.s1 = bx[7];
    } else if (AXIS == 1) {
        g.u0 = bx[6]; g.nu = box_len(bx[6], bx[7]); g.v0 = bx[4]; g.nv = box_len(bx[4], bx[5]);
        g.ustride = 1; g.vstride = mx * m.ny; g.sstride = mx;
        g.l0 = bx[2]; g.l1 = bx[3]; g.s0 = bx[8]; g.s1 = bx[9];
    } else {
        g.u0 = bx[6]; g.nu = box_len(bx[6], bx[7]); g.v0 = bx[8]; g.nv = box_len(bx[8], bx[9]);
        g.ustride = 1; g.vstride = mx; g.sstride = mx * m.ny;
        g.l0 = bx[4]; g.l1 = bx[5]; g.s0 = bx[10]; g.s1 = bx[11];
    }
    if (bx[0] > bx[1]) g.nu = g.nv = 0;  // nothing deposited: no pass
    return g;
}

__device__ __forceinline__ int64_t box_tiles(int axis, const int32_t *__restrict__ bx, int pmax) {
    if (bx[0] > bx[1]) return 0;
    int64_t pen;
    if (axis == 0) pen = (int64_t)box_len(bx[2], bx[3]) * box_len(bx[4], bx[5]);
    else if (axis == 1) pen = (int64_t)box_len(bx[6], bx[7]) * box_len(bx[4], bx[5]);
    else pen = (int64_t)box_len(bx[6], bx[7]) * box_len(bx[8], bx[9]);
    return (pen + pmax - 1) / pmax;
}

// rows (y, z) zeroed before the deposit: those of D, or of E when D is empty
__device__ __forceinline__ int64_t box_zero_rows(const gf_mesh_desc &m, const int32_t *__restrict__ bx) {
    if (m.ptype == kMeshOnChip) return 0;
    const int o = bx[0] <= bx[1] ? 0 : 6;
    return (int64_t)box_len(bx[o + 2], bx[o + 3]) * box_len(bx[o + 4], bx[o + 5]);
}

constexpr int kBoxMaxGroups = 16;
struct BoxPlanGroup {
    const int32_t *halos;
    int64_t *starts;  // ngroup + 1, written here
    int32_t ngroup, axis, pmax;
};
struct BoxPlanArgs {
    int32_t ngroups, nhalo;
    BoxPlanGroup g[kBoxMaxGroups];
    const int32_t *boxes;
    const gf_mesh_desc *mesh;
    int64_t *zstart;  // nhalo + 1, written here: prefix of the rows to zero
};

// Exclusive prefix sums of the per-halo tile counts of every group (block
// g < ngroups) and of the zeroed rows of every mesh (block ngroups).
__global__ void __launch_bounds__(1024) box_plan_kernel(BoxPlanArgs a) {
    __shared__ int64_t part[1024];
    const bool zero = (int)blockIdx.x == a.ngroups;
    const BoxPlanGroup G = zero ? BoxPlanGroup{nullptr, a.zstart, a.nhalo, 0, 1} : a.g[blockIdx.x];
    auto count = [&](int i) -> int64_t {
        if (zero) return box_zero_rows(a.mesh[i], a.boxes + (int64_t)kMeshBoxInts * i);
        return box_tiles(G.axis, a.boxes + (int64_t)kMeshBoxInts * G.halos[i], G.pmax);
    };
    const int cnt = G.ngroup, per = (cnt + 1023) / 1024;
    const int i0 = min(cnt, (int)threadIdx.x * per), i1 = min(cnt, i0 + per);
    int64_t s = 0;
    for (int i = i0; i < i1; i++) s += count(i);
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {  // inclusive scan (Hillis-Steele)
        const int64_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int64_t run = part[threadIdx.x] - s;
    for (int i = i0; i < i1; i++) {
        G.starts[i] = run;
        run += count(i);
    }
    if (threadIdx.x == 1023) G.starts[cnt] = part[1023];
}

// Contiguous share [t0, t1) of `total` items for this block.
__device__ __forceinline__ void block_share(int64_t total, int64_t &t0, int64_t &t1) {
    const int64_t per = (total + gridDim.x - 1) / gridDim.x;
    t0 = min(total, (int64_t)blockIdx.x * per);
    t1 = min(total, t0 + per);
}

// The entry i of a prefix array with starts[i] <= b < starts[i + 1],
// searching upwards from a known lower bound.
__device__ __forceinline__ int prefix_find(const int64_t *__restrict__ starts, int lo, int hi, int64_t b) {
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(starts + mid) <= b) lo = mid; else hi = mid;
    }
    return lo;
}

// Zeroes the rows of every mesh's deposit box (its evaluation box when
// nothing is deposited): each warp takes a contiguous share of all rows
// (balanced whatever the mesh sizes), its lanes store along x.
__global__ void __launch_bounds__(256) zero_box_kernel(float *__restrict__ den, const gf_mesh_desc *__restrict__ mesh,
                                                       const int32_t *__restrict__ boxes,
                                                       const int64_t *__restrict__ zstart, int32_t nhalo) {
    const int64_t total = zstart[nhalo];
    const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t per = (total + nw - 1) / nw;
    int64_t r = min(total, w * per);
    const int64_t r1 = min(total, r + per);
    int h = 0;
    while (r < r1) {
        h = prefix_find(zstart, h, nhalo, r);
        const gf_mesh_desc m = mesh[h];
        const int32_t *bx = boxes + (int64_t)kMeshBoxInts * h;
        const int o = bx[0] <= bx[1] ? 0 : 6;  // D, or E when nothing was deposited
        const int nyb = box_len(bx[o + 2], bx[o + 3]);
        const int64_t local = r - zstart[h];
        int z = bx[o + 4] + (int)(local / nyb);
        int y = bx[o + 2] + (int)(local % nyb);
        const int64_t mx = 2 * (m.nx / 2 + 1);
        const int64_t rend = min(r1, zstart[h + 1]);
        for (; r < rend; r++) {
            float *row = den + m.off + mx * (y + (int64_t)m.ny * z);
            for (int x = bx[o] + lane; x <= bx[o + 1]; x += 32) row[x] = 0.f;
            if (++y > bx[o + 3]) {
                y = bx[o + 2];
                z++;
            }
        }
    }
}

template <int AXIS, int LOGN>
__global__ void __launch_bounds__(FftTile<LOGN>::NT)
smooth_box_kernel(float *__restrict__ den, const gf_mesh_desc *__restrict__ mesh, GroupLaunch g,
                  const AxisTable *__restrict__ axes, const float *__restrict__ tables,
                  const int32_t *__restrict__ boxes) {
    constexpr int N = 1 << LOGN;
    constexpr int P = FftTile<LOGN>::P;
    constexpr int NT = FftTile<LOGN>::NT;
    using L = FftLayout<N>;
    extern __shared__ float2 smem[];
    __shared__ int32_t pb[P];  // offset of each pencil of the tile within its mesh
    float2 *b0 = smem;
    float2 *b1 = smem + (P / 2) * L::SN;
    float *fa = reinterpret_cast<float *>(b0);
    int64_t t0, t1;
    block_share(g.tile_start[g.ngroup], t0, t1);
    int gi = -1;
    for (int64_t tb = t0; tb < t1; tb++) {
        gi = (gi < 0 || __ldg(g.tile_start + gi + 1) <= tb) ? prefix_find(g.tile_start, max(gi, 0), g.ngroup, tb)
                                                           : gi;
        const int h = g.halos[gi];
        const gf_mesh_desc m = mesh[h];
        const BoxGeom q = box_geom<AXIS>(m, boxes + (int64_t)kMeshBoxInts * h);
        const int64_t f0 = (tb - g.tile_start[gi]) * P;
        const int npen = (int)min((int64_t)P, (int64_t)q.nu * q.nv - f0);
        if (threadIdx.x < P) {
            const int64_t f = f0 + threadIdx.x;
            const int v = (int)(f / q.nu), u = (int)(f - (int64_t)v * q.nu);
            pb[threadIdx.x] = (q.u0 + u) * q.ustride + (q.v0 + v) * q.vstride;  // unused beyond npen
        }
        __syncthreads();
        const float *gm = den + m.off;
        const int npair = (npen + 1) >> 1;
        if (AXIS == 0) {  // rows: consecutive threads walk along a row
            constexpr int PER = P * N / NT;
            float v[PER];
#pragma unroll
            for (int r = 0; r < PER; r++) {
                const int e = threadIdx.x + r * NT;
                const int p = e >> LOGN, s = e & (N - 1);
                v[r] = (p < npen && s >= q.l0 && s <= q.l1) ? gm[pb[p] + s] : 0.f;
            }
#pragma unroll
            for (int r = 0; r < PER; r++) {
                const int e = threadIdx.x + r * NT;
                const int p = e >> LOGN, s = e & (N - 1);
                fa[2 * L::at(p >> 1, s) + (p & 1)] = v[r];
            }
        } else {  // columns: consecutive threads take consecutive pencils
            constexpr int NG = NT / P;
            constexpr int PER = N / NG;
            const int p = threadIdx.x % P;
            const int w = threadIdx.x / P;
            float v[PER];
#pragma unroll
            for (int r = 0; r < PER; r++) {
                const int s = w + r * NG;
                v[r] = (p < npen && s >= q.l0 && s <= q.l1) ? gm[pb[p] + s * q.sstride] : 0.f;
            }
#pragma unroll
            for (int r = 0; r < PER; r++) fa[2 * L::at(p >> 1, w + r * NG) + (p & 1)] = v[r];
        }
        __syncthreads();
        const AxisTable at = axes[3 * h + AXIS];
        const float2 *tw = reinterpret_cast<const float2 *>(tables + at.tab_off);
        const float *filt = tables + at.tab_off + 2 * N;
        fft_filter_ifft<LOGN>(b0, b1, npair, tw, filt);
        const float *fs = reinterpret_cast<const float *>(b0);
        float *gd = den + m.off;
        if (AXIS == 0) {
            for (int e = threadIdx.x; e < npen * N; e += NT) {
                const int p = e >> LOGN, s = e & (N - 1);
                if (s >= q.s0 && s <= q.s1) gd[pb[p] + s] = fs[2 * L::at(p >> 1, s) + (p & 1)];
            }
        } else {
            constexpr int NG = NT / P;
            const int p = threadIdx.x % P;
            if (p < npen) {
                for (int s = q.s0 + threadIdx.x / P; s <= q.s1; s += NG)
                    gd[pb[p] + s * q.sstride] = fs[2 * L::at(p >> 1, s) + (p & 1)];
            }
        }
        __syncthreads();  // the tile buffers and pb are reused by the next tile
    }
}

int ilog2_exact(int n) {
    if (n <= 0 || (n & (n - 1))) return -1;
    int l = 0;
    while ((1 << l) < n) l++;
    return l;
}

// Spectral factor of one axis (gsmooth.c:67-86): G(k) = exp(k_s^2 expfac / n^2)
// with k_s the signed frequency, expfac = -(pi RG/cellsize)^2.
double axis_factor(int k, int n, double rg_cells) {
    const double expfac = -(M_PI * rg_cells) * (M_PI * rg_cells);
    long ks = k;
    if (k > n / 2) ks = k - n;
    return exp((double)(ks * ks) * expfac / ((double)n * (double)n));
}

enum PathKind { PATH_FFT8 = 0, PATH_RADIX2 = 1, PATH_DIRECT = 2 };

PathKind path_of(int n) {
    const int l = ilog2_exact(n);
    if (l >= 6 && l <= 9) return PATH_FFT8;
    if (l >= 1) return PATH_RADIX2;
    return PATH_DIRECT;
}

// Table layouts: FFT8: [e^{-2 pi i k/n}, k < n (float2)][G/n (n floats)];
// RADIX2: [e^{-2 pi i k/n}, k < n/2 (float2)][G/n]; DIRECT: [h_n (n floats)].
// Twiddles and filters are evaluated in FP64 and rounded once.

// Floats of the table of an axis of n cells.
int64_t axis_table_floats(int n) {
    const PathKind pk = path_of(n);
    if (pk == PATH_DIRECT) return n;
    return 2 * (int64_t)(pk == PATH_FFT8 ? n : n / 2) + n;
}

// Writes the table of one axis into out[0 .. axis_table_floats(n)).  The
// direct path needs two FP64 work arrays of n entries (g: the spectral
// factors, c: cos(2 pi j / n)); both plan builders pass their own, so the
// allocation-free one can keep them on its stack.
void write_axis_tables(int n, double rg_cells, float *out, double *g, double *c) {
    const PathKind pk = path_of(n);
    int64_t k = 0;
    if (pk != PATH_DIRECT) {
        const int ntw = pk == PATH_FFT8 ? n : n / 2;
        for (int i = 0; i < ntw; i++) {
            const double ang = 2.0 * M_PI * (double)i / (double)n;
            out[k++] = (float)cos(ang);
            out[k++] = (float)-sin(ang);
        }
        for (int i = 0; i < n; i++) out[k++] = (float)(axis_factor(i, n, rg_cells) / n);
    } else {
        // h_m = (1/n) sum_i G_i cos(2 pi (i m mod n) / n): the cosine of each
        // residue is evaluated once (n calls instead of n^2)
        for (int i = 0; i < n; i++) {
            g[i] = axis_factor(i, n, rg_cells);
            c[i] = cos(2.0 * M_PI * (double)i / (double)n);
        }
        for (int mm = 0; mm < n; mm++) {
            double acc = 0.0;
            for (int i = 0; i < n; i++) acc += g[i] * c[((long)i * mm) % n];
            out[k++] = (float)(acc / n);
        }
    }
}

void append_tables(std::vector<float> &tab, int n, double rg_cells, AxisTable &at) {
    // every table starts on a 16-byte boundary: the FFT paths read float2
    // twiddles, and a preceding table may hold an odd number of floats
    while (tab.size() % 4) tab.push_back(0.f);
    at.n = n;
    at.logn = path_of(n) == PATH_DIRECT ? -1 : ilog2_exact(n);
    at.tab_off = (int64_t)tab.size();
    const size_t base = tab.size();
    tab.resize(base + (size_t)axis_table_floats(n));
    std::vector<double> work(path_of(n) == PATH_DIRECT ? 2 * (size_t)n : 0);
    write_axis_tables(n, rg_cells, tab.data() + base, work.data(), work.data() + (work.empty() ? 0 : n));
}

template <int AXIS, int LOGN>
int launch_fft(gf_ctx *ctx, float *den, const gf_mesh_desc *mesh_dev, GroupLaunch g, int64_t ntiles,
               const AxisTable *axes, const float *tables, const int32_t *boxes, int trim) {
    constexpr int N = 1 << LOGN;
    const int threads = FftTile<LOGN>::NT;
    const size_t smem = (size_t)2 * (FftTile<LOGN>::P / 2) * FftLayout<N>::SN * sizeof(float2);
    GF_CUDA_TRY(cudaFuncSetAttribute(smooth_fft_kernel<AXIS, LOGN>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    smooth_fft_kernel<AXIS, LOGN><<<(unsigned)ntiles, threads, smem, ctx->stream>>>(den, mesh_dev, g,
                                                                                   axes, tables, boxes, trim);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

template <int AXIS>
int launch_group(gf_ctx *ctx, float *den, const gf_mesh_desc *mesh_dev, GroupLaunch g,
                 int64_t ntiles, int n, int pmax, const AxisTable *axes, const float *tables,
                 const int32_t *boxes = nullptr, int trim = 0) {
    if (ntiles == 0) return GF_OK;
    if (ntiles > 0x7fffffffLL) {
        set_status(GF_ENOTIMPL, "%lld smoothing tiles exceed one launch", (long long)ntiles);
        return GF_ENOTIMPL;
    }
    if (path_of(n) == PATH_FFT8 && pmax != fft_tile_pencils(n)) {
        // the FFT kernel decodes every tile as fft_tile_pencils(n) pencils: a
        // plan cut for another width would leave pencils unsmoothed
        set_status(GF_EINVAL, "smoothing plan of %d pencils per tile for a %d-cell FFT axis; the "
                   "kernel was built for %d", pmax, n, fft_tile_pencils(n));
        return GF_EINVAL;
    }
    switch (path_of(n) == PATH_FFT8 ? ilog2_exact(n) : 0) {
        case 6: return launch_fft<AXIS, 6>(ctx, den, mesh_dev, g, ntiles, axes, tables, boxes, trim);
        case 7: return launch_fft<AXIS, 7>(ctx, den, mesh_dev, g, ntiles, axes, tables, boxes, trim);
        case 8: return launch_fft<AXIS, 8>(ctx, den, mesh_dev, g, ntiles, axes, tables, boxes, trim);
        case 9: return launch_fft<AXIS, 9>(ctx, den, mesh_dev, g, ntiles, axes, tables, boxes, trim);
        default: break;
    }
    const size_t smem = (size_t)2 * ((pmax + 1) / 2) * n * sizeof(float2);
    GF_CUDA_TRY(cudaFuncSetAttribute(smooth_axis_kernel<AXIS>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    smooth_axis_kernel<AXIS><<<(unsigned)ntiles, kThreads, smem, ctx->stream>>>(den, mesh_dev, g, axes,
                                                                                tables, pmax, boxes, trim);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

}  // namespace

int smooth_plan(int32_t nhalo, const gf_mesh_desc *mesh_host, const OnChipMeshes *onchip, SmoothPlan *plan) {
    *plan = SmoothPlan();
    if (nhalo <= 0) return GF_OK;
    const int32_t non_chip = onchip ? onchip->nmesh : 0;  // meshes on chip
    std::vector<AxisTable> axes(3 * (size_t)nhalo);
    std::vector<float> tables;
    std::map<std::pair<int, double>, AxisTable> cache;
    for (int h = 0; h < nhalo; h++) {
        const gf_mesh_desc &m = mesh_host[h];
        if (m.nx < 1 || m.ny < 1 || m.nz < 1 || !(m.cellsize > 0)) {
            set_status(GF_EINVAL, "halo %d: bad mesh %d x %d x %d", h, m.nx, m.ny, m.nz);
            return GF_EINVAL;
        }
        // gsmooth.c:67 stores RG/cellsize back into the float RG
        const double rg_cells = (double)(float)(m.rg / m.cellsize);
        const int dims[3] = {m.nx, m.ny, m.nz};
        for (int a = 0; a < 3; a++) {
            auto key = std::make_pair(dims[a], rg_cells);
            auto it = cache.find(key);
            if (it == cache.end()) {
                AxisTable at;
                append_tables(tables, dims[a], rg_cells, at);
                it = cache.emplace(key, at).first;
            }
            axes[3 * (size_t)h + a] = it->second;
        }
    }
    // groups: (axis, n) for the FFT path; one group per axis for the rest
    struct Group {
        int axis, n, pmax;
        std::vector<int32_t> halos;
        std::vector<int64_t> start;
    };
    std::vector<Group> groups;
    std::map<std::pair<int, int>, size_t> gidx;
    for (int a = 0; a < 3; a++) {
        for (int h = 0; h < nhalo; h++) {
            const gf_mesh_desc &m = mesh_host[h];
            if (m.ptype == kMeshOnChip) continue;  // smoothed on chip
            const int dims[3] = {m.nx, m.ny, m.nz};
            const int n = dims[a];
            const int key_n = path_of(n) == PATH_FFT8 ? n : -1;
            auto k = std::make_pair(a, key_n);
            auto it = gidx.find(k);
            if (it == gidx.end()) {
                it = gidx.emplace(k, groups.size()).first;
                groups.push_back(Group{a, n, 0, {}, {0}});
            }
            Group &g = groups[it->second];
            g.halos.push_back(h);
            g.n = std::max(g.n, n);
        }
    }
    for (Group &g : groups) {
        if (path_of(g.n) == PATH_FFT8 && g.n == (1 << ilog2_exact(g.n))) {
            g.pmax = fft_tile_pencils(g.n);
        } else {
            int pmax = 32;
            while (pmax > 2 && (size_t)2 * (pmax / 2) * g.n * sizeof(float2) > 200 * 1024) pmax -= 2;
            if ((size_t)2 * (pmax / 2) * g.n * sizeof(float2) > 200 * 1024) {
                set_status(GF_ENOTIMPL, "mesh axis of %d cells exceeds the shared-memory pencil tile", g.n);
                return GF_ENOTIMPL;
            }
            g.pmax = pmax;
        }
        for (int32_t h : g.halos) {
            const gf_mesh_desc &m = mesh_host[h];
            const int64_t cx = (m.nx + g.pmax - 1) / g.pmax;
            int64_t c = g.axis == 0 ? ((int64_t)m.ny * m.nz + g.pmax - 1) / g.pmax
                                    : cx * (g.axis == 1 ? m.nz : m.ny);
            g.start.push_back(g.start.back() + c);
        }
    }
    // the box-restricted passes (smooth_box_launch) cover FFT axes only
    plan->box_ok = groups.size() <= (size_t)kBoxMaxGroups;
    for (const Group &g : groups)
        if (path_of(g.n) != PATH_FFT8 || g.pmax != fft_tile_pencils(g.n)) plan->box_ok = false;
    plan->nhalo = nhalo;
    // one blob: [axes | tables | on-chip halos | per group: halos, starts | zeroed-plane prefix]
    auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
    size_t off = align(axes.size() * sizeof(AxisTable));
    plan->off_tab = off;
    off = align(off + tables.size() * sizeof(float));
    plan->off_chip = off;
    plan->nchip = non_chip;
    off = align(off + (size_t)non_chip * sizeof(int32_t));
    std::vector<size_t> off_h(groups.size()), off_s(groups.size());
    for (size_t i = 0; i < groups.size(); i++) {
        off_h[i] = off;
        off = align(off + groups[i].halos.size() * sizeof(int32_t));
        off_s[i] = off;
        off = align(off + groups[i].start.size() * sizeof(int64_t));
    }
    plan->off_zero = off;
    off = align(off + ((size_t)nhalo + 1) * sizeof(int64_t));
    plan->blob.assign(off, 0);
    char *hbuf = plan->blob.data();
    memcpy(hbuf, axes.data(), axes.size() * sizeof(AxisTable));
    memcpy(hbuf + plan->off_tab, tables.data(), tables.size() * sizeof(float));
    if (non_chip) memcpy(hbuf + plan->off_chip, onchip->halos_host, (size_t)non_chip * sizeof(int32_t));
    for (size_t i = 0; i < groups.size(); i++) {
        memcpy(hbuf + off_h[i], groups[i].halos.data(), groups[i].halos.size() * sizeof(int32_t));
        memcpy(hbuf + off_s[i], groups[i].start.data(), groups[i].start.size() * sizeof(int64_t));
        SmoothGroup sg;
        sg.axis = groups[i].axis;
        sg.n = groups[i].n;
        sg.pmax = groups[i].pmax;
        sg.off_halos = off_h[i];
        sg.off_starts = off_s[i];
        sg.ngroup = (int32_t)groups[i].halos.size();
        sg.ntiles = groups[i].start.back();
        plan->groups.push_back(sg);
    }
    return GF_OK;
}

int smooth_launch(gf_ctx *ctx, const SmoothPlan &plan, const char *dbuf, const gf_mesh_desc *mesh_dev,
                  float *den, const OnChipMeshes *onchip, const MeshBoxes *boxes) {
    if (plan.blob.empty()) return GF_OK;
    const int32_t *bx = boxes ? boxes->dev : nullptr;
    const int trim = boxes && boxes->trim_last ? 1 : 0;
    const AxisTable *d_axes = reinterpret_cast<const AxisTable *>(dbuf);
    const float *d_tab = reinterpret_cast<const float *>(dbuf + plan.off_tab);
    for (const SmoothGroup &g : plan.groups) {
        GroupLaunch gl;
        gl.halos = reinterpret_cast<const int32_t *>(dbuf + g.off_halos);
        gl.tile_start = reinterpret_cast<const int64_t *>(dbuf + g.off_starts);
        gl.ngroup = g.ngroup;
        if (g.axis == 0) GF_TRY(launch_group<0>(ctx, den, mesh_dev, gl, g.ntiles, g.n, g.pmax, d_axes, d_tab, bx, trim));
        else if (g.axis == 1) GF_TRY(launch_group<1>(ctx, den, mesh_dev, gl, g.ntiles, g.n, g.pmax, d_axes, d_tab, bx, trim));
        else GF_TRY(launch_group<2>(ctx, den, mesh_dev, gl, g.ntiles, g.n, g.pmax, d_axes, d_tab, bx, trim));
    }
    if (plan.nchip) {
        OnChipArgs a;
        a.nmesh = plan.nchip;
        a.halos = reinterpret_cast<const int32_t *>(dbuf + plan.off_chip);
        a.ptype = onchip->ptype;
        a.pstart = onchip->pstart;
        a.x = onchip->x;
        a.y = onchip->y;
        a.z = onchip->z;
        a.mass = onchip->mass;
        a.type = onchip->type;
        a.mesh = mesh_dev;
        a.axes = d_axes;
        a.tables = d_tab;
        a.volfold = onchip->volfold;
        a.densph = onchip->densph;
        a.err = ctx->d_err;
        GF_TRY(launch_onchip(ctx, a));
    }
    return GF_OK;
}

int smooth_upload(gf_ctx *ctx, const SmoothPlan &plan, char **dbuf) {
    *dbuf = nullptr;
    if (plan.blob.empty()) return GF_OK;
    const size_t total = plan.blob.size();
    GF_TRY(ctx->smooth_tables.reserve(total));
    GF_TRY(ctx->pin[3].reserve(total));
    // the pinned staging buffer may still feed an earlier asynchronous copy
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    memcpy(ctx->pin[3].ptr, plan.blob.data(), total);
    *dbuf = ctx->smooth_tables.as<char>();
    GF_CUDA_TRY(cudaMemcpyAsync(*dbuf, ctx->pin[3].ptr, total, cudaMemcpyHostToDevice, ctx->stream));
    return GF_OK;
}

int smooth_meshes(gf_ctx *ctx, int32_t nhalo, const gf_mesh_desc *mesh_host,
                  const gf_mesh_desc *mesh_dev, float *den, const OnChipMeshes *onchip,
                  const MeshBoxes *boxes) {
    SmoothPlan plan;
    GF_TRY(smooth_plan(nhalo, mesh_host, onchip, &plan));
    if (plan.blob.empty()) return GF_OK;
    char *dbuf = nullptr;
    GF_TRY(smooth_upload(ctx, plan, &dbuf));
    return smooth_launch(ctx, plan, dbuf, mesh_dev, den, onchip, boxes);
}

namespace {

template <int AXIS, int LOGN>
int launch_box_fft(gf_ctx *ctx, float *den, const gf_mesh_desc *mesh_dev, GroupLaunch g, int64_t max_tiles,
                   const AxisTable *axes, const float *tables, const int32_t *boxes) {
    constexpr int N = 1 << LOGN;
    const int threads = FftTile<LOGN>::NT;
    const size_t smem = (size_t)2 * (FftTile<LOGN>::P / 2) * FftLayout<N>::SN * sizeof(float2);
    auto kern = smooth_box_kernel<AXIS, LOGN>;
    GF_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    GF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    // one resident wave; every block takes a contiguous share of the tiles
    // the device counted (at most max_tiles, the whole-mesh count)
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(max_tiles, (int64_t)sm_count() * std::max(per_sm, 1)));
    kern<<<(unsigned)grid, threads, smem, ctx->stream>>>(den, mesh_dev, g, axes, tables, boxes);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

template <int AXIS>
int launch_box_group(gf_ctx *ctx, float *den, const gf_mesh_desc *mesh_dev, GroupLaunch g, int64_t max_tiles,
                     int n, const AxisTable *axes, const float *tables, const int32_t *boxes) {
    if (max_tiles == 0) return GF_OK;
    switch (ilog2_exact(n)) {
        case 6: return launch_box_fft<AXIS, 6>(ctx, den, mesh_dev, g, max_tiles, axes, tables, boxes);
        case 7: return launch_box_fft<AXIS, 7>(ctx, den, mesh_dev, g, max_tiles, axes, tables, boxes);
        case 8: return launch_box_fft<AXIS, 8>(ctx, den, mesh_dev, g, max_tiles, axes, tables, boxes);
        case 9: return launch_box_fft<AXIS, 9>(ctx, den, mesh_dev, g, max_tiles, axes, tables, boxes);
        default: break;
    }
    set_status(GF_EINVAL, "box-restricted smoothing of a %d-cell axis (FFT axes of 64..512 cells only)", n);
    return GF_EINVAL;
}

}  // namespace

int smooth_box_prepare(gf_ctx *ctx, const SmoothPlan &plan, char *dbuf, const gf_mesh_desc *mesh_dev,
                       float *den, const int32_t *boxes) {
    if (plan.blob.empty() || plan.nhalo <= 0) return GF_OK;
    if (!plan.box_ok) {
        set_status(GF_EINVAL, "the box-restricted mesh passes need FFT axes of 64..512 cells");
        return GF_EINVAL;
    }
    BoxPlanArgs a{};
    a.ngroups = (int32_t)plan.groups.size();
    a.nhalo = plan.nhalo;
    for (size_t i = 0; i < plan.groups.size(); i++) {
        const SmoothGroup &sg = plan.groups[i];
        a.g[i].halos = reinterpret_cast<const int32_t *>(dbuf + sg.off_halos);
        a.g[i].starts = reinterpret_cast<int64_t *>(dbuf + sg.off_starts);
        a.g[i].ngroup = sg.ngroup;
        a.g[i].axis = sg.axis;
        a.g[i].pmax = sg.pmax;
    }
    a.boxes = boxes;
    a.mesh = mesh_dev;
    a.zstart = reinterpret_cast<int64_t *>(dbuf + plan.off_zero);
    box_plan_kernel<<<a.ngroups + 1, 1024, 0, ctx->stream>>>(a);
    GF_LAUNCH_CHECK();
    zero_box_kernel<<<sm_count() * 8, 256, 0, ctx->stream>>>(den, mesh_dev, boxes, a.zstart, plan.nhalo);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

int smooth_box_launch(gf_ctx *ctx, const SmoothPlan &plan, const char *dbuf, const gf_mesh_desc *mesh_dev,
                      float *den, const int32_t *boxes, const OnChipMeshes *onchip) {
    if (plan.blob.empty()) return GF_OK;
    const AxisTable *d_axes = reinterpret_cast<const AxisTable *>(dbuf);
    const float *d_tab = reinterpret_cast<const float *>(dbuf + plan.off_tab);
    // axes in order x, y, z: each pass reads what the previous one wrote
    for (int axis = 0; axis < 3; axis++) {
        for (const SmoothGroup &g : plan.groups) {
            if (g.axis != axis) continue;
            GroupLaunch gl;
            gl.halos = reinterpret_cast<const int32_t *>(dbuf + g.off_halos);
            gl.tile_start = reinterpret_cast<const int64_t *>(dbuf + g.off_starts);
            gl.ngroup = g.ngroup;
            if (axis == 0) GF_TRY(launch_box_group<0>(ctx, den, mesh_dev, gl, g.ntiles, g.n, d_axes, d_tab, boxes));
            else if (axis == 1) GF_TRY(launch_box_group<1>(ctx, den, mesh_dev, gl, g.ntiles, g.n, d_axes, d_tab, boxes));
            else GF_TRY(launch_box_group<2>(ctx, den, mesh_dev, gl, g.ntiles, g.n, d_axes, d_tab, boxes));
        }
    }
    if (plan.nchip) {
        SmoothPlan chip_only;
        chip_only.blob = {0};
        chip_only.off_tab = plan.off_tab;
        chip_only.off_chip = plan.off_chip;
        chip_only.nchip = plan.nchip;
        GF_TRY(smooth_launch(ctx, chip_only, dbuf, mesh_dev, den, onchip, nullptr));
    }
    return GF_OK;
}

}  // namespace gf

// ------------------------------------------------------------------------
// Single-mesh planning into a caller-provided byte buffer (no heap, no device
// allocation) and the matching launches; used by the allocation-free entry
// point in gf_noalloc.cu.
namespace gf {

int smooth_single_build(const gf_mesh_desc &m, unsigned char *blob, size_t cap, SingleMeshPlan *plan) {
    if (m.nx < 1 || m.ny < 1 || m.nz < 1 || !(m.cellsize > 0) || m.nx > kNoAllocMaxAxis ||
        m.ny > kNoAllocMaxAxis || m.nz > kNoAllocMaxAxis) {
        set_status(GF_EINVAL, "mesh %d x %d x %d: every axis must be 1..%d for the allocation-free "
                   "smoothing", m.nx, m.ny, m.nz, kNoAllocMaxAxis);
        return GF_EINVAL;
    }
    auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
    size_t off = 0;
    plan->off_mesh = off;
    off = align(off + sizeof(gf_mesh_desc));
    plan->off_axes = off;
    off = align(off + 3 * sizeof(AxisTable));
    for (int a = 0; a < 3; a++) {
        plan->off_halos[a] = off;
        off = align(off + sizeof(int32_t));
        plan->off_starts[a] = off;
        off = align(off + 2 * sizeof(int64_t));
    }
    plan->off_tables = off;
    if (off > cap) {
        set_status(GF_EINVAL, "allocation-free smoothing: scratch too small");
        return GF_EINVAL;
    }
    gf_mesh_desc md = m;
    md.off = 0;
    memcpy(blob + plan->off_mesh, &md, sizeof(md));
    const double rg_cells = (double)(float)(m.rg / m.cellsize);  // gsmooth.c:67
    const int dims[3] = {m.nx, m.ny, m.nz};
    AxisTable at[3];
    float *tab = reinterpret_cast<float *>(blob + plan->off_tables);
    const int64_t tcap = (int64_t)((cap - plan->off_tables) / sizeof(float));
    int64_t used = 0;
    for (int a = 0; a < 3; a++) {
        const int n = dims[a];
        at[a].n = n;
        at[a].logn = path_of(n) == PATH_DIRECT ? -1 : ilog2_exact(n);
        used = (used + 3) & ~int64_t(3);  // 16-byte aligned tables (float2 twiddles)
        at[a].tab_off = used;
        const int64_t k = axis_table_floats(n);
        if (k > tcap - used) {
            set_status(GF_EINVAL, "allocation-free smoothing: tables exceed the scratch");
            return GF_EINVAL;
        }
        double g[kNoAllocMaxAxis], c[kNoAllocMaxAxis];
        write_axis_tables(n, rg_cells, tab + used, g, c);
        used += k;
        // tiles as smooth_meshes cuts them: the FFT kernel's tile width on the
        // FFT path, else as many as fit in shared memory
        int pmax = fft_tile_pencils(n);
        if (path_of(n) != PATH_FFT8) {
            pmax = 32;
            while (pmax > 2 && (size_t)2 * (pmax / 2) * n * sizeof(float2) > 200 * 1024) pmax -= 2;
        }
        const int64_t cx = (m.nx + pmax - 1) / pmax;
        const int64_t nt = a == 0 ? ((int64_t)m.ny * m.nz + pmax - 1) / pmax
                                  : cx * (a == 1 ? m.nz : m.ny);
        const int32_t h0 = 0;
        const int64_t st[2] = {0, nt};
        memcpy(blob + plan->off_halos[a], &h0, sizeof(h0));
        memcpy(blob + plan->off_starts[a], st, sizeof(st));
        plan->ntiles[a] = nt;
        plan->n[a] = n;
        plan->pmax[a] = pmax;
    }
    memcpy(blob + plan->off_axes, at, sizeof(at));
    plan->bytes = plan->off_tables + (size_t)used * sizeof(float);
    return GF_OK;
}

int smooth_single_launch(gf_ctx *ctx, float *den, const unsigned char *dev_blob,
                         const SingleMeshPlan &plan) {
    const gf_mesh_desc *mesh_dev = reinterpret_cast<const gf_mesh_desc *>(dev_blob + plan.off_mesh);
    const AxisTable *axes = reinterpret_cast<const AxisTable *>(dev_blob + plan.off_axes);
    const float *tables = reinterpret_cast<const float *>(dev_blob + plan.off_tables);
    for (int a = 0; a < 3; a++) {
        GroupLaunch gl;
        gl.halos = reinterpret_cast<const int32_t *>(dev_blob + plan.off_halos[a]);
        gl.tile_start = reinterpret_cast<const int64_t *>(dev_blob + plan.off_starts[a]);
        gl.ngroup = 1;
        if (a == 0) GF_TRY(launch_group<0>(ctx, den, mesh_dev, gl, plan.ntiles[a], plan.n[a], plan.pmax[a], axes, tables));
        else if (a == 1) GF_TRY(launch_group<1>(ctx, den, mesh_dev, gl, plan.ntiles[a], plan.n[a], plan.pmax[a], axes, tables));
        else GF_TRY(launch_group<2>(ctx, den, mesh_dev, gl, plan.ntiles[a], plan.n[a], plan.pmax[a], axes, tables));
    }
    return GF_OK;
}

}  // namespace gf
