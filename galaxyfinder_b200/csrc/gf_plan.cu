// Halo extents, periodic unwrap, FP64 recentring and per-halo mesh planning.
//
// The reference recentres each FoF halo in FP64 by subtracting the per-axis
// minimum (Dump2BP, NewGalFinder/subhaloden.mod6.c:2810-2837) and unwraps
// halos that straddle the periodic box (mklocalize, :79-177).  Here one pass
// over the particles finds, per halo and axis, the min/max of the raw
// coordinate x and of its shifted image x' = x + L for x < L/2; the planner
// keeps whichever representation is more compact (a halo smaller than half
// the box is contiguous in exactly one of them), and the recentring kernel
// writes x - min in FP64 plus the FP32 copy used by the tree, kNN and
// potential kernels.
#include <math.h>

#include <algorithm>
#include <vector>

#include "gf_internal.cuh"

namespace gf {

namespace {

// Order-preserving map double -> uint64 so min/max become integer atomics.
__device__ __forceinline__ unsigned long long dkey(double v) {
    unsigned long long u = __double_as_longlong(v);
    return (u & 0x8000000000000000ULL) ? ~u : (u | 0x8000000000000000ULL);
}
__host__ __device__ inline double dkey_inv(unsigned long long k) {
    unsigned long long u = (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double d;
    memcpy(&d, &u, 8);
    return d;
#endif
}

// ext[h*12 + 4*axis + {0,1,2,3}] = keys of min x, max x, min x', max x'
__global__ void extent_init_kernel(unsigned long long *ext, int64_t nslots) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nslots;
         i += (int64_t)gridDim.x * blockDim.x)
        ext[i] = (i & 1) ? 0ULL : ~0ULL;  // even slots are minima, odd slots maxima
}

// Widens a halo's (min, max, shifted min, shifted max) keys.  The keys only
// move outwards, so a plain read first skips the atomics that would change
// nothing (most warps of a large halo), sparing the contention on its keys.
__device__ __forceinline__ void ext_update(unsigned long long *e, const unsigned long long (&k)[4]) {
    if (k[0] < __ldcg(e + 0)) atomicMin(e + 0, k[0]);
    if (k[1] > __ldcg(e + 1)) atomicMax(e + 1, k[1]);
    if (k[2] < __ldcg(e + 2)) atomicMin(e + 2, k[2]);
    if (k[3] > __ldcg(e + 3)) atomicMax(e + 3, k[3]);
}

__global__ void extent_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const int32_t *__restrict__ hid,
                              double box, unsigned long long *__restrict__ ext) {
    const unsigned lane = threadIdx.x & 31;
    for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) & ~31LL; base < n;
         base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = base + lane;
        const bool valid = p < n;
        const int h = valid ? hid[p] : -1;
        const double c[3] = {valid ? x[p] : 0.0, valid ? y[p] : 0.0, valid ? z[p] : 0.0};
        // lanes sharing lane 0's halo reduce in registers; the rest use atomics
        const int h0 = __shfl_sync(0xffffffffu, h, 0);
        const bool uniform = __all_sync(0xffffffffu, !valid || h == h0);
        for (int a = 0; a < 3; a++) {
            const double v = c[a];
            const double vs = v < 0.5 * box ? v + box : v;
            unsigned long long k[4] = {dkey(v), dkey(v), dkey(vs), dkey(vs)};
            if (!valid) { k[0] = k[2] = ~0ULL; k[1] = k[3] = 0ULL; }
            if (uniform) {
                for (int off = 16; off > 0; off >>= 1) {
                    unsigned long long o0 = __shfl_xor_sync(0xffffffffu, k[0], off);
                    unsigned long long o1 = __shfl_xor_sync(0xffffffffu, k[1], off);
                    unsigned long long o2 = __shfl_xor_sync(0xffffffffu, k[2], off);
                    unsigned long long o3 = __shfl_xor_sync(0xffffffffu, k[3], off);
                    k[0] = min(k[0], o0); k[1] = max(k[1], o1);
                    k[2] = min(k[2], o2); k[3] = max(k[3], o3);
                }
                if (lane == 0 && h0 >= 0) ext_update(ext + (int64_t)h0 * 12 + 4 * a, k);
            } else if (valid) {
                ext_update(ext + (int64_t)h * 12 + 4 * a, k);
            }
        }
    }
}

__global__ void recentre_kernel(int64_t n, const double *__restrict__ x,
                                const double *__restrict__ y, const double *__restrict__ z,
                                const double *__restrict__ mass, const int32_t *__restrict__ hid,
                                const double *__restrict__ frame, double box,
                                double *__restrict__ xr, double *__restrict__ yr,
                                double *__restrict__ zr, float4 *__restrict__ pos) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const double *f = frame + 6 * (int64_t)hid[p];  // (min, shift flag) per axis
        double c[3] = {x[p], y[p], z[p]};
        double r[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            double v = c[a];
            if (f[2 * a + 1] != 0.0 && v < 0.5 * box) v += box;
            r[a] = v - f[2 * a];  // Dump2BP: x - min(x)
        }
        xr[p] = r[0];
        yr[p] = r[1];
        zr[p] = r[2];
        pos[p] = make_float4((float)r[0], (float)r[1], (float)r[2], (float)mass[p]);
    }
}

int grid1d(int64_t n) {
    int64_t g = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, sm_count() * 16));
}

// Frame and extent of one axis from the extent keys (halo_frames' rule).
__host__ __device__ inline void axis_frame(const unsigned long long *k, double box, double &origin,
                                           double &shift, double &extent) {
    const double lo = dkey_inv(k[0]), hi = dkey_inv(k[1]);
    const double los = dkey_inv(k[2]), his = dkey_inv(k[3]);
    const bool sh = box > 0 && (hi - lo) > 0.5 * box && (his - los) < (hi - lo);
    origin = sh ? los : lo;
    shift = sh ? 1.0 : 0.0;
    extent = sh ? his - los : hi - lo;
}

}  // namespace

int halo_frames(gf_ctx *ctx, const gf_batch *b, const int32_t *hid, double box,
                std::vector<double> &frame_host, std::vector<double> &extent_host) {
    const int nh = b->nhalo;
    GF_TRY(ctx->tmp[6].reserve(sizeof(unsigned long long) * 12 * (size_t)nh));
    unsigned long long *ext = ctx->tmp[6].as<unsigned long long>();
    extent_init_kernel<<<grid1d(12 * (int64_t)nh), 256, 0, ctx->stream>>>(ext, 12 * (int64_t)nh);
    GF_LAUNCH_CHECK();
    extent_kernel<<<grid1d(b->nparticle), 256, 0, ctx->stream>>>(b->nparticle, b->x, b->y, b->z,
                                                                  hid, box, ext);
    GF_LAUNCH_CHECK();
    std::vector<unsigned long long> hk(12 * (size_t)nh);
    GF_CUDA_TRY(cudaMemcpyAsync(hk.data(), ext, hk.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    frame_host.assign(6 * (size_t)nh, 0.0);
    extent_host.assign(3 * (size_t)nh, 0.0);
    for (int h = 0; h < nh; h++)
        for (int a = 0; a < 3; a++)
            axis_frame(&hk[12 * (size_t)h + 4 * a], box, frame_host[6 * (size_t)h + 2 * a],
                       frame_host[6 * (size_t)h + 2 * a + 1], extent_host[3 * (size_t)h + a]);
    return GF_OK;
}

int recentre(gf_ctx *ctx, const gf_batch *b, const int32_t *hid, const double *frame_dev,
             double box, double *xr, double *yr, double *zr, float4 *pos) {
    if (b->nparticle <= 0) return GF_OK;
    recentre_kernel<<<grid1d(b->nparticle), 256, 0, ctx->stream>>>(
        b->nparticle, b->x, b->y, b->z, b->mass, hid, frame_dev, box, xr, yr, zr, pos);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

// Mesh of one halo from its recentred extent (min = 0 on every axis).  Host
// and device run the same double arithmetic (this file is compiled with
// --fmad=false), so a mesh planned on the device equals the host's plan.
__host__ __device__ gf_mesh_desc plan_one_mesh(const double ext[3], const gf_mesh_rule &r) {
    gf_mesh_desc m{};
    m.ptype = r.ptype;
    const int nb = r.nbuff;
    // lagFindStellarCore pads the upper bound by 1e-4 of the extent (nnost.c:1050-1052)
    double e[3];
    for (int a = 0; a < 3; a++) e[a] = ext[a] + ext[a] * 0.0001;
    double cs = r.cell;
    int n[3];
    if (r.mode == GF_MESH_REFERENCE) {
        // nnost.c:1053-1055: n = extent/cellsize + nbuff per axis
        for (int a = 0; a < 3; a++) n[a] = (int)(e[a] / cs + nb);
    } else {
        const double w = e[0] > (e[1] > e[2] ? e[1] : e[2]) ? e[0] : (e[1] > e[2] ? e[1] : e[2]);
        int nc;
        if (r.mode == GF_MESH_FIXED) {
            nc = r.nfixed;
            cs = w / (double)(nc - nb);
            if (!(cs > 0)) cs = r.cell;
        } else {  // GF_MESH_POW2: smallest power of two holding extent/cell + nbuff, clamped
            const double need = w / r.cell + nb;
            nc = 1;
            while (nc < need && nc < (1 << 20)) nc <<= 1;
            nc = nc > r.nmin ? nc : r.nmin;
            nc = nc < r.nmax ? nc : r.nmax;
            const double c2 = w / (double)(nc - nb);
            cs = r.cell > c2 ? r.cell : c2;
        }
        n[0] = n[1] = n[2] = nc;
    }
    m.nx = n[0];
    m.ny = n[1];
    m.nz = n[2];
    m.cellsize = cs;
    // nnost.c:1056: the mesh origin sits nbuff/2 cells below the halo minimum
    m.xmin = 0.0 - cs * nb / 2.;
    m.ymin = 0.0 - cs * nb / 2.;
    m.zmin = 0.0 - cs * nb / 2.;
    m.rg = r.rg_in_cells ? r.rg * cs : r.rg;
    return m;
}

namespace {

__global__ void frames_plan_kernel(int32_t nhalo, const unsigned long long *__restrict__ ext, double box,
                                   gf_mesh_rule rule, int do_mesh, const gf_mesh_desc *__restrict__ planned,
                                   double *__restrict__ frame, gf_mesh_desc *__restrict__ mesh, int *err) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nhalo) return;
    double e[3];
    for (int a = 0; a < 3; a++)
        axis_frame(ext + 12 * (int64_t)h + 4 * a, box, frame[6 * (int64_t)h + 2 * a],
                   frame[6 * (int64_t)h + 2 * a + 1], e[a]);
    if (!do_mesh) return;
    gf_mesh_desc m = plan_one_mesh(e, rule);
    const gf_mesh_desc &p = planned[h];
    // the smoothing tables are keyed by the float rg/cellsize (gsmooth.c:67)
    if (m.nx != p.nx || m.ny != p.ny || m.nz != p.nz ||
        (float)(m.rg / m.cellsize) != (float)(p.rg / p.cellsize)) {
        // the captured mesh stays (its shape bounds every access to its
        // cells; particles outside it are flagged by the deposit)
        atomicOr(err, GF_ERRBIT_PLAN);
        mesh[h] = p;
        return;
    }
    m.off = p.off;
    m.ptype = p.ptype;
    mesh[h] = m;
}

}  // namespace

int launch_extents(gf_ctx *ctx, const gf_batch *b, const int32_t *hid, double box) {
    const int nh = b->nhalo;
    GF_TRY(ctx->tmp[6].reserve(sizeof(unsigned long long) * 12 * (size_t)std::max(nh, 1)));
    unsigned long long *ext = ctx->tmp[6].as<unsigned long long>();
    extent_init_kernel<<<grid1d(12 * (int64_t)nh), 256, 0, ctx->stream>>>(ext, 12 * (int64_t)nh);
    GF_LAUNCH_CHECK();
    if (b->nparticle > 0) {
        extent_kernel<<<grid1d(b->nparticle), 256, 0, ctx->stream>>>(b->nparticle, b->x, b->y, b->z, hid, box,
                                                                      ext);
        GF_LAUNCH_CHECK();
    }
    return GF_OK;
}

int launch_frames_plan(gf_ctx *ctx, int32_t nhalo, double box, const gf_mesh_rule &rule, int do_mesh,
                       const gf_mesh_desc *planned, double *frame_dev, gf_mesh_desc *mesh_dev) {
    if (nhalo <= 0) return GF_OK;
    frames_plan_kernel<<<(nhalo + 127) / 128, 128, 0, ctx->stream>>>(
        nhalo, ctx->tmp[6].as<unsigned long long>(), box, rule, do_mesh, planned, frame_dev, mesh_dev, ctx->d_err);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

}  // namespace gf

using namespace gf;

extern "C" int gf_plan_meshes(int32_t nhalo, const double *extent, const gf_mesh_rule *rule,
                              gf_mesh_desc *out, int64_t *total_cells) {
    clear_status();
    if (nhalo < 0 || (nhalo > 0 && (!extent || !out)) || !rule) return GF_EINVAL;
    if (rule->nbuff < 2 || rule->nbuff % 2 || !(rule->cell > 0)) {
        set_status(GF_EINVAL, "mesh rule: nbuff must be even and >= 2, cell > 0");
        return GF_EINVAL;
    }
    int64_t off = 0;
    for (int h = 0; h < nhalo; h++) {
        gf_mesh_desc m = plan_one_mesh(extent + 3 * (size_t)h, *rule);
        if (m.nx < 4 || m.ny < 4 || m.nz < 4) {
            set_status(GF_EINVAL, "halo %d: mesh %d x %d x %d is too small", h, m.nx, m.ny, m.nz);
            return GF_EINVAL;
        }
        m.off = off;
        off += mesh_cells(m);
        off = (off + 63) & ~int64_t(63);  // 256-byte aligned mesh starts
        out[h] = m;
    }
    if (total_cells) *total_cells = off;
    return GF_OK;
}
