// The plain FP64 stage: the same per-halo stage as gf_stage_run, with every
// phase computed in FP64 by straightforward kernels, for the comparison of the
// batched FP32 path with a plain GPU implementation (one halo per call):
//
//   * kNN + SPH density: exact k nearest in FP64 (a warp per query walking
//     the octree with FP64 node boxes, gf_fp64.cuh), W4 density in FP64;
//   * TSC: the exact quadratic spline weights in FP64 (tsc_omp2.c:335-343
//     without its float roundings), FP64 atomics into an FP64 mesh;
//   * smoothing: per-axis FP64 Stockham FFT with the filter factor of
//     gsmooth.c:67-86 (or the exact circular convolution for lengths that
//     are not powers of two), tables evaluated in FP64;
//   * findDen: the 27-point FP64 interpolation;
//   * potential: the Barnes-Hut walk with FP64 node moments and FP64 terms
//     (monopole + quadrupole, exact -m/r), the same opening rule
//     |p - com|^2 < dist2/theta2 and direct sums below ndirect particles.
//
// Compiled with --fmad=false (the FP64 distances are formed as the
// reference's (dx*dx + dy*dy) + dz*dz).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <vector>

#include "gf_fp64.cuh"

namespace gf {

namespace {

int grid_n64(int64_t n, int block) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + block - 1) / block, (int64_t)sm_count() * 16));
}

// ---------------------------------------------------------------- TSC, findDen
__global__ void tsc64_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                             const double *__restrict__ z, const double *__restrict__ mass,
                             const int32_t *__restrict__ type, const int32_t *__restrict__ hid,
                             const gf_mesh_desc *__restrict__ mesh, double *__restrict__ den, double volfact,
                             int *err) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const gf_mesh_desc m = mesh[hid[p]];
        if (m.ptype != GF_TYPE_ALL && (type ? type[p] : GF_TYPE_DM) != m.ptype) continue;
        const Axis64 ax = tsc_axis64(x[p], m.xmin, m.cellsize);
        const Axis64 ay = tsc_axis64(y[p], m.ymin, m.cellsize);
        const Axis64 az = tsc_axis64(z[p], m.zmin, m.cellsize);
        if (!stencil_in(ax, ay, az, m)) {
            atomicOr(err, GF_ERRBIT_RANGE);
            continue;
        }
        const int64_t mx = 2 * (m.nx / 2 + 1);
        const double w = mass[p] * volfact;
        for (int c = 0; c < 3; c++)
            for (int b = 0; b < 3; b++)
                for (int a = 0; a < 3; a++)
                    atomicAdd(den + m.off + (ax.i0 + a) + mx * ((ay.i0 + b) + (int64_t)m.ny * (az.i0 + c)),
                              w * ax.w[a] * ay.w[b] * az.w[c]);
    }
}

__global__ void find_den64_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ z, const int32_t *__restrict__ hid,
                                  const gf_mesh_desc *__restrict__ mesh, const double *__restrict__ den,
                                  float *__restrict__ densph, int *err) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const gf_mesh_desc m = mesh[hid[p]];
        const Axis64 ax = tsc_axis64(x[p], m.xmin, m.cellsize);
        const Axis64 ay = tsc_axis64(y[p], m.ymin, m.cellsize);
        const Axis64 az = tsc_axis64(z[p], m.zmin, m.cellsize);
        if (!stencil_in(ax, ay, az, m)) {
            atomicOr(err, GF_ERRBIT_RANGE);
            densph[p] = 0.f;
            continue;
        }
        const int64_t mx = 2 * (m.nx / 2 + 1);
        double rho = 0.0;
        for (int c = 0; c < 3; c++)
            for (int b = 0; b < 3; b++)
                for (int a = 0; a < 3; a++)
                    rho += den[m.off + (ax.i0 + a) + mx * ((ay.i0 + b) + (int64_t)m.ny * (az.i0 + c))] * ax.w[a] *
                           ay.w[b] * az.w[c];
        densph[p] = (float)rho;
    }
}

// ---------------------------------------------------------------- smoothing
// One axis of one mesh: a block per tile of kP real pencils (two per complex
// pencil).  Power-of-two lengths: radix-2 Stockham FFT, filter G/n, inverse
// FFT; other lengths: the exact n-tap circular convolution with h_n.
constexpr int kP = 8;
constexpr int kT = 256;

template <int AXIS>
__device__ __forceinline__ int64_t elem64(const gf_mesh_desc &m, int64_t mx, int64_t pen, int s) {
    if (AXIS == 0) return m.off + mx * pen + s;  // pen = y + ny z
    if (AXIS == 1) return m.off + (pen % m.nx) + mx * ((int64_t)s + (int64_t)m.ny * (pen / m.nx));  // pen = x + nx z
    return m.off + (pen % m.nx) + mx * ((pen / m.nx) + (int64_t)m.ny * s);  // pen = x + nx y
}

template <int AXIS>
__global__ void __launch_bounds__(kT) smooth64_kernel(double *__restrict__ den, gf_mesh_desc m, int n, int logn,
                                                     const double *__restrict__ tab) {
    extern __shared__ double2 sm64[];
    const int64_t mx = 2 * (m.nx / 2 + 1);
    const int64_t npen = AXIS == 0 ? (int64_t)m.ny * m.nz : (int64_t)m.nx * (AXIS == 1 ? m.nz : m.ny);
    const int64_t pen0 = (int64_t)blockIdx.x * kP;
    const int np = (int)min((int64_t)kP, npen - pen0);
    const int npair = (np + 1) >> 1;
    double2 *A = sm64, *B = sm64 + (kP / 2) * n;
    double *fa = reinterpret_cast<double *>(A);
    for (int e = threadIdx.x; e < 2 * npair * n; e += kT) {
        const int p = e / n, s = e - p * n;
        fa[2 * ((p >> 1) * n + s) + (p & 1)] = p < np ? den[elem64<AXIS>(m, mx, pen0 + p, s)] : 0.0;
    }
    __syncthreads();
    double2 *src = A, *dst = B;
    if (logn >= 0) {
        const double2 *tw = reinterpret_cast<const double2 *>(tab);  // n/2 twiddles e^{-2 pi i k/n}
        const double *filt = tab + n;                                 // n factors G/n
        const int half = n >> 1;
        for (int dir = 0; dir < 2; dir++) {
            const double sgn = dir == 0 ? 1.0 : -1.0;
            for (int ls = 0; ls < logn; ls++) {
                const int smask = (1 << ls) - 1;
                for (int e = threadIdx.x; e < npair * half; e += kT) {
                    const int c = e / half, tt = e - c * half;
                    const int q = tt & smask, pp = tt >> ls;
                    const double2 *xx = src + c * n;
                    double2 *yy = dst + c * n;
                    const double2 a = xx[q + (pp << ls)], b = xx[q + (pp << ls) + half];
                    double2 w = tw[pp << ls];
                    w.y *= sgn;
                    const double2 d = make_double2(a.x - b.x, a.y - b.y);
                    yy[q + (pp << (ls + 1))] = make_double2(a.x + b.x, a.y + b.y);
                    yy[q + (pp << (ls + 1)) + (1 << ls)] = make_double2(d.x * w.x - d.y * w.y, d.x * w.y + d.y * w.x);
                }
                __syncthreads();
                double2 *t = src;
                src = dst;
                dst = t;
            }
            if (dir == 0) {
                for (int e = threadIdx.x; e < npair * n; e += kT) {
                    const double g = filt[e % n];
                    src[e].x *= g;
                    src[e].y *= g;
                }
                __syncthreads();
            }
        }
    } else {
        for (int e = threadIdx.x; e < npair * n; e += kT) {
            const int c = e / n, s = e - c * n;
            const double2 *xx = src + c * n;
            double ar = 0.0, ai = 0.0;
            int idx = s;
            for (int k = 0; k < n; k++) {
                ar += tab[k] * xx[idx].x;
                ai += tab[k] * xx[idx].y;
                idx = idx == 0 ? n - 1 : idx - 1;
            }
            dst[e] = make_double2(ar, ai);
        }
        __syncthreads();
        src = dst;
    }
    const double *fs = reinterpret_cast<const double *>(src);
    for (int e = threadIdx.x; e < 2 * npair * n; e += kT) {
        const int p = e / n, s = e - p * n;
        if (p < np) den[elem64<AXIS>(m, mx, pen0 + p, s)] = fs[2 * ((p >> 1) * n + s) + (p & 1)];
    }
}

int log2_exact(int n) {
    if (n <= 0 || (n & (n - 1))) return -1;
    int l = 0;
    while ((1 << l) < n) l++;
    return l;
}

// FP64 tables of one axis: [n/2 twiddles (re, im)][n factors G/n] for powers
// of two, [h_n (n)] otherwise; G as gsmooth.c:67-86 with RG/cellsize stored
// in a float (gsmooth.c:67).
void tables64(int n, double rg_cells, std::vector<double> &out) {
    const double expfac = -(M_PI * rg_cells) * (M_PI * rg_cells);
    std::vector<double> g(n);
    for (int k = 0; k < n; k++) {
        const long ks = k > n / 2 ? k - n : k;
        g[k] = exp((double)(ks * ks) * expfac / ((double)n * (double)n));
    }
    out.clear();
    if (log2_exact(n) >= 0) {
        for (int k = 0; k < n / 2; k++) {
            const double ang = 2.0 * M_PI * (double)k / (double)n;
            out.push_back(cos(ang));
            out.push_back(-sin(ang));
        }
        for (int k = 0; k < n; k++) out.push_back(g[k] / n);
    } else {
        std::vector<double> c(n);
        for (int j = 0; j < n; j++) c[j] = cos(2.0 * M_PI * (double)j / (double)n);
        for (int mm = 0; mm < n; mm++) {
            double acc = 0.0;
            for (int k = 0; k < n; k++) acc += g[k] * c[((long)k * mm) % n];
            out.push_back(acc / n);
        }
    }
}

template <int AXIS>
int launch_smooth64(gf_ctx *ctx, double *den, const gf_mesh_desc &m, int n, const double *dtab) {
    const int64_t npen = AXIS == 0 ? (int64_t)m.ny * m.nz : (int64_t)m.nx * (AXIS == 1 ? m.nz : m.ny);
    const int64_t tiles = (npen + kP - 1) / kP;
    const size_t smem = (size_t)2 * (kP / 2) * n * sizeof(double2);
    if (smem > 220 * 1024) {
        set_status(GF_ENOTIMPL, "FP64 smoothing of a %d-cell axis exceeds shared memory", n);
        return GF_ENOTIMPL;
    }
    GF_CUDA_TRY(cudaFuncSetAttribute(smooth64_kernel<AXIS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    smooth64_kernel<AXIS><<<(unsigned)tiles, kT, smem, ctx->stream>>>(den, m, n, log2_exact(n), dtab);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

// ---------------------------------------------------------------- potential
// Thread per target in tree order; the 32 targets of a warp walk the preorder
// nodes in lockstep (the smallest next node of the warp), each with its own
// FP64 opening decision; FP64 terms and sums.
__global__ void bh64_kernel(int64_t n, const double4 *__restrict__ tp, const int32_t *__restrict__ perm,
                            const int32_t *__restrict__ phalo, const int32_t *__restrict__ root,
                            const int32_t *__restrict__ rend, const KnnNode *__restrict__ knn,
                            const RefNode *__restrict__ rn, const int32_t *__restrict__ direct,
                            const double *__restrict__ bg, double theta2, double potentfact,
                            float *__restrict__ penergy, float *__restrict__ raw) {
    const int lane = threadIdx.x & 31;
    const int64_t wstride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += wstride) {
        const int64_t t = base + lane;
        const bool valid = t < n;
        int h = 0, my = INT_MAX, my_end = 0, always = 0;
        double4 P = make_double4(0, 0, 0, 0);
        if (valid) {
            h = phalo[t];
            my = root[h];
            my_end = rend[h];
            if (my >= my_end) my = INT_MAX;
            always = direct[h];
            P = tp[t];
        }
        double phi = 0.0;
        while (true) {
            const int i = (int)__reduce_min_sync(0xffffffffu, (unsigned)my);
            if (i == INT_MAX) break;
            if (my == i) {
                const RefNode &r = rn[i];
                const double dx = P.x - r.com[0], dy = P.y - r.com[1], dz = P.z - r.com[2];
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (always || d2 < r.dist2 / theta2) {
                    const KnnNode nd = knn[i];
                    for (int j = nd.lstart; j < nd.lstart + nd.lcount; j++) {
                        const double4 S = tp[j];
                        const double sx = P.x - S.x, sy = P.y - S.y, sz = P.z - S.z;
                        const double r2 = sx * sx + sy * sy + sz * sz;
                        if (r2 > 0.0) phi -= S.w / sqrt(r2);
                    }
                    my = i + 1;
                } else {
                    const double inv = 1.0 / sqrt(d2);
                    const double inv2 = inv * inv, inv3 = inv * inv2;
                    const double qxy = r.q[0] * dx * dx + r.q[1] * dy * dy + r.q[2] * dz * dz +
                                       2.0 * (r.q[3] * dx * dy + r.q[4] * dx * dz + r.q[5] * dy * dz);
                    const double trq = r.q[0] + r.q[1] + r.q[2];
                    phi += -r.mass * inv + 0.5 * trq * inv3 - 1.5 * qxy * inv3 * inv2;
                    my = knn[i].skip;
                }
                if (my >= my_end) my = INT_MAX;
            }
        }
        if (valid) {
            const int64_t o = perm[t];
            if (raw) raw[o] = (float)phi;
            if (penergy) penergy[o] = (float)(phi * potentfact + bg[h]);
        }
    }
}

__global__ void halo_mass64_kernel(int32_t nhalo, const int32_t *__restrict__ root, const RefNode *__restrict__ rn,
                                   const int64_t *__restrict__ pstart, int32_t ndirect, double *__restrict__ mvir,
                                   int32_t *__restrict__ direct) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nhalo) return;
    mvir[h] = rn[root[h]].mass;  // FP64 sum of the halo's float masses
    direct[h] = pstart[h + 1] - pstart[h] < ndirect ? 1 : 0;
}

}  // namespace

int stage_plain_fp64(gf_ctx *ctx, const gf_batch *b, const gf_stage_config *cfg, gf_stage_out *o,
                     const int32_t *hid, const double *xr, const double *yr, const double *zr,
                     const std::vector<gf_mesh_desc> &mesh, const gf_mesh_desc *mesh_dev, int64_t cells,
                     const PotentialParams &pp, float *ms) {
    cudaStream_t s = ctx->stream;
    const int64_t n = b->nparticle;
    const int32_t nh = b->nhalo;
    if (n <= 0) return GF_OK;
    cudaEvent_t ev[5];
    for (auto &e : ev) GF_CUDA_TRY(cudaEventCreate(&e));
    GF_CUDA_TRY(cudaEventRecord(ev[0], s));
    // ---- octree structure (the stage's FP32 build) with FP64 moments and boxes
    const TreeView &t = ctx->last_tree;
    const bool tree = cfg->knn_k > 0 || cfg->do_potential;
    double4 *tp = nullptr;
    RefNode *rn = nullptr;
    if (tree) {
        GF_TRY(ctx->tmp[6].reserve((size_t)n * sizeof(double4) + (size_t)t.nnode * sizeof(RefNode) + 512));
        tp = ctx->tmp[6].as<double4>();
        rn = reinterpret_cast<RefNode *>(tp + n);
        gather_tree_order<<<grid_n64(n, 256), 256, 0, s>>>(n, t.perm, xr, yr, zr, nullptr, b->mass, nullptr, tp,
                                                             nullptr);
        GF_LAUNCH_CHECK();
        ref_node_kernel<<<grid_n64((int64_t)t.nnode * 32, 256), 256, 0, s>>>(t.nnode, t.knn, tp, rn);
        GF_LAUNCH_CHECK();
    }
    // ---- kNN + SPH density
    if (cfg->knn_k > 0) {
        if (!o->nearindex || cfg->knn_k > 32) {
            set_status(GF_EINVAL, "the FP64 stage needs nearindex and knn_k <= 32");
            return GF_EINVAL;
        }
        knn64_kernel<<<grid_n64(n * 32, 128), 128, 0, s>>>(n, xr, yr, zr, hid, cfg->knn_k, t.root, t.rend, t.knn, rn,
                                                           tp, t.perm, b->pstart, o->nearindex, nullptr, nullptr,
                                                           o->dens_sph);
        GF_LAUNCH_CHECK();
    }
    GF_CUDA_TRY(cudaEventRecord(ev[1], s));
    // ---- TSC + smoothing + findDen on FP64 meshes
    if (cfg->do_mesh) {
        GF_TRY(ctx->tmp[7].reserve(sizeof(double) * (size_t)std::max<int64_t>(cells, 1)));
        double *den = ctx->tmp[7].as<double>();
        GF_CUDA_TRY(cudaMemsetAsync(den, 0, sizeof(double) * cells, s));
        tsc64_kernel<<<grid_n64(n, 256), 256, 0, s>>>(n, xr, yr, zr, b->mass, b->type, hid, mesh_dev, den,
                                                      tsc_volfact(), ctx->d_err);
        GF_LAUNCH_CHECK();
        // tables per (n, rg_cells), one device upload
        std::map<std::pair<int, double>, size_t> where;
        std::vector<double> all, one;
        std::vector<size_t> off(3 * (size_t)nh);
        for (int32_t h = 0; h < nh; h++) {
            const gf_mesh_desc &m = mesh[h];
            const double rg_cells = (double)(float)(m.rg / m.cellsize);
            const int dims[3] = {m.nx, m.ny, m.nz};
            for (int a = 0; a < 3; a++) {
                auto key = std::make_pair(dims[a], rg_cells);
                auto it = where.find(key);
                if (it == where.end()) {
                    tables64(dims[a], rg_cells, one);
                    while (all.size() % 2) all.push_back(0.0);
                    it = where.emplace(key, all.size()).first;
                    all.insert(all.end(), one.begin(), one.end());
                }
                off[3 * (size_t)h + a] = it->second;
            }
        }
        GF_TRY(ctx->tmp[5].reserve(all.size() * sizeof(double) + 256));
        GF_CUDA_TRY(cudaMemcpyAsync(ctx->tmp[5].ptr, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        const double *dtab = ctx->tmp[5].as<double>();
        for (int32_t h = 0; h < nh; h++) {
            const gf_mesh_desc &m = mesh[h];
            GF_TRY(launch_smooth64<0>(ctx, den, m, m.nx, dtab + off[3 * (size_t)h]));
            GF_TRY(launch_smooth64<1>(ctx, den, m, m.ny, dtab + off[3 * (size_t)h + 1]));
            GF_TRY(launch_smooth64<2>(ctx, den, m, m.nz, dtab + off[3 * (size_t)h + 2]));
        }
        GF_CUDA_TRY(cudaEventRecord(ev[2], s));
        if (o->dens_mesh) {
            find_den64_kernel<<<grid_n64(n, 256), 256, 0, s>>>(n, xr, yr, zr, hid, mesh_dev, den, o->dens_mesh,
                                                               ctx->d_err);
            GF_LAUNCH_CHECK();
        }
        GF_CUDA_TRY(cudaStreamSynchronize(s));  // the host tables feed the copy above
    } else {
        GF_CUDA_TRY(cudaEventRecord(ev[2], s));
    }
    GF_CUDA_TRY(cudaEventRecord(ev[3], s));
    // ---- potential
    if (cfg->do_potential) {
        GF_TRY(ctx->tmp[4].reserve((size_t)nh * (sizeof(double) * 2 + sizeof(int32_t)) + 512));
        double *mvir = ctx->tmp[4].as<double>();
        double *bg = mvir + nh;
        int32_t *direct = reinterpret_cast<int32_t *>(bg + nh);
        halo_mass64_kernel<<<(nh + 127) / 128, 128, 0, s>>>(nh, t.root, rn, b->pstart, pp.ndirect, mvir, direct);
        GF_LAUNCH_CHECK();
        if (pp.add_bg) {
            GF_TRY(launch_bg_eval(ctx, nh, mvir, pp, bg));
        } else {
            GF_CUDA_TRY(cudaMemsetAsync(bg, 0, (size_t)nh * sizeof(double), s));
        }
        bh64_kernel<<<grid_n64(n, 128), 128, 0, s>>>(n, tp, t.perm, t.phalo, t.root, t.rend, t.knn, rn, direct, bg,
                                                    (double)pp.theta2, pp.potentfact != 0.0 ? pp.potentfact : 1.0,
                                                    o->penergy, o->phi);
        GF_LAUNCH_CHECK();
    }
    GF_CUDA_TRY(cudaEventRecord(ev[4], s));
    GF_CUDA_TRY(cudaEventSynchronize(ev[4]));
    if (ms) {
        for (int i = 0; i < 4; i++) cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return GF_OK;
}

}  // namespace gf
