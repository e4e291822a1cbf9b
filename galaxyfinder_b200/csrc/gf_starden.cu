// starfindsphdensity (NewGalFinder/nnost.c:632-744): the mass-weighted
// stellar SPH density at every particle of a halo and every particle's
// neighbour list.  (The reference's -DADV build reaches stellar densities
// through lagFindStellarCore instead; this is the older entry point.)
//
//   * densph[i] = sum over the NUMNEARDEN (10) nearest STARS j of particle i
//     of W4(|x_i - x_j|, r_10 / 2) * m_j, the W4 of nnost.c:536-555 with
//     r_10 the distance of the last of them, summed in float in distance
//     order (nnost.c:687-700).  Here the stars get libgf's octree with FP64
//     node boxes and moments, and every particle is a query of the exact
//     FP64 k-nearest walk (knn64_kernel, a warp per query, distances rounded
//     as the reference's (dx*dx + dy*dy) + dz*dz, equal distances ordered by
//     star index); a kernel then sums the weights in the reference's float
//     and double types.
//   * nearindex: the Numnear nearest particles of every particle (self
//     included), the lists of the findsphdensity drop-in (nnost.c:702-736).
//
// The reference's star loop assumes at least one star (it links
// ptl[mp - 1]); with none, every density here is 0.  This translation unit is
// compiled with --fmad=false.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "gf_fp64.cuh"

namespace gf {

int findsphdensity_lists(SimpleBasicParticleType *bp, int np, long long *nearindex, int numnear, float *densph);

namespace {

constexpr int kNumNearDen = 10;  // NUMNEARDEN, params.h:73

__global__ void star_pack_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                                 const double *__restrict__ z, const float *__restrict__ m,
                                 float4 *__restrict__ pos) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        pos[i] = make_float4((float)x[i], (float)y[i], (float)z[i], m[i]);
}

// nnost.c:692-699: tmpd2[j] = sqrtf(tmpd2[j]); densph += W4(tmpd2[j],
// neardist/2.) * tmpmass[j], with neardist = sqrtf(d2 of the last neighbour)
// (INSERT, nnost.c:291-292) and the masses stored as float (nnost.c:289).
// Rows of k (the list length, NUMNEARDEN or the star count if smaller).
__global__ void star_density_kernel(int64_t n, int k, const int32_t *__restrict__ idx,
                                    const double *__restrict__ d2, const int32_t *__restrict__ cnt,
                                    const float *__restrict__ smass, float *__restrict__ dens) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int res = cnt[q];
        float rho = 0.f;
        if (res > 0) {
            const float neardist = sqrtf((float)d2[q * k + res - 1]);
            const float hh = (float)((double)neardist / 2.);
            for (int j = 0; j < res; j++) {
                const float dist = sqrtf((float)d2[q * k + j]);
                rho += w4(dist, hh) * smass[idx[q * k + j]];
            }
        }
        dens[q] = rho;
    }
}

int grid_for(int64_t n, int block) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + block - 1) / block, (int64_t)sm_count() * 16));
}

int star_density(SimpleBasicParticleType *bp, int np, float *densph) {
    std::vector<double> sx, sy, sz;
    std::vector<float> sm;
    for (int i = 0; i < np; i++)
        if (bp[i].type == GF_TYPE_STAR) {
            sx.push_back(bp[i].x);
            sy.push_back(bp[i].y);
            sz.push_back(bp[i].z);
            sm.push_back((float)bp[i].mass);
        }
    const int64_t ns = (int64_t)sx.size(), n = np;
    if (ns == 0) {
        memset(densph, 0, sizeof(float) * (size_t)np);
        return GF_OK;
    }
    gf_ctx *ctx = default_ctx();
    if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
    std::lock_guard<std::mutex> g(ctx->lock);
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    // inputs: star x, y, z (FP64), star mass (float), pstart; query x, y, z (FP64)
    const size_t sd = al((size_t)ns * sizeof(double)), sf = al((size_t)ns * sizeof(float));
    const size_t qd = al((size_t)n * sizeof(double));
    const size_t off_m = 3 * sd, off_ps = off_m + sf, off_q = off_ps + 256, in_bytes = off_q + 3 * qd;
    GF_TRY(ctx->pin[0].reserve(in_bytes));
    GF_TRY(ctx->particles.reserve(in_bytes + al((size_t)ns * sizeof(float4))));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // the staging buffer may still feed a copy
    char *h = ctx->pin[0].as<char>();
    memcpy(h, sx.data(), (size_t)ns * sizeof(double));
    memcpy(h + sd, sy.data(), (size_t)ns * sizeof(double));
    memcpy(h + 2 * sd, sz.data(), (size_t)ns * sizeof(double));
    memcpy(h + off_m, sm.data(), (size_t)ns * sizeof(float));
    const int64_t ps[2] = {0, ns};
    memcpy(h + off_ps, ps, sizeof(ps));
    double *hq = reinterpret_cast<double *>(h + off_q);
    for (int64_t i = 0; i < n; i++) {
        hq[i] = bp[i].x;
        hq[qd / sizeof(double) + i] = bp[i].y;
        hq[2 * (qd / sizeof(double)) + i] = bp[i].z;
    }
    char *d = ctx->particles.as<char>();
    GF_CUDA_TRY(cudaMemcpyAsync(d, h, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
    const double *dsx = reinterpret_cast<const double *>(d);
    const double *dsy = reinterpret_cast<const double *>(d + sd);
    const double *dsz = reinterpret_cast<const double *>(d + 2 * sd);
    const float *dsm = reinterpret_cast<const float *>(d + off_m);
    const int64_t *dps = reinterpret_cast<const int64_t *>(d + off_ps);
    const double *dqx = reinterpret_cast<const double *>(d + off_q);
    const double *dqy = dqx + qd / sizeof(double);
    const double *dqz = dqy + qd / sizeof(double);
    float4 *spos = reinterpret_cast<float4 *>(d + in_bytes);
    star_pack_kernel<<<grid_for(ns, 256), 256, 0, ctx->stream>>>(ns, dsx, dsy, dsz, dsm, spos);
    GF_LAUNCH_CHECK();
    // the stars' octree (one halo), then FP64 positions in tree order and FP64 node boxes
    GF_TRY(build_tree(ctx, 1, ns, dps, spos, 0.5f, 0, &ctx->last_tree));
    const TreeView &t = ctx->last_tree;
    GF_TRY(ctx->tmp[2].reserve((size_t)ns * (sizeof(double4) + sizeof(int32_t)) + 512));
    double4 *tp = ctx->tmp[2].as<double4>();
    int32_t *tidx = reinterpret_cast<int32_t *>(tp + ns);
    gather_tree_order<<<grid_for(ns, 256), 256, 0, ctx->stream>>>(ns, t.perm, dsx, dsy, dsz, dsm, nullptr, nullptr,
                                                                   tp, tidx);
    GF_LAUNCH_CHECK();
    GF_TRY(ctx->tmp[3].reserve((size_t)std::max(t.nnode, 1) * sizeof(RefNode)));
    RefNode *rn = ctx->tmp[3].as<RefNode>();
    ref_node_kernel<<<grid_for((int64_t)t.nnode * 32, 256), 256, 0, ctx->stream>>>(t.nnode, t.knn, tp, rn);
    GF_LAUNCH_CHECK();
    // the 10 nearest stars of every particle, then the weighted sum
    const size_t oi = al((size_t)n * kNumNearDen * sizeof(int32_t)), od = al((size_t)n * kNumNearDen * sizeof(double)),
                 on = al((size_t)n * sizeof(int32_t)), of = al((size_t)n * sizeof(float));
    GF_TRY(ctx->tmp[1].reserve(oi + od + on + of));
    char *o = ctx->tmp[1].as<char>();
    int32_t *nidx = reinterpret_cast<int32_t *>(o);
    double *nd2 = reinterpret_cast<double *>(o + oi);
    int32_t *ncnt = reinterpret_cast<int32_t *>(o + oi + od);
    float *dens = reinterpret_cast<float *>(o + oi + od + on);
    const int k = (int)std::min<int64_t>(kNumNearDen, ns);
    knn64_kernel<<<grid_for(n * 32, 128), 128, 0, ctx->stream>>>(n, dqx, dqy, dqz, nullptr, k, t.root, t.rend, t.knn,
                                                                 rn, tp, tidx, nullptr, nidx, nd2, ncnt, nullptr);
    GF_LAUNCH_CHECK();
    star_density_kernel<<<grid_for(n, 256), 256, 0, ctx->stream>>>(n, k, nidx, nd2, ncnt, dsm, dens);
    GF_LAUNCH_CHECK();
    GF_TRY(ctx->pin[2].reserve((size_t)n * sizeof(float)));
    GF_CUDA_TRY(cudaMemcpyAsync(ctx->pin[2].ptr, dens, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost,
                                ctx->stream));
    GF_TRY(check_device_errors(ctx));  // synchronises
    memcpy(densph, ctx->pin[2].ptr, (size_t)n * sizeof(float));
    return GF_OK;
}

}  // namespace

}  // namespace gf

using namespace gf;

extern "C" void starfindsphdensity(SimpleBasicParticleType *bp, int np, long long *nearindex, int Numnear,
                                   float *densph) {
    clear_status();
    int st = GF_OK;
    if (np < 0 || (np > 0 && (!bp || !nearindex || !densph)) || Numnear < 1 || Numnear > 32) {
        set_status(GF_EINVAL, "starfindsphdensity: invalid arguments (1 <= Numnear <= 32)");
        st = GF_EINVAL;
    } else if (np > 0 && np < Numnear) {
        // nnost.c:727-730: every particle must find Numnear neighbours
        set_status(GF_EINVAL, "starfindsphdensity: %d particles, fewer than Numnear = %d", np, Numnear);
        st = GF_EINVAL;
    } else if (np > 0) {
        std::vector<float> sph((size_t)np);
        st = findsphdensity_lists(bp, np, nearindex, Numnear, sph.data());
        if (st == GF_OK) st = star_density(bp, np, densph);
    }
    dropin_exit_on_error(st, "starfindsphdensity");
}
