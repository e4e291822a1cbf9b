// k-nearest-neighbour search and SPH (W4) density on the octree.
//
// The reference (NewGalFinder/nnost.c:375-422 Find_Near, :560-630
// findsphdensity) walks a COM octree per particle and keeps a sorted list of
// the k closest particles, self included.  Here one warp serves one query:
//   * the sorted list (k <= 32) lives in registers, entry j in lane j;
//   * the bound starts at the k-th closest of the 32 particles around the
//     query in tree order (an upper bound on the true k-th distance), so the
//     walk prunes from its first node;
//   * a node is skipped when the exact lower bound of its box distance exceeds
//     the bound; otherwise its loose particles are tested 32 at a time, one per
//     lane, and accepted candidates are inserted by a warp-wide shift.
// Distances are evaluated in double from the FP32 recentred positions,
// (dx*dx + dy*dy) + dz*dz with every operation rounded (this file is compiled
// with --fmad=false), and ties are broken by particle index, so the lists are
// bit-identical to an exact search on the same positions.  The density
// rho_i = sum_j W4(|x_i - x_j|, r_k/2) reproduces nnost.c:609-622 and W4
// (nnost.c:536-555) in the reference's float/double arithmetic, summed in
// list order.
#include <float.h>
#include <limits.h>

#include "gf_tree.cuh"

namespace gf {

namespace {

__device__ __forceinline__ bool key_lt(double da, int ia, double db, int ib) {
    return da < db || (da == db && ia < ib);
}

__device__ __forceinline__ double exact_d2(const float4 &a, const float4 &b) {
    const double dx = (double)a.x - (double)b.x;
    const double dy = (double)a.y - (double)b.y;
    const double dz = (double)a.z - (double)b.z;
    return dx * dx + dy * dy + dz * dz;
}

// Lower bound of the distance^2 from q to any point of the box [lo, hi]; by
// monotonicity of rounding it never exceeds exact_d2 to a particle inside.
__device__ __forceinline__ double box_lb2(const float4 &q, const KnnNode &nd) {
    double g[3];
    const float c[3] = {q.x, q.y, q.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (c[a] < nd.lo[a]) g[a] = (double)nd.lo[a] - (double)c[a];
        else if (c[a] > nd.hi[a]) g[a] = (double)c[a] - (double)nd.hi[a];
        else g[a] = 0.0;
    }
    return g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
}

// W4 kernel, nnost.c:536-555 (float arguments, double constants)
__device__ __forceinline__ float w4(float dist, float h) {
    const float r = dist / h;
    if (r < 1.) {
        return (float)((-0.2387324) * ((2. - (double)r) * (double)r * (double)r - 1.333333) /
                       (double)(h * h * h));
    } else if (r < 2.) {
        const float twomr = (float)((2. - (double)r) / (double)h);
        return (float)(0.07957747 * (double)twomr * (double)twomr * (double)twomr);
    }
    return 0.f;
}

// Ascending bitonic sort of one (d, i) pair per lane.
__device__ __forceinline__ void warp_sort(double &d, int &i) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const double od = __shfl_xor_sync(0xffffffffu, d, stride);
            const int oi = __shfl_xor_sync(0xffffffffu, i, stride);
            const bool up = (lane & size) == 0 || size == 32;
            const bool lower = (lane & stride) == 0;
            const bool mine_lt = key_lt(d, i, od, oi);
            const bool keep = (lower == up) ? mine_lt : !mine_lt;
            if (!keep) {
                d = od;
                i = oi;
            }
        }
    }
}

constexpr double kInf = DBL_MAX;

__global__ void __launch_bounds__(256)
knn_kernel(int64_t n, int k, const float4 *__restrict__ pos, const int32_t *__restrict__ perm,
           const int32_t *__restrict__ phalo, const int64_t *__restrict__ pstart,
           const int32_t *__restrict__ root, const int32_t *__restrict__ rend,
           const KnnNode *__restrict__ nodes, int32_t *__restrict__ nearindex,
           float *__restrict__ dens, int *err) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t q = wid; q < n; q += nwarps) {
        const int h = phalo[q];
        const int64_t hs = pstart[h], he = pstart[h + 1];
        const int nh = (int)(he - hs);
        const int kk = min(k, nh);
        const float4 Q = pos[q];
        // ---- seed: the kk-th closest of up to 32 tree-order neighbours of q
        int64_t w0 = q - 16;
        if (w0 + 32 > he) w0 = he - 32;
        if (w0 < hs) w0 = hs;
        {
            const int64_t j = w0 + lane;
            double d = kInf;
            int id = INT_MAX;
            if (j < he) {
                d = exact_d2(Q, pos[j]);
                id = perm[j];
            }
            warp_sort(d, id);
            d = __shfl_sync(0xffffffffu, d, kk - 1);
            id = __shfl_sync(0xffffffffu, id, kk - 1);
            // bound: accept keys <= (bd, bi)
            double bd = d;
            int bi = id;
            double Ld = kInf;
            int Li = INT_MAX;
            int cnt = 0;
            int node = root[h];
            const int end = rend[h];
            while (node < end) {
                const KnnNode nd = nodes[node];
                if (box_lb2(Q, nd) > bd) {
                    node = nd.skip;
                    continue;
                }
                const int64_t l1 = (int64_t)nd.lstart + nd.lcount;
                for (int64_t base = nd.lstart; base < l1; base += 32) {
                    const int64_t jj = base + lane;
                    double cd = kInf;
                    int ci = INT_MAX;
                    bool acc = false;
                    if (jj < l1) {
                        cd = exact_d2(Q, pos[jj]);
                        ci = perm[jj];
                        acc = !key_lt(bd, bi, cd, ci);  // (cd, ci) <= (bd, bi)
                    }
                    unsigned mask = __ballot_sync(0xffffffffu, acc);
                    while (mask) {
                        const int src = __ffs(mask) - 1;
                        mask &= mask - 1;
                        const double xd = __shfl_sync(0xffffffffu, cd, src);
                        const int xi = __shfl_sync(0xffffffffu, ci, src);
                        if (key_lt(bd, bi, xd, xi)) continue;  // bound tightened meanwhile
                        const int at = __popc(__ballot_sync(0xffffffffu,
                                                            lane < kk && key_lt(Ld, Li, xd, xi)));
                        const double ud = __shfl_up_sync(0xffffffffu, Ld, 1);
                        const int ui = __shfl_up_sync(0xffffffffu, Li, 1);
                        if (lane == at) {
                            Ld = xd;
                            Li = xi;
                        } else if (lane > at) {
                            Ld = ud;
                            Li = ui;
                        }
                        if (cnt < kk) cnt++;
                        if (cnt == kk) {
                            bd = __shfl_sync(0xffffffffu, Ld, kk - 1);
                            bi = __shfl_sync(0xffffffffu, Li, kk - 1);
                        }
                    }
                }
                node = node + 1;
            }
            if (cnt < kk) {
                if (lane == 0) atomicOr(err, GF_ERRBIT_KNN);
                continue;
            }
            // ---- outputs in batch order
            const int qo = perm[q];
            if (lane < k) nearindex[(int64_t)qo * k + lane] = lane < kk ? (int32_t)(Li - hs) : -1;
            // nnost.c:292,415: maxr = sqrtf(maxdist2); W4(sqrtf(d2_j), maxr/2.)
            const float neardist = sqrtf((float)__shfl_sync(0xffffffffu, Ld, kk - 1));
            const float hh = (float)(neardist / 2.);
            const float wj = lane < kk ? w4(sqrtf((float)Ld), hh) : 0.f;
            float rho = 0.f;
            for (int j = 0; j < kk; j++) rho += __shfl_sync(0xffffffffu, wj, j);
            if (lane == 0 && dens) dens[qo] = rho;
        }
    }
}

}  // namespace

int launch_knn(gf_ctx *ctx, const TreeView &t, const int64_t *pstart, int k, int32_t *nearindex,
               float *dens) {
    if (k < 1 || k > 32) {
        set_status(GF_EINVAL, "k = %d: the warp kNN supports 1 <= k <= 32", k);
        return GF_EINVAL;
    }
    if (t.n <= 0) return GF_OK;
    const int block = 256;
    const int64_t warps_needed = t.n;
    int64_t grid = (warps_needed * 32 + block - 1) / block;
    grid = std::min<int64_t>(grid, 148LL * 8 * 4);
    knn_kernel<<<(int)grid, block, 0, ctx->stream>>>(t.n, k, t.pos, t.perm, t.phalo, pstart, t.root,
                                                     t.rend, t.knn, nearindex, dens, ctx->d_err);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

}  // namespace gf
