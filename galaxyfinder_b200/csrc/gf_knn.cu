// k-nearest-neighbour search and SPH (W4) density on the octree.
//
// The reference (NewGalFinder/nnost.c:375-422 Find_Near, :560-630
// findsphdensity) walks a COM octree per particle and keeps a sorted list of
// the k closest particles, self included.  Here one warp serves one query at
// a time, walking a chunk of consecutive tree-order queries:
//   * the sorted list (k <= 32) lives in registers, entry j in lane j;
//   * the bound starts at the k-th closest of the previous query's list (or,
//     for the first query of a chunk, of the 32 tree-order neighbours): any k
//     distinct particles bound the true k-th distance from above, so the walk
//     prunes from its first node;
//   * a node is skipped when the lower bound of its box distance exceeds the
//     bound; otherwise its loose particles are tested 32 at a time, one per
//     lane, and the accepted ones are merged into the list (one warp-wide
//     shift per candidate, or a bitonic sort + merge for a large batch).
// Float distances of the float positions pre-filter nodes and candidates with
// a margin larger than their rounding error; every decision that shapes the
// list uses the exact distance in double, (dx*dx + dy*dy) + dz*dz with every
// operation rounded (this file is compiled with --fmad=false), and ties are
// broken by particle index, so the lists are bit-identical to an exact
// search on the same positions.  The density
// rho_i = sum_j W4(|x_i - x_j|, r_k/2) reproduces nnost.c:609-622 and W4
// (nnost.c:536-555) in the reference's float/double arithmetic, summed in
// list order.
#include <float.h>
#include <limits.h>

#include <algorithm>

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
// Float distances of float positions carry a relative error below 6u
// (u = 2^-24: one rounding per difference, square and sum, all terms
// positive), so a float test against bound * (1 + kSlack) never rejects a
// particle or node that the exact FP64 test would keep.
constexpr float kSlack = 1e-6f;
constexpr int kChunk = 32;  // consecutive tree-order queries per warp task

__device__ __forceinline__ float f_d2(const float4 &a, const float4 &b) {
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ float f_box_lb2(const float4 &q, const KnnNode &nd) {
    const float gx = fmaxf(fmaxf(nd.lo[0] - q.x, q.x - nd.hi[0]), 0.f);
    const float gy = fmaxf(fmaxf(nd.lo[1] - q.y, q.y - nd.hi[1]), 0.f);
    const float gz = fmaxf(fmaxf(nd.lo[2] - q.z, q.z - nd.hi[2]), 0.f);
    return gx * gx + gy * gy + gz * gz;
}

// Merges the candidates of one 32-lane batch (lanes with acc set) into the
// sorted list (Ld, Li, Lt): one insertion per candidate when there are few,
// otherwise a bitonic sort of the batch and a bitonic merge with the list.
__device__ __forceinline__ void merge_batch(unsigned mask, double cd, int ci, int ct, double &Ld,
                                            int &Li, int &Lt, int &cnt, int kk, double &bd,
                                            int &bi) {
    const int lane = threadIdx.x & 31;
    const int m = __popc(mask);
    if (m <= 3) {
        while (mask) {
            const int src = __ffs(mask) - 1;
            mask &= mask - 1;
            const double xd = __shfl_sync(0xffffffffu, cd, src);
            const int xi = __shfl_sync(0xffffffffu, ci, src);
            const int xt = __shfl_sync(0xffffffffu, ct, src);
            if (key_lt(bd, bi, xd, xi)) continue;  // the bound tightened meanwhile
            const int at = __popc(__ballot_sync(0xffffffffu, lane < kk && key_lt(Ld, Li, xd, xi)));
            const double ud = __shfl_up_sync(0xffffffffu, Ld, 1);
            const int ui = __shfl_up_sync(0xffffffffu, Li, 1);
            const int ut = __shfl_up_sync(0xffffffffu, Lt, 1);
            if (lane == at) {
                Ld = xd; Li = xi; Lt = xt;
            } else if (lane > at) {
                Ld = ud; Li = ui; Lt = ut;
            }
            if (cnt < kk) cnt++;
            if (cnt == kk) {
                bd = __shfl_sync(0xffffffffu, Ld, kk - 1);
                bi = __shfl_sync(0xffffffffu, Li, kk - 1);
            }
        }
        return;
    }
    double d = (mask >> lane) & 1 ? cd : kInf;
    int i = (mask >> lane) & 1 ? ci : INT_MAX;
    int t = ct;
    // bitonic sort of the batch, carrying the tree index
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const double od = __shfl_xor_sync(0xffffffffu, d, stride);
            const int oi = __shfl_xor_sync(0xffffffffu, i, stride);
            const int ot = __shfl_xor_sync(0xffffffffu, t, stride);
            const bool up = (lane & size) == 0 || size == 32;
            const bool lower = (lane & stride) == 0;
            const bool lt = key_lt(d, i, od, oi);
            if (!((lower == up) ? lt : !lt)) { d = od; i = oi; t = ot; }
        }
    }
    // the 32 smallest of list and batch: elementwise min with the reversed batch
    const double rd = __shfl_sync(0xffffffffu, d, 31 - lane);
    const int ri = __shfl_sync(0xffffffffu, i, 31 - lane);
    const int rt = __shfl_sync(0xffffffffu, t, 31 - lane);
    if (key_lt(rd, ri, Ld, Li)) { Ld = rd; Li = ri; Lt = rt; }
    // bitonic clean to ascending order
#pragma unroll
    for (int stride = 16; stride > 0; stride >>= 1) {
        const double od = __shfl_xor_sync(0xffffffffu, Ld, stride);
        const int oi = __shfl_xor_sync(0xffffffffu, Li, stride);
        const int ot = __shfl_xor_sync(0xffffffffu, Lt, stride);
        const bool lower = (lane & stride) == 0;
        const bool lt = key_lt(Ld, Li, od, oi);
        if (!(lower ? lt : !lt)) { Ld = od; Li = oi; Lt = ot; }
    }
    cnt = min(cnt + m, 32);
    if (cnt >= kk) {
        bd = __shfl_sync(0xffffffffu, Ld, kk - 1);
        bi = __shfl_sync(0xffffffffu, Li, kk - 1);
    }
}

__global__ void __launch_bounds__(256)
knn_kernel(int64_t n, int k, const float4 *__restrict__ pos, const int32_t *__restrict__ perm,
           const int32_t *__restrict__ phalo, const int64_t *__restrict__ pstart,
           const int32_t *__restrict__ root, const int32_t *__restrict__ rend,
           const KnnNode *__restrict__ nodes, int32_t *__restrict__ nearindex,
           float *__restrict__ dens, int *err) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t ntask = (n + kChunk - 1) / kChunk;
    for (int64_t task = wid; task < ntask; task += nwarps) {
        const int64_t q0 = task * kChunk;
        const int64_t q1 = min(q0 + kChunk, n);
        int prev_h = -1, prev_ok = 0;
        double Ld = kInf;
        int Li = INT_MAX, Lt = 0;
        for (int64_t q = q0; q < q1; q++) {
            const int h = phalo[q];
            const int64_t hs = pstart[h], he = pstart[h + 1];
            const int nh = (int)(he - hs);
            const int kk = min(k, nh);
            const float4 Q = pos[q];
            // ---- seed bound: the kk-th closest of the previous query's list
            // (same halo) or of the 32 tree-order neighbours of q
            double d = kInf;
            int id = INT_MAX;
            if (prev_ok && prev_h == h) {
                if (lane < kk) {
                    d = exact_d2(Q, pos[Lt]);
                    id = Li;
                }
            } else {
                int64_t w0 = q - 16;
                if (w0 + 32 > he) w0 = he - 32;
                if (w0 < hs) w0 = hs;
                const int64_t j = w0 + lane;
                if (j < he) {
                    d = exact_d2(Q, pos[j]);
                    id = perm[j];
                }
            }
            warp_sort(d, id);
            double bd = __shfl_sync(0xffffffffu, d, kk - 1);
            int bi = __shfl_sync(0xffffffffu, id, kk - 1);
            Ld = kInf;
            Li = INT_MAX;
            Lt = 0;
            int cnt = 0;
            int node = root[h];
            const int end = rend[h];
            while (node < end) {
                const KnnNode nd = nodes[node];
                const float bf = (float)bd * (1.f + kSlack);
                if (f_box_lb2(Q, nd) > bf) {
                    node = nd.skip;
                    continue;
                }
                const int l1 = nd.lstart + nd.lcount;
                for (int base = nd.lstart; base < l1; base += 32) {
                    const int jj = base + lane;
                    double cd = kInf;
                    int ci = INT_MAX;
                    bool acc = false;
                    if (jj < l1) {
                        const float4 S = pos[jj];
                        if (f_d2(Q, S) <= (float)bd * (1.f + kSlack)) {
                            cd = exact_d2(Q, S);
                            ci = perm[jj];
                            acc = !key_lt(bd, bi, cd, ci);  // (cd, ci) <= (bd, bi)
                        }
                    }
                    const unsigned mask = __ballot_sync(0xffffffffu, acc);
                    if (mask) merge_batch(mask, cd, ci, jj, Ld, Li, Lt, cnt, kk, bd, bi);
                }
                node = node + 1;
            }
            prev_h = h;
            prev_ok = cnt >= kk;
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
    const int64_t warps_needed = (t.n + kChunk - 1) / kChunk;
    int64_t grid = (warps_needed * 32 + block - 1) / block;
    grid = std::max<int64_t>(1, std::min<int64_t>(grid, 148LL * 8));
    knn_kernel<<<(int)grid, block, 0, ctx->stream>>>(t.n, k, t.pos, t.perm, t.phalo, pstart, t.root,
                                                     t.rend, t.knn, nearindex, dens, ctx->d_err);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

}  // namespace gf
