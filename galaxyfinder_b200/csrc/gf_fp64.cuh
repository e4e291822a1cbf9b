// FP64 octree helpers shared by the reference tree API (gf_reftree.cu) and the
// plain FP64 stage (gf_plain64.cu): node moments and boxes evaluated in FP64
// from FP64 positions on libgf's octree, and an exact FP64 k-nearest search.
// Both translation units are compiled with --fmad=false.
#pragma once

#include <math.h>

#include "gf_tree.cuh"

namespace gf {

// internal linkage: every including translation unit gets its own copy
namespace {

// FP64 moments and box of one preorder node, over its particles.
struct RefNode {
    double com[3];
    double mass;
    double dist2;   // max |x - com|^2
    double q[6];    // xx, yy, zz, xy, xz, yz about the com
    double lo[3], hi[3];
};

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min_d(double v) {
    for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// x, y, z, m of the tree's particles gathered into tree order, and for each
// tree position its index in the caller's numbering (set[p], or p itself).
// Masses are read as float, as divide_node reads them (ost.c:538).
__global__ void gather_tree_order(int64_t n, const int32_t *__restrict__ perm, const double *__restrict__ x,
                                  const double *__restrict__ y, const double *__restrict__ z,
                                  const float *__restrict__ mf, const double *__restrict__ md,
                                  const int32_t *__restrict__ set, double4 *__restrict__ out,
                                  int32_t *__restrict__ tidx) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = perm[t];
        const double m = mf ? (double)mf[p] : (double)(float)md[p];
        out[t] = make_double4(x[p], y[p], z[p], m);
        if (tidx) tidx[t] = set ? set[p] : p;
    }
}

// A warp per node: mass and centre of mass (divide_node, ost.c:545-555:
// float masses summed in double), then size and second moments about it.
__global__ void ref_node_kernel(int32_t nnode, const KnnNode *__restrict__ knn, const double4 *__restrict__ tp,
                                RefNode *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nnode; i += warps) {
        const int a = knn[i].lstart, b = a + knn[i].count;
        double m = 0, sx = 0, sy = 0, sz = 0;
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int j = a + lane; j < b; j += 32) {
            const double4 p = tp[j];
            m += p.w;
            sx += p.w * p.x;
            sy += p.w * p.y;
            sz += p.w * p.z;
            lo[0] = fmin(lo[0], p.x);
            hi[0] = fmax(hi[0], p.x);
            lo[1] = fmin(lo[1], p.y);
            hi[1] = fmax(hi[1], p.y);
            lo[2] = fmin(lo[2], p.z);
            hi[2] = fmax(hi[2], p.z);
        }
        m = warp_sum_d(m);
        sx = warp_sum_d(sx);
        sy = warp_sum_d(sy);
        sz = warp_sum_d(sz);
        for (int c = 0; c < 3; c++) {
            lo[c] = warp_min_d(lo[c]);
            hi[c] = warp_max_d(hi[c]);
        }
        const double cx = sx / m, cy = sy / m, cz = sz / m;
        double d2 = 0, q[6] = {0, 0, 0, 0, 0, 0};
        for (int j = a + lane; j < b; j += 32) {
            const double4 p = tp[j];
            const double dx = p.x - cx, dy = p.y - cy, dz = p.z - cz;
            d2 = fmax(d2, dx * dx + dy * dy + dz * dz);
            q[0] += p.w * dx * dx;
            q[1] += p.w * dy * dy;
            q[2] += p.w * dz * dz;
            q[3] += p.w * dx * dy;
            q[4] += p.w * dx * dz;
            q[5] += p.w * dy * dz;
        }
        d2 = warp_max_d(d2);
        for (int c = 0; c < 6; c++) q[c] = warp_sum_d(q[c]);
        if (lane == 0) {
            RefNode r;
            r.com[0] = cx;
            r.com[1] = cy;
            r.com[2] = cz;
            r.mass = m;
            r.dist2 = d2;
            for (int c = 0; c < 6; c++) r.q[c] = q[c];
            for (int c = 0; c < 3; c++) {
                r.lo[c] = lo[c];
                r.hi[c] = hi[c];
            }
            out[i] = r;
        }
    }
}

// (d2, index) order of the neighbour lists.
__device__ __forceinline__ bool nb_less(double d2a, int32_t ia, double d2b, int32_t ib) {
    return d2a < d2b || (d2a == d2b && ia < ib);
}

// W4 kernel (nnost.c:536-555) in FP64.
__device__ __forceinline__ double w4_64(double r, double h) {
    const double u = r / h;
    if (u < 1.) return (1. - 1.5 * u * u + 0.75 * u * u * u) / (M_PI * h * h * h);
    if (u < 2.) return (2. - u) * (2. - u) * (2. - u) / (4. * M_PI * h * h * h);
    return 0.;
}

// Exact k nearest (k <= 32) of each query point among the particles of its
// halo's tree, a warp per query: lane j keeps the j-th nearest; the walk
// visits the preorder nodes, skipping a subtree whose FP64 box is farther
// than the k-th distance.  Particle distances are (dx*dx + dy*dy) + dz*dz in
// FP64; ties are ordered by the particles' numbers tidx.  qhalo (nullable:
// halo 0) selects the query's tree [root[h], rend[h]); with pstart the
// written indices are relative to the halo's first particle (-1 past a halo
// smaller than k), and with dens the FP64 W4 density of the list (h = r_k/2)
// is written too.
__global__ void knn64_kernel(int64_t nq, const double *__restrict__ qx, const double *__restrict__ qy,
                             const double *__restrict__ qz, const int32_t *__restrict__ qhalo, int k,
                             const int32_t *__restrict__ root, const int32_t *__restrict__ rend,
                             const KnnNode *__restrict__ knn, const RefNode *__restrict__ rn,
                             const double4 *__restrict__ tp, const int32_t *__restrict__ tidx,
                             const int64_t *__restrict__ pstart, int32_t *__restrict__ out_idx,
                             double *__restrict__ out_d2, int32_t *__restrict__ out_n, float *__restrict__ dens) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t q = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; q < nq; q += warps) {
        const int h = qhalo ? qhalo[q] : 0;
        const double px = qx[q], py = qy[q], pz = qz[q];
        double my_d2 = INFINITY;  // lane j: j-th nearest so far
        int32_t my_i = INT32_MAX;
        int filled = 0;
        double kth = INFINITY;
        int32_t kth_i = INT32_MAX;
        const int r1 = rend[h];
        int i = root[h];
        while (i < r1) {
            const KnnNode nd = knn[i];
            if (filled == k) {
                const RefNode &r = rn[i];
                const double dx = fmax(fmax(r.lo[0] - px, px - r.hi[0]), 0.0);
                const double dy = fmax(fmax(r.lo[1] - py, py - r.hi[1]), 0.0);
                const double dz = fmax(fmax(r.lo[2] - pz, pz - r.hi[2]), 0.0);
                if ((dx * dx + dy * dy) + dz * dz > kth) {  // nothing inside can enter the list
                    i = nd.skip;
                    continue;
                }
            }
            for (int c = nd.lstart; c < nd.lstart + nd.lcount; c += 32) {
                const int j = c + lane;
                const bool in = j < nd.lstart + nd.lcount;
                double d2 = INFINITY;
                int32_t id = INT32_MAX;
                if (in) {
                    const double4 s = tp[j];
                    const double tx = px - s.x, ty = py - s.y, tz = pz - s.z;
                    d2 = tx * tx + ty * ty + tz * tz;
                    id = tidx[j];
                }
                unsigned cand = __ballot_sync(0xffffffffu, in && (filled < k || nb_less(d2, id, kth, kth_i)));
                while (cand) {
                    const int src = __ffs(cand) - 1;
                    cand &= cand - 1;
                    const double cd = __shfl_sync(0xffffffffu, d2, src);
                    const int32_t ci = __shfl_sync(0xffffffffu, id, src);
                    if (filled == k && !nb_less(cd, ci, kth, kth_i)) continue;
                    // position of the candidate: the entries before it
                    const unsigned before = __ballot_sync(0xffffffffu, lane < filled && nb_less(my_d2, my_i, cd, ci));
                    const int pos = __popc(before);
                    const double up_d2 = __shfl_up_sync(0xffffffffu, my_d2, 1);
                    const int32_t up_i = __shfl_up_sync(0xffffffffu, my_i, 1);
                    if (lane == pos) {
                        my_d2 = cd;
                        my_i = ci;
                    } else if (lane > pos) {
                        my_d2 = up_d2;
                        my_i = up_i;
                    }
                    if (filled < k) filled++;
                    kth = __shfl_sync(0xffffffffu, my_d2, k - 1);
                    kth_i = __shfl_sync(0xffffffffu, my_i, k - 1);
                }
            }
            i++;  // preorder: the first child, or past this node when it has none
        }
        const int64_t base = pstart ? pstart[h] : 0;
        if (lane < filled) {
            out_idx[q * k + lane] = (int32_t)(my_i - base);
            if (out_d2) out_d2[q * k + lane] = my_d2;
        } else if (lane < k && pstart) {
            out_idx[q * k + lane] = -1;  // a halo smaller than k
        }
        if (lane == 0 && out_n) out_n[q] = filled;
        if (dens && filled > 0) {
            const double hk = sqrt(__shfl_sync(0xffffffffu, my_d2, filled - 1)) / 2.;
            double w = lane < filled ? w4_64(sqrt(my_d2), hk) : 0.;
            w = warp_sum_d(w);
            if (lane == 0) dens[q] = (float)w;
        }
    }
}

}  // namespace

}  // namespace gf
