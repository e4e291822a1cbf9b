// k-nearest-neighbour search and SPH (W4) density on the octree.
//
// The reference (NewGalFinder/nnost.c:375-422 Find_Near, :560-630
// findsphdensity) walks a COM octree per particle and keeps a sorted list of
// the k closest particles, self included.  Three kernels compute the same
// lists (GF_KNN_ALGO selects; the autotuner keeps the fastest):
// knn_bucket_kernel and knn_fbucket_kernel (below) walk once per 32
// tree-order queries with one query per lane (the second with float keys and
// an exact certification); knn_kernel serves one query per warp, walking a
// chunk of consecutive tree-order queries:
//   * the sorted list (k <= 32) lives in registers, entry j in lane j;
//   * the list starts as the k closest of the previous query's list (or,
//     for the first query of a chunk, of the 32 tree-order neighbours), with
//     distances recomputed: any k distinct particles bound the true k-th
//     distance from above, so the walk prunes from its first node, and the
//     walk skips the seeds (a per-warp set in shared memory) so that only new
//     particles are merged;
//   * the walk expands bottom-up from the query's own node (its subtree, then
//     each ancestor's range minus the subtree already walked: its loose
//     particles and other children) and stops once the
//     ball of the bound lies inside the processed subtree's box, so the list
//     fills with close particles first and the bound tightens early;
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
constexpr int kChunk = GF_KNN_CHUNK;  // consecutive tree-order queries per warp task

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
// sorted list (Ld, Li): one insertion per candidate when there are few,
// otherwise a bitonic sort of the batch and a bitonic merge with the list.
__device__ __forceinline__ void merge_batch(unsigned mask, double cd, int ci, double &Ld, int &Li,
                                            int &cnt, int kk, double &bd, int &bi,
                                            unsigned long long &nsingle,
                                            unsigned long long &nbitonic) {
    const int lane = threadIdx.x & 31;
    const int m = __popc(mask);
    if (m <= 3) {
        nsingle += m;
        while (mask) {
            const int src = __ffs(mask) - 1;
            mask &= mask - 1;
            const double xd = __shfl_sync(0xffffffffu, cd, src);
            const int xi = __shfl_sync(0xffffffffu, ci, src);
            if (key_lt(bd, bi, xd, xi)) continue;  // the bound tightened meanwhile
            const int at = __popc(__ballot_sync(0xffffffffu, lane < kk && key_lt(Ld, Li, xd, xi)));
            const double ud = __shfl_up_sync(0xffffffffu, Ld, 1);
            const int ui = __shfl_up_sync(0xffffffffu, Li, 1);
            if (lane == at) {
                Ld = xd; Li = xi;
            } else if (lane > at) {
                Ld = ud; Li = ui;
            }
            if (cnt < kk) cnt++;
            if (cnt == kk) {
                bd = __shfl_sync(0xffffffffu, Ld, kk - 1);
                bi = __shfl_sync(0xffffffffu, Li, kk - 1);
            }
        }
        return;
    }
    nbitonic++;
    double d = (mask >> lane) & 1 ? cd : kInf;
    int i = (mask >> lane) & 1 ? ci : INT_MAX;
    warp_sort(d, i);
    // the 32 smallest of list and batch: elementwise min with the reversed batch
    const double rd = __shfl_sync(0xffffffffu, d, 31 - lane);
    const int ri = __shfl_sync(0xffffffffu, i, 31 - lane);
    if (key_lt(rd, ri, Ld, Li)) { Ld = rd; Li = ri; }
    // bitonic clean to ascending order
#pragma unroll
    for (int stride = 16; stride > 0; stride >>= 1) {
        const double od = __shfl_xor_sync(0xffffffffu, Ld, stride);
        const int oi = __shfl_xor_sync(0xffffffffu, Li, stride);
        const bool lower = (lane & stride) == 0;
        const bool lt = key_lt(Ld, Li, od, oi);
        if (!(lower ? lt : !lt)) { Ld = od; Li = oi; }
    }
    cnt = min(cnt + m, 32);
    if (cnt >= kk) {
        bd = __shfl_sync(0xffffffffu, Ld, kk - 1);
        bi = __shfl_sync(0xffffffffu, Li, kk - 1);
    }
}

struct ListState {
    double Ld;  // list entry of this lane (distance^2)
    int Li;     // list entry of this lane (batch index)
    int cnt;    // entries filled
    int kk;     // neighbours wanted
    double bd;  // bound: accept keys <= (bd, bi)
    int bi;
    int *seeded;  // this warp's set of the seeded list entries (shared memory)
};

// Per-warp open-addressing set (64 slots, -1 = empty) of the batch indices
// the list was seeded with; at most 32 entries, so every probe sequence ends
// within the table.
constexpr int kSetSlots = 64;

__device__ __forceinline__ unsigned set_slot(int id) {
    return ((unsigned)id * 2654435761u) >> 26;  // 6 bits
}

__device__ __forceinline__ void set_insert(int *set, int id) {
    unsigned h = set_slot(id);
    for (int t = 0; t < kSetSlots; t++) {
        const int old = atomicCAS(set + h, -1, id);
        if (old == -1 || old == id) return;
        h = (h + 1) & (kSetSlots - 1);
    }
}

__device__ __forceinline__ bool set_contains(const int *set, int id) {
    unsigned h = set_slot(id);
    for (int t = 0; t < kSetSlots; t++) {
        const int v = set[h];
        if (v == id) return true;
        if (v == -1) return false;
        h = (h + 1) & (kSetSlots - 1);
    }
    return false;
}

template <bool COUNT>
__device__ __forceinline__ void scan_loose(int l0, int l1, const float4 &Q,
                                           const float4 *__restrict__ pos,
                                           const int32_t *__restrict__ perm, ListState &L,
                                           unsigned long long (&ctr)[5]) {
    const int lane = threadIdx.x & 31;
    for (int base = l0; base < l1; base += 32) {
        const int jj = base + lane;
        double cd = kInf;
        int ci = INT_MAX;
        bool acc = false;
        if (jj < l1) {
            const float4 S = pos[jj];
            if (f_d2(Q, S) <= (float)L.bd * (1.f + kSlack)) {
                cd = exact_d2(Q, S);
                ci = perm[jj];
                // (cd, ci) <= (bd, bi), and not already in the list as a seed
                acc = !key_lt(L.bd, L.bi, cd, ci) && !set_contains(L.seeded, ci);
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, acc);
        if (COUNT) {
            ctr[1]++;
            ctr[2] += __popc(mask);
        }
        if (mask) merge_batch(mask, cd, ci, L.Ld, L.Li, L.cnt, L.kk, L.bd, L.bi, ctr[3], ctr[4]);
    }
}

// Visits the preorder nodes [i0, i1) except the subtree [x0, x1), with
// pruning: a node whose box lies beyond the bound hides its subtree (the
// preorder range up to its skip index); every other node's loose particles
// are scanned.  The nodes are read 32 at a time, one per lane.  Which of them
// lie inside a subtree hidden by an earlier node of the window is a prefix
// maximum of the hidden ranges' ends over the lanes (five shuffles), so the
// serial part only steps through the visible nodes that hold loose
// particles, each rechecked against the current (tightening) bound.  A
// child's box lies inside its parent's, so the recheck prunes exactly what
// skipping a subtree hidden later would have pruned.
template <bool COUNT>
__device__ __forceinline__ void walk_range(int i0, int i1, int x0, int x1, const float4 &Q,
                                           const float4 *__restrict__ pos,
                                           const int32_t *__restrict__ perm,
                                           const KnnNode *__restrict__ nodes, ListState &L,
                                           unsigned long long (&ctr)[5]) {
    const int lane = threadIdx.x & 31;
    int wb = i0;
    while (wb < i1) {
        const int j = wb + lane;
        const bool valid = j < i1;
        float lb = __int_as_float(0x7f800000);  // +inf: beyond the range
        int skip = 0, l0 = 0, lc = 0;
        if (valid) {
            const KnnNode nd = nodes[j];
            lb = f_box_lb2(Q, nd);
            skip = nd.skip;
            l0 = nd.lstart;
            lc = nd.lcount;
        }
        // hidden: beyond the bound at the window's start, or the excluded subtree
        bool hides = valid && lb > (float)L.bd * (1.f + kSlack);
        if (j == x0) {
            hides = true;
            skip = x1;
        }
        int cover = hides ? skip : 0;  // inclusive prefix max of the hidden ranges' ends
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, cover, off);
            if (lane >= off) cover = max(cover, o);
        }
        int before = __shfl_up_sync(0xffffffffu, cover, 1);
        if (lane == 0) before = 0;
        const bool visible = valid && before <= j;
        if (COUNT) {
            const unsigned vm = __ballot_sync(0xffffffffu, visible);
            if (lane == 0) ctr[0] += __popc(vm);
        }
        unsigned todo = __ballot_sync(0xffffffffu, visible && !hides && lc > 0);
        while (todo) {
            const int li = __ffs(todo) - 1;
            todo &= todo - 1;
            const float nlb = __shfl_sync(0xffffffffu, lb, li);
            if (nlb > (float)L.bd * (1.f + kSlack)) continue;
            const int s0 = __shfl_sync(0xffffffffu, l0, li);
            const int sc = __shfl_sync(0xffffffffu, lc, li);
            scan_loose<COUNT>(s0, s0 + sc, Q, pos, perm, L, ctr);
        }
        // the next window starts past this one and past every hidden range
        wb = max(wb + 32, __shfl_sync(0xffffffffu, cover, 31));
    }
}

// True when the ball of radius sqrt(bd) around q lies inside the node's box
// (tested in double with a relative and absolute margin).
__device__ __forceinline__ bool ball_inside(const float4 &Q, double bd, const KnnNode &A) {
    const double r = sqrt(bd) * (1.0 + 1e-9) + 1e-12;
    const double qx = Q.x, qy = Q.y, qz = Q.z;
    return qx - r >= (double)A.lo[0] && qx + r <= (double)A.hi[0] && qy - r >= (double)A.lo[1] &&
           qy + r <= (double)A.hi[1] && qz - r >= (double)A.lo[2] && qz + r <= (double)A.hi[2];
}

template <bool COUNT>
__global__ void __launch_bounds__(GF_KNN_BLOCK, GF_KNN_MINB)
knn_kernel(int64_t n, int k, const float4 *__restrict__ pos, const int32_t *__restrict__ perm,
           const float4 *__restrict__ pos_batch, const int32_t *__restrict__ phalo,
           const int64_t *__restrict__ pstart, const int32_t *__restrict__ owner,
           const KnnNode *__restrict__ nodes, int32_t *__restrict__ nearindex,
           float *__restrict__ dens, int *err, unsigned long long *__restrict__ counters,
           const int32_t *__restrict__ qlist, const unsigned *__restrict__ nq_dev = nullptr,
           bool natural_rows = false, int chunk = kChunk) {
    // nq_dev: the query count lives in device memory (qlist filled by an
    // earlier kernel); natural_rows: outputs go to the query's batch row
    // perm[q] rather than to row qi of the list; chunk: list entries per
    // warp task
    if (nq_dev) n = *nq_dev;
    const int lane = threadIdx.x & 31;
    __shared__ int seeded_set[GF_KNN_BLOCK / 32][kSetSlots];
    int *seeded = seeded_set[threadIdx.x >> 5];
    seeded[lane] = -1;
    seeded[lane + 32] = -1;
    __syncwarp();
    // work counters: nodes tested, 32-wide leaf batches, candidates accepted
    // (new and within the bound), candidates inserted one by one, bitonic
    // batch merges
    unsigned long long ctr[5] = {0, 0, 0, 0, 0};
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t ntask = (n + chunk - 1) / chunk;
    for (int64_t task = wid; task < ntask; task += nwarps) {
        const int64_t q0 = task * chunk;
        const int64_t q1 = min(q0 + (int64_t)chunk, n);
        int prev_h = -1, prev_ok = 0;
        ListState L;
        L.Ld = kInf;
        L.Li = INT_MAX;
        for (int64_t qi = q0; qi < q1; qi++) {
            // with a query list, row qi of the outputs is tree position qlist[qi]
            const int64_t q = qlist ? (int64_t)qlist[qi] : qi;
            const int h = phalo[q];
            const int64_t hs = pstart[h], he = pstart[h + 1];
            const int nh = (int)(he - hs);
            const int kk = min(k, nh);
            const float4 Q = pos[q];
            // ---- seed: the list starts as the kk closest of the previous
            // query's list (same halo; distances recomputed) or of the 32
            // tree-order neighbours of q, which also bounds the walk from its
            // first node (kk distinct particles bound the true kk-th
            // distance).  The seeds are remembered so that the walk does not
            // insert them twice.
            double d = kInf;
            int id = INT_MAX;
            if (prev_ok && prev_h == h) {
                if (lane < kk) {
                    d = exact_d2(Q, pos_batch[L.Li]);
                    id = L.Li;
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
            L.Ld = lane < kk ? d : kInf;
            L.Li = lane < kk ? id : INT_MAX;
            L.bd = __shfl_sync(0xffffffffu, d, kk - 1);
            L.bi = __shfl_sync(0xffffffffu, id, kk - 1);
            L.cnt = kk;
            L.kk = kk;
            L.seeded = seeded;
            if (lane < kk) set_insert(seeded, id);
            __syncwarp();
            // ---- bottom-up expanding walk: q's own node's subtree first, then
            // each ancestor's loose particles and other children, until the
            // ball of the bound lies inside the box of the processed subtree
            // (a node's box lies inside its octant region, which holds exactly
            // the subtree's particles, so nothing outside can enter the list).
            // One walk per level: q's own node's subtree, then each
            // ancestor's whole range except the subtree walked before it
            // (one call site keeps the kernel's code small).
            int c = owner[q];
            KnnNode C = nodes[c];
            int w0 = c, w1 = C.skip, x0 = -1, x1 = -1;
            while (true) {
                walk_range<COUNT>(w0, w1, x0, x1, Q, pos, perm, nodes, L, ctr);
                if (C.parent < 0 || (L.cnt >= kk && ball_inside(Q, L.bd, C))) break;
                const int a = C.parent;
                const KnnNode A = nodes[a];
                w0 = a;
                w1 = A.skip;
                x0 = c;
                x1 = C.skip;
                c = a;
                C = A;
            }
            seeded[lane] = -1;
            seeded[lane + 32] = -1;
            __syncwarp();
            prev_h = h;
            prev_ok = L.cnt >= kk;
            if (L.cnt < kk) {
                if (lane == 0) atomicOr(err, GF_ERRBIT_KNN);
                continue;
            }
            // ---- outputs in batch order
            const int64_t qo = qlist && !natural_rows ? qi : (int64_t)perm[q];
            if (lane < k) nearindex[(int64_t)qo * k + lane] = lane < kk ? (int32_t)(L.Li - hs) : -1;
            // nnost.c:292,415: maxr = sqrtf(maxdist2); W4(sqrtf(d2_j), maxr/2.)
            const float neardist = sqrtf((float)__shfl_sync(0xffffffffu, L.Ld, kk - 1));
            const float hh = (float)(neardist / 2.);
            const float wj = lane < kk ? w4(sqrtf((float)L.Ld), hh) : 0.f;
            float rho = 0.f;
            for (int j = 0; j < kk; j++) rho += __shfl_sync(0xffffffffu, wj, j);
            if (lane == 0 && dens) dens[qo] = rho;
        }
    }
    if (COUNT && counters && lane == 0)
        for (int i = 0; i < 5; i++) atomicAdd(counters + i, ctr[i]);
}

// ---------------------------------------------------------------- bucket kNN
// One warp serves a bucket of 32 consecutive tree-order queries, one per
// lane, and walks the tree once for all of them: a node is entered when its
// box lies within the bound of any lane, and each of its loose particles is
// tested by every lane against its own query.  Neighbouring queries share
// most of their candidates, so the walk, the node tests and the particle
// loads are paid once per bucket rather than once per query.  Each lane keeps
// its k closest as a max-heap (GF_KNNB_ARITY children per node) keyed by
// (exact FP64 distance^2, batch index) in its own column of a per-warp
// shared-memory array (column = lane: every access is conflict-free however
// the lanes' heap positions diverge).
//   * Seeds: every lane's heap starts as its query's min(32, halo size)
//     tree-order neighbours (heapified), which bounds its k-th distance before
//     the walk; the walk skips them.
//   * Walk: bottom-up as in knn_kernel, starting at the smallest subtree that
//     holds the whole bucket, then each ancestor's range minus the subtree
//     already walked, until every lane's ball lies inside the processed box.
//   * Output: an in-place heapsort gives the ascending list; the density is
//     summed in list order as in knn_kernel.
// The prefilters and the exact keys are those of knn_kernel, so the lists
// and densities are bit-identical.
constexpr int kHeapBytes = 32 * 32 * (int)(sizeof(double) + sizeof(int));
constexpr int kBucketWarpBytes = kHeapBytes + 32 * (int)sizeof(KnnNode) + 32 * 16 + 32 * 4;
static_assert(sizeof(KnnNode) == 48, "KnnNode is copied as 12 words");

// f_d2 with fused multiply-adds: at most four roundings after the exact-input
// differences, so the relative error stays below the 6u that kSlack covers.
__device__ __forceinline__ float f_d2_fma(const float4 &a, const float4 &b) {
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
}

struct LaneHeap {
    double *D;  // this lane's column: entry e at D[32 * e]
    int *I;
    int kk;
    double bd;  // root key: the bound
    int bi;
    float bf;   // float prefilter bound: (float)bd * (1 + kSlack)
};

constexpr int kArity = GF_KNNB_ARITY;  // children per heap node

// Places (kd, ki) at the hole `pos` and moves it down to restore the max-heap
// over entries [0, size).
__device__ __forceinline__ void heap_sift_down(double *D, int *I, int pos, int size, double kd, int ki) {
    while (true) {
        const int c0 = kArity * pos + 1;
        if (c0 >= size) break;
        int c = c0;
        double cd = D[32 * c0];
        int ci = I[32 * c0];
#pragma unroll
        for (int u = 1; u < kArity; u++) {
            if (c0 + u < size) {
                const double rd = D[32 * (c0 + u)];
                const int ri = I[32 * (c0 + u)];
                if (key_lt(cd, ci, rd, ri)) {
                    c = c0 + u;
                    cd = rd;
                    ci = ri;
                }
            }
        }
        if (!key_lt(kd, ki, cd, ci)) break;
        D[32 * pos] = cd;
        I[32 * pos] = ci;
        pos = c;
    }
    D[32 * pos] = kd;
    I[32 * pos] = ki;
}

__device__ __forceinline__ void heap_set_bound(LaneHeap &H) {
    H.bd = H.D[0];
    H.bi = H.I[0];
    H.bf = (float)H.bd * (1.f + kSlack);
}

// Replaces the root (the largest key) by (kd, ki), which is below it.
__device__ __forceinline__ void heap_put(LaneHeap &H, double kd, int ki) {
    heap_sift_down(H.D, H.I, 0, H.kk, kd, ki);
    heap_set_bound(H);
}

template <bool COUNT>
__global__ void __launch_bounds__(GF_KNNB_BLOCK, GF_KNNB_MINB)
knn_bucket_kernel(int64_t n, int k, const float4 *__restrict__ pos, const int32_t *__restrict__ perm,
                  const int32_t *__restrict__ phalo, const int64_t *__restrict__ pstart,
                  const int32_t *__restrict__ owner, const KnnNode *__restrict__ nodes,
                  int32_t *__restrict__ nearindex, float *__restrict__ dens, int *err,
                  unsigned long long *__restrict__ counters) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    unsigned char *ws = smem + (size_t)(threadIdx.x >> 5) * kBucketWarpBytes;
    double *HD = reinterpret_cast<double *>(ws);
    int *HI = reinterpret_cast<int *>(ws + 32 * 32 * sizeof(double));
    KnnNode *win = reinterpret_cast<KnnNode *>(ws + kHeapBytes);
    float4 *cpos = reinterpret_cast<float4 *>(ws + kHeapBytes + 32 * sizeof(KnnNode));
    int *cid = reinterpret_cast<int *>(cpos + 32);
    int *win_w = reinterpret_cast<int *>(win);
    const int *nodes_w = reinterpret_cast<const int *>(nodes);
    // work counters: node tests, 32-wide particle loads, heap insertions
    // (per lane), warp-wide insertion steps, buckets
    unsigned long long ctr[5] = {0, 0, 0, 0, 0};
    const bool vec_out = k % 4 == 0 && ((uintptr_t)nearindex & 15) == 0;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nbucket = (n + 31) >> 5;
    for (int64_t bucket = wid; bucket < nbucket; bucket += nwarps) {
        const int64_t b = bucket << 5;
        const int64_t q = b + lane;
        const bool valid = q < n;
        const int h = valid ? phalo[q] : -1;
        const float4 Q = valid ? pos[q] : make_float4(0.f, 0.f, 0.f, 0.f);
        const double Qx = Q.x, Qy = Q.y, Qz = Q.z;
        const int myid = valid ? perm[q] : INT_MAX;
        unsigned remaining = __ballot_sync(0xffffffffu, valid);
        // one pass per halo present in the bucket (its lanes are contiguous)
        while (remaining) {
            const int leader = __ffs(remaining) - 1;
            const int hl = __shfl_sync(0xffffffffu, h, leader);
            const unsigned act = __ballot_sync(0xffffffffu, valid && h == hl);
            remaining &= ~act;
            const bool me = (act >> lane) & 1;
            const int qa = (int)(b + leader);
            const int qb = (int)(b + 31 - __clz(act));
            const int64_t hs = pstart[hl];
            const int64_t he = pstart[hl + 1];
            const int kk = (int)min((int64_t)k, he - hs);
            LaneHeap H;
            H.D = HD + lane;
            H.I = HI + lane;
            H.kk = kk;
            // ---- seeds: the min(32, halo size) tree-order neighbours of the
            // lane's query (>= kk particles, so the heap is full and bounds
            // the walk from its first node); the walk skips them
            const int ns = (int)min((int64_t)32, he - hs);
            int64_t sw = q - 16;
            if (sw + ns > he) sw = he - ns;
            if (sw < hs) sw = hs;
            const int sw0 = (int)sw, sw1 = (int)sw + ns;
            if (me) {
                for (int t = 0; t < kk; t++) {
                    H.D[32 * t] = exact_d2(Q, pos[sw0 + t]);
                    H.I[32 * t] = perm[sw0 + t];
                }
                for (int e = (kk - 2) / kArity; e >= 0; e--) heap_sift_down(H.D, H.I, e, kk, H.D[32 * e], H.I[32 * e]);
                heap_set_bound(H);
                for (int t = kk; t < ns; t++) {
                    const double d = exact_d2(Q, pos[sw0 + t]);
                    const int sid = perm[sw0 + t];
                    if (key_lt(d, sid, H.bd, H.bi)) heap_put(H, d, sid);
                }
            } else {
                H.bd = kInf;
                H.bi = INT_MAX;
                H.bf = 0.f;
            }
            // ---- the smallest subtree holding [qa, qb]
            int c = owner[qa];
            KnnNode C = nodes[c];
            while (!(C.lstart <= qa && qb < C.lstart + C.count) && C.parent >= 0) {
                c = C.parent;
                C = nodes[c];
            }
            int w0 = c, w1 = C.skip, x0 = -1, x1 = -1;
            while (true) {
                // ---- stackless preorder walk of [w0, w1) minus [x0, x1)
                int i = w0, wb = INT_MIN / 2;
                while (i < w1) {
                    if (i == x0) {
                        i = x1;
                        continue;
                    }
                    if (i >= wb + 32 || i < wb) {  // window of 32 nodes at i
                        wb = i;
                        const int nw = min(32, w1 - wb) * 12;
                        __syncwarp();
                        for (int t = lane; t < nw; t += 32) win_w[t] = nodes_w[(int64_t)wb * 12 + t];
                        __syncwarp();
                    }
                    const float4 *nv = reinterpret_cast<const float4 *>(win + (i - wb));
                    const float4 n0 = nv[0], n1 = nv[1];
                    const float gx = fmaxf(fmaxf(n0.x - Q.x, Q.x - n0.w), 0.f);
                    const float gy = fmaxf(fmaxf(n0.y - Q.y, Q.y - n1.x), 0.f);
                    const float gz = fmaxf(fmaxf(n0.z - Q.z, Q.z - n1.y), 0.f);
                    const float lb = gx * gx + gy * gy + gz * gz;
                    if (COUNT) ctr[0]++;
                    if (!__any_sync(0xffffffffu, me && lb <= H.bf)) {
                        i = __float_as_int(n1.z);  // skip
                        continue;
                    }
                    const int l0 = __float_as_int(n1.w);
                    const int l1 = l0 + __float_as_int(nv[2].x);
                    for (int base = l0; base < l1; base += 32) {
                        const int j = base + lane;
                        __syncwarp();
                        if (j < l1) {
                            cpos[lane] = pos[j];
                            cid[lane] = perm[j];
                        }
                        __syncwarp();
                        const int m = min(32, l1 - base);
                        if (COUNT) ctr[1] += m;
                        // four candidates in flight: their float distances are
                        // independent; the bound is re-read after each insertion
                        for (int t0 = 0; t0 < m; t0 += 4) {
                            float4 S[4];
                            float f[4];
#pragma unroll
                            for (int u = 0; u < 4; u++) {
                                S[u] = cpos[t0 + u];  // t0 + u <= 31; entries >= m are ignored
                                f[u] = f_d2_fma(Q, S[u]);
                            }
#pragma unroll
                            for (int u = 0; u < 4; u++) {
                                const int p = base + t0 + u;
                                bool ins = false;
                                if (me && t0 + u < m && f[u] <= H.bf && (p < sw0 || p >= sw1)) {
                                    const double dx = Qx - (double)S[u].x;
                                    const double dy = Qy - (double)S[u].y;
                                    const double dz = Qz - (double)S[u].z;
                                    const double d = dx * dx + dy * dy + dz * dz;
                                    const int sid = cid[t0 + u];
                                    if (key_lt(d, sid, H.bd, H.bi)) {
                                        heap_put(H, d, sid);
                                        ins = true;
                                    }
                                }
                                if (COUNT) {
                                    ctr[2] += ins;
                                    ctr[3] += __any_sync(0xffffffffu, ins);
                                }
                            }
                        }
                    }
                    i++;
                }
                const bool done = !me || ball_inside(Q, H.bd, C);
                if (C.parent < 0 || __all_sync(0xffffffffu, done)) break;
                const int a = C.parent;
                const KnnNode A = nodes[a];
                w0 = a;
                w1 = A.skip;
                x0 = c;
                x1 = C.skip;
                c = a;
                C = A;
            }
            if (COUNT) ctr[4]++;
            // ---- outputs in batch order
            if (me) {
                {  // heapsort: ascending keys
                    for (int e = kk - 1; e > 0; e--) {
                        const double td = H.D[32 * e];
                        const int ti = H.I[32 * e];
                        H.D[32 * e] = H.D[0];
                        H.I[32 * e] = H.I[0];
                        heap_sift_down(H.D, H.I, 0, e, td, ti);
                    }
                    int32_t *row = nearindex + (int64_t)myid * k;
                    if (vec_out) {
                        for (int j = 0; j < k; j += 4) {
                            int4 v;
                            v.x = j < kk ? (int32_t)(H.I[32 * j] - hs) : -1;
                            v.y = j + 1 < kk ? (int32_t)(H.I[32 * (j + 1)] - hs) : -1;
                            v.z = j + 2 < kk ? (int32_t)(H.I[32 * (j + 2)] - hs) : -1;
                            v.w = j + 3 < kk ? (int32_t)(H.I[32 * (j + 3)] - hs) : -1;
                            *reinterpret_cast<int4 *>(row + j) = v;
                        }
                    } else {
                        for (int j = 0; j < k; j++) row[j] = j < kk ? (int32_t)(H.I[32 * j] - hs) : -1;
                    }
                    if (dens) {
                        // nnost.c:292,415: maxr = sqrtf(maxdist2); W4(sqrtf(d2_j), maxr/2.)
                        const float neardist = sqrtf((float)H.D[32 * (kk - 1)]);
                        const float hh = (float)(neardist / 2.);
                        float rho = 0.f;
                        for (int j = 0; j < kk; j++) rho += w4(sqrtf((float)H.D[32 * j]), hh);
                        dens[myid] = rho;
                    }
                }
            }
            __syncwarp();
        }
    }
    if (COUNT && counters) {
        for (int off = 16; off; off >>= 1) ctr[2] += __shfl_xor_sync(0xffffffffu, ctr[2], off);
        if (lane == 0) {
            atomicAdd(counters + 0, ctr[0]);
            atomicAdd(counters + 1, ctr[1]);
            atomicAdd(counters + 2, ctr[2]);
            atomicAdd(counters + 3, ctr[3]);
            atomicAdd(counters + 4, ctr[4]);
        }
    }
}

// ------------------------------------------------- bucket kNN, float keys
// As knn_bucket_kernel, but each lane's heap holds packed 64-bit keys
// (float distance^2 bits << 32 | batch index): non-negative float bit
// patterns order like the floats, so one integer compare orders (f, index).
// The walk needs no FP64 and the heaps take 8 KB per warp instead of 12 KB
// (more resident warps).  Float keys can misorder particles whose exact
// distances agree to ~6u, so the result is certified per query: every
// particle not kept has a float distance (or lies in a node whose float box
// distance was) at least frej, or lies outside the box of the processed
// subtree (exact distance >= the box distance dbox), and floats are within
// 6u of the exact value; the kept k are re-ranked by their exact FP64
// distances, and the list is exact when the largest kept exact distance is
// below min(frej (1 - 2e-6), dbox^2).  A query that fails (near-ties at the
// k-th place, duplicate positions) goes to a device list that knn_kernel
// then serves exactly.  The certification, the output row and the density
// (in the arithmetic of knn_kernel) are computed either by every lane for its
// own query (GF_KNNB_LANECERT=1: the lane heapsorts its column, computes the
// exact distances in that order and insertion-sorts only where near-ties
// reversed the float order) or by the warp one query at a time with a
// bitonic sort of the exact keys.
// Nodes of the walk staged per warp in shared memory (GF_KNNB_WIN at a time;
// 0: every node is read from global memory through L1).  A smaller window
// leaves room for more resident warps.
constexpr int kWin = GF_KNNB_WIN;
constexpr int kFBucketWarpBytes = 32 * 32 * 8 + kWin * (int)sizeof(KnnNode) + 32 * 16 + 32 * 4 +
                                  32 * GF_KNNB_QUEUE * 8;

__device__ __forceinline__ uint64_t pack_key(float f, int id) {
    return ((uint64_t)__float_as_uint(f) << 32) | (uint32_t)id;
}
__device__ __forceinline__ float key_f(uint64_t key) { return __uint_as_float((unsigned)(key >> 32)); }

// Max-heap of packed keys in one lane's column (entry e at K[32 e]).  With
// GF_KNNB_HEAPF >= 1 the heap is ordered by the float part alone (one
// 32-bit compare per step; 2 and 3 also move the hole down first, 3 admits
// a particle by its float distance alone): among entries of equal float distance the root is then
// any of them, which the certification already covers (an evicted or
// rejected particle whose float distance equals a kept one's leaves the
// query uncertified, and the exact kernel serves it).
__device__ __forceinline__ void kheap_sift_down(uint64_t *K, int pos, int size, uint64_t key) {
#if GF_KNNB_HEAPF >= 2
    // the hole left at pos descends to a leaf along the larger children (one
    // compare per level, no test against key), then key rises from there to
    // its place below pos
    const unsigned kf = (unsigned)(key >> 32);
    const int top = pos;
    while (true) {
        int c = 2 * pos + 1;
        if (c >= size) break;
        uint64_t ck = K[32 * c];
        if (c + 1 < size) {
            const uint64_t rk = K[32 * (c + 1)];
            if ((unsigned)(rk >> 32) > (unsigned)(ck >> 32)) {
                c++;
                ck = rk;
            }
        }
        K[32 * pos] = ck;
        pos = c;
    }
    while (pos > top) {
        const int p = (pos - 1) >> 1;
        const uint64_t pk = K[32 * p];
        if ((unsigned)(pk >> 32) >= kf) break;
        K[32 * pos] = pk;
        pos = p;
    }
    K[32 * pos] = key;
#else
#if GF_KNNB_HEAPF
    const unsigned kf = (unsigned)(key >> 32);
#endif
    while (true) {
        int c = 2 * pos + 1;
        if (c >= size) break;
        uint64_t ck = K[32 * c];
        if (c + 1 < size) {
            const uint64_t rk = K[32 * (c + 1)];
#if GF_KNNB_HEAPF
            if ((unsigned)(rk >> 32) > (unsigned)(ck >> 32)) {
#else
            if (rk > ck) {
#endif
                c++;
                ck = rk;
            }
        }
#if GF_KNNB_HEAPF
        if (kf >= (unsigned)(ck >> 32)) break;
#else
        if (key > ck) break;
#endif
        K[32 * pos] = ck;
        pos = c;
    }
    K[32 * pos] = key;
#endif
}

template <bool COUNT>
__global__ void __launch_bounds__(GF_KNNB_BLOCK, GF_KNNB_MINB)
knn_fbucket_kernel(int64_t n, int k, const float4 *__restrict__ pos, const int32_t *__restrict__ perm,
                   const float4 *__restrict__ pos_batch, const int32_t *__restrict__ phalo,
                   const int64_t *__restrict__ pstart, const int32_t *__restrict__ owner,
                   const KnnNode *__restrict__ nodes, int32_t *__restrict__ nearindex,
                   float *__restrict__ dens, int32_t *__restrict__ redo, unsigned *__restrict__ nredo,
                   unsigned long long *__restrict__ counters, unsigned long long *__restrict__ work) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    unsigned char *ws = smem + (size_t)(threadIdx.x >> 5) * kFBucketWarpBytes;
    uint64_t *KH = reinterpret_cast<uint64_t *>(ws);
    KnnNode *win = reinterpret_cast<KnnNode *>(ws + 32 * 32 * 8);
    float4 *cpos = reinterpret_cast<float4 *>(ws + 32 * 32 * 8 + kWin * sizeof(KnnNode));
    int *cid = reinterpret_cast<int *>(cpos + 32);
    int *win_w = reinterpret_cast<int *>(win);
    const int *nodes_w = reinterpret_cast<const int *>(nodes);
    uint64_t *K = KH + lane;  // this lane's heap column
    // with GF_KNNB_QUEUE, survivors of the tile filter wait in the lane's
    // queue column and the warp inserts all lanes' queues together, so the
    // lanes sift in the same steps instead of one tile's survivors at a time
    uint64_t *QK = reinterpret_cast<uint64_t *>(cid + 32) + lane;
    int qn = 0;
    // work counters: node tests, particle tests, heap insertions (per lane),
    // warp-wide insertion steps, queries sent to the exact kernel
    unsigned long long ctr[5] = {0, 0, 0, 0, 0};
    const float kInfF = __int_as_float(0x7f800000);
    const bool vec_out = k % 4 == 0 && ((uintptr_t)nearindex & 15) == 0;
    (void)vec_out;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nbucket = (n + 31) >> 5;
    // the warp's next bucket: from the work counter, or grid-stride
    auto next = [&](int64_t stride_bucket) -> int64_t {
        if (!GF_KNNB_DYN || !work) return stride_bucket;
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(work, 1ull);
        return (int64_t)__shfl_sync(0xffffffffu, b, 0);
    };
    for (int64_t bucket = next(wid); bucket < nbucket; bucket = next(bucket + nwarps)) {
        const int64_t b = bucket << 5;
        const int64_t q = b + lane;
        const bool valid = q < n;
        const int h = valid ? phalo[q] : -1;
        const float4 Q = valid ? pos[q] : make_float4(0.f, 0.f, 0.f, 0.f);
        const int myid = valid ? perm[q] : INT_MAX;
        unsigned remaining = __ballot_sync(0xffffffffu, valid);
        while (remaining) {
            const int leader = __ffs(remaining) - 1;
            const int hl = __shfl_sync(0xffffffffu, h, leader);
            const unsigned act = __ballot_sync(0xffffffffu, valid && h == hl);
            remaining &= ~act;
            const bool me = (act >> lane) & 1;
            const int qa = (int)(b + leader);
            const int qb = (int)(b + 31 - __clz(act));
            const int64_t hs = pstart[hl];
            const int64_t he = pstart[hl + 1];
            const int kk = (int)min((int64_t)k, he - hs);
            // ---- seeds: the query's min(GF_KNNB_SEEDS, halo size) tree-order neighbours
            const int ns = (int)min((int64_t)GF_KNNB_SEEDS, he - hs);
            int64_t sw = q - GF_KNNB_SEEDS / 2;
            if (sw + ns > he) sw = he - ns;
            if (sw < hs) sw = hs;
            const int sw0 = (int)sw, sw1 = (int)sw + ns;
            uint64_t rk = ~0ull;  // root key (the bound)
            float bf = 0.f;       // its float distance
            float frej = kInfF;   // least float distance (or box bound) of everything not kept
            if (me) {
                for (int t = 0; t < kk; t++) K[32 * t] = pack_key(f_d2_fma(Q, pos[sw0 + t]), perm[sw0 + t]);
                for (int e = (kk - 2) / 2; e >= 0; e--) kheap_sift_down(K, e, kk, K[32 * e]);
                rk = K[0];
                for (int t = kk; t < ns; t++) {
                    const float f = f_d2_fma(Q, pos[sw0 + t]);
                    const uint64_t key = pack_key(f, perm[sw0 + t]);
                    if (key < rk) {
                        frej = fminf(frej, key_f(rk));
                        kheap_sift_down(K, 0, kk, key);
                        rk = K[0];
                    } else {
                        frej = fminf(frej, f);
                    }
                }
                bf = key_f(rk);
            }
            // every lane inserts its queued survivors
            auto flush_queue = [&]() {
                for (int u = 0; u < qn; u++) {
                    const uint64_t key = QK[32 * u];
                    if (key < rk) {
                        frej = fminf(frej, bf);  // the evicted root
                        kheap_sift_down(K, 0, kk, key);
                        rk = K[0];
                        bf = key_f(rk);
                        if (COUNT) ctr[2]++;
                    } else {
                        frej = fminf(frej, key_f(key));
                    }
                }
                qn = 0;
            };
            (void)flush_queue;
            // ---- the smallest subtree holding [qa, qb]
            int c = owner[qa];
            KnnNode C = nodes[c];
            while (!(C.lstart <= qa && qb < C.lstart + C.count) && C.parent >= 0) {
                c = C.parent;
                C = nodes[c];
            }
            int w0 = c, w1 = C.skip, x0 = -1, x1 = -1;
            double tbox;  // squared distance from the query to the outside of the processed box
            while (true) {
                int i = w0, wb = INT_MIN / 2;
                while (i < w1) {
                    if (i == x0) {
                        i = x1;
                        continue;
                    }
                    const float4 *nv;
                    if (kWin > 0) {
                        if (i >= wb + kWin || i < wb) {
                            wb = i;
                            const int nw = min(kWin, w1 - wb) * 12;
                            __syncwarp();
                            for (int t = lane; t < nw; t += 32) win_w[t] = nodes_w[(int64_t)wb * 12 + t];
                            __syncwarp();
                        }
                        nv = reinterpret_cast<const float4 *>(win + (i - wb));
                    } else {
                        nv = reinterpret_cast<const float4 *>(nodes + i);  // one broadcast line
                    }
                    const float4 n0 = kWin > 0 ? nv[0] : __ldg(nv), n1 = kWin > 0 ? nv[1] : __ldg(nv + 1);
                    const float gx = fmaxf(fmaxf(n0.x - Q.x, Q.x - n0.w), 0.f);
                    const float gy = fmaxf(fmaxf(n0.y - Q.y, Q.y - n1.x), 0.f);
                    const float gz = fmaxf(fmaxf(n0.z - Q.z, Q.z - n1.y), 0.f);
                    const float lb = __fmaf_rn(gx, gx, __fmaf_rn(gy, gy, __fmul_rn(gz, gz)));
                    if (COUNT) ctr[0]++;
                    if (!__any_sync(0xffffffffu, me && lb <= bf)) {
                        frej = fminf(frej, lb);  // the whole subtree lies in this box
                        i = __float_as_int(n1.z);
                        continue;
                    }
                    const int l0 = __float_as_int(n1.w);
                    const int l1 = l0 + __float_as_int(kWin > 0 ? nv[2].x : __ldg(reinterpret_cast<const float *>(nv + 2)));
                    for (int base = l0; base < l1; base += 32) {
                        const int j = base + lane;
                        __syncwarp();
                        if (j < l1) {
                            cpos[lane] = pos[j];
                            cid[lane] = perm[j];
                        } else if (GF_KNNB_FILT) {
                            // a sentinel at infinity: its float distance is
                            // +inf, which neither passes nor lowers frej
                            cpos[lane] = make_float4(kInfF, kInfF, kInfF, 0.f);
                        }
                        __syncwarp();
                        const int m = min(32, l1 - base);
                        if (COUNT) ctr[1] += m;
                        // filter: a branch-free pass over the tile against
                        // the bound at its start (the bound only tightens)
                        unsigned pass = 0;
                        if (me && (base >= sw1 || base + m <= sw0)) {  // none of this lane's seeds here
#if GF_KNNB_FILT
                            // four candidates per step with their own
                            // rejection minima (min is exact, so the order of
                            // the minima does not matter); entries m..m+3 of
                            // the last step are sentinels (t + 3 <= 31)
                            float r1 = kInfF, r2 = kInfF, r3 = kInfF;
                            for (int t = 0; t < m; t += 4) {
                                const float fa = f_d2_fma(Q, cpos[t]), fb = f_d2_fma(Q, cpos[t + 1]);
                                const float fc = f_d2_fma(Q, cpos[t + 2]), fd = f_d2_fma(Q, cpos[t + 3]);
                                const bool oa = fa <= bf, ob = fb <= bf, oc = fc <= bf, od = fd <= bf;
                                pass |= ((unsigned)oa | ((unsigned)ob << 1) | ((unsigned)oc << 2) | ((unsigned)od << 3))
                                        << t;
                                frej = fminf(frej, oa ? kInfF : fa);
                                r1 = fminf(r1, ob ? kInfF : fb);
                                r2 = fminf(r2, oc ? kInfF : fc);
                                r3 = fminf(r3, od ? kInfF : fd);
                            }
                            frej = fminf(fminf(frej, r1), fminf(r2, r3));
#else
#pragma unroll 4
                            for (int t = 0; t < m; t++) {
                                const float f = f_d2_fma(Q, cpos[t]);
                                const bool ok = f <= bf;
                                pass |= (unsigned)ok << t;
                                frej = ok ? frej : fminf(frej, f);
                            }
#endif
                        } else if (me) {
#pragma unroll 4
                            for (int t = 0; t < m; t++) {
                                const float f = f_d2_fma(Q, cpos[t]);
                                const int p = base + t;
                                const bool seed = p >= sw0 && p < sw1;
                                const bool ok = !seed && f <= bf;
                                pass |= (unsigned)ok << t;
                                frej = (ok || seed) ? frej : fminf(frej, f);
                            }
                        }
                        if (COUNT) {
                            ctr[3] += __reduce_max_sync(0xffffffffu, (unsigned)__popc(pass));
                        }
                        // insert the survivors (each lane its own)
#if GF_KNNB_QUEUE
                        while (true) {
                            while (pass && qn < GF_KNNB_QUEUE) {
                                const int t = __ffs(pass) - 1;
                                pass &= pass - 1;
                                const float f = f_d2_fma(Q, cpos[t]);
                                const uint64_t key = pack_key(f, cid[t]);
                                if (key < rk) {
                                    QK[32 * qn] = key;
                                    qn++;
                                } else {
                                    frej = fminf(frej, f);
                                }
                            }
                            if (!__any_sync(0xffffffffu, pass != 0u)) break;
                            flush_queue();  // a lane's queue is full
                        }
#else
                        while (pass) {
                            const int t = __ffs(pass) - 1;
                            pass &= pass - 1;
                            const float f = f_d2_fma(Q, cpos[t]);
#if GF_KNNB_HEAPF == 3
                            // float test: a particle at the root's float
                            // distance stays out and leaves the query
                            // uncertified, as a tie evicted from the heap would
                            if (f < bf) {
                                const uint64_t key = pack_key(f, cid[t]);
#else
                            const uint64_t key = pack_key(f, cid[t]);
                            if (key < rk) {
#endif
                                frej = fminf(frej, bf);  // the evicted root
                                kheap_sift_down(K, 0, kk, key);
                                rk = K[0];
                                bf = key_f(rk);
                                if (COUNT) ctr[2]++;
                            } else {
                                frej = fminf(frej, f);
                            }
                        }
#endif
                    }
                    i++;
                }
#if GF_KNNB_QUEUE
                flush_queue();  // the bound is current before the stopping test
#endif
                // distance from the query to the outside of C's box (exact
                // differences of floats, squared in double)
                const double dbx = fmin((double)Q.x - (double)C.lo[0], (double)C.hi[0] - (double)Q.x);
                const double dby = fmin((double)Q.y - (double)C.lo[1], (double)C.hi[1] - (double)Q.y);
                const double dbz = fmin((double)Q.z - (double)C.lo[2], (double)C.hi[2] - (double)Q.z);
                const double db = fmin(fmin(dbx, dby), dbz);
                tbox = C.parent < 0 ? kInf : (db > 0.0 ? db * db : 0.0);
                const bool done = !me || tbox > (double)bf * (1.0 + 4e-6);
                if (C.parent < 0 || __all_sync(0xffffffffu, done)) break;
                const int a = C.parent;
                const KnnNode A = nodes[a];
                w0 = a;
                w1 = A.skip;
                x0 = c;
                x1 = C.skip;
                c = a;
                C = A;
            }
            // certification threshold: a lower bound of the exact distance^2
            // of every particle not kept
            const double tcert = fmin((double)frej * (1.0 - 2e-6), tbox * (1.0 - 1e-12));
#if GF_KNNB_LANECERT
            // ---- every lane certifies and writes its own query
            if (me) {
                // heapsort of the lane's column: ascending (float distance, index)
                for (int e = kk - 1; e > 0; e--) {
                    const uint64_t last = K[32 * e];
                    K[32 * e] = K[0];
                    kheap_sift_down(K, 0, e, last);
                }
                // exact FP64 distances in that order; the float of each
                // replaces the float key (the density needs nothing else)
                bool sorted = true;
                double dprev = 0.0;
                int iprev = -1;
#pragma unroll 4
                for (int e = 0; e < kk; e++) {
                    const int id = (int)(uint32_t)K[32 * e];
                    const double d = exact_d2(Q, pos_batch[id]);
                    sorted = sorted && (e == 0 || !key_lt(d, id, dprev, iprev));
                    K[32 * e] = pack_key((float)d, id);
                    dprev = d;
                    iprev = id;
                }
                if (!sorted) {
                    // near-ties ordered differently by the float keys:
                    // insertion sort by the exact key (recomputed)
                    for (int e = 1; e < kk; e++) {
                        const uint64_t v = K[32 * e];
                        const int vid = (int)(uint32_t)v;
                        const double vd = exact_d2(Q, pos_batch[vid]);
                        int f = e;
                        for (; f > 0; f--) {
                            const uint64_t u = K[32 * (f - 1)];
                            const int uid = (int)(uint32_t)u;
                            if (!key_lt(vd, vid, exact_d2(Q, pos_batch[uid]), uid)) break;
                            K[32 * f] = u;
                        }
                        K[32 * f] = v;
                    }
                    dprev = exact_d2(Q, pos_batch[(int)(uint32_t)K[32 * (kk - 1)]]);
                }
                if (dprev < tcert) {
                    int32_t *row = nearindex + (int64_t)myid * k;
                    if (vec_out) {
                        for (int j = 0; j < k; j += 4) {
                            int4 v;
                            v.x = j < kk ? (int32_t)((int64_t)(uint32_t)K[32 * j] - hs) : -1;
                            v.y = j + 1 < kk ? (int32_t)((int64_t)(uint32_t)K[32 * (j + 1)] - hs) : -1;
                            v.z = j + 2 < kk ? (int32_t)((int64_t)(uint32_t)K[32 * (j + 2)] - hs) : -1;
                            v.w = j + 3 < kk ? (int32_t)((int64_t)(uint32_t)K[32 * (j + 3)] - hs) : -1;
                            *reinterpret_cast<int4 *>(row + j) = v;
                        }
                    } else {
                        for (int j = 0; j < k; j++)
                            row[j] = j < kk ? (int32_t)((int64_t)(uint32_t)K[32 * j] - hs) : -1;
                    }
                    if (dens) {
                        // nnost.c:292,415: maxr = sqrtf(maxdist2); W4(sqrtf(d2_j), maxr/2.)
                        const float neardist = sqrtf((float)dprev);
                        const float hh = (float)(neardist / 2.);
                        float rho = 0.f;
                        for (int j = 0; j < kk; j++) rho += w4(sqrtf(key_f(K[32 * j])), hh);
                        dens[myid] = rho;
                    }
                } else {
                    redo[atomicAdd(nredo, 1u)] = (int32_t)q;
                    if (COUNT) ctr[4]++;
                }
            }
            __syncwarp();
#else
            // ---- transpose the heaps: entry e of lane l moves to slot
            // 32 e + (l ^ e), so that the warp reads one lane's column
            // without bank conflicts
            for (int e = 0; e < kk; e++) {
                const uint64_t v = KH[32 * e + lane];
                __syncwarp();
                KH[32 * e + (lane ^ e)] = v;
                __syncwarp();
            }
            // ---- one query at a time: exact FP64 re-rank, certify, write
            for (unsigned mm = act; mm; mm &= mm - 1) {
                const int r = __ffs(mm) - 1;
                float4 Qr;
                Qr.x = __shfl_sync(0xffffffffu, Q.x, r);
                Qr.y = __shfl_sync(0xffffffffu, Q.y, r);
                Qr.z = __shfl_sync(0xffffffffu, Q.z, r);
                const double tr = __shfl_sync(0xffffffffu, tcert, r);
                const int rid = __shfl_sync(0xffffffffu, myid, r);
                int id = INT_MAX;
                double d = kInf;
                if (lane < kk) {
                    id = (int)(uint32_t)KH[32 * lane + (r ^ lane)];
                    d = exact_d2(Qr, pos_batch[id]);
                }
                warp_sort(d, id);
                const double dk = __shfl_sync(0xffffffffu, d, kk - 1);
                if (dk < tr) {
                    if (lane < k) nearindex[(int64_t)rid * k + lane] = lane < kk ? (int32_t)(id - hs) : -1;
                    // nnost.c:292,415: maxr = sqrtf(maxdist2); W4(sqrtf(d2_j), maxr/2.)
                    const float neardist = sqrtf((float)dk);
                    const float hh = (float)(neardist / 2.);
                    const float wj = lane < kk ? w4(sqrtf((float)d), hh) : 0.f;
                    float rho = 0.f;
                    for (int j = 0; j < kk; j++) rho += __shfl_sync(0xffffffffu, wj, j);
                    if (lane == 0 && dens) dens[rid] = rho;
                } else if (lane == 0) {
                    redo[atomicAdd(nredo, 1u)] = (int32_t)(b + r);
                    if (COUNT) ctr[4]++;
                }
            }
            __syncwarp();
#endif
        }
    }
    if (COUNT && counters) {
        for (int off = 16; off; off >>= 1) {
            ctr[2] += __shfl_xor_sync(0xffffffffu, ctr[2], off);
            if (GF_KNNB_LANECERT) ctr[4] += __shfl_xor_sync(0xffffffffu, ctr[4], off);
        }
        if (lane == 0) {
            atomicAdd(counters + 0, ctr[0]);
            atomicAdd(counters + 1, ctr[1]);
            atomicAdd(counters + 2, ctr[2]);
            atomicAdd(counters + 3, ctr[3]);
            atomicAdd(counters + 4, ctr[4]);
        }
    }
}

}  // namespace

int launch_knn(gf_ctx *ctx, const TreeView &t, const int64_t *pstart, const float4 *pos_batch, int k,
               int32_t *nearindex, float *dens, unsigned long long *counters,
               const int32_t *qlist, int64_t nq) {
    if (k < 1 || k > 32) {
        set_status(GF_EINVAL, "k = %d: the warp kNN supports 1 <= k <= 32", k);
        return GF_EINVAL;
    }
    const int64_t nquery = qlist ? nq : t.n;
    if (t.n <= 0 || nquery <= 0) return GF_OK;
    if (GF_KNN_ALGO == 2 && !qlist) {
        // scratch: the list of queries the float-key kernel could not certify
        GF_TRY(ctx->tmp[7].reserve((size_t)t.n * sizeof(int32_t) + 256));
        unsigned *nredo = ctx->tmp[7].as<unsigned>();
        int32_t *redo = reinterpret_cast<int32_t *>(ctx->tmp[7].as<char>() + 256);
        GF_CUDA_TRY(cudaMemsetAsync(nredo, 0, sizeof(unsigned), ctx->stream));
        const int block = GF_KNNB_BLOCK;
        const size_t shmem = (size_t)(block / 32) * kFBucketWarpBytes;
        int per_sm = 0;
        auto kern = counters ? knn_fbucket_kernel<true> : knn_fbucket_kernel<false>;
        GF_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
        GF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, shmem));
        const int64_t nbucket = (t.n + 31) / 32;
        int64_t grid = (nbucket * 32 + block - 1) / block;
        grid = std::max<int64_t>(1, std::min<int64_t>(grid, (int64_t)sm_count() * std::max(per_sm, 1)));
        unsigned long long *work = nullptr;
        if (GF_KNNB_DYN) {  // one resident wave; each warp takes its next bucket from a counter
            GF_TRY(ctx->work.reserve(256));
            work = ctx->work.as<unsigned long long>() + 16;  // slot 16: this search
            GF_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(unsigned long long), ctx->stream));
        }
        kern<<<(int)grid, block, shmem, ctx->stream>>>(t.n, k, t.pos, t.perm, pos_batch, t.phalo, pstart, t.owner,
                                                       t.knn, nearindex, dens, redo, nredo, counters, work);
        GF_LAUNCH_CHECK();
        // the uncertified queries, exactly, into their own rows (the count
        // stays on the device; the grid strides over whatever it is)
        knn_kernel<false><<<sm_count() * (2048 / GF_KNN_BLOCK), GF_KNN_BLOCK, 0, ctx->stream>>>(
            t.n, k, t.pos, t.perm, pos_batch, t.phalo, pstart, t.owner, t.knn, nearindex, dens, ctx->d_err,
            nullptr, redo, nredo, true, 1);  // scattered queries: one per warp task
        GF_LAUNCH_CHECK();
        return GF_OK;
    }
    if (GF_KNN_ALGO == 1 && !qlist) {
        const int block = GF_KNNB_BLOCK;
        const size_t shmem = (size_t)(block / 32) * kBucketWarpBytes;
        int per_sm = 0;
        auto kern = counters ? knn_bucket_kernel<true> : knn_bucket_kernel<false>;
        GF_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
        GF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, shmem));
        const int64_t nbucket = (t.n + 31) / 32;
        int64_t grid = (nbucket * 32 + block - 1) / block;
        grid = std::max<int64_t>(1, std::min<int64_t>(grid, (int64_t)sm_count() * std::max(per_sm, 1)));
        kern<<<(int)grid, block, shmem, ctx->stream>>>(t.n, k, t.pos, t.perm, t.phalo, pstart, t.owner, t.knn,
                                                       nearindex, dens, ctx->d_err, counters);
        GF_LAUNCH_CHECK();
        return GF_OK;
    }
    const int block = GF_KNN_BLOCK;
    const int64_t warps_needed = (nquery + kChunk - 1) / kChunk;
    int64_t grid = (warps_needed * 32 + block - 1) / block;
    grid = std::max<int64_t>(1, std::min<int64_t>(grid, (int64_t)sm_count() * (2048 / block)));
    if (counters)
        knn_kernel<true><<<(int)grid, block, 0, ctx->stream>>>(nquery, k, t.pos, t.perm, pos_batch, t.phalo,
                                                               pstart, t.owner, t.knn, nearindex, dens,
                                                               ctx->d_err, counters, qlist);
    else
        knn_kernel<false><<<(int)grid, block, 0, ctx->stream>>>(nquery, k, t.pos, t.perm, pos_batch, t.phalo,
                                                                pstart, t.owner, t.knn, nearindex, dens,
                                                                ctx->d_err, nullptr, qlist);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

}  // namespace gf
