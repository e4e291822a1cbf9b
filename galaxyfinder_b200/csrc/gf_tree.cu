// Level-synchronous GPU build of the centre-of-mass octree of every halo in a
// batch, following the node rules of the reference's tree builders
// (NewGalFinder/ost.c:532-640 divide_node, nnost.c:105-197 new_divide_node_Near):
//   * a node's centre of mass splits its particles into octants by
//     (x > com_x) + 2 (y > com_y) + 4 (z > com_z);
//   * an octant becomes a child node iff it holds >= 10 particles
//     (MIN_CELL_PARTICLE_NUM) and the node's size sqrt(max |x - com|^2)
//     exceeds 0.5e-6 (MINCELLWIDTH/2); smaller octants stay as loose
//     particles of the node;
//   * monopole, second moments and dist2 = max |x - com|^2 are per node.
// Each level processes every still-active particle at once (all halos, all
// nodes of the level): accumulate mass and first moments, finalise the COM,
// accumulate extents/second moments/octant counts, allocate children, and
// scatter the particles into [loose | child 0 | child 1 | ...] order.  After
// the last level the nodes are renumbered in depth-first preorder so the walks
// are stackless: opening node i continues at i + 1, skipping it continues at
// skip[i].
#include <math.h>

#include <algorithm>
#include <vector>

#include "gf_tree.cuh"

namespace gf {

namespace {

constexpr int kMinCell = 10;          // MIN_CELL_PARTICLE_NUM, tree.h:20
constexpr double kMinWidth = 1.E-6;   // MINCELLWIDTH, tree.h:18
constexpr int kBlock = GF_TREE_BLOCK;

// Order-preserving float <-> uint32 map for atomic min/max on any sign.
__device__ __forceinline__ unsigned fkey(float v) {
    unsigned u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(unsigned k) {
    unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// BFS-numbered node arrays used while building.
struct Build {
    int32_t *start, *count, *halo;
    double *m, *mx, *my, *mz;       // mass and first moments, then COM in mx..mz
    unsigned *r2;                   // float bits of max |x - com|^2
    float *q;                       // 6 second moments
    unsigned *box;                  // 6 fkeys: min xyz, max xyz
    int32_t *oct;                   // 8 octant counts
    int32_t *cur;                   // 8 octant cursors
    int32_t *ochild;                // 8 child ids or -1
    int32_t *first, *nchild, *lstart, *lcount;
    int32_t *sub, *pre;             // subtree size, preorder index
    int32_t *par;                   // BFS id of the parent, -1 for roots
    int32_t *counter;               // [0] nodes allocated, [1] overflow flag, [2] blocks done
    int32_t *lev;                   // level L holds BFS nodes [lev[L], lev[L+1])
};

constexpr int kMaxLevels = 4096;

// Grid-stride range of the nodes of level L (bounds in device memory).
#define FOR_LEVEL_NODES(node, L, b)                                                          \
    for (int node = (b).lev[L] + blockIdx.x * blockDim.x + threadIdx.x; node < (b).lev[(L) + 1]; \
         node += gridDim.x * blockDim.x)

__global__ void init_build(int32_t nhalo, Build b) {
    if (threadIdx.x == 0) {
        b.counter[0] = nhalo;  // the roots are nodes 0 .. nhalo-1
        b.counter[1] = 0;
        b.counter[2] = 0;
        b.lev[0] = 0;
        b.lev[1] = nhalo;
    }
}

__global__ void init_roots(int32_t nhalo, const int64_t *__restrict__ pstart, Build b) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nhalo) return;
    b.start[h] = (int32_t)pstart[h];
    b.count[h] = (int32_t)(pstart[h + 1] - pstart[h]);
    b.halo[h] = h;
    b.par[h] = -1;
}

__global__ void init_particles(int64_t n, const int64_t *__restrict__ pstart, int32_t nhalo,
                               const float4 *__restrict__ pos_in, float4 *__restrict__ pos,
                               int32_t *__restrict__ perm, int32_t *__restrict__ pnode) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = nhalo;
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (pstart[mid] <= p) lo = mid; else hi = mid;
        }
        pos[p] = pos_in[p];
        perm[p] = (int32_t)p;
        pnode[p] = lo;  // the root of halo h is node h
    }
}

// Sum of v over the lanes of `mask` that share this lane's key group.
template <class T>
__device__ __forceinline__ T group_sum(unsigned mask, T v) {
    // mask: lanes with the same node; reduce by walking set bits (<= 32 adds)
    T acc = 0;
    for (unsigned m = mask; m; m &= m - 1) acc += __shfl_sync(mask, v, __ffs(m) - 1);
    return acc;
}

// Runs of a warp: lanes with equal node ids are consecutive (a node's active
// particles are contiguous at every level), so a node's lanes form one run.
// Inclusive segmented scans over the runs (five shuffle steps whatever the
// run lengths); each run's last lane holds its reduction.
struct WarpRuns {
    int start;  // first lane of this lane's run
    bool tail;  // last lane of its run
};
__device__ __forceinline__ WarpRuns warp_runs(int node) {
    const int lane = threadIdx.x & 31;
    const int prev = __shfl_up_sync(0xffffffffu, node, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || prev != node);
    WarpRuns r;
    r.start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
    r.tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
    return r;
}
template <class T, class Op>
__device__ __forceinline__ T run_scan(T v, const WarpRuns &r, Op op) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const T u = __shfl_up_sync(0xffffffffu, v, off);
        if (lane - off >= r.start) v = op(v, u);
    }
    return v;
}
struct AddOp {
    template <class T> __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
};
struct MinOp {
    template <class T> __device__ __forceinline__ T operator()(T a, T b) const { return min(a, b); }
};
struct MaxOp {
    template <class T> __device__ __forceinline__ T operator()(T a, T b) const { return max(a, b); }
};
struct FMaxOp {
    __device__ __forceinline__ float operator()(float a, float b) const { return fmaxf(a, b); }
};

// Pass 1: mass and mass-weighted position per node (FP64 accumulation).
__global__ void __launch_bounds__(kBlock)
accum_mass(int64_t n, const float4 *__restrict__ pos, const int32_t *__restrict__ pnode, Build b) {
    __shared__ double s[4][kBlock / 32];
    __shared__ int s_node;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t base = blockIdx.x * (int64_t)kBlock; base < n; base += (int64_t)gridDim.x * kBlock) {
        const int64_t p = base + threadIdx.x;
        const int node = p < n ? pnode[p] : -1;
        double w = 0, wx = 0, wy = 0, wz = 0;
        if (node >= 0) {
            const float4 v = pos[p];
            // ost.c:546-552: mass += ptlmass; mono += ptlmass * x (float mass, FP64 positions)
            w = v.w;
            wx = (double)v.w * (double)v.x;
            wy = (double)v.w * (double)v.y;
            wz = (double)v.w * (double)v.z;
        }
        if (threadIdx.x == 0) s_node = node;
        __syncthreads();
        const bool uniform = __syncthreads_and(node == s_node) && s_node >= 0;
        if (uniform) {
            for (int off = 16; off; off >>= 1) {
                w += __shfl_xor_sync(0xffffffffu, w, off);
                wx += __shfl_xor_sync(0xffffffffu, wx, off);
                wy += __shfl_xor_sync(0xffffffffu, wy, off);
                wz += __shfl_xor_sync(0xffffffffu, wz, off);
            }
            if (lane == 0) { s[0][warp] = w; s[1][warp] = wx; s[2][warp] = wy; s[3][warp] = wz; }
            __syncthreads();
            if (threadIdx.x < 4) {
                double a = 0;
                for (int i = 0; i < kBlock / 32; i++) a += s[threadIdx.x][i];
                double *dst = threadIdx.x == 0 ? b.m : threadIdx.x == 1 ? b.mx : threadIdx.x == 2 ? b.my : b.mz;
                atomicAdd(dst + s_node, a);
            }
        } else if (__all_sync(0xffffffffu, node == __shfl_sync(0xffffffffu, node, 0))) {
            // one node for the whole warp (settled warps add nothing)
            if (node >= 0) {
                for (int off = 16; off; off >>= 1) {
                    w += __shfl_xor_sync(0xffffffffu, w, off);
                    wx += __shfl_xor_sync(0xffffffffu, wx, off);
                    wy += __shfl_xor_sync(0xffffffffu, wy, off);
                    wz += __shfl_xor_sync(0xffffffffu, wz, off);
                }
                if (lane == 0) {
                    atomicAdd(b.m + node, w);
                    atomicAdd(b.mx + node, wx);
                    atomicAdd(b.my + node, wy);
                    atomicAdd(b.mz + node, wz);
                }
            }
        } else {
            // several nodes: segmented sums over the warp's runs, added by
            // each run's last lane (settled runs, node < 0, add nothing)
            const WarpRuns r = warp_runs(node);
            w = run_scan(w, r, AddOp());
            wx = run_scan(wx, r, AddOp());
            wy = run_scan(wy, r, AddOp());
            wz = run_scan(wz, r, AddOp());
            if (r.tail && node >= 0) {
                atomicAdd(b.m + node, w);
                atomicAdd(b.mx + node, wx);
                atomicAdd(b.my + node, wy);
                atomicAdd(b.mz + node, wz);
            }
        }
        __syncthreads();
    }
}

__global__ void finalize_com(int L, Build b) {
    FOR_LEVEL_NODES(node, L, b) {
        const double m = b.m[node];
        if (m > 0) {  // ost.c:553-555
            b.mx[node] /= m;
            b.my[node] /= m;
            b.mz[node] /= m;
        }
    }
}

// Pass 2: extents, max |x - com|^2, second moments and octant counts.
// The 13 reductions (max r2, six moment sums, min and max of the three
// coordinate keys) run over the block when all its particles share a node
// (one atomic per value and block: the top levels of large halos), over the
// warp when it does, else over the warp's runs.
__global__ void __launch_bounds__(kBlock)
accum_moments(int64_t n, const float4 *__restrict__ pos, const int32_t *__restrict__ pnode,
              uint8_t *__restrict__ pkey, int q5_asbuilt, Build b) {
    constexpr int kWarps = kBlock / 32;
    __shared__ float s_f[7][kWarps];
    __shared__ unsigned s_k[6][kWarps];
    __shared__ int s_oct[8];
    __shared__ int s_node;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < 8) s_oct[threadIdx.x] = 0;
    for (int64_t base = blockIdx.x * (int64_t)kBlock; base < n; base += (int64_t)gridDim.x * kBlock) {
        const int64_t p = base + threadIdx.x;
        const int node = p < n ? pnode[p] : -1;
        float v[7] = {0, 0, 0, 0, 0, 0, 0};  // max |x - com|^2, then q0..q5
        unsigned bx[6] = {~0u, ~0u, ~0u, 0u, 0u, 0u};
        int key = 0;
        if (node >= 0) {
            const float4 P = pos[p];
            const double cx = b.mx[node], cy = b.my[node], cz = b.mz[node];
            // ost.c:561-571: float offsets, float moments
            const float tx = (float)((double)P.x - cx);
            const float ty = (float)((double)P.y - cy);
            const float tz = (float)((double)P.z - cz);
            const float m = P.w;
            v[0] = tx * tx + ty * ty + tz * tz;
            v[1] = m * tx * tx;
            v[2] = m * ty * ty;
            v[3] = m * tz * tz;
            v[4] = m * tx * ty;
            v[5] = m * tx * tz;
            v[6] = q5_asbuilt ? m * ty * tx : m * ty * tz;
            bx[0] = bx[3] = fkey(P.x);
            bx[1] = bx[4] = fkey(P.y);
            bx[2] = bx[5] = fkey(P.z);
            // ost.c:589-592: SubCellDicision(x, monox) = x > monox
            key = ((double)P.x > cx ? 1 : 0) | ((double)P.y > cy ? 2 : 0) | ((double)P.z > cz ? 4 : 0);
            pkey[p] = (uint8_t)key;
        }
        if (threadIdx.x == 0) s_node = node;
        __syncthreads();
        const bool block_uniform = __syncthreads_and(node == s_node) && s_node >= 0;
        const bool warp_uniform = __all_sync(0xffffffffu, node == __shfl_sync(0xffffffffu, node, 0));
        if (block_uniform || warp_uniform) {  // butterfly over the warp (none for a settled warp)
            for (int off = 16; node >= 0 && off; off >>= 1) {
                v[0] = fmaxf(v[0], __shfl_xor_sync(0xffffffffu, v[0], off));
                for (int i = 1; i < 7; i++) v[i] += __shfl_xor_sync(0xffffffffu, v[i], off);
                for (int i = 0; i < 3; i++) {
                    bx[i] = min(bx[i], __shfl_xor_sync(0xffffffffu, bx[i], off));
                    bx[3 + i] = max(bx[3 + i], __shfl_xor_sync(0xffffffffu, bx[3 + i], off));
                }
            }
        } else {  // several nodes: segmented over the warp's runs
            const WarpRuns r = warp_runs(node);
            v[0] = run_scan(v[0], r, FMaxOp());
            for (int i = 1; i < 7; i++) v[i] = run_scan(v[i], r, AddOp());
            for (int i = 0; i < 3; i++) {
                bx[i] = run_scan(bx[i], r, MinOp());
                bx[3 + i] = run_scan(bx[3 + i], r, MaxOp());
            }
            if (r.tail && node >= 0) {
                atomicMax(b.r2 + node, __float_as_uint(v[0]));  // non-negative floats
                for (int i = 0; i < 6; i++) atomicAdd(b.q + 6 * (int64_t)node + i, v[1 + i]);
                for (int i = 0; i < 3; i++) {
                    atomicMin(b.box + 6 * (int64_t)node + i, bx[i]);
                    atomicMax(b.box + 6 * (int64_t)node + 3 + i, bx[3 + i]);
                }
            }
        }
        if (block_uniform) {  // then over the block: one atomic per value
            if (lane == 0) {
                for (int i = 0; i < 7; i++) s_f[i][warp] = v[i];
                for (int i = 0; i < 6; i++) s_k[i][warp] = bx[i];
            }
            const unsigned g2 = __match_any_sync(0xffffffffu, key);
            if (lane == __ffs(g2) - 1) atomicAdd(s_oct + key, __popc(g2));
            __syncthreads();
            if (threadIdx.x < 7) {
                const int i = threadIdx.x;
                float a = s_f[i][0];
                for (int w2 = 1; w2 < kWarps; w2++) a = i == 0 ? fmaxf(a, s_f[i][w2]) : a + s_f[i][w2];
                if (i == 0) atomicMax(b.r2 + s_node, __float_as_uint(a));
                else atomicAdd(b.q + 6 * (int64_t)s_node + (i - 1), a);
            } else if (threadIdx.x < 13) {
                const int i = threadIdx.x - 7;
                unsigned a = s_k[i][0];
                for (int w2 = 1; w2 < kWarps; w2++) a = i < 3 ? min(a, s_k[i][w2]) : max(a, s_k[i][w2]);
                if (i < 3) atomicMin(b.box + 6 * (int64_t)s_node + i, a);
                else atomicMax(b.box + 6 * (int64_t)s_node + i, a);
            } else if (threadIdx.x >= 32 && threadIdx.x < 40) {
                const int c = threadIdx.x - 32;
                if (s_oct[c]) atomicAdd(b.oct + 8 * (int64_t)s_node + c, s_oct[c]);
                s_oct[c] = 0;
            }
        } else {
            if (warp_uniform && node >= 0 && lane == 0) {
                atomicMax(b.r2 + node, __float_as_uint(v[0]));
                for (int i = 0; i < 6; i++) atomicAdd(b.q + 6 * (int64_t)node + i, v[1 + i]);
                for (int i = 0; i < 3; i++) {
                    atomicMin(b.box + 6 * (int64_t)node + i, bx[i]);
                    atomicMax(b.box + 6 * (int64_t)node + 3 + i, bx[3 + i]);
                }
            }
            // octant counts: lanes sharing (node, key)
            const unsigned g2 = __match_any_sync(0xffffffffu, node * 8 + key);
            if (node >= 0 && lane == __ffs(g2) - 1) atomicAdd(b.oct + 8 * (int64_t)node + key, __popc(g2));
        }
        __syncthreads();  // s_node, s_f, s_k and s_oct are reused by the next iteration
    }
}

// Decides children, allocates them, and lays out [loose | children] ranges.
// last: the final level of a fixed-depth build, whose nodes keep all their
// particles loose (children there would never be processed); a node that
// would have split flags the build (counter[1]) instead.
__global__ void split_nodes(int L, int32_t ncap, int last, Build b) {
    FOR_LEVEL_NODES(node, L, b) {
    const float r2 = __uint_as_float(b.r2[node]);
    const double nodesize = sqrt((double)r2);           // ost.c:574
    const bool divide = nodesize > 0.5 * kMinWidth;     // divideThisNode, tree.h:36
    int cnt[8], nch = 0;
    for (int c = 0; c < 8; c++) {
        cnt[c] = b.oct[8 * (int64_t)node + c];
        if (divide && cnt[c] >= kMinCell) nch++;
    }
    if (last && nch > 0) {
        atomicOr(b.counter + 1, 2);
        nch = 0;
    }
    int first = -1;
    if (nch > 0) {
        first = atomicAdd(b.counter, nch);
        if (first + nch > ncap) {  // out of node capacity: keep all particles loose
            atomicOr(b.counter + 1, 1);
            nch = 0;
            first = -1;
        }
    }
    int off = b.start[node];
    for (int c = 0; c < 8; c++) {
        const bool child = nch > 0 && divide && cnt[c] >= kMinCell;
        if (!child) {
            b.cur[8 * (int64_t)node + c] = off;
            b.ochild[8 * (int64_t)node + c] = -1;
            off += cnt[c];
        }
    }
    b.lstart[node] = b.start[node];
    b.lcount[node] = off - b.start[node];
    int k = 0;
    for (int c = 0; c < 8; c++) {
        const bool child = nch > 0 && divide && cnt[c] >= kMinCell;
        if (child) {
            const int id = first + k++;
            b.cur[8 * (int64_t)node + c] = off;
            b.ochild[8 * (int64_t)node + c] = id;
            b.start[id] = off;
            b.count[id] = cnt[c];
            b.halo[id] = b.halo[node];
            b.par[id] = node;
            off += cnt[c];
        }
    }
    b.first[node] = first;
    b.nchild[node] = nch;
    }
    // the last block to finish writes the next level's end: the nodes this
    // level allocated (its children are numbered [lev[L+1], lev[L+2]))
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(b.counter + 2, 1) == (int)gridDim.x - 1) {
            b.lev[L + 2] = min(atomicAdd(b.counter, 0), ncap);
            b.counter[2] = 0;  // for the next level's launch
        }
    }
}

// Moves the active particles into [loose | child 0 | child 1 | ...] order.
// A particle that stays loose here has its final tree-order slot: it is
// written once into the final arrays (fpos, fperm) and never copied again;
// its slot, like every earlier-settled one, carries node -1 into the next
// level.
__global__ void scatter_particles(int64_t n, const float4 *__restrict__ pos_in,
                                  const int32_t *__restrict__ perm_in,
                                  const int32_t *__restrict__ pnode_in,
                                  const uint8_t *__restrict__ pkey, float4 *__restrict__ pos_out,
                                  int32_t *__restrict__ perm_out, int32_t *__restrict__ pnode_out,
                                  float4 *__restrict__ fpos, int32_t *__restrict__ fperm, Build b) {
    const int lane = threadIdx.x & 31;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p - lane < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int node = p < n ? pnode_in[p] : -2;
        const int key = node >= 0 ? pkey[p] : 0;
        const unsigned g = __match_any_sync(0xffffffffu, node * 8 + key);
        if (p >= n) continue;
        if (node < 0) {  // settled at an earlier level: already in the final arrays
            pnode_out[p] = -1;
            continue;
        }
        const int leader = __ffs(g) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(b.cur + 8 * (int64_t)node + key, __popc(g));
        base = __shfl_sync(g, base, leader);
        const int dest = base + __popc(g & ((1u << lane) - 1));
        const int child = b.ochild[8 * (int64_t)node + key];
        if (child >= 0) {
            pos_out[dest] = pos_in[p];
            perm_out[dest] = perm_in[p];
        } else {
            fpos[dest] = pos_in[p];
            fperm[dest] = perm_in[p];
        }
        pnode_out[dest] = child;
    }
}

// subtree sizes, deepest level first
__global__ void subtree_sizes(int L, Build b) {
    FOR_LEVEL_NODES(node, L, b) {
        int s = 1;
        const int f = b.first[node];
        for (int c = 0; c < b.nchild[node]; c++) s += b.sub[f + c];
        b.sub[node] = s;
    }
}

// Preorder numbers of the roots: consecutive blocks in halo order (an
// exclusive scan of the roots' subtree sizes, one block).
__global__ void __launch_bounds__(1024) root_preorder(int32_t nhalo, Build b) {
    __shared__ int32_t part[1024];
    const int t = threadIdx.x;
    const int per = (nhalo + 1023) / 1024;
    const int h0 = min(nhalo, t * per), h1 = min(nhalo, h0 + per);
    int32_t sum = 0;
    for (int h = h0; h < h1; h++) sum += b.sub[h];
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {  // inclusive Hillis-Steele scan
        const int32_t v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int32_t acc = part[t] - sum;
    for (int h = h0; h < h1; h++) {
        b.pre[h] = acc;
        acc += b.sub[h];
    }
}

// Flags a fixed-depth build that the batch outgrew: a node of the last level
// that would have split, or the node capacity exceeded.  The tree built is
// consistent either way (those particles stay loose).
__global__ void check_build(Build b, int *err) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && b.counter[1]) atomicOr(err, GF_ERRBIT_PLAN);
}

// preorder numbers, shallowest level first (roots set beforehand)
__global__ void preorder(int L, Build b) {
    FOR_LEVEL_NODES(node, L, b) {
        int p = b.pre[node] + 1;
        const int f = b.first[node];
        for (int c = 0; c < b.nchild[node]; c++) {
            b.pre[f + c] = p;
            p += b.sub[f + c];
        }
    }
}

__global__ void emit_nodes(int nlev, float theta2, Build b, KnnNode *__restrict__ knn,
                           BhNode *__restrict__ bh, int32_t *__restrict__ owner) {
    for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < b.lev[nlev]; node += gridDim.x * blockDim.x) {
    const int i = b.pre[node];
    KnnNode k;
    for (int a = 0; a < 3; a++) {
        k.lo[a] = fkey_inv(b.box[6 * (int64_t)node + a]);
        k.hi[a] = fkey_inv(b.box[6 * (int64_t)node + 3 + a]);
    }
    k.skip = i + b.sub[node];
    k.lstart = b.lstart[node];
    k.lcount = b.lcount[node];
    k.count = b.count[node];
    k.parent = b.par[node] >= 0 ? b.pre[b.par[node]] : -1;
    k.pad = 0;
    for (int j = 0; j < k.lcount; j++) owner[k.lstart + j] = i;
    knn[i] = k;
    BhNode h;
    h.com[0] = b.mx[node];
    h.com[1] = b.my[node];
    h.com[2] = b.mz[node];
    // ost.c:573,80: dist2 = (double)distmax (a float); ratio = dist2/theta2
    h.open_r2 = (double)__uint_as_float(b.r2[node]) / (double)theta2;
    h.mass = (float)b.m[node];
    float q[6];
    for (int a = 0; a < 6; a++) q[a] = b.q[6 * (int64_t)node + a];
    for (int a = 0; a < 6; a++) h.q[a] = q[a];
    h.trq = q[0] + q[1] + q[2];
    h.skip = k.skip;
    h.lstart = k.lstart;
    h.lcount = k.lcount;
    h.count = k.count;
    bh[i] = h;
    }
}

__global__ void emit_roots(int32_t nhalo, Build b, int32_t *__restrict__ root,
                           int32_t *__restrict__ rend) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nhalo) return;
    root[h] = b.pre[h];
    rend[h] = b.pre[h] + b.sub[h];
}

__global__ void particle_halo(int64_t n, const int64_t *__restrict__ pstart, int32_t nhalo,
                              int32_t *__restrict__ phalo) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = nhalo;
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (pstart[mid] <= p) lo = mid; else hi = mid;
        }
        phalo[p] = lo;
    }
}

int grid_n(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + kBlock - 1) / kBlock, sm_count() * 8));
}
int grid_exact(int64_t n, int block) { return (int)std::max<int64_t>(1, (n + block - 1) / block); }

template <class T>
T *carve(char *&p, size_t count) {
    T *r = reinterpret_cast<T *>(p);
    p += (count * sizeof(T) + 255) & ~size_t(255);
    return r;
}

}  // namespace

int build_tree(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
               const float4 *pos_in, float theta2, int q5_asbuilt, TreeView *out,
               const TreeShape *fixed, TreeShape *shape) {
    if (n > 0x7fffffffLL) {
        set_status(GF_ENOTIMPL, "tree build over more than 2^31 particles in one batch");
        return GF_ENOTIMPL;
    }
    if (fixed && (fixed->levels < 1 || fixed->levels > kMaxLevels || fixed->ncap < nhalo)) {
        set_status(GF_EINVAL, "fixed tree shape: %d levels, %lld nodes", fixed ? fixed->levels : 0,
                   fixed ? (long long)fixed->ncap : 0LL);
        return GF_EINVAL;
    }
    int64_t ncap = fixed ? fixed->ncap : n / 2 + 2LL * nhalo + 1024;
    for (int attempt = 0; attempt < (fixed ? 1 : 4); attempt++, ncap *= 2) {
        // ---- particle buffers: pos x2, perm x2, pnode x2, key
        auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
        const size_t pbytes = 3 * al(n * sizeof(float4)) + 5 * al(n * sizeof(int32_t)) + al(n);
        GF_TRY(ctx->tree[0].reserve(pbytes + 256));
        char *pp = ctx->tree[0].as<char>();
        float4 *pos[2] = {carve<float4>(pp, n), carve<float4>(pp, n)};
        int32_t *perm[2] = {carve<int32_t>(pp, n), carve<int32_t>(pp, n)};
        int32_t *pnode[2] = {carve<int32_t>(pp, n), carve<int32_t>(pp, n)};
        uint8_t *pkey = carve<uint8_t>(pp, n);
        float4 *fpos = carve<float4>(pp, n);    // final tree order, written as particles settle
        int32_t *fperm = carve<int32_t>(pp, n);
        // ---- node buffers (BFS numbering): exactly the carves below
        const size_t nc = (size_t)ncap;
        const size_t nbytes = 3 * al(nc * 4) + 4 * al(nc * 8) + al(nc * 4) + al(nc * 24) +
                              al(nc * 24) + 3 * al(nc * 32) + 7 * al(nc * 4) + al(64) +
                              al((kMaxLevels + 2) * sizeof(int32_t));
        GF_TRY(ctx->tree[1].reserve(nbytes + 256));
        char *np_ = ctx->tree[1].as<char>();
        Build b;
        char *zero_begin = np_;
        b.start = carve<int32_t>(np_, nc);
        b.count = carve<int32_t>(np_, nc);
        b.halo = carve<int32_t>(np_, nc);
        b.m = carve<double>(np_, nc);
        b.mx = carve<double>(np_, nc);
        b.my = carve<double>(np_, nc);
        b.mz = carve<double>(np_, nc);
        b.r2 = carve<unsigned>(np_, nc);
        b.q = carve<float>(np_, nc * 6);
        char *zero_end = np_;
        b.box = carve<unsigned>(np_, nc * 6);
        b.oct = carve<int32_t>(np_, nc * 8);
        char *zero2_end = np_;
        b.cur = carve<int32_t>(np_, nc * 8);
        b.ochild = carve<int32_t>(np_, nc * 8);
        b.first = carve<int32_t>(np_, nc);
        b.nchild = carve<int32_t>(np_, nc);
        b.lstart = carve<int32_t>(np_, nc);
        b.lcount = carve<int32_t>(np_, nc);
        b.sub = carve<int32_t>(np_, nc);
        b.pre = carve<int32_t>(np_, nc);
        b.par = carve<int32_t>(np_, nc);
        b.counter = carve<int32_t>(np_, 16);
        b.lev = carve<int32_t>(np_, kMaxLevels + 2);
        cudaStream_t s = ctx->stream;
        GF_CUDA_TRY(cudaMemsetAsync(zero_begin, 0, zero_end - zero_begin, s));
        // box: minima start at all-ones, maxima at zero (per node: 3 min then 3 max)
        GF_CUDA_TRY(cudaMemsetAsync(b.box, 0, nc * 6 * 4, s));
        GF_CUDA_TRY(cudaMemsetAsync(b.oct, 0, zero2_end - (char *)b.oct, s));
        {
            // min slots set to 0xff..: strided pattern, do it with a 2D memset
            GF_CUDA_TRY(cudaMemset2DAsync(b.box, 6 * 4, 0xff, 3 * 4, nc, s));
        }
        init_build<<<1, 32, 0, s>>>(nhalo, b);
        GF_LAUNCH_CHECK();
        if (nhalo > 0) {
            init_roots<<<grid_exact(nhalo, 256), 256, 0, s>>>(nhalo, pstart_dev, b);
            GF_LAUNCH_CHECK();
        }
        init_particles<<<grid_n(n), kBlock, 0, s>>>(n, pstart_dev, nhalo, pos_in, pos[0], perm[0],
                                                    pnode[0]);
        GF_LAUNCH_CHECK();
        // Level by level.  Eagerly, the node count is read back after each
        // level and the build stops at the first level that allocates no
        // children; with a fixed shape it runs fixed->levels levels without
        // a host round trip (the levels past the tree's depth are empty: their
        // particle passes copy settled particles through) and check_build
        // flags a tree that needed more levels or nodes.
        const int fixed_grid = sm_count() * 4;
        std::vector<int32_t> levels = {0, nhalo};  // eager only: the host copy of b.lev
        int cur = 0;
        int32_t hc[2] = {nhalo, 0};
        int nlev = 0;
        for (int L = 0; fixed ? L < fixed->levels : levels[L] < levels[L + 1]; L++) {
            const int gl = fixed ? fixed_grid : grid_exact(levels[L + 1] - levels[L], 256);
            accum_mass<<<grid_n(n), kBlock, 0, s>>>(n, pos[cur], pnode[cur], b);
            GF_LAUNCH_CHECK();
            finalize_com<<<gl, 256, 0, s>>>(L, b);
            GF_LAUNCH_CHECK();
            accum_moments<<<grid_n(n), kBlock, 0, s>>>(n, pos[cur], pnode[cur], pkey, q5_asbuilt, b);
            GF_LAUNCH_CHECK();
            split_nodes<<<gl, 256, 0, s>>>(L, (int32_t)ncap, fixed && L == fixed->levels - 1, b);
            GF_LAUNCH_CHECK();
            scatter_particles<<<grid_n(n), kBlock, 0, s>>>(n, pos[cur], perm[cur], pnode[cur], pkey,
                                                           pos[cur ^ 1], perm[cur ^ 1],
                                                           pnode[cur ^ 1], fpos, fperm, b);
            GF_LAUNCH_CHECK();
            cur ^= 1;
            nlev = L + 1;
            if (fixed) continue;
            GF_CUDA_TRY(cudaMemcpyAsync(hc, b.counter, sizeof(hc), cudaMemcpyDeviceToHost, s));
            GF_CUDA_TRY(cudaStreamSynchronize(s));
            if (hc[1]) break;
            levels.push_back(std::min<int32_t>(hc[0], (int32_t)ncap));
            if (levels.size() > (size_t)kMaxLevels) {
                set_status(GF_EINVAL, "octree deeper than %d levels", kMaxLevels);
                return GF_EINVAL;
            }
        }
        if (hc[1]) continue;  // node capacity exceeded: retry with more nodes
        if (fixed) {
            check_build<<<1, 32, 0, s>>>(b, ctx->d_err);
            GF_LAUNCH_CHECK();
        }
        const int32_t nnode = fixed ? -1 : levels.back();
        for (int L = nlev - 1; L >= 0; L--) {
            subtree_sizes<<<fixed ? fixed_grid : grid_exact(levels[L + 1] - levels[L], 256), 256, 0, s>>>(L, b);
            GF_LAUNCH_CHECK();
        }
        if (nhalo > 0) {
            root_preorder<<<1, 1024, 0, s>>>(nhalo, b);
            GF_LAUNCH_CHECK();
        }
        for (int L = 0; L < nlev; L++) {
            preorder<<<fixed ? fixed_grid : grid_exact(levels[L + 1] - levels[L], 256), 256, 0, s>>>(L, b);
            GF_LAUNCH_CHECK();
        }
        if (shape) {
            shape->levels = nlev;
            shape->ncap = ncap;
            shape->nnode = nnode;
        }
        // ---- output buffers
        const int64_t nout = fixed ? ncap : std::max(nnode, 1);  // node slots written
        const size_t obytes = al((size_t)nout * sizeof(KnnNode)) + al((size_t)nout * sizeof(BhNode)) +
                              2 * al((size_t)std::max(nhalo, 1) * 4) +
                              2 * al((size_t)std::max<int64_t>(n, 1) * 4);
        GF_TRY(ctx->tree[2].reserve(obytes + 256));
        char *op = ctx->tree[2].as<char>();
        KnnNode *knn = carve<KnnNode>(op, (size_t)nout);
        BhNode *bh = carve<BhNode>(op, (size_t)nout);
        int32_t *root = carve<int32_t>(op, std::max(nhalo, 1));
        int32_t *rend = carve<int32_t>(op, std::max(nhalo, 1));
        int32_t *phalo = carve<int32_t>(op, std::max<int64_t>(n, 1));
        int32_t *owner = carve<int32_t>(op, std::max<int64_t>(n, 1));
        if (fixed || nnode > 0) {
            emit_nodes<<<fixed ? fixed_grid : grid_exact(nnode, 256), 256, 0, s>>>(nlev, theta2, b, knn, bh,
                                                                                  owner);
            GF_LAUNCH_CHECK();
            emit_roots<<<grid_exact(nhalo, 256), 256, 0, s>>>(nhalo, b, root, rend);
            GF_LAUNCH_CHECK();
        }
        particle_halo<<<grid_n(n), kBlock, 0, s>>>(n, pstart_dev, nhalo, phalo);
        GF_LAUNCH_CHECK();
        out->nhalo = nhalo;
        out->nnode = nnode;
        out->n = n;
        out->pos = fpos;
        out->perm = fperm;
        out->root = root;
        out->rend = rend;
        out->knn = knn;
        out->bh = bh;
        out->phalo = phalo;
        out->owner = owner;
        return GF_OK;
    }
    set_status(GF_ENOMEM, "octree node capacity exhausted");
    return GF_ENOMEM;
}

int export_tree(gf_ctx *ctx, const TreeView &t, void *knn_host, void *bh_host, float4 *pos_host,
                int32_t *perm_host, int32_t *root_host, int32_t *rend_host) {
    cudaStream_t s = ctx->stream;
    if (knn_host)
        GF_CUDA_TRY(cudaMemcpyAsync(knn_host, t.knn, sizeof(KnnNode) * t.nnode, cudaMemcpyDeviceToHost, s));
    if (bh_host)
        GF_CUDA_TRY(cudaMemcpyAsync(bh_host, t.bh, sizeof(BhNode) * t.nnode, cudaMemcpyDeviceToHost, s));
    if (pos_host)
        GF_CUDA_TRY(cudaMemcpyAsync(pos_host, t.pos, sizeof(float4) * t.n, cudaMemcpyDeviceToHost, s));
    if (perm_host)
        GF_CUDA_TRY(cudaMemcpyAsync(perm_host, t.perm, sizeof(int32_t) * t.n, cudaMemcpyDeviceToHost, s));
    if (root_host)
        GF_CUDA_TRY(cudaMemcpyAsync(root_host, t.root, sizeof(int32_t) * t.nhalo, cudaMemcpyDeviceToHost, s));
    if (rend_host)
        GF_CUDA_TRY(cudaMemcpyAsync(rend_host, t.rend, sizeof(int32_t) * t.nhalo, cudaMemcpyDeviceToHost, s));
    GF_CUDA_TRY(cudaStreamSynchronize(s));
    return GF_OK;
}

}  // namespace gf
