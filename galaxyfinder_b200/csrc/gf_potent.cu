// Barnes-Hut potential on the centre-of-mass octree.
//
// Reference: NewGalFinder/ost.c:226-251 (treeplumpotential) with the cell
// term CELLPLUMPOTENT (:144-176) and the particle term PARTICLEPLUMPOTENT
// (:178-193), opening test treeopen (:72-83): a node is opened when
// |p - com|^2 < dist2/theta2.  The cell term is
//     -M/r + trQ/(2 r^3) - 3 (d.Q.d)/(2 r^5)
// which the reference reads from linearly interpolated tables of -1/x,
// 1/(2x^3) and -3/(2x^5) (force_spline.mod3.c:81-138); here it is evaluated
// directly.  The drivers Self_Halo_Potent / External_Halo_Potent
// (subhaloden.mod6.c:1477-1621) use a direct sum below 100 members (self) or
// 1000 targets (external), then scale by potentfact and add the NFW
// background term of the halo mass (GetBGpotent, :1093-1101).
//
// One thread per target.  The 32 targets of a warp are neighbours in tree
// order and walk the preorder node array in lockstep: every iteration the warp
// takes the smallest next-node index among its lanes, and the lanes waiting
// at that node apply their own opening decision (open: sum the node's loose
// particles and continue at i + 1; accept: add the cell term and continue at
// skip[i]).  Opening decisions use the same FP64 |p - com|^2 as the
// reference, so they are identical to an FP64 walk of the same tree; the
// terms are FP32 evaluated from exact FP64 position differences and summed
// with Kahan compensation.
#include <float.h>
#include <limits.h>
#include <math.h>

#include <algorithm>
#include <type_traits>

#include "gf_tree.cuh"

namespace gf {

namespace {

struct Kahan {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float v) {
        const float y = v - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ float value() const { return s + (-c); }
};

// The sum of a target's FP32 terms: GF_BH_ACC=1 adds them in FP64 (two
// instructions per term, one dependent add), 0 with FP32 Kahan compensation
// (four dependent adds); both round once at the end.
struct Fp64Acc {
    double s = 0.0;
    __device__ __forceinline__ void add(float v) { s += (double)v; }
    __device__ __forceinline__ float value() const { return (float)s; }
};
using BhAcc = std::conditional<GF_BH_ACC == 1, Fp64Acc, Kahan>::type;

// GetBGpotent, subhaloden.mod6.c:1059-1101
__device__ double bg_potent_dev(double mvir, const PotentialParams &pp) {
    const double G = 6.672E-8, RHOC = 2.7755E11;
    const double redshift = (double)(pp.amax / pp.a) - 1.0;
    const double c = 14.5 * pow(mvir / 1.3E13, -0.15) / (1.0 + redshift);
    const double gc = 1. / (log(1.0 + c) - c / (1.0 + c));
    const double om = pp.omep;
    const double vv = 18.0 * M_PI * M_PI + 82.0 * (om - 1.0) - 39.0 * pow(om - 1.0, 2.0);
    const double rvir = pow(3. * mvir / (4.0 * M_PI * vv * RHOC), 0.3333333333333);
    const double vc2 = G * mvir / rvir * pp.potentfact;
    return vc2 * (1 - gc * log(1 + c));
}

// ---- leaf tiles staged by the bulk-copy (TMA) engine, GF_BH_TMA=1
// When lanes open a node whose loose particles fit a slot (at most
// kLeafSlotP float4), one lane has the tensor-memory-access unit copy them
// (cp.async.bulk, global -> this CTA's shared memory, completion counted on
// an mbarrier; no multicast) into the next slot of a per-warp ring, and the
// warp walks on; the opened leaf is summed from shared memory later, when the
// ring is full or the walk ends.  Every wait is bounded: a copy that does not
// complete in time sets GF_ERRBIT_WAIT and the warp falls back to global
// loads for the rest of the launch.
constexpr int kLeafSlots = 4;   // ring slots per warp
constexpr int kLeafSlotP = 32;  // float4 (particles) per slot
constexpr int kWaitTries = 1 << 20;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// bytes: a multiple of 16; src and dst 16-byte aligned
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    uint64_t g;
    asm("cvta.to.global.u64 %0, %1;" : "=l"(g) : "l"(src));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(g), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// the generic-proxy reads of a slot precede the async-proxy write that reuses it
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// COUNT: interaction counters (bench and tests); off in the stage's walk.
template <bool COUNT>
__global__ void __launch_bounds__(GF_BH_BLOCK, GF_BH_MINB)
bh_kernel(int64_t ntarget, const float4 *__restrict__ tpos, const int32_t *__restrict__ thalo,
          const int32_t *__restrict__ tout, const float4 *__restrict__ spos,
          const int32_t *__restrict__ root, const int32_t *__restrict__ rend,
          const BhNode *__restrict__ nodes, const int32_t *__restrict__ direct,
          const double *__restrict__ bg, PotentialParams pp, float *__restrict__ out,
          float *__restrict__ raw, unsigned long long *__restrict__ counters,
          unsigned long long *__restrict__ work, int *__restrict__ err) {
    const int lane = threadIdx.x & 31;
#if GF_BH_TMA
    __shared__ __align__(16) float4 leaf_ring[GF_BH_BLOCK / 32][kLeafSlots][kLeafSlotP];
    __shared__ __align__(8) uint64_t leaf_bar[GF_BH_BLOCK / 32][kLeafSlots];
    float4(*ring)[kLeafSlotP] = leaf_ring[threadIdx.x >> 5];
    uint64_t *bars = leaf_bar[threadIdx.x >> 5];
    if (lane < kLeafSlots) mbar_init(bars + lane);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncwarp();
    uint32_t phases = 0;        // parity each slot's barrier completes next (warp-uniform)
    int head = 0, pending = 0;  // oldest staged slot, staged slots (warp-uniform)
    unsigned qmask = 0;         // in lane s < kLeafSlots: the lanes that opened slot s's leaf
    int qcnt = 0;               // in lane s: the particles in slot s
    bool tma_ok = true;         // cleared by a wait that ran out
#else
    (void)err;
#endif
    const int64_t warp0 = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32;
    const int64_t wstride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long npp = 0, npc = 0;
    // the warp's next 32 targets: from the work counter, or grid-stride
    auto next = [&](int64_t stride_base) -> int64_t {
        if (!GF_BH_DYN || !work) return stride_base;
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(work, 32ull);
        return (int64_t)__shfl_sync(0xffffffffu, b, 0);
    };
    for (int64_t base = next(warp0); base < ntarget; base = next(base + wstride)) {
        const int64_t t = base + lane;
        const bool valid = t < ntarget;
        int h = 0, my = INT_MAX, my_end = 0, always_open = 0;
        float4 P = make_float4(0.f, 0.f, 0.f, 0.f);
        if (valid) {
            h = thalo[t];
            my = root[h];
            my_end = rend[h];
            if (my >= my_end) my = INT_MAX;
            always_open = direct ? direct[h] : 0;
            P = tpos[t];
        }
        const double px = P.x, py = P.y, pz = P.z;
        BhAcc acc;
        // ost.c:186-191: float offsets of the two positions.  For float
        // inputs the FP32 difference is the correctly rounded exact
        // difference, i.e. the same bits as rounding the FP64 difference.
        auto particle_term = [&](const float4 &S) {
            const float fx = P.x - S.x;
            const float fy = P.y - S.y;
            const float fz = P.z - S.z;
            const float r2 = fx * fx + fy * fy + fz * fz;
            if (r2 > 0.f) acc.add(-S.w * rsqrtf(r2));
        };
#if GF_BH_TMA
        // sums the oldest staged leaf once its copy has landed
        auto consume = [&]() {
            const int slot = head;
            const uint32_t par = (phases >> slot) & 1u;
            bool ok = false;
            for (int it = 0; it < kWaitTries && !ok; it++) ok = mbar_try_wait(bars + slot, par);
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) atomicOr(err, GF_ERRBIT_WAIT);
                // the copy may still land in this slot: wait for it once
                // more, then stage no further leaves in this launch
                ok = false;
                for (int it = 0; it < kWaitTries && !ok; it++) ok = mbar_try_wait(bars + slot, par);
                tma_ok = false;
            }
            phases ^= 1u << slot;
            const unsigned m = __shfl_sync(0xffffffffu, qmask, slot);
            const int c = __shfl_sync(0xffffffffu, qcnt, slot);
            if ((m >> lane) & 1u)
                for (int j = 0; j < c; j++) particle_term(ring[slot][j]);
            __syncwarp();  // every lane's reads of the slot precede its next copy
            head = (head + 1) % kLeafSlots;
            pending--;
        };
#endif
        while (true) {
            const int i = (int)__reduce_min_sync(0xffffffffu, (unsigned)my);
            if (i == INT_MAX) break;
            bool stage = false;  // this lane opened a leaf that is staged
            int stage_l0 = 0, stage_n = 0;
            if (my == i) {
                // the node in 16-byte words: (com x, com y), (com z, open_r2),
                // (mass, trq, qxx, qyy), (qzz, qxy, qxz, qyz), (skip, lstart, lcount, count)
                // All five are loaded before the opening test (one broadcast
                // line for the lanes at the node), so the moment loads of an
                // accepted cell overlap the FP64 test instead of following it.
                const double2 *nd2 = reinterpret_cast<const double2 *>(nodes + i);
                const float4 *nf = reinterpret_cast<const float4 *>(nodes + i);
                const double2 c01 = __ldg(nd2), c2r = __ldg(nd2 + 1);
                const float4 mq = __ldg(nf + 2), q = __ldg(nf + 3);  // (mass, trq, q0, q1), (q2..q5)
                const int4 links = __ldg(reinterpret_cast<const int4 *>(nodes + i) + 4);
                const double dx = px - c01.x;
                const double dy = py - c01.y;
                const double dz = pz - c2r.x;
                // separately rounded, as the reference's treeopen (ost.c:79)
                const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                            __dmul_rn(dz, dz));
                if (always_open || d2 < c2r.y) {
#if GF_BH_TMA
                    if (tma_ok && links.z > 0 && links.z <= kLeafSlotP) {
                        stage = true;
                        stage_l0 = links.y;
                        stage_n = links.z;
                    } else
#endif
                    {
                        const int l1 = links.y + links.z;
                        int j = links.y;
#if GF_BH_LEAF4
                        // four loads in flight before the terms, which are
                        // still added in particle order
                        for (; j + 4 <= l1; j += 4) {
                            const float4 s0 = __ldg(spos + j), s1 = __ldg(spos + j + 1);
                            const float4 s2 = __ldg(spos + j + 2), s3 = __ldg(spos + j + 3);
                            particle_term(s0);
                            particle_term(s1);
                            particle_term(s2);
                            particle_term(s3);
                        }
#endif
                        for (; j < l1; j++) particle_term(spos[j]);
                    }
                    if (COUNT) npp += links.z;
                    my = i + 1;
                } else {
                    const float fx = (float)dx, fy = (float)dy, fz = (float)dz;
                    const float r2 = fx * fx + fy * fy + fz * fz;
                    const float inv = rsqrtf(r2);
                    const float inv2 = inv * inv;
                    const float inv3 = inv * inv2;
                    const float qxy = mq.z * fx * fx + mq.w * fy * fy + q.x * fz * fz +
                                      2.f * (q.y * fx * fy + q.z * fx * fz + q.w * fy * fz);
                    acc.add(-mq.x * inv + 0.5f * mq.y * inv3 - 1.5f * qxy * inv3 * inv2);
                    if (COUNT) npc++;
                    my = links.x;
                }
                if (my >= my_end) my = INT_MAX;
            }
#if GF_BH_TMA
            const unsigned om = __ballot_sync(0xffffffffu, stage);
            if (om) {  // the lanes at node i that opened it share its loose particles
                const int src = __ffs(om) - 1;
                const int l0 = __shfl_sync(0xffffffffu, stage_l0, src);
                const int nl = __shfl_sync(0xffffffffu, stage_n, src);
                if (pending == kLeafSlots) consume();
                const int slot = (head + pending) % kLeafSlots;
                if (lane == 0) {
                    fence_proxy_async_smem();
                    mbar_expect_tx(bars + slot, (uint32_t)nl * 16u);
                    bulk_copy_g2s(ring[slot], spos + l0, (uint32_t)nl * 16u, bars + slot);
                }
                if (lane == slot) {
                    qmask = om;
                    qcnt = nl;
                }
                pending++;
            }
#endif
        }
#if GF_BH_TMA
        while (pending) consume();  // the walk's staged leaves, before the outputs
#endif
        if (valid) {
            const int64_t o = tout ? tout[t] : t;
            const float phi = acc.value();
            if (raw) raw[o] = phi;
            if (out) {
                double e = pp.potentfact != 0.0 ? (double)phi * pp.potentfact : (double)phi;
                if (pp.add_bg && bg) e += bg[h];
                out[o] = (float)e;  // penergy = potent*potentfact + halobgpotent
            }
        }
    }
    if (COUNT && counters) {
        for (int off = 16; off; off >>= 1) {
            npp += __shfl_xor_sync(0xffffffffu, npp, off);
            npc += __shfl_xor_sync(0xffffffffu, npc, off);
        }
        if (lane == 0) {
            atomicAdd(counters + 0, npp);
            atomicAdd(counters + 1, npc);
        }
    }
}

// The walk over ntarget targets on a grid of one resident wave.  With
// GF_BH_DYN each warp takes its next 32 targets from a counter in device
// memory, so warps that drew cheap targets keep drawing and the launch ends
// when the work does (with a static grid-stride split, the warps holding the
// costliest targets finish last, alone).
int launch_bh(gf_ctx *ctx, int64_t grid, int64_t ntarget, const float4 *tpos, const int32_t *thalo,
              const int32_t *tout, const float4 *spos, const int32_t *root, const int32_t *rend,
              const BhNode *nodes, const int32_t *direct, const double *bg, const PotentialParams &pp,
              float *out, float *raw, unsigned long long *counters) {
    const int block = GF_BH_BLOCK;
    unsigned long long *work = nullptr;
    // a grid of 1.6 waves (16 blocks per SM requested, 10 resident) would
    // leave 40 % of the SMs' block slots empty in its second wave
    auto kern = counters ? bh_kernel<true> : bh_kernel<false>;
    int per_sm = 0;
    GF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0));
    grid = std::max<int64_t>(1, std::min<int64_t>(grid, (int64_t)sm_count() * std::max(per_sm, 1)));
    if (GF_BH_DYN) {
        GF_TRY(ctx->work.reserve(256));
        work = ctx->work.as<unsigned long long>();  // slot 0: this walk
        GF_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(unsigned long long), ctx->stream));
    }
    kern<<<(int)grid, block, 0, ctx->stream>>>(ntarget, tpos, thalo, tout, spos, root, rend, nodes, direct, bg, pp,
                                               out, raw, counters, work, ctx->d_err);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

// Per-halo total mass (FP64 sum of the float masses, as Self_Halo_Potent's
// Mvir += mass[i]) and background term.  Each halo's particles are summed in
// kMassSplit slices by separate blocks (a large halo no longer holds one
// block for its whole length), then the slices in order.
constexpr int kMassSplit = 16;

__global__ void halo_mass_kernel(int32_t nhalo, const int64_t *__restrict__ pstart,
                                 const float4 *__restrict__ pos, double *__restrict__ part) {
    const int h = blockIdx.x / kMassSplit, sl = blockIdx.x % kMassSplit;
    if (h >= nhalo) return;
    const int64_t a0 = pstart[h], len = pstart[h + 1] - a0;
    const int64_t a = a0 + len * sl / kMassSplit, b = a0 + len * (sl + 1) / kMassSplit;
    double s = 0.0;
    for (int64_t p = a + threadIdx.x; p < b; p += blockDim.x) s += (double)pos[p].w;
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void halo_bg_kernel(int32_t nhalo, const int64_t *__restrict__ pstart,
                               const double *__restrict__ part, PotentialParams pp,
                               const int32_t *__restrict__ ntarget_halo,
                               int32_t ndirect, double *__restrict__ bg,
                               int32_t *__restrict__ direct) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nhalo) return;
    double m = 0.0;
    for (int sl = 0; sl < kMassSplit; sl++) m += part[(int64_t)h * kMassSplit + sl];
    bg[h] = pp.add_bg ? bg_potent_dev(m, pp) : 0.0;
    const int64_t nt = ntarget_halo ? ntarget_halo[h] : pstart[h + 1] - pstart[h];
    direct[h] = nt < ndirect ? 1 : 0;
}

__global__ void bg_eval_kernel(int32_t n, const double *__restrict__ mvir, PotentialParams pp,
                               double *__restrict__ bg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) bg[i] = bg_potent_dev(mvir[i], pp);
}

// bg and direct flags of every halo of t (scratch in ctx->tmp[5]).
int launch_halo_bg(gf_ctx *ctx, const TreeView &t, const int64_t *pstart, const PotentialParams &pp,
                   const int32_t *ntarget_halo, double **bg, int32_t **direct) {
    const size_t nb = (size_t)t.nhalo * sizeof(double);
    const size_t np_ = (size_t)t.nhalo * kMassSplit * sizeof(double);
    GF_TRY(ctx->tmp[5].reserve(nb + np_ + (size_t)t.nhalo * sizeof(int32_t) + 512));
    *bg = ctx->tmp[5].as<double>();
    double *part = *bg + t.nhalo;
    *direct = reinterpret_cast<int32_t *>(part + (size_t)t.nhalo * kMassSplit);
    halo_mass_kernel<<<t.nhalo * kMassSplit, 256, 0, ctx->stream>>>(t.nhalo, pstart, t.pos, part);
    GF_LAUNCH_CHECK();
    halo_bg_kernel<<<(t.nhalo + 127) / 128, 128, 0, ctx->stream>>>(t.nhalo, pstart, part, pp, ntarget_halo,
                                                                   pp.ndirect, *bg, *direct);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

}  // namespace

// The background term of n halo masses as the potential kernels evaluate it.
int launch_bg_eval(gf_ctx *ctx, int32_t n, const double *mvir, const PotentialParams &pp, double *bg) {
    if (n <= 0) return GF_OK;
    bg_eval_kernel<<<(n + 127) / 128, 128, 0, ctx->stream>>>(n, mvir, pp, bg);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

// Potential at every particle of every halo from the halo's own tree
// (self potential); outputs in batch order.
int launch_self_potential(gf_ctx *ctx, const TreeView &t, const int64_t *pstart,
                          const PotentialParams &pp, float *penergy, float *raw,
                          unsigned long long *counters) {
    if (t.n <= 0) return GF_OK;
    // tree-ordered positions carry the masses; halo h is still [pstart[h], pstart[h+1])
    double *bg;
    int32_t *direct;
    GF_TRY(launch_halo_bg(ctx, t, pstart, pp, nullptr, &bg, &direct));
    const int block = GF_BH_BLOCK;
    int64_t grid = (t.n + block - 1) / block;
    grid = std::min<int64_t>(grid, (int64_t)sm_count() * (2048 / block));
    GF_TRY(launch_bh(ctx, grid, t.n, t.pos, t.phalo, t.perm, t.pos, t.root, t.rend, t.bh, direct, bg, pp,
                     penergy, raw, counters));
    return GF_OK;
}

// Potential of one source tree (halo 0 of t) at arbitrary targets.
int launch_external_potential(gf_ctx *ctx, const TreeView &t, const int64_t *pstart_src,
                              int64_t ntarget, const float4 *tpos, const int32_t *thalo,
                              const int32_t *ntarget_halo, const PotentialParams &pp,
                              float *penergy, float *raw) {
    if (ntarget <= 0) return GF_OK;
    double *bg;
    int32_t *direct;
    GF_TRY(launch_halo_bg(ctx, t, pstart_src, pp, ntarget_halo, &bg, &direct));
    const int block = GF_BH_BLOCK;
    int64_t grid = std::min<int64_t>((ntarget + block - 1) / block, (int64_t)sm_count() * (2048 / block));
    GF_TRY(launch_bh(ctx, grid, ntarget, tpos, thalo, nullptr, t.pos, t.root, t.rend, t.bh, direct, bg, pp,
                     penergy, raw, nullptr));
    return GF_OK;
}

}  // namespace gf
