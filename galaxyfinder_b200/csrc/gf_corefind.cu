// Core finding on the kNN graph of one halo: the density peaks of
// finddenpeak (NewGalFinder/subhaloden.mod6.c:416-494) and the core densities
// and core members of FindCoreDensity (:1167-1475).
//
// finddenpeak: particle i is a peak when den[i] > PEAKTHRESHOLD (and it is a
// star, for the stellar path) and no particle of its kNN list is denser;
// peaks in particle order.  One thread per particle, the few peaks sorted on
// the host.
//
// FindCoreDensity, per core c (peak p): the core density is bisected between
// den[p] and minden = max(DENFLOOR, min den); a trial threshold t fails when
// a breadth-first search from p along kNN edges through particles with
// den > t reaches another peak.  The loop
//     t = (up + down)/2; search; fail ? down = t : up = t;
//     while |(up - down)/t| > COREDENRESOLUTION
// then takes up as the core density, and the particles the search from p
// reaches at up are the core's members (none if it reaches another peak).
// Whether a search reaches another peak, and the set it reaches, do not
// depend on the order in which it visits particles, so one block runs each
// search level-synchronously with a shared queue and a visited bitmap.
// Members get haloid = c (a particle reached from several cores keeps the
// highest core index, as the reference's serial loop leaves it) and the
// CORE and BOUND flags; peaks keep the PEAK flag.  starmass is summed in FP64
// and rounded once (the reference adds in float in its search order, so the
// two agree to float rounding).
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gf_internal.cuh"

extern "C" {
// The reference's arena and working-particle array (subhaloden.mod6.c:246-252,
// MAXTHREADS 64, params.h:148), resolved when libgf is linked into the
// reference program; absent (NULL) when libgf is loaded on its own.
void *Realloc(void *a, long long size, void **src) __attribute__((weak));
struct gf_ref_working_particle {
    float den;
    int haloid;
    unsigned char flag;
    unsigned char flag2[64];
};
extern gf_ref_working_particle *wp __attribute__((weak));
}

namespace gf {

namespace {

constexpr double kPeakThreshold = 2000.0;     // PEAKTHRESHOLD 2000.L, params.h:19
constexpr double kCoreDenResolution = 1.e-3;  // COREDENRESOLUTION, params.h:12
constexpr double kDenFloor = 1.;              // DENFLOOR, params.h:109
constexpr int kMaxNumCore = 1000000;          // MAXNUMCORE, params.h:66
constexpr int kNotHaloMember = -9999;         // NOT_HALO_MEMBER, defs.h:29
constexpr unsigned char kWpPeak = 0x01, kWpCore = 0x04, kWpBound = 0x10;  // subhaloden.mod6.c:180-186
constexpr unsigned char kWpVisitedT = 0x01;
constexpr int kStar = 1;                      // TYPE_STAR, tree.h:47
constexpr int kBisectMax = 200;               // the bisection halves its bracket; ends far sooner
constexpr int kCoreBlock = 256;

int grid_for(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sm_count() * 16));
}

__global__ void peak_kernel(int np, int K, const float *__restrict__ den, const int32_t *__restrict__ nbr,
                            const int32_t *__restrict__ type, double thr, int32_t *__restrict__ out,
                            unsigned *__restrict__ count, int cap, int *err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        const float d = den[i];
        if (!((double)d > thr)) continue;
        if (type && type[i] != kStar) continue;
        bool peak = true;
        for (int j = 0; j < K; j++) {
            const int v = nbr[(int64_t)i * K + j];
            if (v < 0 || v >= np) {
                atomicOr(err, GF_ERRBIT_INDEX);
                peak = false;
                break;
            }
            if (den[v] > d) {
                peak = false;
                break;
            }
        }
        if (peak) {
            const unsigned s = atomicAdd(count, 1u);
            if ((int)s < cap) out[s] = i;
        }
    }
}

__device__ __forceinline__ unsigned ordered_bits(float v) {
    const unsigned b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float from_ordered(unsigned o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

__global__ void min_den_kernel(int np, const float *__restrict__ den, unsigned *__restrict__ mn) {
    unsigned m = 0xffffffffu;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x)
        m = min(m, ordered_bits(den[i]));
    for (int off = 16; off; off >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) atomicMin(mn, m);
}

__global__ void fill_kernel(int np, int32_t *__restrict__ a, int32_t v, uint8_t *__restrict__ ispeak) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        a[i] = v;
        ispeak[i] = 0;
    }
}

__global__ void mark_peaks_kernel(int npk, const int32_t *__restrict__ peaks, int np,
                                  uint8_t *__restrict__ ispeak, int *err) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= npk) return;
    const int p = peaks[c];
    if (p < 0 || p >= np) {
        atomicOr(err, GF_ERRBIT_INDEX);
        return;
    }
    ispeak[p] = 1;
}

// One level-synchronous search from pk through particles with den > thr.
// Returns the number of particles reached (queue[0, n)); *brk is set when it
// reaches another peak.  Every thread of the block calls it.
__device__ int core_search(int pk, float thr, int np, int K, const float *__restrict__ den,
                           const int32_t *__restrict__ nbr, const uint8_t *__restrict__ ispeak,
                           unsigned *__restrict__ vis, int32_t *__restrict__ queue, int *s_tail, int *s_brk,
                           int *err) {
    if (threadIdx.x == 0) {
        queue[0] = pk;
        vis[pk >> 5] |= 1u << (pk & 31);
        *s_tail = 1;
        *s_brk = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    int head = 0;
    while (true) {
        const int tail = *s_tail;
        const int brk = *(volatile int *)s_brk;
        __syncthreads();  // everyone has read the level bounds
        if (brk || head >= tail) break;
        const int64_t items = (int64_t)(tail - head) * K;
        for (int64_t it0 = 0; it0 < items; it0 += blockDim.x) {
            const int64_t it = it0 + threadIdx.x;
            bool found = false;
            int v = -1;
            if (it < items) {
                const int u = queue[head + (int)(it / K)];
                v = nbr[(int64_t)u * K + (int)(it % K)];
                if (v < 0 || v >= np) {
                    atomicOr(err, GF_ERRBIT_INDEX);
                } else if (den[v] > thr) {
                    if (ispeak[v]) {
                        if (v != pk) *s_brk = 1;
                    } else {
                        const unsigned bit = 1u << (v & 31);
                        if (!(vis[v >> 5] & bit)) found = !(atomicOr(vis + (v >> 5), bit) & bit);
                    }
                }
            }
            // warp-aggregated append (the loop runs the same trip count on
            // every thread of the block, so whole warps reach the ballot)
            const unsigned want = __ballot_sync(0xffffffffu, found);
            if (want) {
                const int leader = __ffs(want) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(s_tail, __popc(want));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (found) queue[base + __popc(want & ((1u << lane) - 1u))] = v;
            }
        }
        __syncthreads();
        head = tail;
    }
    return *s_tail;
}

// Clears the visited bits of the particles a search reached.
__device__ void clear_search(int n, const int32_t *__restrict__ queue, unsigned *__restrict__ vis) {
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) vis[queue[e] >> 5] = 0u;
    __syncthreads();
}

__global__ void __launch_bounds__(kCoreBlock)
core_density_kernel(int np, int K, const float *__restrict__ den, const int32_t *__restrict__ nbr,
                    const uint8_t *__restrict__ ispeak, const int32_t *__restrict__ peaks, int ncore,
                    const unsigned *__restrict__ minbits, unsigned *__restrict__ vis_all,
                    int32_t *__restrict__ queue_all, int64_t words, const int32_t *__restrict__ type,
                    const double *__restrict__ mass, float *__restrict__ coredensity,
                    int32_t *__restrict__ nummem, int32_t *__restrict__ numstar,
                    float *__restrict__ starmass, int32_t *__restrict__ haloid, int *err) {
    __shared__ int s_tail, s_brk;
    __shared__ double s_mass[kCoreBlock / 32];
    __shared__ int s_cnt[kCoreBlock / 32];
    unsigned *vis = vis_all + (int64_t)blockIdx.x * words;
    int32_t *queue = queue_all + (int64_t)blockIdx.x * np;
    // minden = MAX(DENFLOOR, min den), stored in a float (subhaloden.mod6.c:1178-1180)
    const float minden = (float)fmax(kDenFloor, (double)from_ordered(*minbits));
    for (int c = blockIdx.x; c < ncore; c += gridDim.x) {
        const int pk = peaks[c];
        if (pk < 0 || pk >= np) {
            if (threadIdx.x == 0) atomicOr(err, GF_ERRBIT_INDEX);
            continue;
        }
        float up = den[pk], down = minden, thr;
        int iter = 0;
        do {
            thr = __fadd_rn(up, down) * 0.5f;  // 0.5*(upden+downden): a float sum, halved exactly
            const int n = core_search(pk, thr, np, K, den, nbr, ispeak, vis, queue, &s_tail, &s_brk, err);
            const int brk = s_brk;
            clear_search(n, queue, vis);
            if (brk) down = thr; else up = thr;
            if (++iter > kBisectMax) {
                if (threadIdx.x == 0) atomicOr(err, GF_ERRBIT_WALK);
                break;
            }
        } while (fabs((double)__fdiv_rn(__fsub_rn(up, down), thr)) > kCoreDenResolution);
        // the members: the search at the core density (none if it reaches another peak)
        int n = core_search(pk, up, np, K, den, nbr, ispeak, vis, queue, &s_tail, &s_brk, err);
        const int brk = s_brk;
        clear_search(n, queue, vis);
        if (brk) n = 0;
        double m = 0.0;
        int ns = 0;
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const int v = queue[e];
            if (type[v] == kStar) {
                ns++;
                m += mass[v];
            }
            atomicMax(haloid + v, c);
        }
        for (int off = 16; off; off >>= 1) {
            m += __shfl_xor_sync(0xffffffffu, m, off);
            ns += __shfl_xor_sync(0xffffffffu, ns, off);
        }
        if ((threadIdx.x & 31) == 0) {
            s_mass[threadIdx.x >> 5] = m;
            s_cnt[threadIdx.x >> 5] = ns;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double tm = 0.0;
            int tn = 0;
            for (int w = 0; w < kCoreBlock / 32; w++) {
                tm += s_mass[w];
                tn += s_cnt[w];
            }
            coredensity[c] = up;
            nummem[c] = n;
            numstar[c] = tn;
            starmass[c] = (float)tm;
        }
        __syncthreads();
    }
}

__global__ void core_flags_kernel(int np, const int32_t *__restrict__ haloid, const uint8_t *__restrict__ ispeak,
                                  uint8_t *__restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x)
        flag[i] = (ispeak[i] ? kWpPeak : 0) | (haloid[i] != kNotHaloMember ? (kWpCore | kWpBound) : 0);
}

__global__ void narrow_kernel(int64_t n, const long long *__restrict__ a, int32_t *__restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (a[i] < INT32_MIN || a[i] > INT32_MAX) ? -1 : (int32_t)a[i];
}

int density_peaks(gf_ctx *ctx, int32_t np, int K, const float *den, const int32_t *nbr, const int32_t *type,
                  double threshold, int32_t cap, int32_t *peak, int32_t *npeak) {
    GF_TRY(ctx->tmp[0].reserve(256));
    unsigned *dcount = ctx->tmp[0].as<unsigned>();
    GF_CUDA_TRY(cudaMemsetAsync(dcount, 0, sizeof(unsigned), ctx->stream));
    peak_kernel<<<grid_for(np), 256, 0, ctx->stream>>>(np, K, den, nbr, type, threshold, peak, dcount, cap,
                                                       ctx->d_err);
    GF_LAUNCH_CHECK();
    unsigned count = 0;
    GF_CUDA_TRY(cudaMemcpyAsync(&count, dcount, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // count is a stack variable
    GF_TRY(check_device_errors(ctx));
    *npeak = (int32_t)count;
    const int32_t kept = std::min<int32_t>((int32_t)count, cap);
    if (kept > 1) {  // particle order, as the reference's scan
        std::vector<int32_t> h(kept);
        GF_CUDA_TRY(cudaMemcpyAsync(h.data(), peak, sizeof(int32_t) * kept, cudaMemcpyDeviceToHost, ctx->stream));
        GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        std::sort(h.begin(), h.end());
        GF_CUDA_TRY(cudaMemcpyAsync(peak, h.data(), sizeof(int32_t) * kept, cudaMemcpyHostToDevice, ctx->stream));
        GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // h is a host vector
    }
    if ((int32_t)count > cap) {
        set_status(GF_ERANGE, "gf_density_peaks: %u peaks, room for %d", count, cap);
        return GF_ERANGE;
    }
    return GF_OK;
}

int core_density(gf_ctx *ctx, int32_t np, int K, const float *den, const int32_t *nbr, const int32_t *type,
                 const double *mass, int32_t ncore, const int32_t *peak, float *coredensity, int32_t *nummem,
                 int32_t *numstar, float *starmass, int32_t *haloid, uint8_t *flag) {
    cudaStream_t s = ctx->stream;
    const int64_t words = ((int64_t)np + 31) / 32;
    // concurrent searches: one per block, each with its bitmap and queue,
    // within about 1 GiB of scratch
    const int64_t slot = words * 4 + (int64_t)np * 4;
    const int64_t slots = std::max<int64_t>(1, std::min<int64_t>({(int64_t)ncore, (1LL << 30) / slot, sm_count() * 8}));
    // scratch: [min density | peak flags | bitmaps | queues]
    const size_t head = 256, flags = ((size_t)np + 255) & ~size_t(255);
    GF_TRY(ctx->tmp[1].reserve(head + flags + (size_t)(slots * slot)));
    char *base = ctx->tmp[1].as<char>();
    unsigned *minbits = reinterpret_cast<unsigned *>(base);
    uint8_t *ispeak = reinterpret_cast<uint8_t *>(base + head);
    unsigned *vis = reinterpret_cast<unsigned *>(base + head + flags);
    int32_t *queue = reinterpret_cast<int32_t *>(vis + slots * words);
    GF_CUDA_TRY(cudaMemsetAsync(minbits, 0xff, sizeof(unsigned), s));
    GF_CUDA_TRY(cudaMemsetAsync(vis, 0, (size_t)(slots * words) * 4, s));
    min_den_kernel<<<grid_for(np), 256, 0, s>>>(np, den, minbits);
    GF_LAUNCH_CHECK();
    fill_kernel<<<grid_for(np), 256, 0, s>>>(np, haloid, kNotHaloMember, ispeak);
    GF_LAUNCH_CHECK();
    if (ncore > 0) {
        mark_peaks_kernel<<<(ncore + 255) / 256, 256, 0, s>>>(ncore, peak, np, ispeak, ctx->d_err);
        GF_LAUNCH_CHECK();
        core_density_kernel<<<(int)slots, kCoreBlock, 0, s>>>(np, K, den, nbr, ispeak, peak, ncore, minbits, vis,
                                                              queue, words, type, mass, coredensity, nummem,
                                                              numstar, starmass, haloid, ctx->d_err);
        GF_LAUNCH_CHECK();
    }
    core_flags_kernel<<<grid_for(np), 256, 0, s>>>(np, haloid, ispeak, flag);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

// Host arrays of one halo (the drop-ins' inputs) on the device.
struct HaloCopy {
    float *den = nullptr;
    int32_t *nbr = nullptr;
    int32_t *type = nullptr;
    double *mass = nullptr;
};

int upload_halo(gf_ctx *ctx, int np, int K, const float *den, const long long *neighbor,
                const SimpleBasicParticleType *bp, bool with_type, bool with_mass, HaloCopy &h) {
    const size_t n = (size_t)std::max(np, 1);
    const size_t nk = n * (size_t)std::max(K, 1);
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t bytes = al(n * 4) + al(nk * 8) + al(nk * 4) + al(n * 4) + al(n * 8);
    GF_TRY(ctx->tmp[2].reserve(bytes));
    char *p = ctx->tmp[2].as<char>();
    h.den = reinterpret_cast<float *>(p);
    long long *nbr64 = reinterpret_cast<long long *>(p + al(n * 4));
    h.nbr = reinterpret_cast<int32_t *>(p + al(n * 4) + al(nk * 8));
    h.type = reinterpret_cast<int32_t *>(p + al(n * 4) + al(nk * 8) + al(nk * 4));
    h.mass = reinterpret_cast<double *>(p + al(n * 4) + al(nk * 8) + al(nk * 4) + al(n * 4));
    GF_CUDA_TRY(cudaMemcpyAsync(h.den, den, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(nbr64, neighbor, nk * 8, cudaMemcpyHostToDevice, ctx->stream));
    narrow_kernel<<<grid_for((int64_t)nk), 256, 0, ctx->stream>>>((int64_t)nk, nbr64, h.nbr);
    GF_LAUNCH_CHECK();
    if (with_type || with_mass) {
        std::vector<int32_t> t(n);
        std::vector<double> m(n);
        for (int i = 0; i < np; i++) {
            t[i] = (int32_t)bp[i].type;
            m[i] = bp[i].mass;
        }
        GF_CUDA_TRY(cudaMemcpyAsync(h.type, t.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
        GF_CUDA_TRY(cudaMemcpyAsync(h.mass, m.data(), n * 8, cudaMemcpyHostToDevice, ctx->stream));
        GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // t and m are host vectors
    }
    return GF_OK;
}

int do_finddenpeak(float *den, int numneigh, long long *neighbor, int np, Coretype **Core, int jflag,
                   SimpleBasicParticleType *bp, int *numcore) {
    *numcore = 0;
    if (np <= 0) return GF_OK;
    if (!den || !neighbor || !Core || !*Core || !bp || numneigh < 1) return GF_EINVAL;
    gf_ctx *ctx = default_ctx();
    if (!ctx) return gf_last_status();
    std::lock_guard<std::mutex> g(ctx->lock);
    HaloCopy h;
    GF_TRY(upload_halo(ctx, np, numneigh, den, neighbor, bp, jflag == 1, false, h));
    GF_TRY(ctx->tmp[3].reserve(sizeof(int32_t) * (size_t)np));
    int32_t *dpeak = ctx->tmp[3].as<int32_t>();
    int32_t npeak = 0;
    GF_TRY(density_peaks(ctx, np, numneigh, h.den, h.nbr, jflag == 1 ? h.type : nullptr, kPeakThreshold, np,
                         dpeak, &npeak));
    if (jflag != 1 && npeak > kMaxNumCore) {  // subhaloden.mod6.c:468-471
        set_status(GF_ERANGE, "Error exceeding the number of cores: %d :: %d", kMaxNumCore, np);
        return GF_ERANGE;
    }
    std::vector<int32_t> pk(npeak);
    if (npeak > 0) {
        GF_CUDA_TRY(cudaMemcpyAsync(pk.data(), dpeak, sizeof(int32_t) * npeak, cudaMemcpyDeviceToHost, ctx->stream));
        GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    // the caller's array holds MAXNUMCORE cores; the reference grows it by
    // MAXNUMCORE through the arena when it fills up (:446-450, :480-484)
    if (npeak >= kMaxNumCore - 10) {
        if (!Realloc) {
            set_status(GF_ENOTIMPL, "finddenpeak: %d peaks need the reference's Realloc", npeak);
            return GF_ENOTIMPL;
        }
        const long long want = (long long)sizeof(Coretype) * ((npeak / kMaxNumCore + 1) * (long long)kMaxNumCore);
        *Core = (Coretype *)Realloc(*Core, want, (void **)Core);
    }
    Coretype *core = *Core;
    for (int c = 0; c < npeak; c++) {
        const int i = pk[c];
        core[c].peak = i;
        core[c].cx = (float)bp[i].x;
        core[c].cy = (float)bp[i].y;
        core[c].cz = (float)bp[i].z;
        core[c].density = den[i];
    }
    *numcore = npeak;
    return GF_OK;
}

int do_find_core_density(SimpleBasicParticleType *bp, int np, long long *neighbor, int K, Coretype *core,
                         int numcore) {
    if (np <= 0) return GF_OK;
    if (&wp == nullptr || !wp) {
        set_status(GF_ENOTIMPL, "FindCoreDensity reads the reference's working-particle array wp "
                                "(link libgf into the reference program)");
        return GF_ENOTIMPL;
    }
    if (!bp || !neighbor || (numcore > 0 && !core) || K < 1) return GF_EINVAL;
    gf_ctx *ctx = default_ctx();
    if (!ctx) return gf_last_status();
    std::lock_guard<std::mutex> g(ctx->lock);
    std::vector<float> den(np);
    for (int i = 0; i < np; i++) den[i] = wp[i].den;
    HaloCopy h;
    GF_TRY(upload_halo(ctx, np, K, den.data(), neighbor, bp, true, true, h));
    const size_t nc = (size_t)std::max(numcore, 1);
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    GF_TRY(ctx->tmp[3].reserve(al(nc * 4) * 5 + al((size_t)np * 4) + al((size_t)np)));
    char *p = ctx->tmp[3].as<char>();
    int32_t *dpeak = reinterpret_cast<int32_t *>(p);
    float *dcd = reinterpret_cast<float *>(p + al(nc * 4));
    int32_t *dnm = reinterpret_cast<int32_t *>(p + 2 * al(nc * 4));
    int32_t *dns = reinterpret_cast<int32_t *>(p + 3 * al(nc * 4));
    float *dsm = reinterpret_cast<float *>(p + 4 * al(nc * 4));
    int32_t *dhalo = reinterpret_cast<int32_t *>(p + 5 * al(nc * 4));
    uint8_t *dflag = reinterpret_cast<uint8_t *>(p + 5 * al(nc * 4) + al((size_t)np * 4));
    std::vector<int32_t> pk(nc);
    for (int c = 0; c < numcore; c++) pk[c] = core[c].peak;
    GF_CUDA_TRY(cudaMemcpyAsync(dpeak, pk.data(), nc * 4, cudaMemcpyHostToDevice, ctx->stream));
    GF_TRY(core_density(ctx, np, K, h.den, h.nbr, h.type, h.mass, numcore, dpeak, dcd, dnm, dns, dsm, dhalo,
                        dflag));
    std::vector<float> cd(nc), sm(nc);
    std::vector<int32_t> nm(nc), ns(nc), halo(np);
    std::vector<uint8_t> fl(np);
    GF_CUDA_TRY(cudaMemcpyAsync(cd.data(), dcd, nc * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(nm.data(), dnm, nc * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(ns.data(), dns, nc * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(sm.data(), dsm, nc * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(halo.data(), dhalo, (size_t)np * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(fl.data(), dflag, (size_t)np, cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    GF_TRY(check_device_errors(ctx));
    for (int i = 0; i < np; i++) {
        wp[i].haloid = halo[i];
        wp[i].flag = fl[i];
        for (int t = 0; t < 64; t++) wp[i].flag2[t] &= (unsigned char)~kWpVisitedT;
    }
    for (int c = 0; c < numcore; c++) {
        core[c].coredensity = cd[c];
        core[c].nummem = nm[c];
        core[c].numstar = ns[c];
        core[c].starmass = sm[c];
    }
    return GF_OK;
}

}  // namespace

}  // namespace gf

using namespace gf;

extern "C" {

int gf_density_peaks(gf_ctx *ctx, int32_t np, int numneighbor, const float *den, const int32_t *neighbor,
                     const int32_t *type, double threshold, int32_t cap, int32_t *peak, int32_t *npeak) {
    clear_status();
    if (!ctx || np < 0 || numneighbor < 1 || cap < 0 || !npeak ||
        (np > 0 && (!den || !neighbor || (cap > 0 && !peak)))) {
        set_status(GF_EINVAL, "gf_density_peaks: invalid arguments");
        return GF_EINVAL;
    }
    *npeak = 0;
    if (np == 0) return GF_OK;
    std::lock_guard<std::mutex> g(ctx->lock);
    return density_peaks(ctx, np, numneighbor, den, neighbor, type, threshold, cap, peak, npeak);
}

int gf_core_density(gf_ctx *ctx, int32_t np, int numneighbor, const float *den, const int32_t *neighbor,
                    const int32_t *type, const double *mass, int32_t ncore, const int32_t *peak,
                    float *coredensity, int32_t *nummem, int32_t *numstar, float *starmass, int32_t *haloid,
                    uint8_t *flag) {
    clear_status();
    if (!ctx || np < 0 || numneighbor < 1 || ncore < 0 ||
        (np > 0 && (!den || !neighbor || !type || !mass || !haloid || !flag)) ||
        (ncore > 0 && (!peak || !coredensity || !nummem || !numstar || !starmass))) {
        set_status(GF_EINVAL, "gf_core_density: invalid arguments");
        return GF_EINVAL;
    }
    if (np == 0) return GF_OK;
    std::lock_guard<std::mutex> g(ctx->lock);
    GF_TRY(core_density(ctx, np, numneighbor, den, neighbor, type, mass, ncore, peak, coredensity, nummem,
                        numstar, starmass, haloid, flag));
    return check_device_errors(ctx);
}

int finddenpeak(float *den, int numneigh, long long *neighbor, int np, Coretype **Core, int jflag,
                SimpleBasicParticleType *bp) {
    clear_status();
    int numcore = 0;
    const int st = do_finddenpeak(den, numneigh, neighbor, np, Core, jflag, bp, &numcore);
    if (st == GF_ERANGE && !getenv("GF_NOEXIT")) {  // the reference exits with 999 here
        fprintf(stderr, "%s\n", gf_last_error());
        exit(999);
    }
    dropin_exit_on_error(st, "finddenpeak");
    return numcore;
}

int FindCoreDensity(SimpleBasicParticleType *bp, int np, long long *neighbor, int NumNeighbor, Coretype *core,
                    int numcore) {
    clear_status();
    dropin_exit_on_error(do_find_core_density(bp, np, neighbor, NumNeighbor, core, numcore), "FindCoreDensity");
    return numcore;
}

}  // extern "C"
