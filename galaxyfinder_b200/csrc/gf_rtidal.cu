// NFW tidal-radius table of the reference's OLD_TIDAL build
// (NewGalFinder/mkRtidal.c:7-128): for Nc concentrations, Nd host distances
// (in virial radii) and Nm mass ratios, the tidal radius (in units of the
// distance) at which the NFW host's enclosed-mass difference reaches the
// satellite's mass ratio, found by inverting the tabulated ratio with linear
// interpolation in log space.  AdGetTidalRCenterCore reads it through
// nfw_rtidal when OLD_TIDAL is defined (subhaloden.mod6.c:1913-1916,
// 2007-2017).
//
// The table is built on the GPU, one thread per (concentration, distance)
// row: the 128 mass ratios of the row (getmM, stopping at the first ratio
// above 1, as the reference's break), then the 128 interpolated radii.
// Every operation keeps the reference's operand types (float variables,
// double library calls and double constants); this translation unit is
// compiled with --fmad=false so each one is rounded separately.  The double
// log/log10/pow of the device library may differ from the host C library's
// in the last bit, so a table entry can differ from the reference's in the
// last bits of its float.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "gf_internal.cuh"

namespace gf {

namespace {

constexpr int kNm = 128;  // mass ratios (Nrs = Nm), mkRtidal.c:30-33
constexpr int kNc = 32;   // concentrations
constexpr int kNd = 128;  // distances
constexpr int kCells = kNc * kNd * kNm;

// mkRtidal.c:9-12
__host__ __device__ __forceinline__ float rt_getgc(float c) {
    float res = 1. / (log((double)(1 + c)) - (double)(c / (1 + c)));
    return res;
}

// mkRtidal.c:14-26
__host__ __device__ __forceinline__ float rt_getmM(float c, float dist_over_Rv, float rs_over_dist) {
    const float rs_over_Rv = rs_over_dist * dist_over_Rv;
    const float gc = rt_getgc(c);
    const float s1 = dist_over_Rv - rs_over_Rv;
    const float s2 = dist_over_Rv;
    const float g = gc * rs_over_Rv * rs_over_Rv;
    float mnratio = (double)g * ((double)(-c / s1) / (1. + (double)(c * s1)) +
                                 log(1. + (double)(c * s1)) / (double)s1 / (double)s1);
    const float mnratio2 = (double)g * ((double)(-c / s2) / (1. + (double)(c * s2)) +
                                        log(1. + (double)(c * s2)) / (double)s2 / (double)s2);
    mnratio -= mnratio2;
    return mnratio;
}

// mkRtidal.c:37-50 (np >= 1 for every row of the table)
__host__ __device__ __forceinline__ float rt_interpole(const float *mM, const float *rsdist, int np,
                                                       float massratio) {
    if (massratio < mM[0]) return rsdist[0];
    if (massratio >= mM[np - 1]) return rsdist[np - 1];
    for (int i = 0; i < np - 1; i++) {
        if (massratio >= mM[i] && massratio < mM[i + 1])
            return (rsdist[i + 1] - rsdist[i]) / (mM[i + 1] - mM[i]) * (massratio - mM[i]) + rsdist[i];
    }
    return 0;
}

// mkRtidal.c:60-78: the table cell of (mass ratio, distance / Rvir, c)
__host__ __device__ __forceinline__ int rt_cell(float mM, float dRv, float c) {
    int i = (log10((double)mM) + 4.) / 4. * kNm;
    int j = (log10((double)dRv) + 3.) / 4. * kNd;
    int k = ((double)c - 1.) / 32. * kNc;
    i = i < 0 ? 0 : (i >= kNm ? kNm - 1 : i);
    j = j < 0 ? 0 : (j >= kNd ? kNd - 1 : j);
    k = k < 0 ? 0 : (k >= kNc ? kNc - 1 : k);
    return i + kNm * (j + kNd * k);
}

// mkRtidal.c:80-117, one thread per (k, j) row
__global__ void rtidal_table_kernel(float *__restrict__ table) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= kNc * kNd) return;
    const int k = row / kNd, j = row % kNd;
    const float c = 1. + (32. * k) / kNc;
    float dist_over_Rv = -3. + (double)(4 * j / (float)kNd);
    dist_over_Rv = pow(10., (double)dist_over_Rv);
    float mM[kNm], rsdist[kNm];
    int np = 0;
    for (int i = 0; i < kNm; i++) {
        const float rs_over_dist = (double)((float)(i + 1) / (float)kNm) * 5.;
        const float mratio = rt_getmM(c, dist_over_Rv, rs_over_dist);
        if (mratio > 1) break;
        mM[i] = log10((double)mratio);
        rsdist[i] = log10((double)rs_over_dist);
        np = i + 1;
    }
    for (int i = 0; i < kNm; i++) {
        const float mr = -4 + 4 * (float)i / (float)kNm;
        table[i + kNm * (j + kNd * k)] = pow(10., (double)rt_interpole(mM, rsdist, np, mr));
    }
}

__global__ void rtidal_lookup_kernel(int64_t n, const float *__restrict__ mM, const float *__restrict__ dRv,
                                     const float *__restrict__ c, const float *__restrict__ table,
                                     float *__restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        out[t] = table[rt_cell(mM[t], dRv[t], c[t])];
}

// The drop-ins' copy of the table (host), filled by mkRtidal().
std::mutex g_rt_lock;
std::vector<float> g_rt_host;

}  // namespace

}  // namespace gf

using namespace gf;

extern "C" {

int gf_nfw_rtidal_table(gf_ctx *ctx, float *table) {
    clear_status();
    if (!ctx || !table) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    rtidal_table_kernel<<<(kNc * kNd + 127) / 128, 128, 0, ctx->stream>>>(table);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

int gf_nfw_rtidal_lookup(gf_ctx *ctx, int64_t n, const float *mM, const float *dRv, const float *c,
                         const float *table, float *out) {
    clear_status();
    if (!ctx || n < 0 || (n > 0 && (!mM || !dRv || !c || !table || !out))) return GF_EINVAL;
    if (n == 0) return GF_OK;
    std::lock_guard<std::mutex> g(ctx->lock);
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8);
    rtidal_lookup_kernel<<<(int)blocks, 256, 0, ctx->stream>>>(n, mM, dRv, c, table, out);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

int gf_nfw_rtidal_cells(void) { return kCells; }

// mkRtidal.c:80: builds the table (on the GPU of the default context) into
// the library's host copy that nfw_rtidal reads.
void mkRtidal(void) {
    clear_status();
    gf_ctx *ctx = default_ctx();
    if (!ctx) {
        const int st = last_status() ? last_status() : GF_EDEVICE;
        dropin_exit_on_error(st, "mkRtidal");
        return;
    }
    float *d = nullptr;
    int st = GF_OK;
    std::vector<float> host((size_t)kCells);
    {
        std::lock_guard<std::mutex> g(ctx->lock);
        if (cudaMalloc(&d, sizeof(float) * kCells) != cudaSuccess) st = GF_ENOMEM;
        if (st == GF_OK) {
            rtidal_table_kernel<<<(kNc * kNd + 127) / 128, 128, 0, ctx->stream>>>(d);
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(host.data(), d, sizeof(float) * kCells, cudaMemcpyDeviceToHost, ctx->stream) !=
                    cudaSuccess ||
                cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                st = GF_EDEVICE;
        }
        if (d) cudaFree(d);
    }
    if (st != GF_OK) {
        set_status(st, "mkRtidal: the table could not be built on the device");
        dropin_exit_on_error(st, "mkRtidal");
        return;
    }
    std::lock_guard<std::mutex> g(g_rt_lock);
    g_rt_host.swap(host);
}

// mkRtidal.c:60-78 on the table mkRtidal() built (0 before it is built, as
// the reference's zero-initialised global table).
float nfw_rtidal(float mM, float dRv, float c) {
    std::lock_guard<std::mutex> g(g_rt_lock);
    if (g_rt_host.empty()) return 0.f;
    return g_rt_host[(size_t)rt_cell(mM, dRv, c)];
}

}  // extern "C"
