// Gaussian smoothing of TSC meshes, the operation of NewGalFinder/gsmooth.c:14-115:
//   forward r2c 3-D FFT -> multiply mode (i,j,k) by
//   exp(-(pi RG)^2 (i^2/nx^2 + j^2/ny^2 + k^2/nz^2)) with signed j,k and
//   i in [0, nx/2] -> c2r -> scale 1/(nx ny nz).
//
// The factor is a product of three real, even, per-axis factors, so the 3-D
// operation equals three independent 1-D circular convolutions (one per axis)
// with the real even kernels h_n = IDFT(G_n).  Each pass below loads a tile of
// pencils along one axis into shared memory once, and
//   * for power-of-two lengths runs a Stockham radix-2 FFT, multiplies the
//     spectrum by G_n/n, and runs the inverse FFT, all in shared memory;
//   * for any other length applies the full n-tap circular convolution with
//     the exact h_n (computed in FP64 on the host), so arbitrary sizes such
//     as the reference's extent/cellsize + 10 meshes are exact too.
// Two real pencils are packed into one complex pencil (real and imaginary
// parts): because G_n is real and even, filtering preserves that split.
// Every pass reads and writes each mesh element once (8 B per element per
// axis); twiddles and filters are generated in FP64 on the host.
#include <math.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <utility>

#include "gf_internal.cuh"

namespace gf {

namespace {

struct SmoothTile {
    int32_t halo;
    int32_t base;   // first pencil: row index (x) or first i (y, z)
    int32_t other;  // k (y axis) or j (z axis); unused for x
    int32_t npen;   // pencils in this tile
};

// Tile b of one axis pass -> (halo, pencil range).  tile_start holds the
// per-halo prefix of tile counts for that axis (nhalo+1 entries).
template <int AXIS>
__device__ __forceinline__ SmoothTile decode_tile(int64_t b, const int64_t *__restrict__ tile_start,
                                                  int nhalo, const gf_mesh_desc *__restrict__ mesh,
                                                  int pmax) {
    int lo = 0, hi = nhalo;  // largest h with tile_start[h] <= b
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tile_start[mid] <= b) lo = mid; else hi = mid;
    }
    const int64_t local = b - tile_start[lo];
    const gf_mesh_desc &m = mesh[lo];
    SmoothTile t;
    t.halo = lo;
    if (AXIS == 0) {
        const int rows = m.ny * m.nz;
        t.base = (int)(local * pmax);
        t.other = 0;
        t.npen = min(pmax, rows - t.base);
    } else {
        const int cx = (m.nx + pmax - 1) / pmax;
        t.other = (int)(local / cx);
        t.base = (int)(local - (int64_t)t.other * cx) * pmax;
        t.npen = min(pmax, m.nx - t.base);
    }
    return t;
}

struct AxisTable {
    int32_t n;
    int32_t logn;     // log2(n) for the FFT path, -1 for the direct path
    int64_t tab_off;  // float offset of this axis' tables
};

constexpr int kThreads = 256;

template <int AXIS>
__device__ __forceinline__ int64_t elem_addr(const gf_mesh_desc &m, int64_t mx, const SmoothTile &t,
                                             int p, int s) {
    if (AXIS == 0) return m.off + mx * (int64_t)(t.base + p) + s;
    if (AXIS == 1) return m.off + (t.base + p) + mx * ((int64_t)s + (int64_t)m.ny * t.other);
    return m.off + (t.base + p) + mx * ((int64_t)t.other + (int64_t)m.ny * s);
}

template <int AXIS>
__global__ void __launch_bounds__(kThreads)
smooth_axis_kernel(float *__restrict__ den, const gf_mesh_desc *__restrict__ mesh,
                   const int64_t *__restrict__ tile_start, int nhalo,
                   const AxisTable *__restrict__ axes, const float *__restrict__ tables, int pmax) {
    extern __shared__ float2 smem[];
    const SmoothTile t = decode_tile<AXIS>(blockIdx.x, tile_start, nhalo, mesh, pmax);
    const gf_mesh_desc m = mesh[t.halo];
    const AxisTable at = axes[3 * t.halo + AXIS];
    const int n = at.n;
    const int64_t mx = 2 * (m.nx / 2 + 1);
    const int npair = (t.npen + 1) >> 1;
    float2 *bufA = smem;
    float2 *bufB = smem + (size_t)((pmax + 1) >> 1) * n;
    float *fa = reinterpret_cast<float *>(bufA);

    // ---- load: pencil p -> component (p & 1) of complex pencil p >> 1
    const int total = 2 * npair * n;
    for (int e = threadIdx.x; e < total; e += kThreads) {
        int p, s;
        if (AXIS == 0) { p = e / n; s = e - p * n; }
        else { s = e / (2 * npair); p = e - s * (2 * npair); }
        float v = 0.f;
        if (p < t.npen) v = den[elem_addr<AXIS>(m, mx, t, p, s)];
        fa[2 * ((p >> 1) * n + s) + (p & 1)] = v;
    }
    __syncthreads();

    float2 *src = bufA, *dst = bufB;
    if (at.logn >= 0) {
        const float2 *tw = reinterpret_cast<const float2 *>(tables + at.tab_off);  // n/2 twiddles
        const float *filt = tables + at.tab_off + n;                               // n factors
        const int half = n >> 1;
        const int work = npair * half;
        for (int dir = 0; dir < 2; dir++) {
            const float sgn = dir == 0 ? 1.f : -1.f;  // inverse uses conjugate twiddles
            for (int ls = 0; ls < at.logn; ls++) {
                const int smask = (1 << ls) - 1;
                for (int e = threadIdx.x; e < work; e += kThreads) {
                    const int c = e / half;
                    const int tt = e - c * half;
                    const int q = tt & smask;
                    const int p = tt >> ls;
                    const float2 *x = src + c * n;
                    float2 *y = dst + c * n;
                    const float2 a = x[q + (p << ls)];
                    const float2 b = x[q + (p << ls) + half];
                    float2 w = tw[p << ls];
                    w.y *= sgn;
                    const float2 d = make_float2(a.x - b.x, a.y - b.y);
                    y[q + (p << (ls + 1))] = make_float2(a.x + b.x, a.y + b.y);
                    y[q + (p << (ls + 1)) + (1 << ls)] =
                        make_float2(d.x * w.x - d.y * w.y, d.x * w.y + d.y * w.x);
                }
                __syncthreads();
                float2 *tmp = src; src = dst; dst = tmp;
            }
            if (dir == 0) {
                for (int e = threadIdx.x; e < npair * n; e += kThreads) {
                    const int k = e % n;
                    const float g = filt[k];
                    src[e].x *= g;
                    src[e].y *= g;
                }
                __syncthreads();
            }
        }
    } else {
        // direct n-tap circular convolution with the exact periodic kernel
        const float *h = tables + at.tab_off;
        for (int e = threadIdx.x; e < npair * n; e += kThreads) {
            const int c = e / n;
            const int s = e - c * n;
            const float2 *x = src + c * n;
            float ar = 0.f, ai = 0.f;
            int idx = s;
            for (int mm = 0; mm < n; mm++) {
                const float hv = h[mm];
                const float2 v = x[idx];
                ar = fmaf(hv, v.x, ar);
                ai = fmaf(hv, v.y, ai);
                idx = idx == 0 ? n - 1 : idx - 1;
            }
            dst[e] = make_float2(ar, ai);
        }
        __syncthreads();
        src = dst;
    }

    // ---- store
    const float *fs = reinterpret_cast<const float *>(src);
    for (int e = threadIdx.x; e < total; e += kThreads) {
        int p, s;
        if (AXIS == 0) { p = e / n; s = e - p * n; }
        else { s = e / (2 * npair); p = e - s * (2 * npair); }
        if (p < t.npen) den[elem_addr<AXIS>(m, mx, t, p, s)] = fs[2 * ((p >> 1) * n + s) + (p & 1)];
    }
}

int ilog2_exact(int n) {
    if (n <= 0 || (n & (n - 1))) return -1;
    int l = 0;
    while ((1 << l) < n) l++;
    return l;
}

// Spectral factor of one axis (gsmooth.c:67-86): G(k) = exp(k_s^2 expfac / n^2)
// with k_s the signed frequency, expfac = -(pi RG/cellsize)^2.
double axis_factor(int k, int n, double rg_cells) {
    const double expfac = -(M_PI * rg_cells) * (M_PI * rg_cells);
    long ks = k;
    if (k > n / 2) ks = k - n;
    return exp((double)(ks * ks) * expfac / ((double)n * (double)n));
}

void append_tables(std::vector<float> &tab, int n, double rg_cells, AxisTable &at) {
    at.n = n;
    at.logn = ilog2_exact(n);
    at.tab_off = (int64_t)tab.size();
    if (at.logn >= 0) {
        for (int k = 0; k < n / 2; k++) {  // forward twiddles e^{-2 pi i k/n}
            const double ang = 2.0 * M_PI * (double)k / (double)n;
            tab.push_back((float)cos(ang));
            tab.push_back((float)-sin(ang));
        }
        for (int k = 0; k < n; k++) tab.push_back((float)(axis_factor(k, n, rg_cells) / n));
    } else {
        std::vector<double> g(n);
        for (int k = 0; k < n; k++) g[k] = axis_factor(k, n, rg_cells);
        for (int mm = 0; mm < n; mm++) {
            double acc = 0.0;
            for (int k = 0; k < n; k++) {
                const long km = ((long)k * mm) % n;
                acc += g[k] * cos(2.0 * M_PI * (double)km / (double)n);
            }
            tab.push_back((float)(acc / n));
        }
    }
}

template <int AXIS>
int launch_axis(gf_ctx *ctx, float *den, const gf_mesh_desc *mesh_dev, const int64_t *tile_start,
                int nhalo, int64_t ntiles, const AxisTable *axes, const float *tables, int pmax,
                int nmax) {
    if (ntiles == 0) return GF_OK;
    if (ntiles > 0x7fffffffLL) {
        set_status(GF_ENOTIMPL, "%lld smoothing tiles exceed one launch", (long long)ntiles);
        return GF_ENOTIMPL;
    }
    const size_t smem = (size_t)2 * ((pmax + 1) / 2) * nmax * sizeof(float2);
    GF_CUDA_TRY(cudaFuncSetAttribute(smooth_axis_kernel<AXIS>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    smooth_axis_kernel<AXIS><<<(unsigned)ntiles, kThreads, smem, ctx->stream>>>(
        den, mesh_dev, tile_start, nhalo, axes, tables, pmax);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

}  // namespace

int smooth_meshes(gf_ctx *ctx, int32_t nhalo, const gf_mesh_desc *mesh_host,
                  const gf_mesh_desc *mesh_dev, float *den) {
    if (nhalo <= 0) return GF_OK;
    std::vector<AxisTable> axes(3 * (size_t)nhalo);
    std::vector<float> tables;
    std::map<std::pair<int, double>, AxisTable> cache;
    int nmax = 0;
    for (int h = 0; h < nhalo; h++) {
        const gf_mesh_desc &m = mesh_host[h];
        if (m.nx < 1 || m.ny < 1 || m.nz < 1 || !(m.cellsize > 0)) {
            set_status(GF_EINVAL, "halo %d: bad mesh %d x %d x %d", h, m.nx, m.ny, m.nz);
            return GF_EINVAL;
        }
        // gsmooth.c:67 stores RG/cellsize back into the float RG
        const double rg_cells = (double)(float)(m.rg / m.cellsize);
        const int dims[3] = {m.nx, m.ny, m.nz};
        for (int a = 0; a < 3; a++) {
            auto key = std::make_pair(dims[a], rg_cells);
            auto it = cache.find(key);
            if (it == cache.end()) {
                AxisTable at;
                append_tables(tables, dims[a], rg_cells, at);
                it = cache.emplace(key, at).first;
            }
            axes[3 * (size_t)h + a] = it->second;
            if (dims[a] > nmax) nmax = dims[a];
        }
    }
    // pencils per tile: 32 (a full 128-byte row of a y/z tile) unless the
    // ping-pong buffers would exceed the shared memory of one block
    int pmax = 32;
    while (pmax > 2 && (size_t)2 * (pmax / 2) * nmax * sizeof(float2) > 200 * 1024) pmax -= 2;
    if ((size_t)2 * (pmax / 2) * nmax * sizeof(float2) > 200 * 1024) {
        set_status(GF_ENOTIMPL, "mesh axis of %d cells exceeds the shared-memory pencil tile", nmax);
        return GF_ENOTIMPL;
    }
    std::vector<int64_t> tstart[3];
    for (int a = 0; a < 3; a++) tstart[a].assign((size_t)nhalo + 1, 0);
    for (int h = 0; h < nhalo; h++) {
        const gf_mesh_desc &m = mesh_host[h];
        const int64_t cx = (m.nx + pmax - 1) / pmax;
        tstart[0][h + 1] = tstart[0][h] + ((int64_t)m.ny * m.nz + pmax - 1) / pmax;
        tstart[1][h + 1] = tstart[1][h] + cx * m.nz;
        tstart[2][h + 1] = tstart[2][h] + cx * m.ny;
    }
    // stage everything in one device buffer: [axes | tables | starts x | starts y | starts z]
    auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t off_tab = align(axes.size() * sizeof(AxisTable));
    const size_t off_s0 = align(off_tab + tables.size() * sizeof(float));
    const size_t sbytes = ((size_t)nhalo + 1) * sizeof(int64_t);
    const size_t off_s1 = align(off_s0 + sbytes);
    const size_t off_s2 = align(off_s1 + sbytes);
    const size_t total = off_s2 + sbytes;
    GF_TRY(ctx->smooth_tables.reserve(total));
    GF_TRY(ctx->pin[3].reserve(total));
    char *hbuf = ctx->pin[3].as<char>();
    // the pinned staging buffer may still feed an earlier asynchronous copy
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    memcpy(hbuf, axes.data(), axes.size() * sizeof(AxisTable));
    memcpy(hbuf + off_tab, tables.data(), tables.size() * sizeof(float));
    memcpy(hbuf + off_s0, tstart[0].data(), sbytes);
    memcpy(hbuf + off_s1, tstart[1].data(), sbytes);
    memcpy(hbuf + off_s2, tstart[2].data(), sbytes);
    char *dbuf = ctx->smooth_tables.as<char>();
    GF_CUDA_TRY(cudaMemcpyAsync(dbuf, hbuf, total, cudaMemcpyHostToDevice, ctx->stream));
    const AxisTable *d_axes = reinterpret_cast<const AxisTable *>(dbuf);
    const float *d_tab = reinterpret_cast<const float *>(dbuf + off_tab);
    GF_TRY(launch_axis<0>(ctx, den, mesh_dev, reinterpret_cast<const int64_t *>(dbuf + off_s0),
                          nhalo, tstart[0][nhalo], d_axes, d_tab, pmax, nmax));
    GF_TRY(launch_axis<1>(ctx, den, mesh_dev, reinterpret_cast<const int64_t *>(dbuf + off_s1),
                          nhalo, tstart[1][nhalo], d_axes, d_tab, pmax, nmax));
    GF_TRY(launch_axis<2>(ctx, den, mesh_dev, reinterpret_cast<const int64_t *>(dbuf + off_s2),
                          nhalo, tstart[2][nhalo], d_axes, d_tab, pmax, nmax));
    return GF_OK;
}

}  // namespace gf
