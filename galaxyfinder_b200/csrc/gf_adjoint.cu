// Adjoints of the density stage with respect to particle positions and
// masses, the kNN of a list of query particles, and the mesh peak scan.
//
//   TSC deposit   den[c] = volfact * sum_p m_p W(x_p - c)      tsc_omp2.c:166-506
//   findDen       rho_p  = sum_c S[c] W(x_p - c)               tsc_omp2.c:40-163
//   W4 density    rho_i  = sum_j W4(|x_i - x_j|, r_k,i / 2)    nnost.c:536-630
//   mesh peaks    strict 26-neighbour maxima above a threshold nnost.c:1176-1200
//
// W is the product of three quadratic B-splines (TSC), which is C1 in the
// positions, so its gradient is the product rule over the 27 stencil cells.
// The Gaussian smoothing (gsmooth.c:14-115) is a real, even filter applied as
// a circular convolution: its matrix is symmetric and it is its own adjoint,
// so gf_gaussian_smooth applied to a mesh gradient is the smoothing adjoint.
// All gradients are accumulated in FP64 (outputs are added to, not set).
#include <math.h>

#include <algorithm>
#include <vector>

#include "gf_tree.cuh"

namespace gf {

namespace {

int grid_for(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sm_count() * 16));
}

// dL/dm_p = volfact sum_c G[c] W_c,  dL/dx_p = volfact m_p sum_c G[c] dW_c/dx
__global__ void tsc_adjoint_kernel(int64_t n, const double *__restrict__ x,
                                   const double *__restrict__ y, const double *__restrict__ z,
                                   const double *__restrict__ mass,
                                   const int32_t *__restrict__ type,
                                   const int32_t *__restrict__ hid,
                                   const gf_mesh_desc *__restrict__ mesh,
                                   const float *__restrict__ G, double volfact,
                                   double *__restrict__ gx, double *__restrict__ gy,
                                   double *__restrict__ gz, double *__restrict__ gm, int *err) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const gf_mesh_desc m = mesh[hid ? hid[p] : 0];
        if (m.ptype != GF_TYPE_ALL && (type ? type[p] : GF_TYPE_DM) != m.ptype) continue;
        const Axis64 ax = tsc_axis64(x[p], m.xmin, m.cellsize);
        const Axis64 ay = tsc_axis64(y[p], m.ymin, m.cellsize);
        const Axis64 az = tsc_axis64(z[p], m.zmin, m.cellsize);
        if (!stencil_in(ax, ay, az, m)) {
            atomicOr(err, GF_ERRBIT_RANGE);
            continue;
        }
        const int64_t mx = 2 * (m.nx / 2 + 1);
        const float *g = G + m.off;
        double s0 = 0, sx = 0, sy = 0, sz = 0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const float *row = g + ax.i0 + mx * ((ay.i0 + b) + (int64_t)m.ny * (az.i0 + c));
                const double wyz = ay.w[b] * az.w[c];
                const double dyz = ay.dw[b] * az.w[c];
                const double ydz = ay.w[b] * az.dw[c];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const double v = __ldg(row + a);
                    s0 += v * ax.w[a] * wyz;
                    sx += v * ax.dw[a] * wyz;
                    sy += v * ax.w[a] * dyz;
                    sz += v * ax.w[a] * ydz;
                }
            }
        }
        const double mp = mass[p];
        if (gm) gm[p] += volfact * s0;
        gx[p] += volfact * mp * sx;
        gy[p] += volfact * mp * sy;
        gz[p] += volfact * mp * sz;
    }
}

// rho_p = sum_c S[c] W_c(x_p): dL/dS[c] += g_p W_c (scattered), dL/dx_p += g_p sum_c S[c] dW_c/dx
__global__ void find_den_adjoint_kernel(int64_t n, const double *__restrict__ x,
                                        const double *__restrict__ y,
                                        const double *__restrict__ z,
                                        const int32_t *__restrict__ hid,
                                        const gf_mesh_desc *__restrict__ mesh,
                                        const float *__restrict__ S,
                                        const double *__restrict__ gd, float *__restrict__ gS,
                                        double *__restrict__ gx, double *__restrict__ gy,
                                        double *__restrict__ gz, int *err) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const double gp = gd[p];
        if (gp == 0.0) continue;
        const gf_mesh_desc m = mesh[hid ? hid[p] : 0];
        const Axis64 ax = tsc_axis64(x[p], m.xmin, m.cellsize);
        const Axis64 ay = tsc_axis64(y[p], m.ymin, m.cellsize);
        const Axis64 az = tsc_axis64(z[p], m.zmin, m.cellsize);
        if (!stencil_in(ax, ay, az, m)) {
            atomicOr(err, GF_ERRBIT_RANGE);
            continue;
        }
        const int64_t mx = 2 * (m.nx / 2 + 1);
        double sx = 0, sy = 0, sz = 0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const int64_t row = m.off + ax.i0 + mx * ((ay.i0 + b) + (int64_t)m.ny * (az.i0 + c));
                const double wyz = ay.w[b] * az.w[c];
                const double dyz = ay.dw[b] * az.w[c];
                const double ydz = ay.w[b] * az.dw[c];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    if (gS) atomicAdd(gS + row + a, (float)(gp * ax.w[a] * wyz));
                    if (S) {
                        const double v = __ldg(S + row + a);
                        sx += v * ax.dw[a] * wyz;
                        sy += v * ax.w[a] * dyz;
                        sz += v * ax.w[a] * ydz;
                    }
                }
            }
        }
        if (S) {
            gx[p] += gp * sx;
            gy[p] += gp * sy;
            gz[p] += gp * sz;
        }
    }
}

// W4 of nnost.c:536-555 in FP64 and its derivatives: W(r; h) = f(r/h)/h^3,
// dW/dr = f'(q)/h^4, dW/dh = -(3 W + r dW/dr)/h.
struct W4d {
    double w, wr, wh;
};

__device__ __forceinline__ W4d w4_grad(double r, double h) {
    const double A1 = -0.2387324, A2 = 0.07957747;  // AMPW41, AMPW42 (nnost.c:534-535)
    const double q = r / h, h3 = h * h * h, h4 = h3 * h;
    W4d o{0, 0, 0};
    if (q < 1.) {
        o.w = A1 * ((2. - q) * q * q - 1.333333) / h3;
        o.wr = A1 * (4. * q - 3. * q * q) / h4;
    } else if (q < 2.) {
        const double t = 2. - q;
        o.w = A2 * t * t * t / h3;
        o.wr = -3. * A2 * t * t / h4;
    }
    o.wh = -(3. * o.w + r * o.wr) / h;
    return o;
}

__device__ __forceinline__ int halo_of(int64_t i, int32_t nhalo, const int64_t *pstart) {
    int lo = 0, hi = nhalo;  // largest h with pstart[h] <= i
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pstart[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// One warp per query i, neighbour j of its list in lane j (FP64 positions):
//   d rho_i / d x_i  = sum_j W_r(d_ij) (x_i - x_j)/d_ij + (sum_j W_h) dh/dx_i
//   d rho_i / d x_j  = -W_r(d_ij) (x_i - x_j)/d_ij           (+ the h term for the k-th)
// with h = r_k / 2 and r_k = |x_i - x_K| the k-th (last) neighbour's distance.
__global__ void knn_density_adjoint_kernel(int64_t nq, const int64_t *__restrict__ qidx, int64_t n,
                                           const double *__restrict__ px,
                                           const double *__restrict__ py,
                                           const double *__restrict__ pz, int32_t nhalo,
                                           const int64_t *__restrict__ pstart, int k,
                                           const int32_t *__restrict__ nearindex,
                                           const double *__restrict__ gd,
                                           double *__restrict__ gx, double *__restrict__ gy,
                                           double *__restrict__ gz, int *err) {
    const int lane = threadIdx.x & 31;
    const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t q = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; q < nq; q += nwarp) {
        const double g = gd[q];
        const int64_t i = qidx ? qidx[q] : q;
        if (g == 0.0) continue;
        if (i < 0 || i >= n) {
            if (lane == 0) atomicOr(err, GF_ERRBIT_INDEX);
            continue;
        }
        const int h = halo_of(i, nhalo, pstart);
        const int64_t hs = pstart[h];
        const int64_t nh = pstart[h + 1] - hs;
        const int kk = (int)(nh < k ? nh : k);
        const double xi = px[i], yi = py[i], zi = pz[i];
        int64_t J = -1;
        bool bad = false;
        if (lane < kk) {
            const int32_t jl = nearindex[q * k + lane];
            if (jl < 0 || jl >= nh) bad = true;
            else J = hs + jl;
        }
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) atomicOr(err, GF_ERRBIT_INDEX);
            continue;
        }
        double dx = 0, dy = 0, dz = 0, d = 0;
        if (J >= 0) {
            dx = xi - px[J];
            dy = yi - py[J];
            dz = zi - pz[J];
            d = sqrt(dx * dx + dy * dy + dz * dz);
        }
        const double rk = __shfl_sync(0xffffffffu, d, kk - 1);
        if (!(rk > 0.0)) continue;  // degenerate list: the density is not differentiable
        const double hh = 0.5 * rk;
        W4d w{0, 0, 0};
        if (J >= 0) w = w4_grad(d, hh);
        double sum_wh = w.wh;
        for (int off = 16; off; off >>= 1) sum_wh += __shfl_xor_sync(0xffffffffu, sum_wh, off);
        double cx = 0, cy = 0, cz = 0;
        if (J >= 0 && d > 0.0) {
            const double f = g * w.wr / d;
            cx = f * dx;
            cy = f * dy;
            cz = f * dz;
            atomicAdd(gx + J, -cx);
            atomicAdd(gy + J, -cy);
            atomicAdd(gz + J, -cz);
        }
        // h = |x_i - x_K| / 2: dh/dx_i = (x_i - x_K) / (2 r_k) = -dh/dx_K
        if (lane == kk - 1) {
            const double f = g * sum_wh / (2.0 * rk);
            cx += f * dx;
            cy += f * dy;
            cz += f * dz;
            atomicAdd(gx + J, -f * dx);
            atomicAdd(gy + J, -f * dy);
            atomicAdd(gz + J, -f * dz);
        }
        for (int off = 16; off; off >>= 1) {
            cx += __shfl_xor_sync(0xffffffffu, cx, off);
            cy += __shfl_xor_sync(0xffffffffu, cy, off);
            cz += __shfl_xor_sync(0xffffffffu, cz, off);
        }
        if (lane == 0) {
            atomicAdd(gx + i, cx);
            atomicAdd(gy + i, cy);
            atomicAdd(gz + i, cz);
        }
    }
}

__global__ void invert_perm_kernel(int64_t n, const int32_t *__restrict__ perm,
                                   int32_t *__restrict__ inv) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        inv[perm[t]] = (int32_t)t;
}

__global__ void query_list_kernel(int64_t nq, const int64_t *__restrict__ qidx, int64_t n,
                                  const int32_t *__restrict__ inv, int32_t *__restrict__ qlist,
                                  int *err) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nq;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = qidx[q];
        if (i < 0 || i >= n) {
            atomicOr(err, GF_ERRBIT_INDEX);
            qlist[q] = 0;
        } else {
            qlist[q] = inv[i];
        }
    }
}

// Strict 26-neighbour maxima above a threshold in the interior
// [margin, n - margin) of every mesh (nnost.c:1176-1200: a cell is not a peak
// when den <= any neighbour).  blockIdx.y selects the halo.
__global__ void mesh_peaks_kernel(const gf_mesh_desc *__restrict__ mesh,
                                  const float *__restrict__ den, int margin, float threshold,
                                  int64_t cap, int32_t *__restrict__ out_halo,
                                  int64_t *__restrict__ out_cell, float *__restrict__ out_val,
                                  unsigned long long *__restrict__ count) {
    const int h = blockIdx.y;
    const gf_mesh_desc m = mesh[h];
    const int64_t ix = m.nx - 2 * margin, iy = m.ny - 2 * margin, iz = m.nz - 2 * margin;
    if (ix <= 0 || iy <= 0 || iz <= 0) return;
    const int64_t ncell = ix * iy * iz;
    const int64_t mx = 2 * (m.nx / 2 + 1);
    const float *d = den + m.off;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = margin + c % ix;
        const int64_t j = margin + (c / ix) % iy;
        const int64_t k = margin + c / (ix * iy);
        const int64_t o = i + mx * (j + (int64_t)m.ny * k);
        const float v = d[o];
        if (!(v > threshold)) continue;
        bool peak = true;
        for (int dk = -1; dk <= 1 && peak; dk++)
            for (int dj = -1; dj <= 1 && peak; dj++)
                for (int di = -1; di <= 1; di++) {
                    if (!di && !dj && !dk) continue;
                    if (v <= d[o + di + mx * (dj + (int64_t)m.ny * dk)]) {
                        peak = false;
                        break;
                    }
                }
        if (!peak) continue;
        const unsigned long long at = atomicAdd(count, 1ull);
        if ((int64_t)at < cap) {
            out_halo[at] = h;
            out_cell[at] = o;
            out_val[at] = v;
        }
    }
}

}  // namespace

int launch_mesh_peaks(gf_ctx *ctx, int32_t nhalo, int64_t maxcell, const gf_mesh_desc *mesh_dev,
                      const float *den, int margin, float threshold, int64_t cap, int32_t *out_halo,
                      int64_t *out_cell, float *out_val, unsigned long long *dcount) {
    GF_CUDA_TRY(cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), ctx->stream));
    const int64_t gx = std::min<int64_t>((maxcell + 255) / 256, sm_count() * 8);
    dim3 grid((unsigned)std::max<int64_t>(gx, 1), (unsigned)nhalo);
    mesh_peaks_kernel<<<grid, 256, 0, ctx->stream>>>(mesh_dev, den, margin, threshold, cap, out_halo,
                                                    out_cell, out_val, dcount);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

}  // namespace gf

using namespace gf;

extern "C" {

int gf_knn_query(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                 const float *pos4_dev, int k, int64_t nq, const int64_t *qidx_dev,
                 int32_t *nearindex, float *dens) {
    clear_status();
    if (!ctx || nhalo < 0 || n < 0 || nq < 0 || n > INT32_MAX ||
        (n > 0 && (!pstart_dev || !pos4_dev)) || (nq > 0 && (!qidx_dev || !nearindex))) {
        set_status(GF_EINVAL, "gf_knn_query: invalid arguments");
        return GF_EINVAL;
    }
    if (n == 0 || nq == 0) return GF_OK;
    std::lock_guard<std::mutex> g(ctx->lock);
    const float4 *pos = reinterpret_cast<const float4 *>(pos4_dev);
    GF_TRY(build_tree(ctx, nhalo, n, pstart_dev, pos, 0.5f, 0, &ctx->last_tree));
    const size_t inv_bytes = ((size_t)n * sizeof(int32_t) + 255) & ~size_t(255);
    GF_TRY(ctx->tmp[2].reserve(inv_bytes + (size_t)nq * sizeof(int32_t)));
    int32_t *inv = ctx->tmp[2].as<int32_t>();
    int32_t *qlist = reinterpret_cast<int32_t *>(ctx->tmp[2].as<char>() + inv_bytes);
    invert_perm_kernel<<<grid_for(n), 256, 0, ctx->stream>>>(n, ctx->last_tree.perm, inv);
    GF_LAUNCH_CHECK();
    query_list_kernel<<<grid_for(nq), 256, 0, ctx->stream>>>(nq, qidx_dev, n, inv, qlist, ctx->d_err);
    GF_LAUNCH_CHECK();
    GF_TRY(check_device_errors(ctx));
    GF_TRY(launch_knn(ctx, ctx->last_tree, pstart_dev, pos, k, nearindex, dens, nullptr, qlist, nq));
    return check_device_errors(ctx);
}

int gf_knn_density_adjoint(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                           const double *x, const double *y, const double *z, int k, int64_t nq,
                           const int64_t *qidx_dev, const int32_t *nearindex, const double *gdens,
                           double *gx, double *gy, double *gz) {
    clear_status();
    if (!ctx || nhalo <= 0 || n < 0 || nq < 0 || k < 1 || k > 32 ||
        (nq > 0 && (!pstart_dev || !x || !y || !z || !nearindex || !gdens || !gx || !gy || !gz))) {
        set_status(GF_EINVAL, "gf_knn_density_adjoint: invalid arguments");
        return GF_EINVAL;
    }
    if (nq == 0 || n == 0) return GF_OK;
    std::lock_guard<std::mutex> g(ctx->lock);
    const int64_t blocks = std::min<int64_t>((nq * 32 + 255) / 256, sm_count() * 16);
    knn_density_adjoint_kernel<<<(int)std::max<int64_t>(blocks, 1), 256, 0, ctx->stream>>>(
        nq, qidx_dev, n, x, y, z, nhalo, pstart_dev, k, nearindex, gdens, gx, gy, gz, ctx->d_err);
    GF_LAUNCH_CHECK();
    return check_device_errors(ctx);
}

int gf_tsc_adjoint(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev, const float *gden,
                   double *gx, double *gy, double *gz, double *gm) {
    clear_status();
    if (!ctx || !b || (b->nparticle > 0 && (!mesh_dev || !gden || !gx || !gy || !gz || !b->x ||
                                            !b->y || !b->z || !b->mass || !b->pstart))) {
        set_status(GF_EINVAL, "gf_tsc_adjoint: invalid arguments");
        return GF_EINVAL;
    }
    if (b->nparticle == 0) return GF_OK;
    std::lock_guard<std::mutex> g(ctx->lock);
    const int32_t *hid = nullptr;
    if (b->nhalo > 1) {
        GF_TRY(ctx->hid.reserve((size_t)b->nparticle * sizeof(int32_t)));
        GF_TRY(compute_hid(ctx, b->nhalo, b->nparticle, b->pstart, ctx->hid.as<int32_t>()));
        hid = ctx->hid.as<int32_t>();
    }
    tsc_adjoint_kernel<<<grid_for(b->nparticle), 256, 0, ctx->stream>>>(
        b->nparticle, b->x, b->y, b->z, b->mass, b->type, hid, mesh_dev, gden, tsc_volfact(), gx, gy,
        gz, gm, ctx->d_err);
    GF_LAUNCH_CHECK();
    return check_device_errors(ctx);
}

int gf_find_den_adjoint(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev,
                        const float *den, const double *gdens, float *gden, double *gx,
                        double *gy, double *gz) {
    clear_status();
    if (!ctx || !b || (b->nparticle > 0 && (!mesh_dev || !gdens || !b->x || !b->y || !b->z ||
                                            !b->pstart || (den && (!gx || !gy || !gz))))) {
        set_status(GF_EINVAL, "gf_find_den_adjoint: invalid arguments");
        return GF_EINVAL;
    }
    if (b->nparticle == 0) return GF_OK;
    std::lock_guard<std::mutex> g(ctx->lock);
    const int32_t *hid = nullptr;
    if (b->nhalo > 1) {
        GF_TRY(ctx->hid.reserve((size_t)b->nparticle * sizeof(int32_t)));
        GF_TRY(compute_hid(ctx, b->nhalo, b->nparticle, b->pstart, ctx->hid.as<int32_t>()));
        hid = ctx->hid.as<int32_t>();
    }
    find_den_adjoint_kernel<<<grid_for(b->nparticle), 256, 0, ctx->stream>>>(
        b->nparticle, b->x, b->y, b->z, hid, mesh_dev, den, gdens, gden, gx, gy, gz, ctx->d_err);
    GF_LAUNCH_CHECK();
    return check_device_errors(ctx);
}

int gf_mesh_peaks(gf_ctx *ctx, int32_t nhalo, const gf_mesh_desc *mesh_host,
                  const gf_mesh_desc *mesh_dev, const float *den, int margin, float threshold,
                  int64_t cap, int32_t *out_halo, int64_t *out_cell, float *out_val,
                  int64_t *npeak) {
    clear_status();
    if (!ctx || nhalo < 0 || nhalo > 65535 || margin < 1 || cap < 0 || !npeak ||
        (nhalo > 0 && (!mesh_host || !mesh_dev || !den)) ||
        (cap > 0 && (!out_halo || !out_cell || !out_val))) {
        set_status(GF_EINVAL, "gf_mesh_peaks: invalid arguments");
        return GF_EINVAL;
    }
    *npeak = 0;
    if (nhalo == 0) return GF_OK;
    std::lock_guard<std::mutex> g(ctx->lock);
    int64_t maxcell = 1;
    for (int h = 0; h < nhalo; h++)
        maxcell = std::max<int64_t>(maxcell, (int64_t)mesh_host[h].nx * mesh_host[h].ny * mesh_host[h].nz);
    GF_TRY(ctx->tmp[3].reserve(sizeof(unsigned long long)));
    unsigned long long *dcount = ctx->tmp[3].as<unsigned long long>();
    GF_TRY(launch_mesh_peaks(ctx, nhalo, maxcell, mesh_dev, den, margin, threshold, cap, out_halo,
                             out_cell, out_val, dcount));
    unsigned long long hcount = 0;
    GF_CUDA_TRY(cudaMemcpyAsync(&hcount, dcount, sizeof(hcount), cudaMemcpyDeviceToHost, ctx->stream));
    GF_TRY(check_device_errors(ctx));
    *npeak = (int64_t)hcount;
    return GF_OK;
}

}  // extern "C"
