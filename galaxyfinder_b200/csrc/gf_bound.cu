// Boundedness test, tidal radius and tidal cut of NewGalFinder's member
// iteration (the callers of the potential), on the GPU.
//
//   CheckSelfTE        subhaloden.mod6.c:1730-1820
//   CheckExternalTE    subhaloden.mod6.c:1622-1704
//   AdGetTidalRCenterCore + get_tidal_ellipse   :1910-2035, :1102-1165
//   tidal cut of GetMemberRestParticleList / GetShellParticleFromRestParticleLIST
//                      :2734-2745, :532-541
//
// This file is compiled with --fmad=false: the kinetic energies, distances
// and comparisons follow the reference's float/double sequence operation by
// operation.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gf_tree.cuh"

namespace gf {

namespace {

int grid_for(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sm_count() * 16));
}

// KE_i = 1/2 |(x_i - c) r1 + (v_i - v_c) r2|^2 (subhaloden.mod6.c:1787-1795,
// 1667-1675), bound iff not KE > -PE; counts the bound particles.
__global__ void energy_flag_kernel(int n, const double *__restrict__ r, const float *__restrict__ v,
                                   const float *__restrict__ penergy, double cx, double cy,
                                   double cz, double cvx, double cvy, double cvz, double r1k,
                                   double r2k, unsigned char *__restrict__ flag,
                                   int *__restrict__ nbound) {
    int local = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float distx = (float)((r[3 * i] - cx) * r1k);
        const float disty = (float)((r[3 * i + 1] - cy) * r1k);
        const float distz = (float)((r[3 * i + 2] - cz) * r1k);
        const float tvx = (float)((double)distx + ((double)v[3 * i] - cvx) * r2k);
        const float tvy = (float)((double)disty + ((double)v[3 * i + 1] - cvy) * r2k);
        const float tvz = (float)((double)distz + ((double)v[3 * i + 2] - cvz) * r2k);
        const float ke = (float)(0.5 * (double)(tvx * tvx + tvy * tvy + tvz * tvz));
        const bool unbound = ke > -penergy[i];
        flag[i] = unbound ? GF_UNBOUND : GF_BOUND;
        local += unbound ? 0 : 1;
    }
    for (int off = 16; off; off >>= 1) local += __shfl_xor_sync(0xffffffffu, local, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(nbound, local);
}

// ------------------------------------------------------------------ tidal radius
constexpr double kMaxTidalR = 2.e5;  // MAX_TIDAL_R, subhaloden.mod6.c:34
constexpr int kNumMass = 10000;      // NUM_MASS, header.h:97

// get_tidal_ellipse, subhaloden.mod6.c:1102-1165, on the host: a handful of
// transcendental calls per core pair, in the reference's operand types (the
// core offsets are float differences, Mvir is float, the NFW helpers mix in
// long double).
double tidal_ellipse(const Coretype &my, const Coretype &other, float mvir, double mratio,
                     double bmass) {
    const gf_physics &ph = physics();
    const double dx = my.cx - other.cx, dy = my.cy - other.cy, dz = my.cz - other.cz;
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    const double dvx = my.cvx - other.cvx, dvy = my.cvy - other.cvy, dvz = my.cvz - other.cvz;
    const double v2 = dvx * dvx + dvy * dvy + dvz * dvz;
    const double wx = dy * dvz - dz * dvy, wy = dz * dvx - dx * dvz, wz = dx * dvy - dy * dvx;
    const double w2 = (wx * wx + wy * wy + wz * wz) / (dist * dist);
    const double pot = mvir / dist;
    const double kpdratio = ph.r2kineticfact * ph.r2kineticfact / ph.potentfact;
    double ellipse = w2 / pot * kpdratio;
    const double rvir = nfw_rvir(mvir);
    const double s = dist / rvir;
    const double nfwc = nfw_concentration(bmass);
    if (s > 1) {
        const double fact = v2 / (bmass / rvir) * kpdratio;
        if (fact > 2.0) ellipse = 0.0;
    } else {
        const double fact = v2 * s / (nfw_gnfw(nfwc) * log((double)(1.0L + nfwc * s)) * bmass / rvir) * kpdratio;
        if (fact > 2.0) ellipse = 0.0;
    }
    const double alpha = nfw_alpha(nfwc, s);
    return pow(mratio / (ellipse + alpha), (double)0.33333333333333L);
}

// Distance^2 of every member slot from its own core's (float) centre, in FP64
// (subhaloden.mod6.c:1973-1976), and the member's mass as float (:1941).
// midx lists each core's members in particle order.
__global__ void member_d2_kernel(int64_t nmem, const int32_t *__restrict__ midx,
                                 const int32_t *__restrict__ mcore, const double *__restrict__ x,
                                 const double *__restrict__ y, const double *__restrict__ z,
                                 const double *__restrict__ mass, const float *__restrict__ cxyz,
                                 double *__restrict__ md2, float *__restrict__ mmass) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nmem;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int i = midx[k], j = mcore[k];
        const double tx = x[i] - (double)cxyz[3 * j];
        const double ty = y[i] - (double)cxyz[3 * j + 1];
        const double tz = z[i] - (double)cxyz[3 * j + 2];
        md2[k] = tx * tx + ty * ty + tz * tz;
        mmass[k] = (float)mass[i];
    }
}

// Mass (Mvir) and number (inum) of core j's members closer to core j's centre
// than core i, for every pair (:1970-1982).  The reference accumulates Mvir
// in float, member by member in particle order; a warp walks the members 32
// at a time and adds the selected masses in that order through a shuffle
// chain, so the float sum is the reference's bit for bit.  One warp per pair.
__global__ void enclosed_kernel(int npair, const int32_t *__restrict__ pair_j,
                                const double *__restrict__ pair_r2,
                                const int64_t *__restrict__ mstart, const double *__restrict__ md2,
                                const float *__restrict__ mmass, float *__restrict__ encl_mass,
                                int *__restrict__ encl_num) {
    const int lane = threadIdx.x & 31;
    const int nwarp = (gridDim.x * blockDim.x) >> 5;
    for (int pr = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; pr < npair; pr += nwarp) {
        const int j = pair_j[pr];
        const double r2 = pair_r2[pr];
        const int64_t a = mstart[j], b = mstart[j + 1];
        float m = 0.f;
        int c = 0;
        for (int64_t base = a; base < b; base += 32) {
            const int64_t k = base + lane;
            float mk = 0.f;
            bool in = false;
            if (k < b) {
                in = md2[k] < r2;  // :1978
                mk = mmass[k];
            }
            unsigned bal = __ballot_sync(0xffffffffu, in);
            c += __popc(bal);
            while (bal) {
                const int src = __ffs(bal) - 1;
                m = m + __shfl_sync(0xffffffffu, mk, src);
                bal &= bal - 1;
            }
        }
        if (lane == 0) {
            encl_mass[pr] = m;
            encl_num[pr] = c;
        }
    }
}

// Tidal cut: flags of |x - c|^2 < Rt^2 in the reference's float arithmetic
// (:2738-2741: float offsets of FP64 positions from the float centre).
__global__ void tidal_flag_kernel(int n, const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ z, const int32_t *__restrict__ plist,
                                  float cx, float cy, float cz, float rt2,
                                  unsigned char *__restrict__ flag, int *__restrict__ block_count) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int f = 0;
    if (i < n) {
        const int k = plist ? plist[i] : i;
        const float tx = (float)(x[k] - (double)cx);
        const float ty = (float)(y[k] - (double)cy);
        const float tz = (float)(z[k] - (double)cz);
        const float d2 = tx * tx + ty * ty + tz * tz;
        f = d2 < rt2 ? 1 : 0;
        flag[i] = (unsigned char)f;
    }
    const unsigned b = __ballot_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(&cnt, __popc(b));
    __syncthreads();
    if (threadIdx.x == 0) block_count[blockIdx.x] = cnt;
}

// Order-preserving compaction of the flagged entries given each block's
// exclusive offset.
__global__ void tidal_compact_kernel(int n, const int32_t *__restrict__ plist,
                                     const unsigned char *__restrict__ flag,
                                     const int *__restrict__ block_off, int32_t *__restrict__ out) {
    __shared__ int warp_base[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = i < n ? flag[i] : 0;
    const unsigned b = __ballot_sync(0xffffffffu, f);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_base[w] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            const int c = warp_base[k];
            warp_base[k] = acc;
            acc += c;
        }
    }
    __syncthreads();
    if (f) out[block_off[blockIdx.x] + warp_base[w] + __popc(b & ((1u << lane) - 1))] = plist ? plist[i] : i;
}

}  // namespace

int energy_check(const Kptype *tkp, int tnp, unsigned char *bndflag, const Kptype *skp, int snp,
                 bool self, const double c[6]) {
    gf_ctx *ctx = default_ctx();
    if (!ctx) return -1;
    std::lock_guard<std::mutex> g(ctx->lock);
    std::vector<Vector3d> tr((size_t)tnp), sr;
    std::vector<float> v(3 * (size_t)tnp), smass;
    for (int i = 0; i < tnp; i++) {
        tr[i].x = tkp[i].x;
        tr[i].y = tkp[i].y;
        tr[i].z = tkp[i].z;
        v[3 * i] = tkp[i].vx;
        v[3 * i + 1] = tkp[i].vy;
        v[3 * i + 2] = tkp[i].vz;
    }
    const Kptype *src = self ? tkp : skp;
    const int ns = self ? tnp : snp;
    sr.resize((size_t)ns);
    smass.resize((size_t)ns);
    for (int i = 0; i < ns; i++) {
        sr[i].x = src[i].x;
        sr[i].y = src[i].y;
        sr[i].z = src[i].z;
        smass[i] = src[i].mass;
    }
    float *dpe = nullptr;
    const double *dr = nullptr;
    if (potent_device(ctx, tnp, tr.data(), ns, sr.data(), smass.data(), self, &dpe, &dr) != GF_OK)
        return -1;
    const size_t vbytes = 3 * (size_t)tnp * sizeof(float);
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    if (ctx->tmp[1].reserve(al(vbytes) + al((size_t)tnp) + 256) != GF_OK) return -1;
    float *dv = ctx->tmp[1].as<float>();
    unsigned char *dflag = ctx->tmp[1].as<unsigned char>() + al(vbytes);
    int *dcount = reinterpret_cast<int *>(dflag + al((size_t)tnp));
    if (cudaMemcpyAsync(dv, v.data(), vbytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(dcount, 0, sizeof(int), ctx->stream) != cudaSuccess) {
        set_status(GF_EDEVICE, "energy check: copy failed");
        return -1;
    }
    const gf_physics &ph = physics();
    energy_flag_kernel<<<grid_for(tnp), 256, 0, ctx->stream>>>(
        tnp, dr, dv, dpe, c[0], c[1], c[2], c[3], c[4], c[5], ph.r1kineticfact, ph.r2kineticfact,
        dflag, dcount);
    count_launch();
    if (cudaGetLastError() != cudaSuccess) {
        set_status(GF_EDEVICE, "energy check: launch failed");
        return -1;
    }
    int nbound = 0;
    if (cudaMemcpyAsync(bndflag, dflag, (size_t)tnp, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaMemcpyAsync(&nbound, dcount, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) {
        set_status(GF_EDEVICE, "energy check: copy back failed");
        return -1;
    }
    if (check_device_errors(ctx) != GF_OK) return -1;
    return nbound;
}

}  // namespace gf

using namespace gf;

extern "C" {

int CheckSelfTE(Kptype *kp, int np, unsigned char *bndflag, Coretype *icore) {
    clear_status();
    (void)icore;
    if (np < 0 || (np > 0 && (!kp || !bndflag))) {
        set_status(GF_EINVAL, "CheckSelfTE: invalid arguments");
        return 0;
    }
    if (np == 0) return 0;
    // subhaloden.mod6.c:1770-1784: mass-weighted centre of the member stars
    double c[6] = {0, 0, 0, 0, 0, 0}, tmass = 0;
    for (int i = 0; i < np; i++) {
        if (kp[i].bp && kp[i].bp->type == GF_TYPE_STAR) {
            c[0] += kp[i].x * kp[i].mass;
            c[1] += kp[i].y * kp[i].mass;
            c[2] += kp[i].z * kp[i].mass;
            c[3] += (double)kp[i].vx * kp[i].mass;
            c[4] += (double)kp[i].vy * kp[i].mass;
            c[5] += (double)kp[i].vz * kp[i].mass;
            tmass += kp[i].mass;
        }
    }
    for (int a = 0; a < 6; a++) c[a] = c[a] / tmass;  // no stars: 0/0 as in the reference
    const int nb = energy_check(kp, np, bndflag, nullptr, 0, true, c);
    return nb < 0 ? 0 : nb;
}

int CheckExternalTE(Kptype *tkp, int tnp, unsigned char *bndflag, Kptype *skp, int snp,
                    Coretype *icore) {
    clear_status();
    if (tnp < 0 || snp < 0 || !icore || (tnp > 0 && (!tkp || !bndflag)) || (snp > 0 && !skp)) {
        set_status(GF_EINVAL, "CheckExternalTE: invalid arguments");
        return 0;
    }
    if (tnp == 0) return 0;
    // subhaloden.mod6.c:1661-1662: the core's centre and velocity
    const double c[6] = {icore->cx, icore->cy, icore->cz, icore->cvx, icore->cvy, icore->cvz};
    if (snp == 0) {
        set_status(GF_EINVAL, "CheckExternalTE: no source particles");
        return 0;
    }
    const int nb = energy_check(tkp, tnp, bndflag, skp, snp, false, c);
    return nb < 0 ? 0 : nb;
}

int gf_tidal_radius(Coretype *core, int numcore, const int32_t *score_core, int ncore,
                    const SimpleBasicParticleType *bp, const int32_t *haloid, int np) {
    clear_status();
    if (numcore < 0 || ncore < 0 || np < 0 || (numcore > 0 && !core) ||
        (ncore > 0 && !score_core) || (np > 0 && (!bp || !haloid))) {
        set_status(GF_EINVAL, "gf_tidal_radius: invalid arguments");
        return GF_EINVAL;
    }
    if (numcore == 0 || ncore == 0) return GF_OK;
    for (int i = 0; i < ncore; i++)
        if (score_core[i] < 0 || score_core[i] >= numcore) {
            set_status(GF_EINVAL, "gf_tidal_radius: core id out of range");
            return GF_EINVAL;
        }
    for (int i = 0; i < np; i++)
        if (haloid[i] >= numcore) {
            set_status(GF_EINVAL, "gf_tidal_radius: particle core id out of range");
            return GF_EINVAL;
        }
    // core2member (:1918-1949): members per core in particle order and the
    // core's float mass sum, accumulated as the reference does
    std::vector<int64_t> mstart((size_t)numcore + 1, 0);
    std::vector<float> tmass((size_t)numcore, 0.f);
    for (int i = 0; i < np; i++)
        if (haloid[i] >= 0) {
            mstart[haloid[i] + 1]++;
            tmass[haloid[i]] = (float)((double)tmass[haloid[i]] + bp[i].mass);
        }
    for (int c = 0; c < numcore; c++) mstart[c + 1] += mstart[c];
    const int64_t nmem = mstart[numcore];
    // pairs (core ranked a, every core ranked after it) with members on both sides
    std::vector<int32_t> pj, pair_start((size_t)ncore + 1, 0);
    std::vector<double> pr2;
    for (int a = 0; a < ncore; a++) {
        const int ci = score_core[a];
        pair_start[a] = (int32_t)pj.size();
        if (mstart[ci + 1] == mstart[ci]) continue;
        const double cx = core[ci].cx, cy = core[ci].cy, cz = core[ci].cz;
        for (int b = a + 1; b < ncore; b++) {
            const int cj = score_core[b];
            if (mstart[cj + 1] == mstart[cj]) continue;
            const double bx = core[cj].cx, by = core[cj].cy, bz = core[cj].cz;
            pj.push_back(cj);
            pr2.push_back((bx - cx) * (bx - cx) + (by - cy) * (by - cy) + (bz - cz) * (bz - cz));
        }
    }
    pair_start[ncore] = (int32_t)pj.size();
    if (pj.size() > (size_t)INT32_MAX) {
        set_status(GF_EINVAL, "gf_tidal_radius: too many core pairs");
        return GF_EINVAL;
    }
    const int npair = (int)pj.size();
    std::vector<float> encl_mass((size_t)npair);
    std::vector<int> encl_num((size_t)npair);
    if (npair > 0) {
        gf_ctx *ctx = default_ctx();
        if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
        std::lock_guard<std::mutex> g(ctx->lock);
        std::vector<int32_t> midx((size_t)nmem), mcore((size_t)nmem);
        {
            std::vector<int64_t> cur(mstart.begin(), mstart.end() - 1);
            for (int i = 0; i < np; i++)
                if (haloid[i] >= 0) {
                    const int64_t at = cur[haloid[i]]++;
                    midx[at] = i;
                    mcore[at] = haloid[i];
                }
        }
        std::vector<float> cxyz(3 * (size_t)numcore);
        for (int c = 0; c < numcore; c++) {
            cxyz[3 * c] = core[c].cx;
            cxyz[3 * c + 1] = core[c].cy;
            cxyz[3 * c + 2] = core[c].cz;
        }
        const size_t np_ = (size_t)np;
        std::vector<double> xyzm(4 * np_);
        for (size_t i = 0; i < np_; i++) {
            xyzm[i] = bp[i].x;
            xyzm[np_ + i] = bp[i].y;
            xyzm[2 * np_ + i] = bp[i].z;
            xyzm[3 * np_ + i] = bp[i].mass;
        }
        auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
        const size_t nm = (size_t)nmem, npr = (size_t)npair;
        size_t off = 0;
        const size_t o_xyz = off; off += al(4 * np_ * sizeof(double));
        const size_t o_mi = off; off += al(nm * sizeof(int32_t));
        const size_t o_mc = off; off += al(nm * sizeof(int32_t));
        const size_t o_c = off; off += al(3 * (size_t)numcore * sizeof(float));
        const size_t o_ms = off; off += al(((size_t)numcore + 1) * sizeof(int64_t));
        const size_t o_d2 = off; off += al(nm * sizeof(double));
        const size_t o_mm = off; off += al(nm * sizeof(float));
        const size_t o_pj = off; off += al(npr * sizeof(int32_t));
        const size_t o_pr = off; off += al(npr * sizeof(double));
        const size_t o_em = off; off += al(npr * sizeof(float));
        const size_t o_en = off; off += al(npr * sizeof(int));
        GF_TRY(ctx->particles.reserve(off));
        char *d = ctx->particles.as<char>();
        cudaStream_t s = ctx->stream;
        GF_CUDA_TRY(cudaMemcpyAsync(d + o_xyz, xyzm.data(), 4 * np_ * sizeof(double), cudaMemcpyHostToDevice, s));
        GF_CUDA_TRY(cudaMemcpyAsync(d + o_mi, midx.data(), nm * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        GF_CUDA_TRY(cudaMemcpyAsync(d + o_mc, mcore.data(), nm * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        GF_CUDA_TRY(cudaMemcpyAsync(d + o_c, cxyz.data(), cxyz.size() * sizeof(float), cudaMemcpyHostToDevice, s));
        GF_CUDA_TRY(cudaMemcpyAsync(d + o_ms, mstart.data(), mstart.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        GF_CUDA_TRY(cudaMemcpyAsync(d + o_pj, pj.data(), npr * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        GF_CUDA_TRY(cudaMemcpyAsync(d + o_pr, pr2.data(), npr * sizeof(double), cudaMemcpyHostToDevice, s));
        const double *dx = reinterpret_cast<const double *>(d + o_xyz);
        member_d2_kernel<<<grid_for(nmem), 256, 0, s>>>(
            nmem, reinterpret_cast<const int32_t *>(d + o_mi), reinterpret_cast<const int32_t *>(d + o_mc),
            dx, dx + np_, dx + 2 * np_, dx + 3 * np_, reinterpret_cast<const float *>(d + o_c),
            reinterpret_cast<double *>(d + o_d2), reinterpret_cast<float *>(d + o_mm));
        GF_LAUNCH_CHECK();
        const int warps_per_block = 8;
        const int blocks = (int)std::min<int64_t>((npair + warps_per_block - 1) / warps_per_block, sm_count() * 32);
        enclosed_kernel<<<blocks, 32 * warps_per_block, 0, s>>>(
            npair, reinterpret_cast<const int32_t *>(d + o_pj), reinterpret_cast<const double *>(d + o_pr),
            reinterpret_cast<const int64_t *>(d + o_ms), reinterpret_cast<const double *>(d + o_d2),
            reinterpret_cast<const float *>(d + o_mm), reinterpret_cast<float *>(d + o_em),
            reinterpret_cast<int *>(d + o_en));
        GF_LAUNCH_CHECK();
        GF_CUDA_TRY(cudaMemcpyAsync(encl_mass.data(), d + o_em, npr * sizeof(float), cudaMemcpyDeviceToHost, s));
        GF_CUDA_TRY(cudaMemcpyAsync(encl_num.data(), d + o_en, npr * sizeof(int), cudaMemcpyDeviceToHost, s));
        GF_TRY(check_device_errors(ctx));
    }
    // Rtidal over the cores ranked after each core (:1956-2029)
    for (int a = 0; a < ncore; a++) {
        const int ci = score_core[a];
        const int64_t npc = mstart[ci + 1] - mstart[ci];
        core[ci].nummem = (int)npc;
        if (npc == 0) {
            core[ci].Rtidal = 0.f;
            continue;
        }
        float rt = (float)kMaxTidalR;
        for (int p = pair_start[a]; p < pair_start[a + 1]; p++) {
            const int cj = pj[p];
            const double r2 = pr2[p];
            if (encl_num[p] == 0) {
                rt = ((double)rt < kMaxTidalR) ? rt : (float)kMaxTidalR;
                continue;
            }
            const float mvir = encl_mass[p];
            // int mtmp = tmass / Mvir * NUM_MASS: a float quotient converted to
            // int; out of int range (or NaN) the x86 conversion gives INT_MIN
            const float q = tmass[ci] / mvir * (float)kNumMass;
            const bool outweighs = q >= (float)kNumMass && q < 2147483648.f;
            if (outweighs) {
                rt = (float)(sqrt(r2) * 0.5);
            } else {
                const double mratio = (double)(tmass[ci] / mvir);
                double tr = tidal_ellipse(core[ci], core[cj], mvir, mratio, (double)tmass[cj]);
                tr = tr < 0.5 ? tr : 0.5;
                const double cand = sqrt(r2) * tr;
                rt = ((double)rt < cand) ? rt : (float)cand;
            }
        }
        core[ci].Rtidal = rt;
    }
    return GF_OK;
}

int gf_tidal_select(const SimpleBasicParticleType *bp, int np, const int32_t *plist, int nlist,
                    float cx, float cy, float cz, float rtidal, int32_t *out, int *nout) {
    clear_status();
    const int n = plist ? nlist : np;
    if (np < 0 || n < 0 || !nout || (n > 0 && (!bp || !out))) {
        set_status(GF_EINVAL, "gf_tidal_select: invalid arguments");
        return GF_EINVAL;
    }
    *nout = 0;
    if (n == 0) return GF_OK;
    if (plist)
        for (int i = 0; i < n; i++)
            if (plist[i] < 0 || plist[i] >= np) {
                set_status(GF_EINVAL, "gf_tidal_select: list entry out of range");
                return GF_EINVAL;
            }
    gf_ctx *ctx = default_ctx();
    if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
    std::lock_guard<std::mutex> g(ctx->lock);
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    const int nb = (n + 255) / 256;
    size_t off = 0;
    const size_t o_xyz = off; off += al((size_t)np * 3 * sizeof(double));
    const size_t o_pl = off; off += al((size_t)n * sizeof(int32_t));
    const size_t o_fl = off; off += al((size_t)n);
    const size_t o_bc = off; off += al((size_t)nb * sizeof(int));
    const size_t o_out = off; off += al((size_t)n * sizeof(int32_t));
    GF_TRY(ctx->particles.reserve(off));
    char *d = ctx->particles.as<char>();
    std::vector<double> xyz(3 * (size_t)np);
    for (int i = 0; i < np; i++) {
        xyz[i] = bp[i].x;
        xyz[(size_t)np + i] = bp[i].y;
        xyz[2 * (size_t)np + i] = bp[i].z;
    }
    cudaStream_t s = ctx->stream;
    GF_CUDA_TRY(cudaMemcpyAsync(d + o_xyz, xyz.data(), xyz.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    if (plist) GF_CUDA_TRY(cudaMemcpyAsync(d + o_pl, plist, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    const double *dx = reinterpret_cast<const double *>(d + o_xyz);
    const float rt2 = rtidal * rtidal;  // :2732
    tidal_flag_kernel<<<nb, 256, 0, s>>>(n, dx, dx + np, dx + 2 * (size_t)np,
                                         plist ? reinterpret_cast<const int32_t *>(d + o_pl) : nullptr,
                                         cx, cy, cz, rt2, reinterpret_cast<unsigned char *>(d + o_fl),
                                         reinterpret_cast<int *>(d + o_bc));
    GF_LAUNCH_CHECK();
    std::vector<int> bc((size_t)nb);
    GF_CUDA_TRY(cudaMemcpyAsync(bc.data(), d + o_bc, (size_t)nb * sizeof(int), cudaMemcpyDeviceToHost, s));
    GF_CUDA_TRY(cudaStreamSynchronize(s));
    int total = 0;
    for (int b = 0; b < nb; b++) {
        const int c = bc[b];
        bc[b] = total;
        total += c;
    }
    GF_CUDA_TRY(cudaMemcpyAsync(d + o_bc, bc.data(), (size_t)nb * sizeof(int), cudaMemcpyHostToDevice, s));
    tidal_compact_kernel<<<nb, 256, 0, s>>>(n, plist ? reinterpret_cast<const int32_t *>(d + o_pl) : nullptr,
                                            reinterpret_cast<const unsigned char *>(d + o_fl),
                                            reinterpret_cast<const int *>(d + o_bc),
                                            reinterpret_cast<int32_t *>(d + o_out));
    GF_LAUNCH_CHECK();
    GF_CUDA_TRY(cudaMemcpyAsync(out, d + o_out, (size_t)total * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    GF_TRY(check_device_errors(ctx));
    *nout = total;
    return GF_OK;
}

}  // extern "C"
