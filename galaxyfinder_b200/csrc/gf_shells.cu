// One shell of the boundedness loop of subhalo_den
// (NewGalFinder/subhaloden.mod6.c:3033-3101), batched over the shell's cores.
//
// The reference takes the shell's cores one after another (in the order of
// its qsort by member count).  For core j it collects the targets
// (GetShellParticleFromRestParticleLIST, :516-543: the shell's particles not
// yet bound, then every REMAINING particle, both cut at the core's tidal
// radius) and the sources (GetMemCandidateList, :544-560: the core's members,
// then the particles of the later shells that hold the core), tests every
// target against the sources (MULTIHALOSHELL -> CheckExternalTE, :1622-1721)
// and marks the bound ones as the core's members and the others REMAINING;
// after the last core the shell's unbound particles become REMAINING
// (UnboundShellP2Rest, :2111-2121).
//
// Within a shell a target never is a member of any core (targets have no
// halo id: the shell's particles lose theirs when the shell is formed, and a
// REMAINING particle always is NOT_HALO_MEMBER), so every core's sources stay
// fixed while the shell runs, and a particle's energy test depends only on
// the particle, the core and its sources.  The targets of core j are the
// candidates of j at the start of the shell minus those bound by earlier
// cores (plus second copies of the shell particles that earlier cores found
// unbound, which are candidates already).  So all cores' candidates are
// tested in one batched pass on the GPU (one source octree per core, one
// potential launch, one energy launch) and the loop is replayed on the host
// with the reference's order and counts.  The external potential sums
// directly below 1000 targets (subhaloden.mod6.c:1545): the batch uses the
// candidate count, and a core whose replayed target count falls on the other
// side of 1000 is retested alone with its exact target list, as the
// one-call-per-core path would.
//
// This file is compiled with --fmad=false: the tidal cut and the kinetic
// energies follow the reference's float/double sequence.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gf_tree.cuh"

namespace gf {

namespace {

constexpr unsigned char kWpBound = 0x10, kWpRemaining = 0x20;  // WP_BOUND, WP_REMAINING, :185-186
constexpr int32_t kNotMember = -9999;  // NOT_HALO_MEMBER, defs.h:29
constexpr int kDirectBelow = 1000;     // External_Halo_Potent's direct-sum bound, :1545

__global__ void pos_kernel(int64_t n, const double *__restrict__ r, const float *__restrict__ m,
                           float4 *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = make_float4((float)r[3 * i], (float)r[3 * i + 1], (float)r[3 * i + 2], m ? m[i] : 0.f);
}

// energy_flag_kernel's test with the core of each target (gf_bound.cu,
// subhaloden.mod6.c:1667-1675, 1693-1700).
__global__ void energy_cores_kernel(int64_t n, const double *__restrict__ r, const float *__restrict__ v,
                                    const float *__restrict__ penergy, const int32_t *__restrict__ tcore,
                                    const double *__restrict__ centre, double r1k, double r2k,
                                    unsigned char *__restrict__ flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double *c = centre + 6 * (int64_t)tcore[i];
        const float distx = (float)((r[3 * i] - c[0]) * r1k);
        const float disty = (float)((r[3 * i + 1] - c[1]) * r1k);
        const float distz = (float)((r[3 * i + 2] - c[2]) * r1k);
        const float tvx = (float)((double)distx + ((double)v[3 * i] - c[3]) * r2k);
        const float tvy = (float)((double)disty + ((double)v[3 * i + 1] - c[4]) * r2k);
        const float tvz = (float)((double)distz + ((double)v[3 * i + 2] - c[5]) * r2k);
        const float ke = (float)(0.5 * (double)(tvx * tvx + tvy * tvy + tvz * tvz));
        flag[i] = ke > -penergy[i] ? GF_UNBOUND : GF_BOUND;
    }
}

int grid_of(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 16));
}

// The tidal cut of GetShellParticleFromRestParticleLIST (:532-541): float
// offsets from the float centre, float squared distance against Rtidal^2.
inline bool within(const SimpleBasicParticleType &p, const Coretype &c) {
    const float tmpx = (float)(p.x - c.cx);
    const float tmpy = (float)(p.y - c.cy);
    const float tmpz = (float)(p.z - c.cz);
    const float dist2 = tmpx * tmpx + tmpy * tmpy + tmpz * tmpz;
    const float tidalr2 = c.Rtidal * c.Rtidal;
    return dist2 < tidalr2;
}

struct CoreWork {
    int core = 0;
    std::vector<int32_t> cand;     // candidates at the start of the shell (batch targets)
    std::vector<int32_t> src;      // sources (members, then later shells' particles)
    int64_t toff = 0;              // offset of the candidates in the batch
};

// One core's energy test on its exact target list (Kptype as DumpKPfromBP fills it).
int retest_core(const SimpleBasicParticleType *bp, const std::vector<int32_t> &tl, const std::vector<int32_t> &sl,
                const Coretype &c, std::vector<unsigned char> &flag_out) {
    std::vector<Kptype> tkp(tl.size()), skp(sl.size());
    auto dump = [&](std::vector<Kptype> &kp, const std::vector<int32_t> &l) {
        for (size_t i = 0; i < l.size(); i++) {
            const SimpleBasicParticleType &p = bp[l[i]];
            kp[i].x = p.x;
            kp[i].y = p.y;
            kp[i].z = p.z;
            kp[i].vx = (float)p.vx;
            kp[i].vy = (float)p.vy;
            kp[i].vz = (float)p.vz;
            kp[i].mass = (float)p.mass;
            kp[i].bp = const_cast<SimpleBasicParticleType *>(&p);
        }
    };
    dump(tkp, tl);
    dump(skp, sl);
    flag_out.assign(tl.size(), GF_BOUND);
    const double cc[6] = {c.cx, c.cy, c.cz, c.cvx, c.cvy, c.cvz};
    const int nb = energy_check(tkp.data(), (int)tl.size(), flag_out.data(), skp.data(), (int)sl.size(), false, cc);
    return nb < 0 ? (last_status() ? last_status() : GF_EDEVICE) : GF_OK;
}

}  // namespace

}  // namespace gf

using namespace gf;

extern "C" int gf_shell_bound(const SimpleBasicParticleType *bp, int np, unsigned char *flag, int32_t *haloid,
                              const int32_t *shellp, const int32_t *shellp_start, const int32_t *shellc,
                              const int32_t *shellc_start, int nshell, int ishell, const Coretype *core,
                              int numcore, const int32_t *order, int norder, int32_t *nmem_out,
                              int32_t *nretest_out) {
    clear_status();
    if (np < 0 || nshell < 0 || ishell < 0 || ishell >= nshell || numcore < 0 || norder < 0 ||
        (np > 0 && (!bp || !flag || !haloid)) || !shellp_start || !shellc_start ||
        (norder > 0 && (!order || !core))) {
        set_status(GF_EINVAL, "gf_shell_bound: invalid arguments");
        return GF_EINVAL;
    }
    for (int j = 0; j < norder; j++)
        if (order[j] < 0 || order[j] >= numcore) {
            set_status(GF_EINVAL, "gf_shell_bound: core id out of range");
            return GF_EINVAL;
        }
    if (nretest_out) *nretest_out = 0;
    const int32_t *sp = shellp + shellp_start[ishell];
    const int nsp = shellp_start[ishell + 1] - shellp_start[ishell];
    // ---- candidates and sources of every core, at the start of the shell
    std::vector<CoreWork> w((size_t)norder);
    std::vector<int32_t> rem;  // REMAINING particles, index order
    for (int i = 0; i < np; i++)
        if (flag[i] & kWpRemaining) rem.push_back(i);
    std::vector<std::vector<int32_t>> members((size_t)numcore);
    for (int i = 0; i < np; i++)
        if (haloid[i] >= 0 && haloid[i] < numcore) members[haloid[i]].push_back(i);
    int64_t ntgt = 0, nsrc = 0;
    for (int j = 0; j < norder; j++) {
        CoreWork &cw = w[j];
        cw.core = order[j];
        const Coretype &c = core[cw.core];
        for (int t = 0; t < nsp; t++)
            if (!(flag[sp[t]] & kWpBound) && within(bp[sp[t]], c)) cw.cand.push_back(sp[t]);
        for (int32_t t : rem)
            if (within(bp[t], c)) cw.cand.push_back(t);
        cw.src = members[cw.core];
        for (int s = ishell + 1; s < nshell; s++)
            for (int q = shellc_start[s]; q < shellc_start[s + 1]; q++)
                if (shellc[q] == cw.core) {
                    cw.src.insert(cw.src.end(), shellp + shellp_start[s], shellp + shellp_start[s + 1]);
                    break;
                }
        if (!cw.cand.empty() && cw.src.empty()) {
            set_status(GF_EINVAL, "gf_shell_bound: core %d has targets but no source particles", cw.core);
            return GF_EINVAL;
        }
        cw.toff = ntgt;
        ntgt += (int64_t)cw.cand.size();
        nsrc += cw.cand.empty() ? 0 : (int64_t)cw.src.size();
    }
    // ---- one batched energy test of every (candidate, core) pair
    std::vector<unsigned char> bflag((size_t)ntgt);
    if (ntgt > 0) {
        gf_ctx *ctx = default_ctx();
        if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
        std::lock_guard<std::mutex> lk(ctx->lock);
        // the cores with targets, as the "halos" of a batch of source sets
        std::vector<int> live;
        for (int j = 0; j < norder; j++)
            if (!w[j].cand.empty()) live.push_back(j);
        const int nl = (int)live.size();
        std::vector<int64_t> ps((size_t)nl + 1, 0);
        std::vector<int32_t> ntg((size_t)nl), tcore((size_t)ntgt);
        std::vector<double> sr((size_t)nsrc * 3), tr((size_t)ntgt * 3), centre((size_t)nl * 6);
        std::vector<float> sm((size_t)nsrc), tv((size_t)ntgt * 3);
        int64_t so = 0;
        for (int l = 0; l < nl; l++) {
            const CoreWork &cw = w[live[l]];
            for (int32_t s : cw.src) {
                sr[3 * so] = bp[s].x;
                sr[3 * so + 1] = bp[s].y;
                sr[3 * so + 2] = bp[s].z;
                sm[so] = (float)bp[s].mass;  // Kptype.mass
                so++;
            }
            ps[l + 1] = so;
            ntg[l] = (int32_t)cw.cand.size();
            for (size_t t = 0; t < cw.cand.size(); t++) {
                const SimpleBasicParticleType &p = bp[cw.cand[t]];
                const int64_t i = cw.toff + (int64_t)t;
                tr[3 * i] = p.x;
                tr[3 * i + 1] = p.y;
                tr[3 * i + 2] = p.z;
                tv[3 * i] = (float)p.vx;
                tv[3 * i + 1] = (float)p.vy;
                tv[3 * i + 2] = (float)p.vz;
                tcore[i] = l;
            }
            const Coretype &c = core[cw.core];
            const double cc[6] = {c.cx, c.cy, c.cz, c.cvx, c.cvy, c.cvz};
            for (int a = 0; a < 6; a++) centre[6 * l + a] = cc[a];
        }
        auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
        const size_t b_ps = al(ps.size() * 8), b_ntg = al(ntg.size() * 4), b_tc = al(tcore.size() * 4),
                     b_sr = al(sr.size() * 8), b_tr = al(tr.size() * 8), b_ce = al(centre.size() * 8),
                     b_sm = al(sm.size() * 4), b_tv = al(tv.size() * 4);
        const size_t hbytes = b_ps + b_ntg + b_tc + b_sr + b_tr + b_ce + b_sm + b_tv;
        const size_t dbytes = hbytes + al((size_t)nsrc * 16) + al((size_t)ntgt * 16) + al((size_t)ntgt * 4) +
                              al((size_t)ntgt) + 512;
        GF_TRY(ctx->pin[2].reserve(hbytes));
        GF_TRY(ctx->particles.reserve(dbytes));
        GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // the pinned buffer may feed an earlier copy
        char *h = ctx->pin[2].as<char>();
        size_t off = 0;
        auto put = [&](const void *src, size_t bytes, size_t cap) {
            memcpy(h + off, src, bytes);
            const size_t at = off;
            off += cap;
            return at;
        };
        const size_t o_ps = put(ps.data(), ps.size() * 8, b_ps), o_ntg = put(ntg.data(), ntg.size() * 4, b_ntg),
                     o_tc = put(tcore.data(), tcore.size() * 4, b_tc), o_sr = put(sr.data(), sr.size() * 8, b_sr),
                     o_tr = put(tr.data(), tr.size() * 8, b_tr), o_ce = put(centre.data(), centre.size() * 8, b_ce),
                     o_sm = put(sm.data(), sm.size() * 4, b_sm), o_tv = put(tv.data(), tv.size() * 4, b_tv);
        char *d = ctx->particles.as<char>();
        GF_CUDA_TRY(cudaMemcpyAsync(d, h, hbytes, cudaMemcpyHostToDevice, ctx->stream));
        float4 *spos = reinterpret_cast<float4 *>(d + hbytes);
        float4 *tpos = reinterpret_cast<float4 *>(d + hbytes + al((size_t)nsrc * 16));
        float *dpe = reinterpret_cast<float *>(d + hbytes + al((size_t)nsrc * 16) + al((size_t)ntgt * 16));
        unsigned char *dflag = reinterpret_cast<unsigned char *>(dpe) + al((size_t)ntgt * 4);
        const int64_t *dps = reinterpret_cast<const int64_t *>(d + o_ps);
        pos_kernel<<<grid_of(nsrc), 256, 0, ctx->stream>>>(nsrc, reinterpret_cast<const double *>(d + o_sr),
                                                            reinterpret_cast<const float *>(d + o_sm), spos);
        GF_LAUNCH_CHECK();
        pos_kernel<<<grid_of(ntgt), 256, 0, ctx->stream>>>(ntgt, reinterpret_cast<const double *>(d + o_tr),
                                                            nullptr, tpos);
        GF_LAUNCH_CHECK();
        const float theta2 = 0.5f;  // subhaloden.mod6.c:1541
        GF_TRY(build_tree(ctx, nl, nsrc, dps, spos, theta2, 0, &ctx->last_tree));
        const gf_physics &ph = physics();
        const PotentialParams pp = potential_params(theta2, kDirectBelow, ph.potentfact, 1);
        GF_TRY(launch_external_potential(ctx, ctx->last_tree, dps, ntgt, tpos,
                                         reinterpret_cast<const int32_t *>(d + o_tc),
                                         reinterpret_cast<const int32_t *>(d + o_ntg), pp, dpe, nullptr));
        energy_cores_kernel<<<grid_of(ntgt), 256, 0, ctx->stream>>>(
            ntgt, reinterpret_cast<const double *>(d + o_tr), reinterpret_cast<const float *>(d + o_tv), dpe,
            reinterpret_cast<const int32_t *>(d + o_tc), reinterpret_cast<const double *>(d + o_ce),
            ph.r1kineticfact, ph.r2kineticfact, dflag);
        GF_LAUNCH_CHECK();
        GF_CUDA_TRY(cudaMemcpyAsync(bflag.data(), dflag, (size_t)ntgt, cudaMemcpyDeviceToHost, ctx->stream));
        GF_TRY(check_device_errors(ctx));
    }
    // ---- the reference's loop, replayed in its order
    std::vector<int32_t> tl, pos_of;
    std::vector<unsigned char> fl;
    for (int j = 0; j < norder; j++) {
        CoreWork &cw = w[j];
        const Coretype &c = core[cw.core];
        // GetShellParticleFromRestParticleLIST now: shell particles not bound,
        // then REMAINING ones (a shell particle an earlier core left unbound is
        // both), cut at the tidal radius
        tl.clear();
        for (int t = 0; t < nsp; t++)
            if (!(flag[sp[t]] & kWpBound) && within(bp[sp[t]], c)) tl.push_back(sp[t]);
        for (int i = 0; i < np; i++)
            if ((flag[i] & kWpRemaining) && within(bp[i], c)) tl.push_back(i);
        if (nmem_out) nmem_out[j] = 0;
        if (tl.empty()) continue;
        const bool direct_now = (int)tl.size() < kDirectBelow;
        const bool direct_batch = (int)cw.cand.size() < kDirectBelow;
        if (direct_now != direct_batch) {
            GF_TRY(retest_core(bp, tl, cw.src, c, fl));
            if (nretest_out) (*nretest_out)++;
        } else {
            // every target is a candidate of the start of the shell: its test
            // from the batch (candidates are unique, in cw.cand order)
            fl.resize(tl.size());
            // candidate position by particle index
            pos_of.assign((size_t)np, -1);
            for (size_t q = 0; q < cw.cand.size(); q++) pos_of[cw.cand[q]] = (int32_t)q;
            for (size_t t = 0; t < tl.size(); t++) {
                const int32_t q = pos_of[tl[t]];
                if (q < 0) {
                    set_status(GF_EDEVICE, "gf_shell_bound: a target of core %d was not a candidate", cw.core);
                    return GF_EDEVICE;
                }
                fl[t] = bflag[(size_t)(cw.toff + q)];
            }
        }
        // MULTIHALOSHELL (:1708-1721), then the caller's marking (:3090-3095)
        int nmem = 0;
        for (size_t t = 0; t < tl.size(); t++) {
            const int32_t b = tl[t];
            if (fl[t] == GF_BOUND) {
                flag[b] |= kWpBound;
                nmem++;
            } else {
                flag[b] |= kWpRemaining;
                flag[b] &= (unsigned char)~kWpBound;
                haloid[b] = kNotMember;
            }
        }
        for (size_t t = 0; t < tl.size(); t++)
            if (fl[t] == GF_BOUND) {
                flag[tl[t]] |= kWpBound;
                flag[tl[t]] &= (unsigned char)~kWpRemaining;
                haloid[tl[t]] = cw.core;
            }
        if (nmem_out) nmem_out[j] = nmem;
    }
    // UnboundShellP2Rest (:2111-2121)
    for (int t = 0; t < nsp; t++)
        if (!(flag[sp[t]] & kWpBound)) {
            haloid[sp[t]] = kNotMember;
            flag[sp[t]] |= kWpRemaining;
        }
    return GF_OK;
}

// ------------------------------------------------------------------ BOUNDITER
// One pass of subhalo_den's BOUNDITER loop over the cores
// (subhaloden.mod6.c:3118-3172).  For core j (in the order of the pass's
// qsort by member count; cores without members are skipped)
// GetMemberRestParticleList (:2722-2768) takes every particle within Rtidal
// that is free, the core's own, or a non-core member of a core later in the
// order, and releases the core's own members beyond Rtidal; SINGLEHALO
// (:1859-1880) tests the list against its own potential (CheckSelfTE,
// :1730-1820: Self_Halo_Potent and the KE about the list's stellar centre)
// and moves the bound particles to the core and its unbound members out.
// A core's list depends on the cores before it, so the lists are predicted
// from the state at the start of a batch, every predicted list is tested in
// one GPU pass (one octree per list), and the loop is replayed in the
// reference's order: a core whose actual list equals its prediction takes
// the batch's result; at the first core whose list changed, a new batch
// starts from that core (its prediction is then exact, so every batch
// settles at least one core).
namespace gf {

namespace {

constexpr unsigned char kWpCoreBit = 0x04;  // WP_CORE, :183

bool within_f(const SimpleBasicParticleType &p, float cx, float cy, float cz, float rt2) {
    const float tmpx = (float)(p.x - cx);
    const float tmpy = (float)(p.y - cy);
    const float tmpz = (float)(p.z - cz);
    const float dist2 = tmpx * tmpx + tmpy * tmpy + tmpz * tmpz;
    return dist2 < rt2;
}

// GetMemberRestParticleList (:2722-2768); `release` applies its side effect
// (the core's own members beyond Rtidal become free and REMAINING).
void member_rest_list(const SimpleBasicParticleType *bp, int np, unsigned char *flag, int32_t *haloid,
                      const Coretype &c, int hid, const std::vector<int> &later_rank, int now, bool release,
                      std::vector<int32_t> &list) {
    const float rt2 = c.Rtidal * c.Rtidal;
    list.clear();
    for (int i = 0; i < np; i++) {
        if (within_f(bp[i], c.cx, c.cy, c.cz, rt2)) {
            list.push_back(i);
        } else if (release && haloid[i] == hid) {
            haloid[i] = kNotMember;
            flag[i] |= kWpRemaining;
        }
    }
    size_t keep = 0;
    for (size_t q = 0; q < list.size(); q++) {
        const int32_t i = list[q];
        const int32_t id = haloid[i];
        bool ok = id == kNotMember || id == hid;
        // a non-core member of a core later in the order (:2758-2763)
        if (!ok && !(flag[i] & kWpCoreBit) && id >= 0 && id < (int32_t)later_rank.size() && later_rank[id] > now)
            ok = true;
        if (ok) list[keep++] = i;
    }
    list.resize(keep);
}

}  // namespace

}  // namespace gf

extern "C" int gf_bound_pass(const SimpleBasicParticleType *bp, int np, unsigned char *flag, int32_t *haloid,
                             const Coretype *core, int numcore, const int32_t *order, const int32_t *nmem,
                             int norder, int32_t *nbound_out, int32_t *nbatch_out) {
    clear_status();
    if (np < 0 || numcore < 0 || norder < 0 || (np > 0 && (!bp || !flag || !haloid)) ||
        (norder > 0 && (!order || !nmem || !core))) {
        set_status(GF_EINVAL, "gf_bound_pass: invalid arguments");
        return GF_EINVAL;
    }
    // rank of each core in the order (score index); -1 for cores not in it
    std::vector<int> rank((size_t)numcore, -1);
    for (int j = 0; j < norder; j++) {
        if (order[j] < 0 || order[j] >= numcore) {
            set_status(GF_EINVAL, "gf_bound_pass: core id out of range");
            return GF_EINVAL;
        }
        rank[order[j]] = j;
    }
    if (nbatch_out) *nbatch_out = 0;
    for (int j = 0; j < norder; j++)
        if (nbound_out) nbound_out[j] = 0;
    std::vector<std::vector<int32_t>> pred((size_t)norder);
    std::vector<int64_t> poff((size_t)norder, -1);
    std::vector<int32_t> actual;
    std::vector<unsigned char> bflag;
    int start = 0;
    while (start < norder) {
        // ---- predicted lists of the cores from `start`, from the current state
        int64_t ntot = 0;
        std::vector<int> live;
        for (int j = start; j < norder; j++) {
            pred[j].clear();
            poff[j] = -1;
            if (nmem[j] == 0) continue;
            member_rest_list(bp, np, flag, haloid, core[order[j]], order[j], rank, j, false, pred[j]);
            if (pred[j].empty()) continue;
            poff[j] = ntot;
            ntot += (int64_t)pred[j].size();
            live.push_back(j);
        }
        if (live.empty()) break;
        // ---- one GPU pass: self potential of every list, KE about its stellar centre
        bflag.assign((size_t)ntot, GF_BOUND);
        {
            gf_ctx *ctx = default_ctx();
            if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
            std::lock_guard<std::mutex> lk(ctx->lock);
            const int nl = (int)live.size();
            std::vector<int64_t> ps((size_t)nl + 1, 0);
            std::vector<int32_t> tcore((size_t)ntot);
            std::vector<double> r((size_t)ntot * 3), centre((size_t)nl * 6);
            std::vector<float> m((size_t)ntot), v((size_t)ntot * 3);
            for (int l = 0; l < nl; l++) {
                const std::vector<int32_t> &L = pred[live[l]];
                // CheckSelfTE's centre (:1770-1784): the list's stars, mass
                // weighted, in list order (0/0 without stars, as the reference)
                double c[6] = {0, 0, 0, 0, 0, 0}, tmass = 0;
                for (size_t q = 0; q < L.size(); q++) {
                    const SimpleBasicParticleType &p = bp[L[q]];
                    const int64_t i = poff[live[l]] + (int64_t)q;
                    const float mf = (float)p.mass, vx = (float)p.vx, vy = (float)p.vy, vz = (float)p.vz;
                    r[3 * i] = p.x;
                    r[3 * i + 1] = p.y;
                    r[3 * i + 2] = p.z;
                    m[i] = mf;
                    v[3 * i] = vx;
                    v[3 * i + 1] = vy;
                    v[3 * i + 2] = vz;
                    tcore[i] = l;
                    if (p.type == GF_TYPE_STAR) {
                        c[0] += p.x * mf;
                        c[1] += p.y * mf;
                        c[2] += p.z * mf;
                        c[3] += (double)vx * mf;
                        c[4] += (double)vy * mf;
                        c[5] += (double)vz * mf;
                        tmass += mf;
                    }
                }
                for (int a = 0; a < 6; a++) centre[6 * l + a] = c[a] / tmass;
                ps[l + 1] = ps[l] + (int64_t)L.size();
            }
            auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
            const size_t b_ps = al(ps.size() * 8), b_tc = al(tcore.size() * 4), b_r = al(r.size() * 8),
                         b_ce = al(centre.size() * 8), b_m = al(m.size() * 4), b_v = al(v.size() * 4);
            const size_t hbytes = b_ps + b_tc + b_r + b_ce + b_m + b_v;
            const size_t dbytes = hbytes + al((size_t)ntot * 16) + al((size_t)ntot * 4) + al((size_t)ntot) + 512;
            GF_TRY(ctx->pin[2].reserve(hbytes));
            GF_TRY(ctx->particles.reserve(dbytes));
            GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // the pinned buffer may feed an earlier copy
            char *h = ctx->pin[2].as<char>();
            size_t off = 0;
            auto put = [&](const void *src, size_t bytes, size_t cap) {
                memcpy(h + off, src, bytes);
                const size_t at = off;
                off += cap;
                return at;
            };
            const size_t o_ps = put(ps.data(), ps.size() * 8, b_ps), o_tc = put(tcore.data(), tcore.size() * 4, b_tc),
                         o_r = put(r.data(), r.size() * 8, b_r), o_ce = put(centre.data(), centre.size() * 8, b_ce),
                         o_m = put(m.data(), m.size() * 4, b_m), o_v = put(v.data(), v.size() * 4, b_v);
            char *d = ctx->particles.as<char>();
            GF_CUDA_TRY(cudaMemcpyAsync(d, h, hbytes, cudaMemcpyHostToDevice, ctx->stream));
            float4 *pos = reinterpret_cast<float4 *>(d + hbytes);
            float *dpe = reinterpret_cast<float *>(d + hbytes + al((size_t)ntot * 16));
            unsigned char *dflag = reinterpret_cast<unsigned char *>(dpe) + al((size_t)ntot * 4);
            const int64_t *dps = reinterpret_cast<const int64_t *>(d + o_ps);
            pos_kernel<<<grid_of(ntot), 256, 0, ctx->stream>>>(ntot, reinterpret_cast<const double *>(d + o_r),
                                                                reinterpret_cast<const float *>(d + o_m), pos);
            GF_LAUNCH_CHECK();
            const float theta2 = 0.5f;  // subhaloden.mod6.c:1481
            GF_TRY(build_tree(ctx, nl, ntot, dps, pos, theta2, 0, &ctx->last_tree));
            const gf_physics &ph = physics();
            // Self_Halo_Potent sums directly below 100 particles (:1485)
            const PotentialParams pp = potential_params(theta2, 100, ph.potentfact, 1);
            GF_TRY(launch_self_potential(ctx, ctx->last_tree, dps, pp, dpe, nullptr, nullptr));
            energy_cores_kernel<<<grid_of(ntot), 256, 0, ctx->stream>>>(
                ntot, reinterpret_cast<const double *>(d + o_r), reinterpret_cast<const float *>(d + o_v), dpe,
                reinterpret_cast<const int32_t *>(d + o_tc), reinterpret_cast<const double *>(d + o_ce),
                ph.r1kineticfact, ph.r2kineticfact, dflag);
            GF_LAUNCH_CHECK();
            GF_CUDA_TRY(cudaMemcpyAsync(bflag.data(), dflag, (size_t)ntot, cudaMemcpyDeviceToHost, ctx->stream));
            GF_TRY(check_device_errors(ctx));
        }
        if (nbatch_out) (*nbatch_out)++;
        // ---- the reference's order
        int next = norder;
        for (int j = start; j < norder; j++) {
            if (nmem[j] == 0) continue;
            const int hid = order[j];
            member_rest_list(bp, np, flag, haloid, core[hid], hid, rank, j, true, actual);
            if (actual.empty()) continue;
            if (actual != pred[j]) {  // an earlier core changed this list: a new batch from here
                next = j;
                break;
            }
            int nb = 0;
            for (size_t q = 0; q < actual.size(); q++) {  // SINGLEHALO's marking (:1868-1877)
                const int32_t i = actual[q];
                if (bflag[(size_t)(poff[j] + (int64_t)q)] == GF_BOUND) {
                    haloid[i] = hid;
                    flag[i] &= (unsigned char)~kWpRemaining;
                    nb++;
                } else if (haloid[i] == hid) {
                    haloid[i] = kNotMember;
                    flag[i] |= kWpRemaining;
                }
            }
            if (nbound_out) nbound_out[j] = nb;
        }
        start = next;
    }
    return GF_OK;
}
