// The reference's per-particle tree API, on the GPU:
//
//   new_Make_Tree_Near (NewGalFinder/nnost.c:199-254)  kNN tree build
//   Find_Near          (nnost.c:375-422)               k nearest of one point
//   Make_Tree          (ost.c:642-699)                 potential tree build
//   treeplumpotential  (ost.c:226-251)                 tree potential at one point
//
// The builders build libgf's centre-of-mass octree of the caller's particles
// on the device (the reference's node rule: octants split at the centre of
// mass, a child node for >= 10 particles when the node is larger than
// 0.5e-6) and write it into the caller's TStruct array in the reference's
// threaded layout, relinking the caller's TPtlStruct siblings, so that the
// reference's own walks work on it.  Node moments (mass, centre of mass,
// size, second moments) are evaluated in FP64 from the caller's FP64
// positions; node sizes therefore bound every particle of the node.
//
// The per-point queries are called by the reference inside OpenMP loops over
// every particle of the tree (findsphdensity, nnost.c:609-628; the potential
// drivers).  The first query on a tree answers every particle of the tree in
// one launch and keeps the rows on the host; later queries at a particle's
// position (matched by its exact FP64 coordinates) copy their row, and any
// other point runs a one-point launch.  All of it is serialised by one mutex,
// so the entry points are safe to call from many threads.
//
//   * Find_Near: exact k nearest (k <= 32) in FP64 from the FP64 positions,
//     distances rounded as the reference's (dx*dx + dy*dy) + dz*dz; a warp per
//     query walks the octree with FP64 node boxes.  Equal distances are
//     ordered by particle index (the reference keeps its walk order).
//   * treeplumpotential: the Barnes-Hut kernel of the stage (gf_potent.cu) on
//     the same octree: FP64 opening decisions |p - com|^2 < dist2/theta2,
//     exact cell and particle terms, compensated sums.
//
// This translation unit is compiled with --fmad=false.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "gf_fp64.cuh"
#include "gf_ref_types.h"

namespace gf {

namespace {

static_assert(sizeof(TPtlStruct) == 56, "TPtlStruct layout (tree.h:72-77)");
static_assert(sizeof(TStruct) == 176, "TStruct layout (tree.h:79-91)");
static_assert(sizeof(particle) == 40, "particle layout (tree.h:145-149)");

constexpr int kMaxNear = 32;  // MAX_NUM_NEAR, tree.h:20

__global__ void pack_f4(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, const float *__restrict__ m, float4 *__restrict__ out) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        out[p] = make_float4((float)x[p], (float)y[p], (float)z[p], m ? m[p] : 0.f);
}

int grid_for(int64_t n, int block) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + block - 1) / block, (int64_t)sm_count() * 16));
}

// ---------------------------------------------------------------- tree cache
struct PosKey {
    uint64_t x, y, z;
    bool operator==(const PosKey &o) const { return x == o.x && y == o.y && z == o.z; }
};
struct PosHash {
    size_t operator()(const PosKey &k) const {
        uint64_t h = k.x * 0x9E3779B97F4A7C15ull;
        h ^= (k.y + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2));
        h ^= (k.z + 0x85EBCA77C2B2AE63ull + (h << 6) + (h >> 2));
        return (size_t)h;
    }
};
PosKey key_of(double x, double y, double z) {
    PosKey k;
    memcpy(&k.x, &x, 8);
    memcpy(&k.y, &y, 8);
    memcpy(&k.z, &z, 8);
    return k;
}

// A tree the per-point queries answer from: the caller's arrays it belongs
// to, its particle set (indices into the caller's TPtlStruct array), a
// fingerprint of its root node, and the rows answered so far.
struct Entry {
    const void *tree = nullptr, *ptl = nullptr;
    std::vector<int32_t> set;            // set order -> index into ptl
    std::vector<double> x, y, z;         // FP64 positions, set order
    std::vector<float> m;                // float masses, set order
    unsigned char fp[64];                // fingerprint of the caller's root node
    std::unordered_map<PosKey, int32_t, PosHash> where;  // position -> set index
    int knn_k = 0;                       // k of the cached kNN rows (0: none)
    std::vector<int32_t> knn_idx, knn_n; // rows (indices into ptl) and their lengths
    std::vector<double> knn_d2;
    float pot_theta2 = -1.f;             // theta2 of the cached potentials (<0: none)
    std::vector<float> pot;
    uint64_t serial = 0;
};

struct State {
    std::mutex lock;
    gf_ctx *ctx = nullptr;               // device tree of the resident entry
    std::vector<Entry *> entries;        // most recent first
    Entry *resident = nullptr;           // entry whose tree is on the device
    float resident_theta2 = 0.f;
    int32_t root = 0, rend = 0, nnode = 0;
    DevBuf dpos, dnodes, dq, dout;       // FP64 particles (tree order), RefNodes, queries, outputs
    HostPinned hstage;
    uint64_t serial = 0;
};
State &state() {
    static State s;
    return s;
}
constexpr size_t kMaxEntries = 4;
constexpr int64_t kMaxCachedRowEntries = int64_t(1) << 25;  // rows kept on the host: n*k <= 32M

void fingerprint(const TStruct *t, unsigned char *fp) {
    memset(fp, 0, 64);
    memcpy(fp, &t->daughter, sizeof(void *));
    memcpy(fp + 8, &t->mass, 8);
    memcpy(fp + 16, &t->monox, 8);
    memcpy(fp + 24, &t->monoy, 8);
    memcpy(fp + 32, &t->monoz, 8);
    memcpy(fp + 40, &t->Nparticle, 4);
    memcpy(fp + 48, &t->dist, 8);
}

int ensure_ctx(State &S) {
    if (S.ctx) {
        GF_CUDA_TRY(cudaSetDevice(S.ctx->device));
        return GF_OK;
    }
    gf_ctx *d = default_ctx();  // picks the device the drop-ins use
    if (!d) return last_status() ? last_status() : GF_EDEVICE;
    GF_TRY(gf_ctx_create(&S.ctx, d->device, nullptr));
    return GF_OK;
}

// Builds the device octree of entry e (FP32 positions, as the stage) with its
// FP64 node moments; leaves knn nodes in S.ctx->last_tree and RefNodes in S.dnodes.
int build_device_tree(State &S, Entry *e, float theta2) {
    gf_ctx *ctx = S.ctx;
    const int64_t n = (int64_t)e->set.size();
    // host staging: x, y, z (FP64), mass (float), pstart
    const size_t dbytes = (size_t)n * sizeof(double);
    const size_t fbytes = (size_t)n * sizeof(float);
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t off_m = 3 * al(dbytes), off_ps = off_m + al(fbytes), off_set = off_ps + 256,
                 total = off_set + al((size_t)n * sizeof(int32_t));
    GF_TRY(S.hstage.reserve(total));
    GF_TRY(ctx->particles.reserve(total + al((size_t)n * sizeof(float4))));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // the staging buffer may feed a copy
    char *h = S.hstage.as<char>();
    memcpy(h, e->x.data(), dbytes);
    memcpy(h + al(dbytes), e->y.data(), dbytes);
    memcpy(h + 2 * al(dbytes), e->z.data(), dbytes);
    memcpy(h + off_m, e->m.data(), fbytes);
    int64_t ps[2] = {0, n};
    memcpy(h + off_ps, ps, sizeof(ps));
    memcpy(h + off_set, e->set.data(), (size_t)n * sizeof(int32_t));
    char *d = ctx->particles.as<char>();
    GF_CUDA_TRY(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, ctx->stream));
    const double *dx = reinterpret_cast<const double *>(d);
    const double *dy = reinterpret_cast<const double *>(d + al(dbytes));
    const double *dz = reinterpret_cast<const double *>(d + 2 * al(dbytes));
    const float *dm = reinterpret_cast<const float *>(d + off_m);
    const int64_t *dps = reinterpret_cast<const int64_t *>(d + off_ps);
    const int32_t *dset = reinterpret_cast<const int32_t *>(d + off_set);
    float4 *pos = reinterpret_cast<float4 *>(d + total);
    pack_f4<<<grid_for(n, 256), 256, 0, ctx->stream>>>(n, dx, dy, dz, dm, pos);
    GF_LAUNCH_CHECK();
    GF_TRY(build_tree(ctx, 1, n, dps, pos, theta2, 0, &ctx->last_tree));
    const TreeView &t = ctx->last_tree;
    GF_TRY(S.dpos.reserve((size_t)n * sizeof(double4) + (size_t)n * sizeof(int32_t) + 512));
    double4 *tp = S.dpos.as<double4>();
    int32_t *tidx = reinterpret_cast<int32_t *>(tp + n);
    gather_tree_order<<<grid_for(n, 256), 256, 0, ctx->stream>>>(n, t.perm, dx, dy, dz, dm, nullptr, dset,
                                                                   tp, tidx);
    GF_LAUNCH_CHECK();
    GF_TRY(S.dnodes.reserve((size_t)t.nnode * sizeof(RefNode)));
    ref_node_kernel<<<grid_for((int64_t)t.nnode * 32, 256), 256, 0, ctx->stream>>>(
        t.nnode, t.knn, tp, S.dnodes.as<RefNode>());
    GF_LAUNCH_CHECK();
    int32_t rr[2];
    GF_CUDA_TRY(cudaMemcpyAsync(&rr[0], t.root, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(&rr[1], t.rend, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    GF_TRY(check_device_errors(ctx));  // synchronises
    S.root = rr[0];
    S.rend = rr[1];
    S.nnode = t.nnode;
    S.resident = e;
    S.resident_theta2 = theta2;
    return GF_OK;
}

// Writes the resident device tree into the caller's arrays in the reference's
// threaded layout (see the file comment); returns the node count.
int export_tree(State &S, Entry *e, TStruct *T, size_t nnode_cap, TPtlStruct *ptl, double thetasq) {
    gf_ctx *ctx = S.ctx;
    const int nn = S.rend - S.root;
    if ((size_t)nn > nnode_cap) {
        set_status(GF_ENOMEM, "the tree of %zu particles has %d nodes; the caller's TStruct array holds %zu",
                   e->set.size(), nn, nnode_cap);
        return GF_ENOMEM;
    }
    const int64_t n = (int64_t)e->set.size();
    std::vector<KnnNode> kn(nn);
    std::vector<RefNode> rn(nn);
    std::vector<int32_t> perm(n);
    const TreeView &t = ctx->last_tree;
    GF_CUDA_TRY(cudaMemcpyAsync(kn.data(), t.knn + S.root, nn * sizeof(KnnNode), cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(rn.data(), S.dnodes.as<RefNode>() + S.root, nn * sizeof(RefNode),
                                cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(perm.data(), t.perm, n * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    auto ptl_of = [&](int32_t tree_pos) { return ptl + e->set[perm[tree_pos]]; };
    for (int64_t j = 0; j < n; j++) ptl[e->set[j]].type = GF_TYPE_PTL;
    T[0].sibling = nullptr;
    for (int i = 0; i < nn; i++) {
        TStruct &N = T[i];
        const KnnNode &k = kn[i];
        const RefNode &r = rn[i];
        N.type = GF_TYPE_TREE;
        N.L = 0;
        N.x0 = N.y0 = N.z0 = 0;
        N.mass = r.mass;
        N.Nparticle = k.count;
        N.monox = r.com[0];
        N.monoy = r.com[1];
        N.monoz = r.com[2];
        N.dist2 = r.dist2;
        N.dist = sqrt(r.dist2);
        for (int c = 0; c < 6; c++) N.quad[c] = r.q[c];
        N.trQ = r.q[0] + r.q[1] + r.q[2];
        N.dist_over_thetasq = thetasq > 0 ? r.dist2 / thetasq : 0.0;
        // offspring: loose particles, then child nodes (preorder i+1, then by skip)
        void *first = nullptr;
        void **link = &first;
        for (int j = 0; j < k.lcount; j++) {
            TPtlStruct *p = ptl_of(k.lstart + j);
            *link = p;
            link = &p->sibling;
        }
        const int skip = k.skip - S.root;
        for (int c = i + 1; c < skip; c = kn[c].skip - S.root) {
            *link = &T[c];
            link = &T[c].sibling;
        }
        *link = N.sibling;  // the last offspring continues at the node's own sibling
        N.daughter = first;
    }
    fingerprint(&T[0], e->fp);
    return nn;
}

void drop_entry(State &S, Entry *e) {
    if (S.resident == e) S.resident = nullptr;
    delete e;
}

Entry *new_entry(State &S, const void *tree, const void *ptl) {
    // a new tree of the same arrays replaces the old one; the oldest go beyond the limit
    for (auto it = S.entries.begin(); it != S.entries.end();) {
        if ((*it)->tree == tree && (*it)->ptl == ptl) {
            drop_entry(S, *it);
            it = S.entries.erase(it);
        } else {
            ++it;
        }
    }
    while (S.entries.size() >= kMaxEntries) {
        drop_entry(S, S.entries.back());
        S.entries.pop_back();
    }
    Entry *e = new Entry();
    e->tree = tree;
    e->ptl = ptl;
    e->serial = ++S.serial;
    S.entries.insert(S.entries.begin(), e);
    return e;
}

void fill_particles(Entry *e, const TPtlStruct *ptl) {
    const size_t n = e->set.size();
    e->x.resize(n);
    e->y.resize(n);
    e->z.resize(n);
    e->m.resize(n);
    e->where.clear();
    e->where.reserve(n * 2);
    for (size_t j = 0; j < n; j++) {
        const TPtlStruct &p = ptl[e->set[j]];
        e->x[j] = p.x;
        e->y[j] = p.y;
        e->z[j] = p.z;
        e->m[j] = (float)p.mass;  // divide_node reads float ptlmass (ost.c:538)
        e->where.emplace(key_of(p.x, p.y, p.z), (int32_t)j);
    }
}

int make_tree(TStruct *T, size_t nnode, TPtlStruct *ptl, size_t np, double thetasq, const char *who) {
    clear_status();
    if (!T || !ptl || np < 1 || nnode < 1 || np > 0x7fffffffULL) {
        set_status(GF_EINVAL, "%s: invalid arguments (np = %zu, nnode = %zu)", who, np, nnode);
        return GF_EINVAL;
    }
    State &S = state();
    std::lock_guard<std::mutex> g(S.lock);
    GF_TRY(ensure_ctx(S));
    Entry *e = new_entry(S, T, ptl);
    e->set.resize(np);
    for (size_t j = 0; j < np; j++) e->set[j] = (int32_t)j;
    fill_particles(e, ptl);
    const float th = thetasq > 0 ? (float)thetasq : 0.5f;
    GF_TRY(build_device_tree(S, e, th));
    const int nn = export_tree(S, e, T, nnode, ptl, thetasq);
    return nn < 0 ? nn : GF_OK;
}

// The entry of a tree the caller passes to a query: one built here (matched
// by its arrays and root fingerprint), or else the particle set gathered by
// walking the caller's threaded tree (built by other code).
Entry *entry_for(State &S, TStruct *tree, TPtlStruct *ptl) {
    unsigned char fp[64];
    fingerprint(tree, fp);
    for (size_t i = 0; i < S.entries.size(); i++) {
        Entry *e = S.entries[i];
        if (e->tree == tree && e->ptl == ptl && memcmp(e->fp, fp, 64) == 0) {
            if (i) std::rotate(S.entries.begin(), S.entries.begin() + i, S.entries.begin() + i + 1);
            return e;
        }
    }
    Entry *e = new_entry(S, tree, ptl);
    // every offspring once: open every node
    const void *p = tree;
    while (p) {
        if (static_cast<const TStruct *>(p)->type == GF_TYPE_TREE) {
            p = static_cast<const TStruct *>(p)->daughter;
        } else {
            const TPtlStruct *q = static_cast<const TPtlStruct *>(p);
            e->set.push_back((int32_t)(q - ptl));
            p = q->sibling;
        }
    }
    fill_particles(e, ptl);
    memcpy(e->fp, fp, 64);
    return e;
}

// kNN rows of n query points (FP64) on the resident tree; host outputs.
int run_knn(State &S, Entry *e, int64_t n, const double *qx, const double *qy, const double *qz, int k,
            int32_t *idx, double *d2, int32_t *cnt) {
    gf_ctx *ctx = S.ctx;
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t qb = al((size_t)n * sizeof(double));
    const size_t ob_i = al((size_t)n * k * sizeof(int32_t)), ob_d = al((size_t)n * k * sizeof(double)),
                 ob_n = al((size_t)n * sizeof(int32_t));
    GF_TRY(S.dq.reserve(3 * qb));
    GF_TRY(S.dout.reserve(ob_i + ob_d + ob_n));
    GF_TRY(S.hstage.reserve(std::max(3 * qb, ob_i + ob_d + ob_n)));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    char *h = S.hstage.as<char>();
    memcpy(h, qx, n * sizeof(double));
    memcpy(h + qb, qy, n * sizeof(double));
    memcpy(h + 2 * qb, qz, n * sizeof(double));
    char *dq = S.dq.as<char>();
    GF_CUDA_TRY(cudaMemcpyAsync(dq, h, 3 * qb, cudaMemcpyHostToDevice, ctx->stream));
    const int64_t np = (int64_t)e->set.size();
    const int32_t *tidx = reinterpret_cast<const int32_t *>(S.dpos.as<double4>() + np);
    char *dout = S.dout.as<char>();
    int32_t *oi = reinterpret_cast<int32_t *>(dout);
    double *od = reinterpret_cast<double *>(dout + ob_i);
    int32_t *on = reinterpret_cast<int32_t *>(dout + ob_i + ob_d);
    const int64_t threads = n * 32;
    knn64_kernel<<<grid_for(threads, 128), 128, 0, ctx->stream>>>(
        n, reinterpret_cast<const double *>(dq), reinterpret_cast<const double *>(dq + qb),
        reinterpret_cast<const double *>(dq + 2 * qb), nullptr, k, ctx->last_tree.root, ctx->last_tree.rend,
        ctx->last_tree.knn, S.dnodes.as<RefNode>(), S.dpos.as<double4>(), tidx, nullptr, oi, od, on, nullptr);
    GF_LAUNCH_CHECK();
    GF_CUDA_TRY(cudaMemcpyAsync(h, dout, ob_i + ob_d + ob_n, cudaMemcpyDeviceToHost, ctx->stream));
    GF_TRY(check_device_errors(ctx));
    memcpy(idx, h, (size_t)n * k * sizeof(int32_t));
    memcpy(d2, h + ob_i, (size_t)n * k * sizeof(double));
    memcpy(cnt, h + ob_i + ob_d, (size_t)n * sizeof(int32_t));
    return GF_OK;
}

// Raw tree potential at n FP32 target points (float4, w unused) or, with
// targets == nullptr, at every particle of the resident tree (set order).
int run_potential(State &S, Entry *e, int64_t n, const float4 *targets, float theta2, float *out) {
    gf_ctx *ctx = S.ctx;
    const TreeView &t = ctx->last_tree;
    PotentialParams pp{};
    pp.theta2 = theta2;
    pp.ndirect = 0;
    pp.potentfact = 0.0;
    pp.add_bg = 0;
    const int64_t *dps = nullptr;
    // pstart of the one halo: the build staged it after the positions
    {
        const int64_t np = (int64_t)e->set.size();
        auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
        const size_t dbytes = (size_t)np * sizeof(double), fbytes = (size_t)np * sizeof(float);
        dps = reinterpret_cast<const int64_t *>(ctx->particles.as<char>() + 3 * al(dbytes) + al(fbytes));
    }
    GF_TRY(S.dout.reserve((size_t)n * sizeof(float) + 512));
    float *draw = S.dout.as<float>();
    if (!targets) {
        GF_TRY(launch_self_potential(ctx, t, dps, pp, nullptr, draw, nullptr));
    } else {
        GF_TRY(S.dq.reserve((size_t)n * (sizeof(float4) + sizeof(int32_t)) + 512));
        float4 *dt = S.dq.as<float4>();
        int32_t *dh = reinterpret_cast<int32_t *>(dt + n);
        GF_CUDA_TRY(cudaMemcpyAsync(dt, targets, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream));
        GF_CUDA_TRY(cudaMemsetAsync(dh, 0, (size_t)n * sizeof(int32_t), ctx->stream));
        GF_TRY(launch_external_potential(ctx, t, dps, n, dt, dh, nullptr, pp, nullptr, draw));
    }
    GF_CUDA_TRY(cudaMemcpyAsync(out, draw, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    return check_device_errors(ctx);
}

int find_near(particle *point, int k, TStruct *tree, TPtlStruct *ptl, float *maxr, long long *nearindx,
              double *DIST2, float *MASS, int *nfound) {
    clear_status();
    *nfound = 0;
    if (!point || !tree || !ptl || !maxr || !nearindx || !DIST2 || !MASS || k < 1 || k > kMaxNear) {
        set_status(GF_EINVAL, "Find_Near: invalid arguments (1 <= Num_neighbor <= %d)", kMaxNear);
        return GF_EINVAL;
    }
    State &S = state();
    std::lock_guard<std::mutex> g(S.lock);
    GF_TRY(ensure_ctx(S));
    Entry *e = entry_for(S, tree, ptl);
    if (e->set.empty()) return GF_OK;
    const int64_t np = (int64_t)e->set.size();
    const bool cache_rows = np * (int64_t)k <= kMaxCachedRowEntries;
    if (cache_rows && e->knn_k != k) {
        if (S.resident != e) GF_TRY(build_device_tree(S, e, 0.5f));
        e->knn_idx.resize((size_t)np * k);
        e->knn_d2.resize((size_t)np * k);
        e->knn_n.resize(np);
        GF_TRY(run_knn(S, e, np, e->x.data(), e->y.data(), e->z.data(), k, e->knn_idx.data(),
                       e->knn_d2.data(), e->knn_n.data()));
        e->knn_k = k;
    }
    int32_t rowi[kMaxNear];
    double rowd[kMaxNear];
    int32_t cnt = 0;
    auto it = cache_rows ? e->where.find(key_of(point->x, point->y, point->z)) : e->where.end();
    if (it != e->where.end()) {
        const int64_t r = it->second;
        cnt = e->knn_n[r];
        memcpy(rowi, &e->knn_idx[r * k], cnt * sizeof(int32_t));
        memcpy(rowd, &e->knn_d2[r * k], cnt * sizeof(double));
    } else {
        if (S.resident != e) GF_TRY(build_device_tree(S, e, 0.5f));
        GF_TRY(run_knn(S, e, 1, &point->x, &point->y, &point->z, k, rowi, rowd, &cnt));
    }
    for (int j = 0; j < cnt; j++) {
        nearindx[j] = rowi[j];
        DIST2[j] = rowd[j];
        MASS[j] = (float)ptl[rowi[j]].mass;
    }
    // INSERT's maxdist = sqrtf(maxdist2) (nnost.c:291): float square root of
    // the k-th squared distance rounded to float
    if (cnt > 0) *maxr = sqrtf((float)rowd[cnt - 1]);
    *nfound = cnt;
    return GF_OK;
}

int plum_potential(particle *p, float theta2, TStruct *tree, TPtlStruct *ptl, float *out) {
    clear_status();
    *out = 0.f;
    if (!p || !tree || !ptl || !(theta2 > 0)) {
        set_status(GF_EINVAL, "treeplumpotential: invalid arguments");
        return GF_EINVAL;
    }
    State &S = state();
    std::lock_guard<std::mutex> g(S.lock);
    GF_TRY(ensure_ctx(S));
    Entry *e = entry_for(S, tree, ptl);
    if (e->set.empty()) return GF_OK;
    const int64_t np = (int64_t)e->set.size();
    if (S.resident != e || S.resident_theta2 != theta2) GF_TRY(build_device_tree(S, e, theta2));
    if (e->pot_theta2 != theta2) {
        e->pot.resize(np);
        GF_TRY(run_potential(S, e, np, nullptr, theta2, e->pot.data()));
        e->pot_theta2 = theta2;
    }
    auto it = e->where.find(key_of(p->x, p->y, p->z));
    if (it != e->where.end()) {
        *out = e->pot[it->second];
        return GF_OK;
    }
    const float4 t = make_float4((float)p->x, (float)p->y, (float)p->z, 0.f);
    return run_potential(S, e, 1, &t, theta2, out);
}

}  // namespace

}  // namespace gf

using namespace gf;

extern "C" {

void new_Make_Tree_Near(TStruct *TREE_START, size_t nnode, TPtlStruct *ptl, size_t np, int recursiveflag) {
    (void)recursiveflag;  // the build is the same for every threading mode
    dropin_exit_on_error(make_tree(TREE_START, nnode, ptl, np, 0.0, "new_Make_Tree_Near"), "new_Make_Tree_Near");
}

void Make_Tree(TStruct *TREE_START, size_t nnode, TPtlStruct *ptl, size_t np, float thetasq, int recursiveflag) {
    (void)recursiveflag;
    if (!(thetasq > 0)) {
        clear_status();
        set_status(GF_EINVAL, "Make_Tree: thetasq must be positive");
        dropin_exit_on_error(GF_EINVAL, "Make_Tree");
        return;
    }
    dropin_exit_on_error(make_tree(TREE_START, nnode, ptl, np, (double)thetasq, "Make_Tree"), "Make_Tree");
}

int Find_Near(particle *point, int Num_neighbor, TStruct *tree, TPtlStruct *ptl, float *maxr,
              long long *nearindx, double *DIST2, float *MASS) {
    int n = 0;
    dropin_exit_on_error(find_near(point, Num_neighbor, tree, ptl, maxr, nearindx, DIST2, MASS, &n), "Find_Near");
    return n;
}

float treeplumpotential(particle *p, float theta2, TStruct *tree, TPtlStruct *ptl) {
    float v = 0.f;
    dropin_exit_on_error(plum_potential(p, theta2, tree, ptl, &v), "treeplumpotential");
    return v;
}

}  // extern "C"
