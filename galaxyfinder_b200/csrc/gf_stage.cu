// The batched density-and-potential stage and the remaining C-ABI entry
// points (kNN/SPH density, tree potential, their reference-signature drop-ins).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gf_tree.cuh"

namespace gf {

namespace {

__global__ void pack_pos_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                                const double *__restrict__ z, const float *__restrict__ mf,
                                const double *__restrict__ md, float4 *__restrict__ pos) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        pos[p] = make_float4((float)x[p], (float)y[p], (float)z[p],
                             mf ? mf[p] : (md ? (float)md[p] : 1.f));
}

__global__ void vec3_pos_kernel(int64_t n, const double *__restrict__ r, const float *__restrict__ m,
                                float4 *__restrict__ pos) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        pos[p] = make_float4((float)r[3 * p], (float)r[3 * p + 1], (float)r[3 * p + 2], m ? m[p] : 0.f);
}

int grid1(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sm_count() * 16)); }


struct EventTimer {
    cudaStream_t s;
    bool on;
    cudaEvent_t ev[16];
    int n = 0;
    EventTimer(cudaStream_t s_, bool on_) : s(s_), on(on_) {
        if (on)
            for (auto &e : ev) cudaEventCreate(&e);
    }
    ~EventTimer() {
        if (on)
            for (auto &e : ev) cudaEventDestroy(e);
    }
    void mark() {
        if (on && n < 16) cudaEventRecord(ev[n++], s);
    }
    float ms(int i) {
        float t = 0;
        if (on && i + 1 < n) cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
        return t;
    }
};

}  // namespace

PotentialParams potential_params(float theta2, int ndirect, double potentfact, int add_bg) {
    const gf_physics &ph = physics();
    PotentialParams pp;
    pp.theta2 = theta2;
    pp.ndirect = ndirect;
    pp.potentfact = potentfact;
    pp.add_bg = add_bg;
    pp.amax = ph.amax;
    pp.a = ph.a;
    pp.omep = ph.omep;
    return pp;
}

}  // namespace gf

using namespace gf;

extern "C" {

int gf_tree_build(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                  const float *pos4_dev, float theta2, int q5_asbuilt, gf_tree_info *info) {
    clear_status();
    if (!ctx || (n > 0 && (!pstart_dev || !pos4_dev)) || nhalo < 0) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    GF_TRY(build_tree(ctx, nhalo, n, pstart_dev, reinterpret_cast<const float4 *>(pos4_dev), theta2,
                      q5_asbuilt, &ctx->last_tree));
    if (info) {
        info->nnode = ctx->last_tree.nnode;
        info->nparticle = n;
        info->nhalo = nhalo;
    }
    return check_device_errors(ctx);
}

int gf_tree_export(gf_ctx *ctx, void *bh_nodes, void *knn_nodes, float *pos4, int32_t *perm,
                   int32_t *root, int32_t *rend) {
    clear_status();
    if (!ctx) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    return export_tree(ctx, ctx->last_tree, knn_nodes, bh_nodes, reinterpret_cast<float4 *>(pos4),
                       perm, root, rend);
}

int gf_knn_density(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                   const float *pos4_dev, int k, int32_t *nearindex, float *dens) {
    clear_status();
    if (!ctx || (n > 0 && (!pstart_dev || !pos4_dev || !nearindex))) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    GF_TRY(build_tree(ctx, nhalo, n, pstart_dev, reinterpret_cast<const float4 *>(pos4_dev), 0.5f,
                      0, &ctx->last_tree));
    GF_TRY(launch_knn(ctx, ctx->last_tree, pstart_dev, reinterpret_cast<const float4 *>(pos4_dev), k,
                      nearindex, dens));
    return check_device_errors(ctx);
}

int gf_bg_potent_device(gf_ctx *ctx, int32_t n, const double *mvir_dev, double *bg_dev) {
    clear_status();
    if (!ctx || n < 0 || (n > 0 && (!mvir_dev || !bg_dev))) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    const PotentialParams pp = potential_params(0.5f, 0, physics().potentfact, 1);
    GF_TRY(launch_bg_eval(ctx, n, mvir_dev, pp, bg_dev));
    return check_device_errors(ctx);
}

int gf_self_potential(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                      const float *pos4_dev, float theta2, int32_t ndirect, double potentfact,
                      int add_bg, float *penergy, float *raw) {
    clear_status();
    if (!ctx || (n > 0 && (!pstart_dev || !pos4_dev))) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    GF_TRY(build_tree(ctx, nhalo, n, pstart_dev, reinterpret_cast<const float4 *>(pos4_dev), theta2,
                      0, &ctx->last_tree));
    PotentialParams pp = potential_params(theta2, ndirect, potentfact, add_bg);
    GF_TRY(launch_self_potential(ctx, ctx->last_tree, pstart_dev, pp, penergy, raw, nullptr));
    return check_device_errors(ctx);
}

}  // extern "C"

namespace gf {

// The stage on ctx (its lock held); `plan`, when given, receives what a
// captured pass needs: the meshes, their cell counts and the octree's shape.
int stage_run_locked(gf_ctx *ctx, const gf_batch *b, const gf_stage_config *cfg, gf_stage_out *o,
                     gf_stage_stats *st, StagePlan *plan) {
    const int64_t n = b->nparticle;
    const int32_t nh = b->nhalo;
    cudaStream_t s = ctx->stream;
    EventTimer tm(s, st != nullptr);
    tm.mark();  // 0
    // ---- 1. halo frames + FP64 recentring (Dump2BP / periodic unwrap)
    GF_TRY(ctx->hid.reserve(sizeof(int32_t) * std::max<int64_t>(n, 1)));
    int32_t *hid = ctx->hid.as<int32_t>();
    GF_TRY(compute_hid(ctx, nh, n, b->pstart, hid));
    std::vector<double> frame, extent;
    GF_TRY(halo_frames(ctx, b, hid, cfg->box, frame, extent));
    const size_t nn = (size_t)std::max<int64_t>(n, 1);
    const size_t dbytes = (nn * sizeof(double) + 255) & ~size_t(255);
    GF_TRY(ctx->tmp[2].reserve(3 * dbytes + nn * sizeof(float4) + 256));
    char *t2 = ctx->tmp[2].as<char>();
    double *xr = o->xr ? o->xr : reinterpret_cast<double *>(t2);
    double *yr = o->yr ? o->yr : reinterpret_cast<double *>(t2 + dbytes);
    double *zr = o->zr ? o->zr : reinterpret_cast<double *>(t2 + 2 * dbytes);
    float4 *pos = reinterpret_cast<float4 *>(t2 + 3 * dbytes);  // 256-byte aligned
    // mesh plan from the recentred extents
    std::vector<gf_mesh_desc> mesh((size_t)std::max(nh, 1));
    int64_t cells = 0, dev_cells = 0;
    std::vector<int32_t> onchip_halos;
    if (cfg->do_mesh) {
        int sp = gf_plan_meshes(nh, extent.data(), &cfg->mesh, mesh.data(), &cells);
        if (sp != GF_OK) return sp;
        // 64^3 meshes run their whole mesh stage on chip; the others are laid
        // out in device memory
        for (int32_t h = 0; h < nh; h++) {
            gf_mesh_desc &m = mesh[h];
            if (cfg->mesh_onchip && !cfg->plain_fp64 && m.nx == kOnChipMesh && m.ny == kOnChipMesh && m.nz == kOnChipMesh) {
                m.ptype = kMeshOnChip;
                m.off = 0;
                onchip_halos.push_back(h);
                continue;
            }
            m.off = dev_cells;
            dev_cells += mesh_cells(m);
            dev_cells = (dev_cells + 63) & ~int64_t(63);  // 256-byte aligned mesh starts
        }
    }
    const size_t frame_bytes = frame.size() * sizeof(double);
    const size_t mesh_bytes = mesh.size() * sizeof(gf_mesh_desc);
    GF_TRY(ctx->mesh.reserve(frame_bytes + mesh_bytes + 512));
    GF_TRY(ctx->pin[1].reserve(frame_bytes + mesh_bytes + 512));
    memcpy(ctx->pin[1].ptr, frame.data(), frame_bytes);
    memcpy(ctx->pin[1].as<char>() + ((frame_bytes + 255) & ~size_t(255)), mesh.data(), mesh_bytes);
    GF_CUDA_TRY(cudaMemcpyAsync(ctx->mesh.ptr, ctx->pin[1].ptr,
                                ((frame_bytes + 255) & ~size_t(255)) + mesh_bytes,
                                cudaMemcpyHostToDevice, s));
    const double *frame_dev = ctx->mesh.as<double>();
    const gf_mesh_desc *mesh_dev =
        reinterpret_cast<const gf_mesh_desc *>(ctx->mesh.as<char>() + ((frame_bytes + 255) & ~size_t(255)));
    GF_TRY(recentre(ctx, b, hid, frame_dev, cfg->box, xr, yr, zr, pos));
    tm.mark();  // 1
    // ---- 2. octree
    const bool need_tree = cfg->knn_k > 0 || cfg->do_potential;
    if (need_tree)
        GF_TRY(build_tree(ctx, nh, n, b->pstart, pos, cfg->theta2, cfg->q5_asbuilt, &ctx->last_tree, nullptr,
                          plan ? &plan->tree : nullptr));
    if (plan) {
        plan->need_tree = need_tree;
        plan->mesh = mesh;
        plan->cells = cells;
        plan->dev_cells = dev_cells;
        plan->onchip = !onchip_halos.empty();
    }
    tm.mark();  // 2
    if (cfg->plain_fp64) {
        const double pf = cfg->potentfact != 0.0 ? cfg->potentfact : physics().potentfact;
        const PotentialParams pp = potential_params(cfg->theta2, cfg->ndirect, pf, cfg->add_bg);
        float ms4[4] = {0, 0, 0, 0};
        GF_TRY(stage_plain_fp64(ctx, b, cfg, o, hid, xr, yr, zr, mesh, mesh_dev, cells, pp, st ? ms4 : nullptr));
        tm.mark();  // 3: the FP64 phases are timed inside
        int status = check_device_errors(ctx);
        if (st) {
            memset(st, 0, sizeof(*st));
            st->nparticle = n;
            st->nhalo = nh;
            st->nnode = need_tree ? ctx->last_tree.nnode : 0;
            st->mesh_cells = cells;
            st->mesh_cells_device = cells;
            st->ms_recentre = tm.ms(0);
            st->ms_tree = tm.ms(1);
            st->ms_knn = ms4[0];
            st->ms_smooth = ms4[1];
            st->ms_findden = ms4[2];
            st->ms_potential = ms4[3];
        }
        return status;
    }
    // ---- 3. kNN + SPH density
    if (cfg->knn_k > 0) {
        if (!o->nearindex) {
            set_status(GF_EINVAL, "knn_k > 0 needs nearindex");
            return GF_EINVAL;
        }
        unsigned long long *kc = nullptr;
        if (st && cfg->count_work) {
            GF_TRY(ctx->tmp[4].reserve(128));
            kc = ctx->tmp[4].as<unsigned long long>() + 4;
            GF_CUDA_TRY(cudaMemsetAsync(kc, 0, 5 * sizeof(unsigned long long), s));
        }
        GF_TRY(launch_knn(ctx, ctx->last_tree, b->pstart, pos, cfg->knn_k, o->nearindex, o->dens_sph, kc));
    }
    tm.mark();  // 3
    // ---- 4. TSC mesh -> smoothing -> findDen
    bool used_box_mode = false;
    if (cfg->do_mesh) {
        GF_TRY(ctx->tmp[3].reserve(sizeof(float) * (size_t)std::max<int64_t>(dev_cells, 1)));
        float *den = ctx->tmp[3].as<float>();
        const double vf = tsc_volfact();
        GF_TRY(ctx->mesh_boxes.reserve(sizeof(int32_t) * kMeshBoxInts * (size_t)std::max(nh, 1)));
        int32_t *boxes = ctx->mesh_boxes.as<int32_t>();
        OnChipMeshes oc;
        if (!onchip_halos.empty()) {
            if (!o->dens_mesh || !volfact_folds(vf)) {
                set_status(GF_EINVAL, "on-chip meshes need dens_mesh and a power-of-two volfact");
                return GF_EINVAL;
            }
            oc.nmesh = (int32_t)onchip_halos.size();
            oc.halos_host = onchip_halos.data();
            oc.ptype = cfg->mesh.ptype;
            oc.pstart = b->pstart;
            oc.x = xr;
            oc.y = yr;
            oc.z = zr;
            oc.mass = b->mass;
            oc.type = b->type;
            oc.volfold = (float)vf;
            oc.densph = o->dens_mesh;
        }
        SmoothPlan sp;
        GF_TRY(smooth_plan(nh, mesh.data(), onchip_halos.empty() ? nullptr : &oc, &sp));
        // only findDen reads the stage's meshes: with FFT axes and a folding
        // volfact the passes run over the occupied boxes, and only the deposit
        // boxes are zeroed (the rest of den is never read)
        const bool box_mode = sp.box_ok && volfact_folds(vf) && !sp.blob.empty();
        used_box_mode = box_mode;
        char *dbuf = nullptr;
        if (box_mode) {
            GF_TRY(smooth_upload(ctx, sp, &dbuf));
            GF_TRY(launch_mesh_boxes(ctx, n, xr, yr, zr, b->type, hid, nh, mesh_dev, boxes));
            GF_TRY(smooth_box_prepare(ctx, sp, dbuf, mesh_dev, den, boxes));
        } else {
            GF_CUDA_TRY(cudaMemsetAsync(den, 0, sizeof(float) * dev_cells, s));
        }
        // batch order: the deposit's float sums in octree order were faster
        // (2.73 -> 2.34 ms) but put the densest cells of the 5e7-particle
        // cluster 1.04e-5 from an FP64 deposit, past the 1e-5 target
        // the occupied boxes let the smoothing skip all-zero pencils, and its
        // last pass the columns no particle's findDen stencil reads
        GF_TRY(launch_stage_deposit(ctx, n, xr, yr, zr, b->mass, b->type, hid, b->pstart,
                                    need_tree ? ctx->last_tree.perm : nullptr,
                                    need_tree ? ctx->last_tree.phalo : nullptr, nh, mesh_dev, den, vf,
                                    box_mode ? nullptr : boxes));
        if (!volfact_folds(vf)) GF_TRY(launch_scale(ctx, den, dev_cells, vf));
        tm.mark();  // 4
        if (box_mode) {
            GF_TRY(smooth_box_launch(ctx, sp, dbuf, mesh_dev, den, boxes, &oc));
        } else {
            MeshBoxes mb;
            mb.dev = boxes;
            mb.trim_last = true;  // den is read only by find_den below
            GF_TRY(smooth_meshes(ctx, nh, mesh.data(), mesh_dev, den, &oc, &mb));
        }
        tm.mark();  // 5
        if (o->dens_mesh)
            GF_TRY(launch_find_den(ctx, n, xr, yr, zr, hid, mesh_dev, den, o->dens_mesh,
                                   need_tree ? ctx->last_tree.perm : nullptr));
        tm.mark();  // 6
    } else {
        tm.mark();
        tm.mark();
        tm.mark();
    }
    // ---- 5. potential
    unsigned long long *counters = nullptr;
    if (cfg->do_potential) {
        if (st && cfg->count_work) {
            GF_TRY(ctx->tmp[4].reserve(128));
            counters = ctx->tmp[4].as<unsigned long long>();
            GF_CUDA_TRY(cudaMemsetAsync(counters, 0, 16, s));
        }
        const double pf = cfg->potentfact != 0.0 ? cfg->potentfact : physics().potentfact;
        PotentialParams pp = potential_params(cfg->theta2, cfg->ndirect, pf, cfg->add_bg);
        GF_TRY(launch_self_potential(ctx, ctx->last_tree, b->pstart, pp, o->penergy, o->phi, counters));
    }
    tm.mark();  // 7
    int status = check_device_errors(ctx);
    if (st) {
        memset(st, 0, sizeof(*st));
        st->nparticle = n;
        st->nhalo = nh;
        st->nnode = need_tree ? ctx->last_tree.nnode : 0;
        st->mesh_cells = cells;
        st->mesh_cells_device = dev_cells;
        st->onchip_meshes = (int64_t)onchip_halos.size();
        if (cfg->do_mesh && dev_cells > 0 && ctx->mesh_boxes.ptr) {
            // cells of the pencils the three smoothing passes filter, by the
            // rule of the smoothing's tile test at pencil granularity
            std::vector<int32_t> bx((size_t)kMeshBoxInts * nh);
            cudaMemcpy(bx.data(), ctx->mesh_boxes.ptr, bx.size() * sizeof(int32_t), cudaMemcpyDeviceToHost);
            auto len = [](int32_t lo, int32_t hi) { return hi >= lo ? (int64_t)hi - lo + 1 : 0; };
            for (int32_t h = 0; h < nh; h++) {
                const gf_mesh_desc &m = mesh[h];
                if (m.ptype == kMeshOnChip) continue;
                const int32_t *q = &bx[(size_t)kMeshBoxInts * h];
                st->mesh_pass_cells += (int64_t)m.nx * len(q[2], q[3]) * len(q[4], q[5]);  // x pass
                if (used_box_mode) {  // y pass over the evaluation box's x only
                    if (q[0] > q[1]) continue;  // nothing deposited: no pass
                    st->mesh_pass_cells += (int64_t)m.ny * len(q[6], q[7]) * len(q[4], q[5]);
                } else {
                    st->mesh_pass_cells += (int64_t)m.ny * m.nx * len(q[4], q[5]);
                }
                st->mesh_pass_cells += (int64_t)m.nz * len(q[6], q[7]) * len(q[8], q[9]);  // z pass, trimmed
            }
        }
        std::vector<int64_t> ps_host;
        if (!onchip_halos.empty()) {
            ps_host.resize((size_t)nh + 1);
            cudaMemcpy(ps_host.data(), b->pstart, ps_host.size() * sizeof(int64_t), cudaMemcpyDeviceToHost);
            for (int32_t h : onchip_halos) st->onchip_particles += ps_host[h + 1] - ps_host[h];
        }
        st->ms_recentre = tm.ms(0);
        st->ms_tree = tm.ms(1);
        st->ms_knn = tm.ms(2);
        st->ms_tsc = tm.ms(3);
        st->ms_smooth = tm.ms(4);
        st->ms_findden = tm.ms(5);
        st->ms_potential = tm.ms(6);
        if (cfg->count_work && ctx->tmp[4].ptr) {
            unsigned long long hcnt[9] = {0};
            cudaMemcpy(hcnt, ctx->tmp[4].ptr, sizeof(hcnt), cudaMemcpyDeviceToHost);
            if (counters) {
                st->pp_interactions = hcnt[0];
                st->pc_interactions = hcnt[1];
            }
            if (cfg->knn_k > 0) {
                st->knn_nodes = hcnt[4];
                st->knn_batches = hcnt[5];
                st->knn_candidates = hcnt[6];
                st->knn_single_inserts = hcnt[7];
                st->knn_bitonic_merges = hcnt[8];
            }
        }
    }
    return status;
}

}  // namespace gf

extern "C" {

int gf_stage_run(gf_ctx *ctx, const gf_batch *b, const gf_stage_config *cfg, gf_stage_out *o,
                 gf_stage_stats *st) {
    clear_status();
    if (!ctx || !b || !cfg || !o || b->nhalo < 0 || b->nparticle < 0) return GF_EINVAL;
    if (b->nparticle > 0 && (!b->pstart || !b->x || !b->y || !b->z || !b->mass)) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    return stage_run_locked(ctx, b, cfg, o, st, nullptr);
}

}  // extern "C"

// ------------------------------------------------------------------ stage graph
// The stage captured as one CUDA graph.  An eager run plans it (meshes from
// the halo extents, the octree's depth and node count); the captured pass
// then computes the frames and meshes on the device from the same extents,
// builds the octree with a fixed depth (two levels more than planned) and
// node capacity (a quarter more) and replays every kernel of the stage with
// no host round trip.  A replay is valid for any contents of the batch's
// input buffers whose meshes keep the planned shapes and whose octree fits
// the fixed shape; otherwise the pass flags GF_ERRBIT_PLAN and the replay
// reports GF_ESTALE (gf_stage_graph_run then re-plans and re-captures).
namespace gf {

struct StageGraph {
    gf_ctx *ctx = nullptr;
    gf_batch b{};
    gf_stage_config cfg{};
    gf_stage_out o{};
    StagePlan plan;
    TreeShape fixed;
    SmoothPlan smooth;
    DevBuf planned;       // the planned mesh descriptors (device)
    DevBuf smooth_blob;   // the smoothing plan (device)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<void *> bufs;  // context buffers the graph reads and writes
    int32_t replans = 0;
};

namespace {

std::vector<void *> context_buffers(gf_ctx *c) {
    std::vector<void *> v = {c->hid.ptr, c->mesh.ptr, c->mesh_boxes.ptr, c->smooth_tables.ptr, c->particles.ptr,
                             c->work.ptr};
    for (auto &t : c->tmp) v.push_back(t.ptr);
    for (auto &t : c->tree) v.push_back(t.ptr);
    return v;
}

// The stage with every launch shape from the graph's plan: capturable.
int stage_pass_graph(StageGraph &g) {
    gf_ctx *ctx = g.ctx;
    const gf_batch *b = &g.b;
    const gf_stage_config *cfg = &g.cfg;
    gf_stage_out *o = &g.o;
    const int64_t n = b->nparticle;
    const int32_t nh = b->nhalo;
    cudaStream_t s = ctx->stream;
    GF_TRY(ctx->hid.reserve(sizeof(int32_t) * std::max<int64_t>(n, 1)));
    int32_t *hid = ctx->hid.as<int32_t>();
    GF_TRY(compute_hid(ctx, nh, n, b->pstart, hid));
    GF_TRY(launch_extents(ctx, b, hid, cfg->box));
    const size_t nn = (size_t)std::max<int64_t>(n, 1);
    const size_t dbytes = (nn * sizeof(double) + 255) & ~size_t(255);
    GF_TRY(ctx->tmp[2].reserve(3 * dbytes + nn * sizeof(float4) + 256));
    char *t2 = ctx->tmp[2].as<char>();
    double *xr = o->xr ? o->xr : reinterpret_cast<double *>(t2);
    double *yr = o->yr ? o->yr : reinterpret_cast<double *>(t2 + dbytes);
    double *zr = o->zr ? o->zr : reinterpret_cast<double *>(t2 + 2 * dbytes);
    float4 *pos = reinterpret_cast<float4 *>(t2 + 3 * dbytes);
    const size_t frame_bytes = (6 * (size_t)std::max(nh, 1) * sizeof(double) + 255) & ~size_t(255);
    GF_TRY(ctx->mesh.reserve(frame_bytes + (size_t)std::max(nh, 1) * sizeof(gf_mesh_desc) + 512));
    double *frame_dev = ctx->mesh.as<double>();
    gf_mesh_desc *mesh_dev = reinterpret_cast<gf_mesh_desc *>(ctx->mesh.as<char>() + frame_bytes);
    GF_TRY(launch_frames_plan(ctx, nh, cfg->box, cfg->mesh, cfg->do_mesh, g.planned.as<gf_mesh_desc>(), frame_dev,
                              mesh_dev));
    GF_TRY(recentre(ctx, b, hid, frame_dev, cfg->box, xr, yr, zr, pos));
    if (g.plan.need_tree)
        GF_TRY(build_tree(ctx, nh, n, b->pstart, pos, cfg->theta2, cfg->q5_asbuilt, &ctx->last_tree, &g.fixed));
    if (cfg->knn_k > 0)
        GF_TRY(launch_knn(ctx, ctx->last_tree, b->pstart, pos, cfg->knn_k, o->nearindex, o->dens_sph, nullptr));
    if (cfg->do_mesh) {
        const int64_t dev_cells = g.plan.dev_cells;
        GF_TRY(ctx->tmp[3].reserve(sizeof(float) * (size_t)std::max<int64_t>(dev_cells, 1)));
        float *den = ctx->tmp[3].as<float>();
        const double vf = tsc_volfact();
        GF_TRY(ctx->mesh_boxes.reserve(sizeof(int32_t) * kMeshBoxInts * (size_t)std::max(nh, 1)));
        int32_t *boxes = ctx->mesh_boxes.as<int32_t>();
        // as the eager stage: passes over the occupied boxes, only the deposit
        // boxes zeroed; the tile counts are recounted on the device each replay
        const bool box_mode = g.smooth.box_ok && volfact_folds(vf) && !g.smooth.blob.empty();
        if (box_mode) {
            GF_TRY(launch_mesh_boxes(ctx, n, xr, yr, zr, b->type, hid, nh, mesh_dev, boxes));
            GF_TRY(smooth_box_prepare(ctx, g.smooth, g.smooth_blob.as<char>(), mesh_dev, den, boxes));
        } else {
            GF_CUDA_TRY(cudaMemsetAsync(den, 0, sizeof(float) * dev_cells, s));
        }
        GF_TRY(launch_stage_deposit(ctx, n, xr, yr, zr, b->mass, b->type, hid, b->pstart,
                                    g.plan.need_tree ? ctx->last_tree.perm : nullptr,
                                    g.plan.need_tree ? ctx->last_tree.phalo : nullptr, nh, mesh_dev, den, vf,
                                    box_mode ? nullptr : boxes));
        if (!volfact_folds(vf)) GF_TRY(launch_scale(ctx, den, dev_cells, vf));
        if (box_mode) {
            GF_TRY(smooth_box_launch(ctx, g.smooth, g.smooth_blob.as<char>(), mesh_dev, den, boxes));
        } else {
            MeshBoxes mb;
            mb.dev = boxes;
            mb.trim_last = true;  // den is read only by find_den below
            GF_TRY(smooth_launch(ctx, g.smooth, g.smooth_blob.as<char>(), mesh_dev, den, nullptr, &mb));
        }
        if (o->dens_mesh)
            GF_TRY(launch_find_den(ctx, n, xr, yr, zr, hid, mesh_dev, den, o->dens_mesh,
                                   g.plan.need_tree ? ctx->last_tree.perm : nullptr));
    }
    if (cfg->do_potential) {
        const double pf = cfg->potentfact != 0.0 ? cfg->potentfact : physics().potentfact;
        PotentialParams pp = potential_params(cfg->theta2, cfg->ndirect, pf, cfg->add_bg);
        GF_TRY(launch_self_potential(ctx, ctx->last_tree, b->pstart, pp, o->penergy, o->phi, nullptr));
    }
    return GF_OK;
}

void release_graph(StageGraph &g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g.exec = nullptr;
    g.graph = nullptr;
}

// Plans with an eager run (whose outputs are the batch's results), runs the
// fixed-shape pass once uncaptured (it reserves every buffer), then captures.
int capture_graph(StageGraph &g) {
    gf_ctx *ctx = g.ctx;
    release_graph(g);
    g.plan = StagePlan();
    GF_TRY(stage_run_locked(ctx, &g.b, &g.cfg, &g.o, nullptr, &g.plan));
    if (g.plan.onchip) {
        set_status(GF_ENOTIMPL, "a stage graph does not capture on-chip meshes (mesh_onchip)");
        return GF_ENOTIMPL;
    }
    g.fixed.levels = g.plan.tree.levels + 2;
    g.fixed.ncap = g.plan.tree.ncap + g.plan.tree.ncap / 4 + 64;
    const int32_t nh = g.b.nhalo;
    GF_TRY(g.planned.reserve(sizeof(gf_mesh_desc) * (size_t)std::max(nh, 1)));
    if (nh > 0 && g.cfg.do_mesh)
        GF_CUDA_TRY(cudaMemcpy(g.planned.ptr, g.plan.mesh.data(), sizeof(gf_mesh_desc) * nh, cudaMemcpyHostToDevice));
    if (g.cfg.do_mesh) {
        GF_TRY(smooth_plan(nh, g.plan.mesh.data(), nullptr, &g.smooth));
        GF_TRY(g.smooth_blob.reserve(std::max<size_t>(g.smooth.blob.size(), 256)));
        if (!g.smooth.blob.empty())
            GF_CUDA_TRY(cudaMemcpy(g.smooth_blob.ptr, g.smooth.blob.data(), g.smooth.blob.size(),
                                   cudaMemcpyHostToDevice));
    }
    GF_TRY(stage_pass_graph(g));
    GF_TRY(check_device_errors(ctx));
    g.bufs = context_buffers(ctx);
    GF_CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int st = stage_pass_graph(g);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
    if (st != GF_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (ce != cudaSuccess) {
        set_status(GF_EDEVICE, "stage graph capture: %s", cudaGetErrorString(ce));
        return GF_EDEVICE;
    }
    g.graph = graph;
    GF_CUDA_TRY(cudaGraphInstantiate(&g.exec, g.graph, 0));
    if (context_buffers(ctx) != g.bufs) {  // a buffer grew during capture: the graph holds stale pointers
        set_status(GF_EDEVICE, "stage graph capture reallocated a scratch buffer");
        return GF_EDEVICE;
    }
    return GF_OK;
}

}  // namespace

}  // namespace gf

struct gf_stage_graph : gf::StageGraph {};

extern "C" {

int gf_stage_graph_create(gf_ctx *ctx, const gf_batch *b, const gf_stage_config *cfg, gf_stage_out *o,
                          gf_stage_graph **out) {
    clear_status();
    if (!ctx || !b || !cfg || !o || !out || b->nhalo < 0 || b->nparticle < 0) return GF_EINVAL;
    if (b->nparticle > 0 && (!b->pstart || !b->x || !b->y || !b->z || !b->mass)) return GF_EINVAL;
    if (cfg->plain_fp64 || cfg->mesh_onchip) {
        set_status(GF_ENOTIMPL, "a stage graph captures the batched FP32 stage with device-memory meshes");
        return GF_ENOTIMPL;
    }
    *out = nullptr;
    auto *g = new gf_stage_graph();
    g->ctx = ctx;
    g->b = *b;
    g->cfg = *cfg;
    g->o = *o;
    std::lock_guard<std::mutex> lk(ctx->lock);
    const int st = capture_graph(*g);
    if (st != GF_OK) {
        release_graph(*g);
        delete g;
        return st;
    }
    *out = g;
    return GF_OK;
}

int gf_stage_graph_launch(gf_stage_graph *g) {
    clear_status();
    if (!g || !g->exec) return GF_EINVAL;
    std::lock_guard<std::mutex> lk(g->ctx->lock);
    if (context_buffers(g->ctx) != g->bufs) {
        set_status(GF_ESTALE, "the context's scratch buffers moved since the capture");
        return GF_ESTALE;
    }
    GF_CUDA_TRY(cudaGraphLaunch(g->exec, g->ctx->stream));
    return GF_OK;
}

int gf_stage_graph_sync(gf_stage_graph *g) {
    clear_status();
    if (!g) return GF_EINVAL;
    std::lock_guard<std::mutex> lk(g->ctx->lock);
    return check_device_errors(g->ctx);
}

int gf_stage_graph_run(gf_stage_graph *g, int32_t *replanned) {
    if (replanned) *replanned = 0;
    int st = gf_stage_graph_launch(g);
    if (st == GF_OK) st = gf_stage_graph_sync(g);
    if (st != GF_ESTALE) return st;
    clear_status();
    std::lock_guard<std::mutex> lk(g->ctx->lock);
    g->replans++;
    if (replanned) *replanned = 1;
    return capture_graph(*g);  // its eager run leaves this batch's results
}

int gf_stage_graph_replans(const gf_stage_graph *g) { return g ? g->replans : -1; }

int gf_stage_graph_nodes(const gf_stage_graph *g, int32_t *kernels, int32_t *nodes) {
    clear_status();
    if (!g || !g->graph) return GF_EINVAL;
    size_t n = 0;
    GF_CUDA_TRY(cudaGraphGetNodes(g->graph, nullptr, &n));
    std::vector<cudaGraphNode_t> v(n);
    GF_CUDA_TRY(cudaGraphGetNodes(g->graph, v.data(), &n));
    int32_t k = 0;
    for (cudaGraphNode_t nd : v) {
        cudaGraphNodeType t;
        GF_CUDA_TRY(cudaGraphNodeGetType(nd, &t));
        k += t == cudaGraphNodeTypeKernel;
    }
    if (kernels) *kernels = k;
    if (nodes) *nodes = (int32_t)n;
    return GF_OK;
}

void gf_stage_graph_destroy(gf_stage_graph *g) {
    if (!g) return;
    {
        std::lock_guard<std::mutex> lk(g->ctx->lock);
        cudaStreamSynchronize(g->ctx->stream);
        release_graph(*g);
    }
    delete g;
}

}  // extern "C"

// ------------------------------------------------------------------ drop-ins
namespace {

int do_findsphdensity(SimpleBasicParticleType *bp, int np, long long *nearindex, int numnear,
                      float *densph) {
    if (np < 0 || (np > 0 && (!bp || !nearindex || !densph)) || numnear < 1 || numnear > 32) {
        set_status(GF_EINVAL, "findsphdensity: invalid arguments (1 <= Numnear <= 32)");
        return GF_EINVAL;
    }
    if (np == 0) return GF_OK;
    gf_ctx *ctx = default_ctx();
    if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
    std::lock_guard<std::mutex> g(ctx->lock);
    const size_t n = (size_t)np;
    // stage x, y, z, mass (FP64) and pstart in one pinned buffer
    const size_t hbytes = n * 4 * sizeof(double) + 2 * sizeof(int64_t);
    GF_TRY(ctx->pin[0].reserve(hbytes));
    GF_TRY(ctx->particles.reserve(hbytes + n * (sizeof(float4) + sizeof(int32_t) + sizeof(float)) + 1024));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    double *h = ctx->pin[0].as<double>();
    for (size_t i = 0; i < n; i++) {
        h[i] = bp[i].x;
        h[n + i] = bp[i].y;
        h[2 * n + i] = bp[i].z;
        h[3 * n + i] = bp[i].mass;
    }
    int64_t *hp = reinterpret_cast<int64_t *>(h + 4 * n);
    hp[0] = 0;
    hp[1] = np;
    char *d = ctx->particles.as<char>();
    GF_CUDA_TRY(cudaMemcpyAsync(d, h, hbytes, cudaMemcpyHostToDevice, ctx->stream));
    const double *dx = reinterpret_cast<const double *>(d);
    const int64_t *dpstart = reinterpret_cast<const int64_t *>(dx + 4 * n);
    float4 *pos = reinterpret_cast<float4 *>(d + ((hbytes + 255) & ~size_t(255)));
    GF_TRY(ctx->tmp[1].reserve(n * (size_t)numnear * sizeof(int32_t) + n * sizeof(float) + 512));
    int32_t *near32 = ctx->tmp[1].as<int32_t>();
    float *dens = reinterpret_cast<float *>(near32 + n * numnear);
    pack_pos_kernel<<<grid1(np), 256, 0, ctx->stream>>>(np, dx, dx + n, dx + 2 * n, nullptr, dx + 3 * n, pos);
    GF_LAUNCH_CHECK();
    GF_TRY(build_tree(ctx, 1, np, dpstart, pos, 0.5f, 0, &ctx->last_tree));
    GF_TRY(launch_knn(ctx, ctx->last_tree, dpstart, pos, numnear, near32, dens));
    GF_TRY(ctx->pin[2].reserve(n * (size_t)numnear * sizeof(int32_t) + n * sizeof(float)));
    int32_t *hn = ctx->pin[2].as<int32_t>();
    GF_CUDA_TRY(cudaMemcpyAsync(hn, near32, n * (size_t)numnear * sizeof(int32_t) + n * sizeof(float),
                                cudaMemcpyDeviceToHost, ctx->stream));
    GF_TRY(check_device_errors(ctx));  // synchronises
    for (size_t i = 0; i < n * (size_t)numnear; i++) nearindex[i] = hn[i];
    memcpy(densph, hn + n * numnear, n * sizeof(float));
    return GF_OK;
}

}  // namespace

namespace gf {
// The findsphdensity drop-in's lists and densities for another drop-in
// (starfindsphdensity, gf_starden.cu).
int findsphdensity_lists(SimpleBasicParticleType *bp, int np, long long *nearindex, int numnear,
                         float *densph) {
    return do_findsphdensity(bp, np, nearindex, numnear, densph);
}
}  // namespace gf

namespace gf {

// Potential of the sources (sr, smass) at the targets r (self: r == sr) on
// the device of ctx; leaves penergy in device memory (*dout) and the FP64
// target positions (Vector3d AoS) at *dtargets.  Caller holds ctx->lock.
int potent_device(gf_ctx *ctx, int nend, const Vector3d *r, int snp, const Vector3d *sr,
                  const float *smass, bool self, float **dout_ret, const double **dtargets) {
    const size_t ns = (size_t)snp, nt = (size_t)nend;
    // pinned staging: sources (3 doubles + mass), targets (3 doubles), pstart, target count
    const size_t hbytes = ns * 3 * sizeof(double) + ns * sizeof(float) + (self ? 0 : nt * 3 * sizeof(double)) +
                          4 * sizeof(int64_t);
    GF_TRY(ctx->pin[0].reserve(hbytes + 64));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    char *h = ctx->pin[0].as<char>();
    size_t off = 0;
    memcpy(h + off, sr, ns * 3 * sizeof(double));
    const size_t off_sr = off;
    off += ns * 3 * sizeof(double);
    memcpy(h + off, smass, ns * sizeof(float));
    const size_t off_sm = off;
    off += ns * sizeof(float);
    off = (off + 7) & ~size_t(7);
    const size_t off_tr = off;
    if (!self) {
        memcpy(h + off, r, nt * 3 * sizeof(double));
        off += nt * 3 * sizeof(double);
    }
    const size_t off_ps = off;
    int64_t *ps = reinterpret_cast<int64_t *>(h + off);
    ps[0] = 0;
    ps[1] = snp;
    reinterpret_cast<int32_t *>(ps + 2)[0] = nend;  // target count of the single source halo
    off += 4 * sizeof(int64_t);
    const size_t dbytes = off + ns * sizeof(float4) + nt * (sizeof(float4) + sizeof(int32_t) + sizeof(float)) + 2048;
    GF_TRY(ctx->particles.reserve(dbytes));
    char *d = ctx->particles.as<char>();
    GF_CUDA_TRY(cudaMemcpyAsync(d, h, off, cudaMemcpyHostToDevice, ctx->stream));
    char *q = d + ((off + 255) & ~size_t(255));
    float4 *spos = reinterpret_cast<float4 *>(q);
    q += ((ns * sizeof(float4) + 255) & ~size_t(255));
    float4 *tpos = reinterpret_cast<float4 *>(q);
    q += ((nt * sizeof(float4) + 255) & ~size_t(255));
    int32_t *thalo = reinterpret_cast<int32_t *>(q);
    q += ((nt * sizeof(int32_t) + 255) & ~size_t(255));
    float *dout = reinterpret_cast<float *>(q);
    const int64_t *dps = reinterpret_cast<const int64_t *>(d + off_ps);
    vec3_pos_kernel<<<grid1(snp), 256, 0, ctx->stream>>>(snp, reinterpret_cast<const double *>(d + off_sr),
                                                         reinterpret_cast<const float *>(d + off_sm), spos);
    GF_LAUNCH_CHECK();
    const float theta2 = 0.5f;  // subhaloden.mod6.c:1481,1541
    GF_TRY(build_tree(ctx, 1, snp, dps, spos, theta2, 0, &ctx->last_tree));
    const gf_physics &ph = physics();
    if (self) {
        PotentialParams pp = potential_params(theta2, 100, ph.potentfact, 1);
        GF_TRY(launch_self_potential(ctx, ctx->last_tree, dps, pp, dout, nullptr, nullptr));
    } else {
        // targets: FP32 positions, all looking into halo 0 (the one source tree);
        // their masses do not enter the potential
        GF_CUDA_TRY(cudaMemsetAsync(thalo, 0, nt * sizeof(int32_t), ctx->stream));
        vec3_pos_kernel<<<grid1(nend), 256, 0, ctx->stream>>>(
            nend, reinterpret_cast<const double *>(d + off_tr), nullptr, tpos);
        GF_LAUNCH_CHECK();
        // External_Halo_Potent sums directly below 1000 targets (subhaloden.mod6.c:1545)
        PotentialParams pp = potential_params(theta2, 1000, ph.potentfact, 1);
        const int32_t *ntarget_dev = reinterpret_cast<const int32_t *>(dps + 2);
        GF_TRY(launch_external_potential(ctx, ctx->last_tree, dps, nend, tpos, thalo, ntarget_dev,
                                         pp, dout, nullptr));
    }
    *dout_ret = dout;
    if (dtargets)
        *dtargets = reinterpret_cast<const double *>(d + (self ? off_sr : off_tr));
    return GF_OK;
}

}  // namespace gf

namespace {

int potent_common(int nend, Vector3d *r, float *penergy, int snp, Vector3d *sr, float *smass,
                  bool self) {
    gf_ctx *ctx = default_ctx();
    if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
    std::lock_guard<std::mutex> g(ctx->lock);
    float *dout = nullptr;
    GF_TRY(potent_device(ctx, nend, r, snp, sr, smass, self, &dout, nullptr));
    GF_CUDA_TRY(cudaMemcpyAsync(penergy, dout, (size_t)nend * sizeof(float), cudaMemcpyDeviceToHost,
                                ctx->stream));
    return check_device_errors(ctx);  // synchronises
}

}  // namespace

extern "C" {

void findsphdensity(SimpleBasicParticleType *bp, int np, long long *nearindex, int Numnear,
                    float *densph) {
    clear_status();
    dropin_exit_on_error(do_findsphdensity(bp, np, nearindex, Numnear, densph), "findsphdensity");
}

void Self_Halo_Potent(int np, Vector3d *r, float *mass, float *penergy) {
    clear_status();
    if (np < 0 || (np > 0 && (!r || !mass || !penergy))) {
        set_status(GF_EINVAL, "Self_Halo_Potent: invalid arguments");
        dropin_exit_on_error(GF_EINVAL, "Self_Halo_Potent");
        return;
    }
    if (np == 0) return;
    dropin_exit_on_error(potent_common(np, r, penergy, np, r, mass, true), "Self_Halo_Potent");
}

void External_Halo_Potent(int nend, Vector3d *r, float *mass, float *penergy, int snp,
                          Vector3d *sr, float *smass) {
    clear_status();
    (void)mass;
    if (nend < 0 || snp < 0 || (nend > 0 && (!r || !penergy)) || (snp > 0 && (!sr || !smass))) {
        set_status(GF_EINVAL, "External_Halo_Potent: invalid arguments");
        dropin_exit_on_error(GF_EINVAL, "External_Halo_Potent");
        return;
    }
    if (nend == 0) return;
    if (snp == 0) {  // no sources: only the background term of a zero mass
        for (int i = 0; i < nend; i++) penergy[i] = 0.f;
        return;
    }
    dropin_exit_on_error(potent_common(nend, r, penergy, snp, sr, smass, false), "External_Halo_Potent");
}

}  // extern "C"
