// Centre-of-mass octree shared by the kNN search and the Barnes-Hut potential.
#pragma once

#include "gf_internal.cuh"

namespace gf {

// W4 kernel, nnost.c:536-555 (float arguments, double constants); the
// translation units that use it are compiled with --fmad=false.
__device__ __forceinline__ float w4(float dist, float h) {
    const float r = dist / h;
    if (r < 1.) {
        return (float)((-0.2387324) * ((2. - (double)r) * (double)r * (double)r - 1.333333) /
                       (double)(h * h * h));
    } else if (r < 2.) {
        const float twomr = (float)((2. - (double)r) / (double)h);
        return (float)(0.07957747 * (double)twomr * (double)twomr * (double)twomr);
    }
    return 0.f;
}

// Builds the octree of every halo of a batch.  pos (batch order, halo h is
// [pstart[h], pstart[h+1])) holds recentred FP32 positions and masses.
// theta2 fills BhNode::open_r2; q5_asbuilt reproduces ost.c:571 (m*y*x in
// place of m*y*z).  Buffers live in ctx->tree[]; the view stays valid until
// the next build on ctx.
// Shape of a built octree: levels processed, node capacity and node count
// (-1 for a build with a fixed shape, whose count stays on the device).
struct TreeShape {
    int32_t levels = 0;
    int64_t ncap = 0;
    int32_t nnode = 0;
};
// The energy test of CheckSelfTE / CheckExternalTE (gf_bound.cu) on the
// default context: bndflag per target, the bound count, or -1 with the status
// set.  c: the centre and velocity of the KE (x, y, z, vx, vy, vz).
int energy_check(const Kptype *tkp, int tnp, unsigned char *bndflag, const Kptype *skp, int snp, bool self,
                 const double c[6]);

// What a captured stage pass takes from an eager run of the stage.
struct StagePlan {
    bool need_tree = false, onchip = false;
    std::vector<gf_mesh_desc> mesh;  // planned meshes (offsets into the mesh buffer)
    int64_t cells = 0, dev_cells = 0;
    TreeShape tree;                  // the octree the eager run built
};
int stage_run_locked(gf_ctx *ctx, const gf_batch *b, const gf_stage_config *cfg, gf_stage_out *o,
                     gf_stage_stats *st, StagePlan *plan);

// With `fixed`, the build runs fixed->levels levels over fixed->ncap node
// slots with no host round trip (capturable in a CUDA graph) and flags
// GF_ERRBIT_PLAN when the batch needs more; `shape` receives the shape built.
int build_tree(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
               const float4 *pos, float theta2, int q5_asbuilt, TreeView *out,
               const TreeShape *fixed = nullptr, TreeShape *shape = nullptr);

// Potential walk parameters (see gf_potent.cu).
struct PotentialParams {
    float theta2;
    int32_t ndirect;      // halos with fewer targets than this use the direct sum
    double potentfact;    // 0 -> raw potential
    int32_t add_bg;       // add the NFW background term of the halo mass
    float amax, a, omep;  // cosmology for the background term
};

// The walk parameters with the cosmology of the background term (gf_stage.cu).
PotentialParams potential_params(float theta2, int ndirect, double potentfact, int add_bg);

// pos_batch: the same FP32 positions in batch order (seeds re-read them by
// batch index).
int launch_knn(gf_ctx *ctx, const TreeView &t, const int64_t *pstart, const float4 *pos_batch, int k,
               int32_t *nearindex, float *dens, unsigned long long *counters = nullptr,
               const int32_t *qlist = nullptr, int64_t nq = 0);
int launch_self_potential(gf_ctx *ctx, const TreeView &t, const int64_t *pstart,
                          const PotentialParams &pp, float *penergy, float *raw,
                          unsigned long long *counters);
int launch_bg_eval(gf_ctx *ctx, int32_t n, const double *mvir, const PotentialParams &pp, double *bg);
int launch_external_potential(gf_ctx *ctx, const TreeView &t, const int64_t *pstart_src,
                              int64_t ntarget, const float4 *tpos, const int32_t *thalo,
                              const int32_t *ntarget_halo, const PotentialParams &pp,
                              float *penergy, float *raw);
// Strict 26-neighbour maxima above threshold in the interior of every mesh
// (gf_adjoint.cu); *dcount (device) receives the number found.
int launch_mesh_peaks(gf_ctx *ctx, int32_t nhalo, int64_t maxcell, const gf_mesh_desc *mesh_dev,
                      const float *den, int margin, float threshold, int64_t cap, int32_t *out_halo,
                      int64_t *out_cell, float *out_val, unsigned long long *dcount);
const gf_physics &physics();
double bg_potent(double mvir);
// Host NFW helpers (get_concentration, get_alpha, gnfw, GetRvir of
// subhaloden.mod6.c:1059-1092) in the reference's float/double/long double mix.
double nfw_concentration(double mass);
double nfw_alpha(double c, double s);
double nfw_gnfw(double c);
double nfw_rvir(double mvir);

// Tree (or direct) potential of the sources (sr, smass) at targets r (self:
// r == sr) on ctx's device, as Self_Halo_Potent / External_Halo_Potent:
// penergy = phi * potentfact + GetBGpotent(source mass), left in device memory
// at *dout; *dtargets (optional) receives the device copy of the FP64 target
// positions (Vector3d AoS).  The caller holds ctx->lock.
int potent_device(gf_ctx *ctx, int nend, const Vector3d *r, int snp, const Vector3d *sr,
                  const float *smass, bool self, float **dout, const double **dtargets);

// The whole stage in FP64 (gf_plain64.cu) after recentring and the octree
// build on ctx: kNN + SPH density, meshes, potential.  ms (optional) receives
// the kNN, TSC + smoothing, findDen and potential times.
int stage_plain_fp64(gf_ctx *ctx, const gf_batch *b, const gf_stage_config *cfg, gf_stage_out *o,
                     const int32_t *hid, const double *xr, const double *yr, const double *zr,
                     const std::vector<gf_mesh_desc> &mesh, const gf_mesh_desc *mesh_dev, int64_t cells,
                     const PotentialParams &pp, float *ms);

// Copies the preorder node arrays and particle order to the host (tests).
int export_tree(gf_ctx *ctx, const TreeView &t, void *knn_host, void *bh_host, float4 *pos_host,
                int32_t *perm_host, int32_t *root_host, int32_t *rend_host);

}  // namespace gf
