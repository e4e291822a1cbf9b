/* libgf — B200-native density-and-potential stage of the PGalF galaxy finder
 * (NewGalFinder's per-halo kNN/SPH density, TSC mass assignment, FFT Gaussian
 * smoothing, mesh-density interpolation and Barnes-Hut potential).
 *
 * Two layers, both plain C ABI (no C++ or torch types in any signature):
 *
 *  1. Drop-in entry points with the reference's exact C signatures.  A
 *     reference build links libgf's objects in place of its own definitions
 *     (the reference objects with these symbols weakened, linked with the
 *     whole libgf.a archive) and the calls from subhalo_den() land here.  They take
 *     the reference's host buffers, copy them to the GPU, run the kernels and
 *     copy results back before returning, so no host pointer is kept across
 *     calls (the reference's Memory2.c arena may move blocks between calls,
 *     Memory2.c:173-195).  The status is kept in gf_last_status() /
 *     gf_last_error(); where the reference prints and calls exit(99), the
 *     void entry points do the same unless GF_NOEXIT is set in the
 *     environment.
 *
 *  2. The native batched API (gf_*): device pointers, many halos per call,
 *     stream-ordered, returning an int status.
 *
 * Status codes: */
#ifndef GF_H
#define GF_H

#include <stddef.h>
#include <stdint.h>

#include "gf_ref_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define GF_OK 0
#define GF_EINVAL 1    /* bad argument (size, pointer, mesh too small for the particles) */
#define GF_ENOMEM 2    /* device or host allocation failed */
#define GF_EDEVICE 3   /* CUDA error or no usable device */
#define GF_ETIMEOUT 4  /* a device-side bounded wait gave up */
#define GF_ERANGE 5    /* a particle fell outside its mesh (the reference would write out of bounds) */
#define GF_ENOTIMPL 6
#define GF_ESTALE 7    /* a captured stage graph's plan no longer fits the batch: re-plan */

const char *gf_status_string(int status);
/* Status and message of the most recent call made by this host thread. */
int gf_last_status(void);
const char *gf_last_error(void);
/* Select the CUDA device the drop-in entry points use (default: 0, or the
 * GF_DEVICE environment variable).  Returns a status. */
int gf_set_device(int device);
/* Number of kernels this process has launched through libgf (for tests that
 * must prove the GPU path ran). */
uint64_t gf_kernel_launch_count(void);
/* Compile-time launch parameter `name` of the loaded library (GF_KNN_ALGO,
 * GF_KNNB_BLOCK, GF_KNNB_ARITY, GF_KNNB_SEEDS, GF_KNNB_QUEUE, GF_KNNB_LANECERT,
 * GF_KNN_BLOCK, GF_KNN_MINB, GF_KNN_CHUNK, GF_BH_BLOCK, GF_BH_MINB, GF_BH_DYN, GF_BH_ACC, GF_KNNB_DYN,
 * GF_FFT_PENCILS, GF_FFT_PENCILS_64, GF_FFT_PENCILS_128, GF_TSC_TILE,
 * GF_TREE_BLOCK) in *value.
 * Returns GF_EINVAL for an unknown name. */
int gf_tuning_value(const char *name, int64_t *value);

/* ------------------------------------------------------------------------
 * Physics constants used by the potential drivers.  They are the values the
 * reference computes in physical_parameters() (NewGalFinder/gfind.c:842-890)
 * and reads as globals (potentfact, r1kineticfact, r2kineticfact, amax, a,
 * omep).  Defaults: amax = a = 1, omep = 0.3, omeplam = 0.7, hubble = 70.
 * ---------------------------------------------------------------------- */
typedef struct gf_physics {
    float amax, a, omep, omeplam, hubble;
    double potentfact, r1kineticfact, r2kineticfact;
} gf_physics;

/* Recompute potentfact/r1kineticfact/r2kineticfact from the cosmology in
 * `ph` (gfind.c:842-890) and store it for the drop-in potential drivers. */
int gf_set_cosmology(float amax, float a, float omep, float omeplam, float hubble);
int gf_get_physics(gf_physics *out);
/* NFW background potential of a halo of mass mvir (subhaloden.mod6.c:1093). */
double gf_bg_potent(double mvir);

/* ------------------------------------------------------------------------
 * Drop-in entry points (reference signatures; host pointers; synchronous).
 * ---------------------------------------------------------------------- */

/* NewGalFinder/tsc_omp2.c:166.  den holds mx*ny*nz floats, mx = 2(nx/2+1). */
void assign_density_TSC(SimpleBasicParticleType *bp, int np, float *den, int nx, int ny, int nz,
                        double Xmin, double Ymin, double Zmin, double cellsize, int ptype);
/* NewGalFinder/tsc_omp2.c:40 */
void findDen(SimpleBasicParticleType *bp, int np, float *densph, double xmin, double ymin,
             double zmin, double cellsize, float *den, int nx, int ny, int nz);
/* NewGalFinder/gsmooth.c:14.  In place on mx*ny*nz floats. */
void gaussian_Smoothing(float *denGrid, int nx, int ny, int nz, double cellsize, float RG);
/* NewGalFinder/nnost.c:560.  nearindex holds np*Numnear indices into bp. */
void findsphdensity(SimpleBasicParticleType *bp, int np, long long *nearindex, int Numnear,
                    float *densph);
/* NewGalFinder/nnost.c:632.  densph[i]: W4-weighted mass of the 10 nearest
 * stars (type 1) of particle i (0 when the halo has none); nearindex: the
 * Numnear nearest particles of every particle, as findsphdensity. */
void starfindsphdensity(SimpleBasicParticleType *bp, int np, long long *nearindex, int Numnear,
                        float *densph);
/* NewGalFinder/nnost.c:991.  Mesh density (TSC of the ptype particles,
 * Gaussian smoothing, findDen at every particle -> densph), the mesh peak
 * cores (*Core, *NumCore; at most maxnumcore before merging) and the kNN of
 * every particle (nearindex, np*Numnear) on the GPU.  More than 10 cores are
 * merged by the reference's own MergingPeak (subhaloden.mod6.c:341) and the
 * core array is resized with its arena Realloc (Memory2.c:217); both are
 * resolved when libgf is linked into the reference program.  Without
 * MergingPeak, more than 10 cores is an error (GF_ENOTIMPL); without Realloc
 * the array keeps its size. */
void lagFindStellarCore(SimpleBasicParticleType *bp, int np, int Numnear, float *densph,
                        Coretype **Core, int *NumCore, int maxnumcore, long long *nearindex,
                        int ptype);
/* NewGalFinder/nnost.c:199 (new_Make_Tree_Near) and ost.c:642 (Make_Tree).
 * Build libgf's centre-of-mass octree of ptl[0..np) on the GPU and write it
 * into TREE_START[0..nnode) in the reference's threaded layout (tree.h:72-91),
 * relinking ptl[].sibling: a node's daughter is its first offspring (its
 * loose particles first, then its child nodes), each offspring's sibling the
 * next, the last one's sibling the node's sibling.  mass, monox/y/z, dist
 * (= max |x - com|), dist2, quad, trQ and Nparticle are FP64 moments of the
 * node's particles; Make_Tree also sets dist_over_thetasq = dist2/thetasq.
 * The node count must fit nnode (GF_ENOMEM otherwise).  recursiveflag is
 * accepted and ignored: the build is the same for every mode. */
void new_Make_Tree_Near(TStruct *TREE_START, size_t nnode, TPtlStruct *ptl, size_t np,
                        int recursiveflag);
void Make_Tree(TStruct *TREE_START, size_t nnode, TPtlStruct *ptl, size_t np, float thetasq,
               int recursiveflag);
/* NewGalFinder/nnost.c:375.  The Num_neighbor (<= 32) nearest particles of
 * *point among the tree's particles, self included: indices into ptl,
 * squared distances (FP64, (dx*dx + dy*dy) + dz*dz) and masses in ascending
 * distance (equal distances by index), *maxr = sqrtf(k-th squared distance);
 * returns their number.  Thread safe.  The first call on a tree answers every
 * particle of the tree in one launch; calls at a particle's exact position
 * then copy its row, other points run a one-point launch.  A tree the caller
 * built by other code is read by walking its threads. */
int Find_Near(particle *point, int Num_neighbor, TStruct *tree, TPtlStruct *ptl, float *maxr,
              long long *nearindx, double *DIST2, float *MASS);
/* NewGalFinder/ost.c:226.  Raw Barnes-Hut potential of the tree's particles
 * at *p (opening |p - com|^2 < dist2/theta2, particle terms with r > 0, no
 * potentfact), on the GPU with the same batching as Find_Near.  Thread safe. */
float treeplumpotential(particle *p, float theta2, TStruct *tree, TPtlStruct *ptl);
/* NewGalFinder/subhaloden.mod6.c:416.  Density peaks on the kNN graph:
 * particles with den > PEAKTHRESHOLD (stars only when jflag is 1) whose kNN
 * list (neighbor, np*numneigh) holds no denser particle, written to *Core in
 * particle order (peak, cx, cy, cz, density); returns their number.  The
 * caller's array holds MAXNUMCORE cores; more peaks grow it by MAXNUMCORE
 * through the reference's arena Realloc (the reference's static maxnumcore is
 * not updated).  More than MAXNUMCORE peaks on the all-particle path exit
 * with 999, as the reference does (GF_ERANGE with GF_NOEXIT). */
int finddenpeak(float *den, int numneigh, long long *neighbor, int np, Coretype **Core, int jflag,
                SimpleBasicParticleType *bp);
/* NewGalFinder/subhaloden.mod6.c:1167.  Core density and core members of each
 * core on the kNN graph (see gf_core_density).  Reads the densities from and
 * writes haloid and flag to the reference's working-particle array wp,
 * resolved when libgf is linked into the reference program (GF_ENOTIMPL
 * otherwise); fills coredensity, nummem, numstar and starmass of core[].
 * Returns numcore. */
int FindCoreDensity(SimpleBasicParticleType *bp, int np, long long *neighbor, int NumNeighbor,
                    Coretype *core, int numcore);
/* NewGalFinder/subhaloden.mod6.c:1477 */
void Self_Halo_Potent(int np, Vector3d *r, float *mass, float *penergy);
/* NewGalFinder/subhaloden.mod6.c:1537 */
void External_Halo_Potent(int nend, Vector3d *r, float *mass, float *penergy, int snp,
                          Vector3d *sr, float *smass);
/* NewGalFinder/subhaloden.mod6.c:1730.  Bound flags (GF_BOUND/GF_UNBOUND) of
 * the members kp[np]: kinetic energy about the stars' centre of mass against
 * the self potential (Self_Halo_Potent).  Returns the number bound. */
int CheckSelfTE(Kptype *kp, int np, unsigned char *bndflag, Coretype *icore);
/* NewGalFinder/subhaloden.mod6.c:1622.  Bound flags of the targets tkp[tnp]
 * against the potential of the sources skp[snp] (External_Halo_Potent), kinetic
 * energy about the core's centre and velocity.  Returns the number bound. */
int CheckExternalTE(Kptype *tkp, int tnp, unsigned char *bndflag, Kptype *skp, int snp,
                    Coretype *icore);
/* NewGalFinder/force_spline.mod3.c:81.  The GPU potential evaluates the
 * kernel -1/r and its quadrupole terms exactly, so no table is built; the
 * call only initialises the device. */
void i_potent_spline(void);
/* NewGalFinder/mkRtidal.c:80.  Builds the NFW tidal-radius table of the
 * OLD_TIDAL build (32 concentrations x 128 distances x 128 mass ratios) on
 * the GPU into the library's copy that nfw_rtidal reads. */
void mkRtidal(void);
/* NewGalFinder/mkRtidal.c:60.  The table entry of (satellite / host mass
 * ratio, distance in host virial radii, host concentration): the tidal radius
 * in units of the distance; 0 before mkRtidal has run. */
float nfw_rtidal(float mM, float dRv, float c);

/* Tidal radius of every core: AdGetTidalRCenterCore (subhaloden.mod6.c:1910-2035)
 * with get_tidal_ellipse (:1102-1165).  The reference reads each particle's
 * core from its file-global working array (wp[i].haloid); here it is passed
 * as haloid[np] (negative: no core), and score_core[ncore] lists the core ids
 * in the reference's score order (increasing member count).  Fills
 * core[].Rtidal and core[].nummem.  Host pointers, synchronous. */
/* One shell of subhalo_den's boundedness loop (subhaloden.mod6.c:3033-3101),
 * batched over the shell's cores: for each core of `order` (the shell's
 * cores after the loop's qsort by member count) the shell's particles not yet
 * bound and every REMAINING particle within the core's Rtidal are tested
 * against the core's members and the later shells that hold the core
 * (CheckExternalTE); the bound ones join the core, the others become
 * REMAINING; then the shell's unbound particles become REMAINING
 * (UnboundShellP2Rest).  A core's sources do not change during its shell, so
 * every core's candidates are tested in one GPU pass and the loop is
 * replayed in the reference's order; a core whose replayed target count
 * crosses the 1000-target direct-sum bound is retested alone
 * (*nretest_out counts them).
 * bp[np]: the halo's particles; flag[np], haloid[np]: wp[].flag (WP_BOUND
 * 0x10, WP_REMAINING 0x20) and wp[].haloid, updated in place; shellp with
 * shellp_start[nshell+1] and shellc with shellc_start[nshell+1]: the
 * SHELL2P and SHELL2C lists; core[numcore] with Rtidal set; nmem_out[norder]
 * (may be NULL): MULTIHALOSHELL's bound count per core of `order`.  Host
 * arrays; synchronous. */
int gf_shell_bound(const SimpleBasicParticleType *bp, int np, unsigned char *flag, int32_t *haloid,
                   const int32_t *shellp, const int32_t *shellp_start, const int32_t *shellc,
                   const int32_t *shellc_start, int nshell, int ishell, const Coretype *core, int numcore,
                   const int32_t *order, int norder, int32_t *nmem_out, int32_t *nretest_out);
/* One pass of subhalo_den's BOUNDITER loop over the cores
 * (subhaloden.mod6.c:3118-3172), batched: for each core of `order` (all
 * cores after the pass's qsort by member count; nmem[] their member counts
 * at the start of the pass, cores with none skipped; Rtidal set by
 * gf_tidal_radius) GetMemberRestParticleList and SINGLEHALO (CheckSelfTE:
 * the list's self potential, the KE about its stellar centre).  The lists
 * are predicted from the state at the start of a batch and tested in one GPU
 * pass; the replay in the reference's order keeps a core's result when its
 * actual list equals the prediction and starts a new batch at the first core
 * whose list changed (*nbatch_out: GPU passes used).  flag[np] and
 * haloid[np] (wp[].flag, wp[].haloid) are updated in place; nbound_out[norder]
 * (may be NULL): SINGLEHALO's bound count per core.  Host arrays;
 * synchronous. */
int gf_bound_pass(const SimpleBasicParticleType *bp, int np, unsigned char *flag, int32_t *haloid,
                  const Coretype *core, int numcore, const int32_t *order, const int32_t *nmem, int norder,
                  int32_t *nbound_out, int32_t *nbatch_out);
int gf_tidal_radius(Coretype *core, int numcore, const int32_t *score_core, int ncore,
                    const SimpleBasicParticleType *bp, const int32_t *haloid, int np);
/* Tidal cut of GetMemberRestParticleList (subhaloden.mod6.c:2734-2745) and
 * GetShellParticleFromRestParticleLIST (:532-541): the entries of plist[nlist]
 * (all np particles if plist is NULL) whose float distance^2 from (cx, cy, cz)
 * is below rtidal^2, in list order, into out[]; *nout receives the count. */
int gf_tidal_select(const SimpleBasicParticleType *bp, int np, const int32_t *plist, int nlist,
                    float cx, float cy, float cz, float rtidal, int32_t *out, int *nout);

/* ------------------------------------------------------------------------
 * Native batched API.
 * ---------------------------------------------------------------------- */
typedef struct gf_ctx gf_ctx;

/* stream: a cudaStream_t (NULL = legacy default stream). */
int gf_ctx_create(gf_ctx **ctx, int device, void *stream);
int gf_ctx_destroy(gf_ctx *ctx);
int gf_ctx_set_stream(gf_ctx *ctx, void *stream);

/* Per-halo mesh description (device array, one entry per halo).  The mesh of
 * halo h occupies den[off, off + mx*ny*nz) with mx = 2(nx/2+1), laid out as
 * den[i + mx*(j + ny*k)] (tsc_omp2.c:16).  Positions handed to the mesh
 * kernels are in the same frame as (xmin, ymin, zmin). */
typedef struct gf_mesh_desc {
    int64_t off;
    int32_t nx, ny, nz;
    int32_t ptype;          /* TSC particle filter; GF_TYPE_ALL = every particle */
    double xmin, ymin, zmin;
    double cellsize;
    double rg;              /* Gaussian smoothing length (same unit as cellsize) */
} gf_mesh_desc;

/* Particle batch in device memory: halos are contiguous ranges
 * [pstart[h], pstart[h+1]) of the particle arrays. */
typedef struct gf_batch {
    int32_t nhalo;
    int64_t nparticle;
    const int64_t *pstart;   /* device, nhalo+1 */
    const double *x, *y, *z; /* device, FP64 positions (cMpc/h) */
    const double *mass;      /* device, FP64 (Msun/h) */
    const int32_t *type;     /* device, may be NULL (all GF_TYPE_DM) */
} gf_batch;

/* Per-halo mesh sizing rules (the mesh of a halo is planned from its
 * recentred extent; the origin is nbuff/2 cells below the halo minimum and
 * the upper bound is padded by 1e-4 of the extent, nnost.c:1040-1056). */
#define GF_MESH_REFERENCE 0 /* n = extent/cell + nbuff per axis (nnost.c:1053-1055) */
#define GF_MESH_FIXED 1     /* cubic n = nfixed; cell = max extent / (n - nbuff) */
#define GF_MESH_POW2 2      /* cubic n = clamp(next_pow2(extent/cell + nbuff), nmin, nmax);
                               cell grows beyond `cell` when the halo needs more than nmax */
typedef struct gf_mesh_rule {
    int32_t mode;
    int32_t nfixed, nmin, nmax;
    int32_t nbuff;          /* NCELLBUFF (params.h:115), 10 */
    int32_t ptype;          /* TSC particle filter */
    int32_t rg_in_cells;    /* 1: rg is in units of the planned cell size */
    int32_t reserved;
    double cell;            /* TSC_CELL_SIZE (params.h:92), 0.004 cMpc/h */
    double rg;              /* Gaussian_Smoothing_Length (params.h:104), 0.008 cMpc/h */
} gf_mesh_rule;

/* Plans one mesh per halo from extent[3*h + axis] (recentred extents,
 * cMpc/h); writes desc[h] with consecutive, 256-byte aligned offsets and
 * returns the total float count in *total_cells.  Host-only. */
int gf_plan_meshes(int32_t nhalo, const double *extent, const gf_mesh_rule *rule,
                   gf_mesh_desc *desc, int64_t *total_cells);

/* Gaussian smoothing of one caller-owned device mesh (mx*ny*nz floats, in
 * place) on the caller's stream, allocating nothing.  No counterpart in the
 * reference: it serves callers that cannot allocate device memory (a fixed
 * budget owned by another allocator, or a path that cannot afford an
 * allocation's synchronisation).  Its scratch is a 64 KiB static device array
 * that every GPU loading libgf holds until exit; each axis must be at most
 * 1024 cells (GF_EINVAL otherwise).  The first call on a device looks up the
 * array's device address with that device current, so make it before any
 * stream capture.  All calls share the array: calls that may overlap on the
 * GPU (different streams without ordering) race and must be serialised.
 * Every call plans on the host; an axis whose length is not a power of two
 * takes its exact n-tap filter from an O(n^2) FP64 sum there. */
int gf_gaussian_smooth_noalloc(float *den, int nx, int ny, int nz, double cellsize, float RG,
                               void *stream);

/* Mesh stage on a batch whose meshes are already described: zero + TSC
 * deposit (tsc_omp2.c:166), Gaussian smoothing (gsmooth.c:14) and the
 * interpolation back to every particle (tsc_omp2.c:40).  den must hold the
 * sum of all meshes; densph one float per particle.  If smoothed_only is 0
 * the raw deposit is left in den and densph is not written. */
int gf_mesh_stage(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev,
                  const gf_mesh_desc *mesh_host, float *den, float *densph, int smooth);

/* Individual batched mesh kernels (device pointers). */
int gf_tsc_deposit(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev,
                   const gf_mesh_desc *mesh_host, float *den);
int gf_gaussian_smooth(gf_ctx *ctx, int32_t nhalo, const gf_mesh_desc *mesh_host,
                       const gf_mesh_desc *mesh_dev, float *den);
int gf_find_den(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev, const float *den,
                float *densph);

/* Adjoints (no reference counterpart: the reference has no derivatives).
 * Gradients are FP64 device arrays that these calls ADD to.
 *   gf_tsc_adjoint: the deposit of tsc_omp2.c:166 with respect to positions
 *     and masses, given dL/dden in gden (padded mesh layout); gm may be NULL.
 *   gf_find_den_adjoint: the interpolation of tsc_omp2.c:40 given dL/drho_p
 *     in gdens: adds g_p * W to the mesh gradient gden (float, may be NULL)
 *     and, when den (the interpolated mesh) is given, g_p * dW/dx * den to
 *     the position gradients.
 * The Gaussian smoothing of gsmooth.c:14 is self-adjoint (a real, even
 * filter): gf_gaussian_smooth of a mesh gradient is its adjoint. */
int gf_tsc_adjoint(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev, const float *gden,
                   double *gx, double *gy, double *gz, double *gm);
int gf_find_den_adjoint(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev,
                        const float *den, const double *gdens, float *gden, double *gx,
                        double *gy, double *gz);

/* Galaxy-centre refinement (no reference counterpart; compared with the
 * search of GalCenter/find_centers.c:25-104): gradient ascent of each centre
 * (cx, cy, cz: FP64 device arrays, in the frame of its halo's mesh, updated
 * in place) on that halo's smoothed density den (halo_dev[c]; may be NULL
 * for one halo): up to max_steps moves of step_frac times the mesh's
 * smoothing length along the gradient; a move that does not raise the
 * density is not taken and halves the step.  rho receives the final density
 * and moves the number of moves taken.  One launch for all centres. */
int gf_refine_centres(gf_ctx *ctx, int32_t nhalo, const gf_mesh_desc *mesh_dev, const float *den,
                      int32_t ncentre, const int32_t *halo_dev, double *cx, double *cy, double *cz,
                      int max_steps, double step_frac, double *rho, int32_t *moves);

/* Density peaks of one halo's kNN graph (finddenpeak,
 * NewGalFinder/subhaloden.mod6.c:416-494): particles with den > threshold
 * (and type == GF_TYPE_STAR when type is not NULL) whose kNN list holds no
 * denser particle.  den (np), neighbor (np*numneighbor, halo-local int32) and
 * type are device arrays; up to cap peak indices go to peak (device) in
 * particle order; *npeak (host) receives the number found (GF_ERANGE when it
 * exceeds cap). */
int gf_density_peaks(gf_ctx *ctx, int32_t np, int numneighbor, const float *den, const int32_t *neighbor,
                     const int32_t *type, double threshold, int32_t cap, int32_t *peak, int32_t *npeak);
/* Core densities and core members (FindCoreDensity,
 * NewGalFinder/subhaloden.mod6.c:1167-1475), all arrays on the device: per
 * core c (peak[c]) the density threshold is bisected between den[peak] and
 * max(DENFLOOR, min den) until |(up - down)/t| <= COREDENRESOLUTION, a trial
 * t failing when a breadth-first search from the peak along kNN edges through
 * particles with den > t reaches another peak; coredensity[c] = up, and the
 * particles reached at up are the members (none if another peak is reached):
 * nummem, numstar (GF_TYPE_STAR members), starmass (their mass, summed in
 * FP64 and rounded to float; the reference adds in float in its search
 * order).  haloid[i] = the highest core index that reached i, -9999
 * (NOT_HALO_MEMBER) for none; flag[i] = PEAK (0x01) for peaks | CORE|BOUND
 * (0x14) for members.  Uses up to about 1 GiB of scratch for concurrent
 * searches. */
int gf_core_density(gf_ctx *ctx, int32_t np, int numneighbor, const float *den, const int32_t *neighbor,
                    const int32_t *type, const double *mass, int32_t ncore, const int32_t *peak,
                    float *coredensity, int32_t *nummem, int32_t *numstar, float *starmass, int32_t *haloid,
                    uint8_t *flag);

/* Strict 26-neighbour maxima of every mesh above threshold, in the interior
 * [margin, n - margin) of each axis (the mesh peak test of nnost.c:1176-1200;
 * lagFindStellarCore uses margin NCELLBUFF/2 and PEAKTHRESHOLD).  Up to cap
 * peaks are written (halo, cell offset within the halo's mesh, value) in no
 * particular order; *npeak receives the number found (may exceed cap). */
int gf_mesh_peaks(gf_ctx *ctx, int32_t nhalo, const gf_mesh_desc *mesh_host,
                  const gf_mesh_desc *mesh_dev, const float *den, int margin, float threshold,
                  int64_t cap, int32_t *out_halo, int64_t *out_cell, float *out_val,
                  int64_t *npeak);

/* ------------------------------------------------------------------------
 * Centre-of-mass octree (ost.c:532-699 Make_Tree / divide_node, nnost.c:105-254
 * new_Make_Tree_Near), kNN + SPH density (nnost.c:375-422 Find_Near,
 * :560-630 findsphdensity) and Barnes-Hut potential (ost.c:226-251
 * treeplumpotential; subhaloden.mod6.c:1477-1621) on device buffers.
 * pos4: float4 (x, y, z, mass) per particle, recentred per halo; halo h is
 * [pstart[h], pstart[h+1]).  Outputs are in input (batch) order.
 * ---------------------------------------------------------------------- */
typedef struct gf_tree_info {
    int64_t nparticle;
    int32_t nhalo;
    int32_t nnode;
} gf_tree_info;

/* Builds the octree (kept in ctx until the next build). */
int gf_tree_build(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                  const float *pos4_dev, float theta2, int q5_asbuilt, gf_tree_info *info);
/* Copies the last tree to host memory: preorder potential nodes (80 bytes
 * each), kNN nodes (48 bytes each), tree-ordered float4 positions, the
 * tree-order -> batch-index permutation and each halo's preorder root/end.
 * Any pointer may be NULL. */
int gf_tree_export(gf_ctx *ctx, void *bh_nodes, void *knn_nodes, float *pos4, int32_t *perm,
                   int32_t *root, int32_t *rend);
/* k nearest neighbours (self included, k <= 32, ordered by distance then
 * index; halo-local indices, -1 past a halo's size) and W4 density. */
int gf_knn_density(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                   const float *pos4_dev, int k, int32_t *nearindex, float *dens);
/* The same search for the nq particles listed in qidx (batch indices):
 * row q of nearindex (halo-local indices) and dens belongs to qidx[q]. */
int gf_knn_query(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                 const float *pos4_dev, int k, int64_t nq, const int64_t *qidx_dev,
                 int32_t *nearindex, float *dens);
/* Adjoint of the W4 density rho_i = sum_j W4(|x_i - x_j|, r_k/2)
 * (nnost.c:536-630) with respect to the FP64 positions x, y, z (batch
 * order): for each row q (particle qidx[q], or q when qidx is NULL) with its
 * neighbour list nearindex[q*k ..] (halo-local, from the forward search) and
 * upstream gradient gdens[q], adds to gx/gy/gz the terms of the pair
 * distances and of the kernel width h = r_k/2. */
int gf_knn_density_adjoint(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                           const double *x, const double *y, const double *z, int k, int64_t nq,
                           const int64_t *qidx_dev, const int32_t *nearindex, const double *gdens,
                           double *gx, double *gy, double *gz);
/* The same term as the stage's potential kernels evaluate it on the device,
 * for n halo masses (device arrays; stream ordered on ctx).  The device has no
 * x87 long double, so its intermediates are double where the reference's
 * (and gf_bg_potent's) are long double. */
int gf_bg_potent_device(gf_ctx *ctx, int32_t n, const double *mvir_dev, double *bg_dev);
/* The NFW tidal-radius table of mkRtidal (mkRtidal.c:80-128) into a device
 * buffer of gf_nfw_rtidal_cells() floats, laid out as the reference's
 * tidal_den (mass ratio fastest, then distance, then concentration); and
 * nfw_rtidal (mkRtidal.c:60-78) for n (mass ratio, distance / Rvir, c)
 * triples of device arrays on such a table.  Stream ordered on ctx. */
int gf_nfw_rtidal_cells(void);
int gf_nfw_rtidal_table(gf_ctx *ctx, float *table_dev);
int gf_nfw_rtidal_lookup(gf_ctx *ctx, int64_t n, const float *mM_dev, const float *dRv_dev,
                         const float *c_dev, const float *table_dev, float *out_dev);
/* Self potential of every halo: penergy = phi * potentfact + bg(halo mass)
 * (bg only if add_bg); halos with fewer than ndirect particles are summed
 * directly.  raw (optional) receives phi itself. */
int gf_self_potential(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
                      const float *pos4_dev, float theta2, int32_t ndirect, double potentfact,
                      int add_bg, float *penergy, float *raw);

/* ------------------------------------------------------------------------
 * The whole per-halo stage on a batch: FP64 recentring (Dump2BP) with
 * periodic unwrap, octree, kNN + SPH density, TSC mesh + smoothing + findDen,
 * and the self potential of every halo.
 * ---------------------------------------------------------------------- */
typedef struct gf_stage_config {
    gf_mesh_rule mesh;
    double box;            /* periodic box size, cMpc/h (0: no unwrap) */
    int32_t knn_k;         /* neighbours per particle incl. self (0: skip kNN) */
    int32_t do_mesh;       /* TSC + smoothing + findDen */
    int32_t do_potential;  /* tree potential */
    int32_t ndirect;       /* direct-sum threshold (Self_Halo_Potent: 100) */
    float theta2;          /* opening parameter (0.5 in the reference) */
    int32_t add_bg;        /* add GetBGpotent of each halo's mass */
    int32_t q5_asbuilt;    /* reproduce ost.c:571's y*x in place of y*z */
    int32_t count_work;    /* with stats: also count kNN/potential work (slower) */
    double potentfact;     /* 0: from gf_get_physics() */
    int32_t mesh_onchip;   /* 1: 64^3 meshes run their whole mesh stage (TSC, smoothing,
                              findDen) in one thread-block cluster's distributed shared
                              memory; 0: every mesh through device memory (faster on the
                              benchmark catalogue: 18.2 vs 32.2 ms of smoothing) */
    int32_t plain_fp64;    /* 1: the plain FP64 stage (every phase in FP64 by straightforward
                              kernels, meshes in device memory), the baseline the batched
                              FP32 stage is compared with */
} gf_stage_config;

typedef struct gf_stage_out {
    int32_t *nearindex;    /* device, n*knn_k halo-local indices */
    float *dens_sph;       /* device, n (may be NULL) */
    float *dens_mesh;      /* device, n (may be NULL) */
    float *penergy;        /* device, n (may be NULL) */
    double *xr, *yr, *zr;  /* device, n recentred positions (may be NULL) */
    float *phi;            /* device, n raw tree potential before potentfact and the
                              background term, i.e. penergy = (float)(phi*potentfact + bg)
                              (may be NULL) */
} gf_stage_out;

typedef struct gf_stage_stats {
    int64_t nparticle, nnode, mesh_cells;
    int32_t nhalo, reserved;
    uint64_t pp_interactions, pc_interactions;
    float ms_recentre, ms_tree, ms_knn, ms_tsc, ms_smooth, ms_findden, ms_potential, ms_pad;
    /* kNN work: nodes tested, 32-wide leaf batches, candidates passing the
     * float filter, candidates inserted one by one, bitonic batch merges */
    uint64_t knn_nodes, knn_batches, knn_candidates, knn_single_inserts, knn_bitonic_merges;
    /* meshes: floats laid out in device memory (mesh_cells counts every
     * planned mesh), and the meshes and particles of the on-chip path */
    int64_t mesh_cells_device, onchip_meshes, onchip_particles;
    /* cells of the pencils the three smoothing passes filtered, summed over
     * the passes (3 * mesh_cells_device without the occupied-box skips) */
    int64_t mesh_pass_cells;
} gf_stage_stats;

/* stats may be NULL; when given, per-phase CUDA-event times are filled in. */
int gf_stage_run(gf_ctx *ctx, const gf_batch *b, const gf_stage_config *cfg, gf_stage_out *out,
                 gf_stage_stats *stats);

/* The stage captured as one CUDA graph on ctx's stream (no reference
 * counterpart: the reference runs the stage per halo on the host).
 * gf_stage_graph_create runs gf_stage_run once to plan (the meshes from the
 * halo extents, the octree's depth and node count; its outputs are this
 * batch's results), then captures a pass that computes the frames and meshes
 * on the device, builds the octree with a fixed depth (two levels above the
 * planned one) and node capacity (a quarter above), and runs every kernel of
 * the stage with no host round trip.  The batch, config and output structs
 * are copied: the device buffers they point to must stay allocated and are
 * read and written by every replay.
 *
 * gf_stage_graph_launch replays the graph asynchronously on the batch's
 * current contents; gf_stage_graph_sync waits and reports GF_ESTALE when a
 * replay no longer fitted the plan (a mesh changed shape or the octree
 * outgrew the fixed depth or capacity: its outputs are then not valid) or
 * when the context's scratch buffers moved (another call on ctx needed more).
 * gf_stage_graph_run launches, waits and, on GF_ESTALE, re-plans and
 * re-captures (the eager planning run leaves valid outputs) and sets
 * *replanned.  Graphs capture the batched FP32 stage with device-memory
 * meshes (GF_ENOTIMPL for plain_fp64 or mesh_onchip); stats are not kept. */
typedef struct gf_stage_graph gf_stage_graph;
int gf_stage_graph_create(gf_ctx *ctx, const gf_batch *b, const gf_stage_config *cfg, gf_stage_out *out,
                          gf_stage_graph **graph);
int gf_stage_graph_launch(gf_stage_graph *graph);
int gf_stage_graph_sync(gf_stage_graph *graph);
int gf_stage_graph_run(gf_stage_graph *graph, int32_t *replanned);
int gf_stage_graph_replans(const gf_stage_graph *graph);
/* Kernel nodes and all nodes of the captured graph. */
int gf_stage_graph_nodes(const gf_stage_graph *graph, int32_t *kernels, int32_t *nodes);
void gf_stage_graph_destroy(gf_stage_graph *graph);

#ifdef __cplusplus
}
#endif
#endif
