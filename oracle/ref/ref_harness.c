/* Harness around the reference's own hot-path functions (compiled unmodified
 * from NewGalFinder/*.c by oracle/ref/Makefile).  It defines the globals the
 * reference expects from gfind.c (cosmology, potentfact, rank ids), sets up
 * the reference's stack arena (Memory2.c:Make_Total_Memory) and the potential
 * spline table (force_spline.mod3.c:81), and exposes plain-array entry points
 * that ctypes can call.
 *
 * Test infrastructure only: used to generate golden fixtures, to pin the
 * oracle restatement, and as the CPU baseline ("reference" kind).  Never
 * linked into the product library. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "Memory.h"
#include "ramses.h"
#include "tree.h"
#include "defs.h"
#include "params.h"

/* ---- globals normally defined by gfind.c (names renamed by defs.h) ---- */
int myid = 0, nid = 1;
double onesolarmass = 1.0;
double com2real, real2com, potentfact, pntmass, r1kineticfact, r2kineticfact;
float amax = 1.f, a = 1.f, rng = 1.f, size = 100.f, hubble = 70.f;
int ng = 0, nspace = 1, nx = 0, ny = 0, nz = 0;
float omep = 0.3f, omeplam = 0.7f, acoeff[8];
float epsilon = 0.f;
float m_tidal[10000], r_tidal[10000]; /* NUM_MASS, header.h:97 */

/* ---- reference functions (signatures from the cited files) ---- */
typedef struct Vector3d { double x, y, z; } Vector3d; /* subhaloden.mod6.c:70 */
void i_potent_spline(void);                                          /* force_spline.mod3.c:81 */
void findsphdensity(SimpleBasicParticleType *, int, long long *, int, float *); /* nnost.c:560 */
void starfindsphdensity(SimpleBasicParticleType *, int, long long *, int, float *); /* nnost.c:632 */
void lagFindStellarCore(SimpleBasicParticleType *, int, int, float *, Coretype **, int *, int,
                        long long *, int);                           /* nnost.c:991 */
void assign_density_TSC(SimpleBasicParticleType *, int, float *, int, int, int, double, double,
                        double, double, int);                        /* tsc_omp2.c:166 */
void findDen(SimpleBasicParticleType *, int, float *, double, double, double, double, float *,
             int, int, int);                                         /* tsc_omp2.c:40 */
void gaussian_Smoothing(float *, int, int, int, double, float);      /* gsmooth.c:14 */
void new_Make_Tree_Near(TStruct *, size_t, TPtlStruct *, size_t, int); /* nnost.c:199 */
int Find_Near(particle *, int, TStruct *, TPtlStruct *, float *, long long *, dptype *, float *);
void Self_Halo_Potent(int, Vector3d *, float *, float *);            /* subhaloden.mod6.c:1477 */
void External_Halo_Potent(int, Vector3d *, float *, float *, int, Vector3d *, float *);
double GetBGpotent(double);                                          /* subhaloden.mod6.c:1093 */

static int g_ready = 0;

/* gfind.c:842-890 (physical_parameters), second assignment block, which is
 * the one that takes effect. */
static void set_physics(void) {
    float omepk = 1.f - omep - omeplam;
    float h0 = hubble / 100.f;
    float Hsub = sqrt(omep * pow(amax / a, 3) + omeplam + omepk * pow(amax / a, 2));
    com2real = 1.L / h0 * a / amax * Mpc;
    real2com = 1.L / com2real;
    pntmass = Msun / h0;
    potentfact = 6.672E-8L * pntmass / com2real; /* G from header.h:1 */
    r1kineticfact = 100.E5L * Hsub * a / amax;
    r2kineticfact = 1.E5L;
}

int ref_init(long long megabytes) {
    if (g_ready) return 0;
    if (!Make_Total_Memory(megabytes * MEGABYTE)) return -1;
    i_potent_spline();
    set_physics();
    g_ready = 1;
    return 0;
}

void ref_set_cosmology(float amax_, float a_, float omep_, float omeplam_, float hubble_) {
    amax = amax_; a = a_; omep = omep_; omeplam = omeplam_; hubble = hubble_;
    set_physics();
}

double ref_get_potentfact(void) { return potentfact; }
double ref_get_r1kineticfact(void) { return r1kineticfact; }
double ref_get_r2kineticfact(void) { return r2kineticfact; }
double ref_GetBGpotent(double mvir) { return GetBGpotent(mvir); }

static SimpleBasicParticleType *make_bp(int np, const int *type, const double *x, const double *y,
                                        const double *z, const double *mass) {
    SimpleBasicParticleType *bp = NULL;
    bp = (SimpleBasicParticleType *)Malloc(sizeof(SimpleBasicParticleType) * (size_t)np, PPTR(bp));
    for (int i = 0; i < np; i++) {
        memset(&bp[i], 0, sizeof(bp[i]));
        bp[i].type = type ? (unsigned)type[i] : TYPE_DM;
        bp[i].mass = mass ? mass[i] : 1.0;
        bp[i].x = x[i];
        bp[i].y = y[i];
        bp[i].z = z[i];
        bp[i].indx = i;
    }
    return bp;
}

int ref_findsphdensity(int np, const double *x, const double *y, const double *z,
                       const double *mass, long long *nearindex, int k, float *dens) {
    if (!g_ready) return -1;
    SimpleBasicParticleType *bp = make_bp(np, NULL, x, y, z, mass);
    findsphdensity(bp, np, nearindex, k, dens);
    Free(bp);
    return 0;
}

/* starfindsphdensity: stellar density (10 nearest stars, mass weighted) and
 * the neighbour lists; the particles' types select the stars. */
int ref_starfindsphdensity(int np, const int *type, const double *x, const double *y, const double *z,
                           const double *mass, long long *nearindex, int k, float *dens) {
    if (!g_ready) return -1;
    SimpleBasicParticleType *bp = make_bp(np, type, x, y, z, mass);
    starfindsphdensity(bp, np, nearindex, k, dens);
    Free(bp);
    return 0;
}

/* Runs lagFindStellarCore and returns the per-particle mesh density, the
 * neighbour lists and the mesh-peak cores (peak index, x, y, z, density). */
int ref_lagFindStellarCore(int np, const int *type, const double *x, const double *y,
                           const double *z, const double *mass, int k, float *dens,
                           long long *nearindex, int ptype, int maxcore, int *ncore,
                           int *core_peak, float *core_xyzd) {
    if (!g_ready) return -1;
    SimpleBasicParticleType *bp = make_bp(np, type, x, y, z, mass);
    Coretype *core = NULL;
    core = (Coretype *)Malloc(sizeof(Coretype) * (size_t)maxcore, PPTR(core));
    int numcore = 0;
    lagFindStellarCore(bp, np, k, dens, &core, &numcore, maxcore, nearindex, ptype);
    *ncore = numcore;
    for (int c = 0; c < numcore; c++) {
        core_peak[c] = core[c].peak;
        core_xyzd[4 * c + 0] = core[c].cx;
        core_xyzd[4 * c + 1] = core[c].cy;
        core_xyzd[4 * c + 2] = core[c].cz;
        core_xyzd[4 * c + 3] = core[c].density;
    }
    if (numcore > 0) Free(core);
    Free(bp);
    return 0;
}

int ref_assign_density_TSC(int np, const int *type, const double *x, const double *y,
                           const double *z, const double *mass, float *den, int nx_, int ny_,
                           int nz_, double xmin, double ymin, double zmin, double cellsize,
                           int ptype) {
    if (!g_ready) return -1;
    SimpleBasicParticleType *bp = make_bp(np, type, x, y, z, mass);
    assign_density_TSC(bp, np, den, nx_, ny_, nz_, xmin, ymin, zmin, cellsize, ptype);
    Free(bp);
    return 0;
}

int ref_findDen(int np, const double *x, const double *y, const double *z, float *densph,
                double xmin, double ymin, double zmin, double cellsize, float *den, int nx_,
                int ny_, int nz_) {
    if (!g_ready) return -1;
    SimpleBasicParticleType *bp = make_bp(np, NULL, x, y, z, NULL);
    findDen(bp, np, densph, xmin, ymin, zmin, cellsize, den, nx_, ny_, nz_);
    Free(bp);
    return 0;
}

int ref_gaussian_Smoothing(float *den, int nx_, int ny_, int nz_, double cellsize, float rg) {
    if (!g_ready) return -1;
    gaussian_Smoothing(den, nx_, ny_, nz_, cellsize, rg);
    return 0;
}

/* new_Make_Tree_Near + Find_Near for every particle (the findsphdensity
 * inner loop without the density), returning the raw lists. */
int ref_find_near_all(int np, const double *x, const double *y, const double *z,
                      const double *mass, int k, long long *idx, double *d2, float *maxr) {
    if (!g_ready) return -1;
    particle *p = NULL;
    TPtlStruct *ptl = NULL;
    TStruct *tree = NULL;
    p = (particle *)Malloc(sizeof(particle) * (size_t)np, PPTR(p));
    ptl = (TPtlStruct *)Malloc(sizeof(TPtlStruct) * (size_t)np, PPTR(ptl));
    size_t nnode = (size_t)(np / 2 > 650000 ? np / 2 : 650000);
    tree = (TStruct *)Malloc(sizeof(TStruct) * nnode, PPTR(tree));
    for (int i = 0; i < np; i++) {
        p[i].x = x[i]; p[i].y = y[i]; p[i].z = z[i];
        ptl[i].type = TYPE_PTL;
        ptl[i].x = x[i]; ptl[i].y = y[i]; ptl[i].z = z[i];
        ptl[i].mass = mass ? mass[i] : 1.0;
    }
    new_Make_Tree_Near(tree, nnode, ptl, (size_t)np, RECURSIVE);
#pragma omp parallel for schedule(guided)
    for (int i = 0; i < np; i++) {
        float mass_k[MAX_NUM_NEAR];
        Find_Near(p + i, k, tree, ptl, maxr + i, idx + (size_t)i * k, d2 + (size_t)i * k, mass_k);
    }
    Free(tree);
    Free(ptl);
    Free(p);
    return 0;
}

int ref_Self_Halo_Potent(int np, const double *x, const double *y, const double *z,
                         float *mass, float *penergy) {
    if (!g_ready) return -1;
    Vector3d *r = NULL;
    r = (Vector3d *)Malloc(sizeof(Vector3d) * (size_t)np, PPTR(r));
    for (int i = 0; i < np; i++) { r[i].x = x[i]; r[i].y = y[i]; r[i].z = z[i]; }
    Self_Halo_Potent(np, r, mass, penergy);
    Free(r);
    return 0;
}

int ref_External_Halo_Potent(int nend, const double *x, const double *y, const double *z,
                             float *mass, float *penergy, int snp, const double *sx,
                             const double *sy, const double *sz, float *smass) {
    if (!g_ready) return -1;
    Vector3d *r = NULL, *sr = NULL;
    r = (Vector3d *)Malloc(sizeof(Vector3d) * (size_t)nend, PPTR(r));
    sr = (Vector3d *)Malloc(sizeof(Vector3d) * (size_t)snp, PPTR(sr));
    for (int i = 0; i < nend; i++) { r[i].x = x[i]; r[i].y = y[i]; r[i].z = z[i]; }
    for (int i = 0; i < snp; i++) { sr[i].x = sx[i]; sr[i].y = sy[i]; sr[i].z = sz[i]; }
    External_Halo_Potent(nend, r, mass, penergy, snp, sr, smass);
    Free(sr);
    Free(r);
    return 0;
}

/* Make_Tree (SERIALIZED, as Self_Halo_Potent builds it) + treeplumpotential at
 * every particle: the raw tree potential before potentfact and the NFW term. */
void Make_Tree(TStruct *, size_t, TPtlStruct *, size_t, float, int);
float treeplumpotential(particle *, float, TStruct *, TPtlStruct *);
int ref_tree_potential(int np, const double *x, const double *y, const double *z,
                       const float *mass, float theta2, float *phi) {
    if (!g_ready) return -1;
    TPtlStruct *ptl = NULL;
    TStruct *tree = NULL;
    size_t nnode = (size_t)(np / 2 > 650000 ? np / 2 : 650000);
    tree = (TStruct *)Malloc(sizeof(TStruct) * nnode, PPTR(tree));
    ptl = (TPtlStruct *)Malloc(sizeof(TPtlStruct) * (size_t)np, PPTR(ptl));
    for (int i = 0; i < np; i++) {
        ptl[i].type = TYPE_PTL;
        ptl[i].x = x[i]; ptl[i].y = y[i]; ptl[i].z = z[i];
        ptl[i].mass = mass[i];
    }
    Make_Tree(tree, nnode, ptl, (size_t)np, theta2, SERIALIZED);
#pragma omp parallel for schedule(guided)
    for (int i = 0; i < np; i++) {
        particle p;
        p.x = x[i]; p.y = y[i]; p.z = z[i];
        phi[i] = treeplumpotential(&p, theta2, tree, ptl);
    }
    Free(ptl);
    Free(tree);
    return 0;
}

/* ---- boundedness test and tidal radius (subhaloden.mod6.c) ---- */
typedef struct Kptype_h {
    double x, y, z;
    float vx, vy, vz, mass;
    SimpleBasicParticleType *bp;
} Kptype_h;                                                      /* subhaloden.mod6.c:73-77 */
typedef struct Coresorttype_h { int nmem; Coretype *core; } Coresorttype_h; /* :298-301 */
typedef struct WorkingParticle_h {
    float den;
    int haloid;
    unsigned char flag;
    unsigned char flag2[64];
} WorkingParticle_h;                                             /* :246-251, MAXTHREADS 64 */
extern WorkingParticle_h *wp;
int CheckSelfTE(Kptype_h *, int, unsigned char *, Coretype *);
int CheckExternalTE(Kptype_h *, int, unsigned char *, Kptype_h *, int, Coretype *);
void AdGetTidalRCenterCore(Coretype *, int, Coresorttype_h *, int, SimpleBasicParticleType *, int);

static Kptype_h *make_kp(int n, const double *x, const double *y, const double *z, const float *vx,
                         const float *vy, const float *vz, const float *mass,
                         SimpleBasicParticleType *bp) {
    Kptype_h *kp = (Kptype_h *)malloc(sizeof(Kptype_h) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) {
        kp[i].x = x[i]; kp[i].y = y[i]; kp[i].z = z[i];
        kp[i].vx = vx[i]; kp[i].vy = vy[i]; kp[i].vz = vz[i];
        kp[i].mass = mass[i];
        kp[i].bp = bp ? bp + i : NULL;
    }
    return kp;
}

int ref_CheckSelfTE(int np, const double *x, const double *y, const double *z, const float *vx,
                    const float *vy, const float *vz, const float *mass, const int *type,
                    unsigned char *flag) {
    if (!g_ready) return -1;
    SimpleBasicParticleType *bp = make_bp(np, type, x, y, z, NULL);
    Kptype_h *kp = make_kp(np, x, y, z, vx, vy, vz, mass, bp);
    int nb = CheckSelfTE(kp, np, flag, NULL);
    free(kp);
    Free(bp);
    return nb;
}

int ref_CheckExternalTE(int tnp, const double *x, const double *y, const double *z,
                        const float *vx, const float *vy, const float *vz, const float *mass,
                        int snp, const double *sx, const double *sy, const double *sz,
                        const float *smass, const float *core6, unsigned char *flag) {
    if (!g_ready) return -1;
    Kptype_h *tkp = make_kp(tnp, x, y, z, vx, vy, vz, mass, NULL);
    float *zero = (float *)calloc((size_t)(snp > 0 ? snp : 1), sizeof(float));
    Kptype_h *skp = make_kp(snp, sx, sy, sz, zero, zero, zero, smass, NULL);
    Coretype core;
    memset(&core, 0, sizeof(core));
    core.cx = core6[0]; core.cy = core6[1]; core.cz = core6[2];
    core.cvx = core6[3]; core.cvy = core6[4]; core.cvz = core6[5];
    int nb = CheckExternalTE(tkp, tnp, flag, skp, snp, &core);
    free(skp); free(zero); free(tkp);
    return nb;
}

int ref_AdGetTidalRCenterCore(int np, const double *x, const double *y, const double *z,
                              const double *mass, const int *haloid, int numcore,
                              const float *core6, int ncore, const int *score_core,
                              float *rtidal, int *nummem) {
    if (!g_ready) return -1;
    SimpleBasicParticleType *bp = make_bp(np, NULL, x, y, z, mass);
    WorkingParticle_h *w = (WorkingParticle_h *)calloc((size_t)(np > 0 ? np : 1), sizeof(WorkingParticle_h));
    for (int i = 0; i < np; i++) w[i].haloid = haloid[i];
    WorkingParticle_h *saved = wp;
    wp = w;
    Coretype *core = (Coretype *)calloc((size_t)numcore, sizeof(Coretype));
    for (int c = 0; c < numcore; c++) {
        core[c].cx = core6[6 * c]; core[c].cy = core6[6 * c + 1]; core[c].cz = core6[6 * c + 2];
        core[c].cvx = core6[6 * c + 3]; core[c].cvy = core6[6 * c + 4]; core[c].cvz = core6[6 * c + 5];
    }
    Coresorttype_h *score = (Coresorttype_h *)calloc((size_t)(ncore > 0 ? ncore : 1), sizeof(Coresorttype_h));
    for (int a = 0; a < ncore; a++) { score[a].core = core + score_core[a]; score[a].nmem = 0; }
    AdGetTidalRCenterCore(core, numcore, score, ncore, bp, np);
    for (int c = 0; c < numcore; c++) { rtidal[c] = core[c].Rtidal; nummem[c] = core[c].nummem; }
    wp = saved;
    free(score); free(core); free(w);
    Free(bp);
    return 0;
}

/* ---- core finding on the kNN graph (subhaloden.mod6.c:416-494, 1167-1475) ---- */
int finddenpeak(float *, int, long long *, int, Coretype **, int, SimpleBasicParticleType *);
int FindCoreDensity(SimpleBasicParticleType *, int, long long *, int, Coretype *, int);
void omp_set_num_threads(int);
int omp_get_max_threads(void);

/* finddenpeak on given densities and kNN lists; peak[] receives the peak
 * particles in the reference's order, xyzd[4 c] their float cx, cy, cz and
 * density.  Returns the number of peaks (at most maxcore are written). */
int ref_finddenpeak(int np, const float *den, const long long *neighbor, int numneigh, const int *type,
                    const double *x, const double *y, const double *z, int jflag, int maxcore,
                    int *peak, float *xyzd) {
    if (!g_ready) return -1;
    SimpleBasicParticleType *bp = make_bp(np, type, x, y, z, NULL);
    Coretype *core = NULL;
    core = (Coretype *)Malloc(sizeof(Coretype) * (size_t)MAXNUMCORE, PPTR(core));
    int nc = finddenpeak((float *)den, numneigh, (long long *)neighbor, np, &core, jflag, bp);
    for (int c = 0; c < nc && c < maxcore; c++) {
        peak[c] = core[c].peak;
        xyzd[4 * c] = core[c].cx; xyzd[4 * c + 1] = core[c].cy;
        xyzd[4 * c + 2] = core[c].cz; xyzd[4 * c + 3] = core[c].density;
    }
    Free(core);
    Free(bp);
    return nc;
}

/* FindCoreDensity on one thread (its member ids then follow the core order)
 * for the given densities, kNN lists and core peaks.  Outputs per core
 * (coredensity, nummem, numstar, starmass) and per particle (haloid, flag). */
int ref_FindCoreDensity(int np, const float *den, const long long *neighbor, int numneigh,
                        const int *type, const double *mass, int numcore, const int *peak,
                        float *coredensity, int *nummem, int *numstar, float *starmass,
                        int *haloid, unsigned char *flag) {
    if (!g_ready) return -1;
    double *zero = (double *)calloc((size_t)(np > 0 ? np : 1), sizeof(double));
    SimpleBasicParticleType *bp = make_bp(np, type, zero, zero, zero, mass);
    WorkingParticle_h *w = (WorkingParticle_h *)calloc((size_t)(np > 0 ? np : 1), sizeof(WorkingParticle_h));
    for (int i = 0; i < np; i++) w[i].den = den[i];
    WorkingParticle_h *saved = wp;
    wp = w;
    Coretype *core = (Coretype *)calloc((size_t)(numcore > 0 ? numcore : 1), sizeof(Coretype));
    for (int c = 0; c < numcore; c++) core[c].peak = peak[c];
    int nth = omp_get_max_threads();
    omp_set_num_threads(1);
    int r = FindCoreDensity(bp, np, (long long *)neighbor, numneigh, core, numcore);
    omp_set_num_threads(nth);
    for (int c = 0; c < numcore; c++) {
        coredensity[c] = core[c].coredensity; nummem[c] = core[c].nummem;
        numstar[c] = core[c].numstar; starmass[c] = core[c].starmass;
    }
    for (int i = 0; i < np; i++) { haloid[i] = w[i].haloid; flag[i] = w[i].flag; }
    wp = saved;
    free(core); free(w); free(zero);
    Free(bp);
    return r;
}

/* ---- the reference's per-halo pipeline (subhaloden.mod6.c:2861) ---- */
int subhalo_den(FoFTPtlStruct *, int, int *); /* lint is int, header.h:74 */

/* Runs subhalo_den on one FoF halo given as arrays (comoving positions in the
 * periodic box, velocities, masses, types; linking lengths from the masses as
 * gfind.c does); p2halo receives each particle's galaxy id (NOT_HALO_MEMBER
 * for none).  Returns subhalo_den's result (the number of galaxies). */
int ref_subhalo_den(int np, const int *type, const double *x, const double *y, const double *z,
                    const double *vx, const double *vy, const double *vz, const double *mass,
                    int *p2halo) {
    if (!g_ready) return -1;
    FoFTPtlStruct *rbp = (FoFTPtlStruct *)calloc((size_t)(np > 0 ? np : 1), sizeof(FoFTPtlStruct));
    for (int i = 0; i < np; i++) {
        rbp[i].type = (unsigned)type[i];
        rbp[i].x = x[i]; rbp[i].y = y[i]; rbp[i].z = z[i];
        rbp[i].vx = vx[i]; rbp[i].vy = vy[i]; rbp[i].vz = vz[i];
        rbp[i].mass = mass[i];
        rbp[i].indx = i;
        /* the FoF linking length of each particle, as gfind.c:49-88 sets it */
        rbp[i].link02 = 0.2 * pow(mass[i] / 2.7755e11L / omep, 0.33333333333333333333L);
    }
    int res = subhalo_den(rbp, np, p2halo);
    free(rbp);
    return res;
}
