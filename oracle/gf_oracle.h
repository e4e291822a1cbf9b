/* CPU restatement of the reference's density-and-potential stage — the oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this library, and only to check results
 * (or the timed CPU baseline); the product path never calls it.
 *
 * Every function cites the reference file:line it restates.  Pinned by
 * tests/test_oracle_pin.py against golden fixtures produced by the
 * reference's own code (tests/golden/make_golden.py). */
#ifndef GF_ORACLE_H
#define GF_ORACLE_H
#include <stdint.h>

/* tsc_omp2.c:166-506.  acc_double = 0: float accumulation in the order the
 * reference run with `ref_threads` OpenMP threads uses (bit-identical to it);
 * 1: double accumulation rounded once at the end. */
int or_tsc(int64_t np, const double *x, const double *y, const double *z, const double *mass,
           const int32_t *type, float *den, int nx, int ny, int nz, double xmin, double ymin,
           double zmin, double cellsize, int ptype, int acc_double, int ref_threads);

/* tsc_omp2.c:40-163 */
int or_find_den(int64_t np, const double *x, const double *y, const double *z, float *densph,
                double xmin, double ymin, double zmin, double cellsize, const float *den, int nx,
                int ny, int nz);

/* gsmooth.c:14-115 evaluated in FP64 (exact separable spectral filter, see
 * gf_oracle.c); den is float in/out, out64 (optional) receives the FP64
 * result on the logical mx*ny*nz layout. */
int or_smooth(float *den, int nx, int ny, int nz, double cellsize, float rg, double *out64);

/* Exact k nearest neighbours (self included) of every particle by brute
 * force, ordered by (d^2, index).  Positions are the FP32 recentred values;
 * d^2 is evaluated in double with separately rounded operations
 * (dx*dx + dy*dy) + dz*dz, the order of nnost.c:405-408. */
int or_knn_brute(int64_t np, const float *x, const float *y, const float *z, int k,
                 int64_t *idx, double *d2);

/* Cell-list exact kNN, same result as or_knn_brute, for larger np. */
int or_knn_grid(int64_t np, const float *x, const float *y, const float *z, int k,
                int64_t *idx, double *d2);

/* findsphdensity's density (nnost.c:609-622) from sorted d^2 lists:
 * rho_i = sum_j W4(sqrtf(d2_ij), sqrtf(d2_ik)/2) in the reference's float/double
 * arithmetic (W4: nnost.c:536-555). */
int or_sph_density(int64_t np, int k, const double *d2, float *dens);
int or_star_density(int64_t np, int k, const double *d2, const int64_t *sidx, const int32_t *cnt,
                    const float *smass, float *dens);



/* FP64 walk of a tree exported by libgf (same opening decisions, exact
 * terms): ost.c:72-83 (treeopen), :144-193 (cell/particle terms), :226-251.
 * nodes: preorder records of gf_tree_export (80 bytes each); sources in tree
 * order; topen[t] != 0 opens every node (direct sum). */
int or_tree_potential(int32_t nnode, const void *nodes, int64_t nsrc, const float *sx,
                      const float *sy, const float *sz, const float *sm, int64_t ntgt,
                      const float *tx, const float *ty, const float *tz, const int32_t *troot,
                      const int32_t *trend, const int32_t *topen, double *phi);

/* FP64 direct-sum potential (subhaloden.mod6.c:1493-1503 in double). */
int or_direct_potential(int64_t nsrc, const float *sx, const float *sy, const float *sz,
                        const float *sm, int64_t ntgt, const float *tx, const float *ty,
                        const float *tz, double *phi);
#endif
