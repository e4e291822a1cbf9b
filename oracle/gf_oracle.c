/* CPU restatement of the reference's density stage — the oracle.
 * TEST INFRASTRUCTURE ONLY (see gf_oracle.h): never linked into libgf.
 *
 * Built with -ffp-contract=off so that every float/double operation is
 * rounded separately, as in the reference built the same way. */
#include "gf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* --------------------------------------------------------------------- TSC */

typedef struct {
    long long i[3], j[3], k[3];
    float wx[3], wy[3], wz[3];
} stencil_t;

/* tsc_omp2.c:303-314 / :51-71: double mesh coordinate, rint, float offset */
static void axis(double pos, double origin, double cellsize, long long *n3, float *d1) {
    double xp = (pos - origin) / cellsize;
    long long nr = (long long)rint(xp);
    float rem = (float)(xp - (double)nr);
    long long sg = (long long)copysignf(1.f, rem);
    n3[0] = nr;
    n3[1] = nr + sg;
    n3[2] = nr - sg;
    *d1 = fabsf(rem);
}

static int stencil_ok(const stencil_t *s, int nx, int ny, int nz) {
    return s->i[0] >= 1 && s->i[0] + 1 < nx && s->j[0] >= 1 && s->j[0] + 1 < ny && s->k[0] >= 1 &&
           s->k[0] + 1 < nz;
}

int or_tsc(int64_t np, const double *x, const double *y, const double *z, const double *mass,
           const int32_t *type, float *den, int nx, int ny, int nz, double xmin, double ymin,
           double zmin, double cellsize, int ptype, int acc_double, int ref_threads) {
    const long long mx = 2 * (nx / 2 + 1);
    const long long ncell = mx * ny * nz;
    double *acc = NULL;
    if (acc_double) acc = (double *)calloc((size_t)ncell, sizeof(double));
    for (long long c = 0; c < ncell; c++) den[c] = 0.f;
    int bad = 0;
    /* tsc_omp2.c:210-270: the reference deposits in two passes over the
     * particles; a particle goes to pass 1 or 2 by its slab position along
     * the longest mesh axis, split among `mthreads` threads.  Within one pass
     * a cell is touched by one thread only, so its float sum runs over the
     * pass-1 particles in index order, then the pass-2 particles. */
    int nxyz = nx > ny ? nx : ny;
    nxyz = nxyz > nz ? nxyz : nz;
    int nthreads = ref_threads < 1 ? 1 : ref_threads, mthreads;
    double xwidth = (double)nxyz / (double)nthreads;
    if (0.5 * xwidth < 5) mthreads = (int)((double)nxyz / (2 * 5.));
    else mthreads = nthreads;
    double Xwidth = (double)nxyz / (double)mthreads;
    signed char *target = (signed char *)malloc((size_t)np + 1);
    for (int64_t p = 0; p < np; p++) {
        double xp;
        if (nxyz == nx) xp = (x[p] - xmin) / cellsize;
        else if (nxyz == ny) xp = (y[p] - ymin) / cellsize;
        else xp = (z[p] - zmin) / cellsize;
        int j = (int)(xp / Xwidth) + 1;
        int k = (int)((long double)(xp / Xwidth) + 0.5L) + 1;
        if (j >= mthreads + 1) target[p] = (signed char)mthreads;
        else if (k == j) target[p] = (signed char)-j;
        else target[p] = (signed char)j;
    }
    for (int pass = 0; pass < 2; pass++)
    for (int64_t p = 0; p < np; p++) {
        if (ptype != 5 && (type ? type[p] : 2) != ptype) continue;
        if ((pass == 0) != (target[p] < 0)) continue;
        stencil_t s;
        float xd1, yd1, zd1;
        axis(x[p], xmin, cellsize, s.i, &xd1);
        axis(y[p], ymin, cellsize, s.j, &yd1);
        axis(z[p], zmin, cellsize, s.k, &zd1);
        if (!stencil_ok(&s, nx, ny, nz)) { bad = 1; continue; }
        /* tsc_omp2.c:335-343 */
        double pmas0 = mass[p], p05 = pmas0 * 0.5;
        s.wx[0] = (float)((0.75 - (double)(xd1 * xd1)) * pmas0);
        s.wy[0] = (float)(0.75 - (double)(yd1 * yd1));
        s.wz[0] = (float)(0.75 - (double)(zd1 * zd1));
        s.wx[2] = (float)(p05 * (0.25 + (double)xd1 * ((double)xd1 - 1.)));
        s.wx[1] = (float)((double)s.wx[2] + pmas0 * (double)xd1);
        s.wy[2] = (float)(0.5 * (0.25 + (double)yd1 * ((double)yd1 - 1.)));
        s.wy[1] = s.wy[2] + yd1;
        s.wz[2] = (float)(0.5 * (0.25 + (double)zd1 * ((double)zd1 - 1.)));
        s.wz[1] = s.wz[2] + zd1;
        /* tsc_omp2.c:354-382: z planes in order 1,2,3; y rows 1,2,3; x 1,2,3 */
        for (int c = 0; c < 3; c++)
            for (int b = 0; b < 3; b++)
                for (int a = 0; a < 3; a++) {
                    float wxy = s.wx[a] * s.wy[b];
                    float w = wxy * s.wz[c];
                    long long o = s.i[a] + mx * (s.j[b] + (long long)ny * s.k[c]);
                    if (acc_double) acc[o] += (double)w;
                    else den[o] += w;
                }
    }
    free(target);
    /* tsc_omp2.c:188,497: den *= volfact, volfact = (0.001/0.004)^3 */
    const double r = 0.001 / 0.004;
    const double volfact = r * r * r;
    for (long long c = 0; c < ncell; c++) {
        if (acc_double) den[c] = (float)(acc[c] * volfact);
        else den[c] = (float)(den[c] * volfact);
    }
    free(acc);
    return bad;
}

int or_find_den(int64_t np, const double *x, const double *y, const double *z, float *densph,
                double xmin, double ymin, double zmin, double cellsize, const float *den, int nx,
                int ny, int nz) {
    const long long mx = 2 * (nx / 2 + 1);
    int bad = 0;
    for (int64_t p = 0; p < np; p++) {
        stencil_t s;
        float xd1, yd1, zd1;
        axis(x[p], xmin, cellsize, s.i, &xd1);
        axis(y[p], ymin, cellsize, s.j, &yd1);
        axis(z[p], zmin, cellsize, s.k, &zd1);
        if (!stencil_ok(&s, nx, ny, nz)) { bad = 1; densph[p] = 0.f; continue; }
        /* tsc_omp2.c:75-83 */
        s.wx[0] = (float)(0.75 - (double)(xd1 * xd1));
        s.wy[0] = (float)(0.75 - (double)(yd1 * yd1));
        s.wz[0] = (float)(0.75 - (double)(zd1 * zd1));
        s.wx[2] = (float)(0.5 * (0.25 + (double)xd1 * ((double)xd1 - 1.)));
        s.wx[1] = s.wx[2] + xd1;
        s.wy[2] = (float)(0.5 * (0.25 + (double)yd1 * ((double)yd1 - 1.)));
        s.wy[1] = s.wy[2] + yd1;
        s.wz[2] = (float)(0.5 * (0.25 + (double)zd1 * ((double)zd1 - 1.)));
        s.wz[1] = s.wz[2] + zd1;
        /* tsc_omp2.c:95-127: density += (den * wxwy) * wz, same term order */
        float density = 0.f;
        for (int c = 0; c < 3; c++)
            for (int b = 0; b < 3; b++)
                for (int a = 0; a < 3; a++) {
                    float wxy = s.wx[a] * s.wy[b];
                    float v = den[s.i[a] + mx * (s.j[b] + (long long)ny * s.k[c])];
                    density += (v * wxy) * s.wz[c];
                }
        densph[p] = density;
    }
    return bad;
}

/* -------------------------------------------------------------- smoothing */
/* gsmooth.c multiplies the r2c spectrum of the (nz, ny, nx) mesh by
 * exp(expfac (k^2/nz^2 + j^2/ny^2 + i^2/nx^2)), expfac = -(pi RG/cellsize)^2,
 * signed k, j and i in [0, nx/2], then c2r and 1/(nx ny nz).  That factor is
 * a product of real even per-axis factors, so the result is the mesh
 * circularly convolved along each axis with h_n[m] = (1/n) sum_k G_n(k)
 * cos(2 pi k m/n).  Evaluated here in FP64 with the exact kernels. */
static void kernel_h(int n, double rg_cells, double *h) {
    const double expfac = -(M_PI * rg_cells) * (M_PI * rg_cells);
    double *g = (double *)malloc(sizeof(double) * n);
    for (int k = 0; k < n; k++) {
        long ks = k > n / 2 ? k - n : k;
        g[k] = exp((double)(ks * ks) * expfac / ((double)n * (double)n));
    }
    for (int m = 0; m < n; m++) {
        double acc = 0.0;
        for (int k = 0; k < n; k++) acc += g[k] * cos(2.0 * M_PI * (double)(((long)k * m) % n) / n);
        h[m] = acc / n;
    }
    free(g);
}

static void conv_axis(double *a, int n, long long stride, long long count_outer,
                      long long outer_stride, long long count_inner, long long inner_stride,
                      const double *h) {
    double *in = (double *)malloc(sizeof(double) * n);
    for (long long o = 0; o < count_outer; o++)
        for (long long q = 0; q < count_inner; q++) {
            double *base = a + o * outer_stride + q * inner_stride;
            for (int s = 0; s < n; s++) in[s] = base[s * stride];
            for (int s = 0; s < n; s++) {
                double acc = 0.0;
                for (int m = 0; m < n; m++) {
                    int idx = s - m;
                    if (idx < 0) idx += n;
                    acc += h[m] * in[idx];
                }
                base[s * stride] = acc;
            }
        }
    free(in);
}

int or_smooth(float *den, int nx, int ny, int nz, double cellsize, float rg, double *out64) {
    const long long mx = 2 * (nx / 2 + 1);
    const long long ncell = mx * ny * nz;
    const double rg_cells = (double)(float)(rg / cellsize); /* gsmooth.c:67 */
    double *a = (double *)malloc(sizeof(double) * ncell);
    for (long long c = 0; c < ncell; c++) a[c] = den[c];
    double *h = (double *)malloc(sizeof(double) * (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)));
    kernel_h(nx, rg_cells, h);
    conv_axis(a, nx, 1, (long long)ny * nz, mx, 1, 0, h);           /* rows */
    kernel_h(ny, rg_cells, h);
    conv_axis(a, ny, mx, nz, mx * ny, nx, 1, h);                     /* y pencils */
    kernel_h(nz, rg_cells, h);
    conv_axis(a, nz, mx * ny, ny, mx, nx, 1, h);                     /* z pencils */
    for (long long k = 0; k < nz; k++)
        for (long long j = 0; j < ny; j++)
            for (long long i = 0; i < nx; i++) {
                long long o = i + mx * (j + (long long)ny * k);
                den[o] = (float)a[o];
                if (out64) out64[o] = a[o];
            }
    free(h);
    free(a);
    return 0;
}

/* -------------------------------------------------------------------- kNN */
/* d^2 in the operation order of nnost.c:405-408, each op rounded */
static inline double dist2(const float *x, const float *y, const float *z, int64_t i, int64_t j) {
    double dx = (double)x[i] - (double)x[j];
    double dy = (double)y[i] - (double)y[j];
    double dz = (double)z[i] - (double)z[j];
    return dx * dx + dy * dy + dz * dz;
}

static inline int key_less(double da, int64_t ia, double db, int64_t ib) {
    return da < db || (da == db && ia < ib);
}

/* insert (d, j) into the sorted list of length *cnt (capacity k) */
static inline void list_insert(double *ld, int64_t *li, int *cnt, int k, double d, int64_t j) {
    if (*cnt == k && !key_less(d, j, ld[k - 1], li[k - 1])) return;
    int pos = *cnt < k ? *cnt : k - 1;
    while (pos > 0 && key_less(d, j, ld[pos - 1], li[pos - 1])) {
        ld[pos] = ld[pos - 1];
        li[pos] = li[pos - 1];
        pos--;
    }
    ld[pos] = d;
    li[pos] = j;
    if (*cnt < k) (*cnt)++;
}

int or_knn_brute(int64_t np, const float *x, const float *y, const float *z, int k,
                 int64_t *idx, double *d2) {
    if (k > np) return 1;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < np; i++) {
        double *ld = d2 + i * k;
        int64_t *li = idx + i * k;
        int cnt = 0;
        for (int64_t j = 0; j < np; j++) list_insert(ld, li, &cnt, k, dist2(x, y, z, i, j), j);
    }
    return 0;
}

/* cell list with ring search: exact because a ring is only skipped once the
 * k-th distance is below the ring's minimum distance */
int or_knn_grid(int64_t np, const float *x, const float *y, const float *z, int k,
                int64_t *idx, double *d2) {
    if (k > np) return 1;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    const float *c[3] = {x, y, z};
    for (int64_t i = 0; i < np; i++)
        for (int a = 0; a < 3; a++) {
            if (c[a][i] < lo[a]) lo[a] = c[a][i];
            if (c[a][i] > hi[a]) hi[a] = c[a][i];
        }
    double ext = 0;
    for (int a = 0; a < 3; a++) ext = fmax(ext, hi[a] - lo[a]);
    int g = (int)cbrt((double)np / 4.0);
    if (g < 1) g = 1;
    if (g > 256) g = 256;
    double cell = ext / g * 1.000001 + 1e-300;
    int dim[3];
    for (int a = 0; a < 3; a++) {
        dim[a] = (int)((hi[a] - lo[a]) / cell) + 1;
    }
    long long ncell = (long long)dim[0] * dim[1] * dim[2];
    int64_t *head = (int64_t *)malloc(sizeof(int64_t) * (ncell + 1));
    int64_t *order = (int64_t *)malloc(sizeof(int64_t) * np);
    int *cid = (int *)malloc(sizeof(int) * np * 3);
    memset(head, 0, sizeof(int64_t) * (ncell + 1));
    for (int64_t i = 0; i < np; i++) {
        int q[3];
        for (int a = 0; a < 3; a++) {
            q[a] = (int)((c[a][i] - lo[a]) / cell);
            if (q[a] >= dim[a]) q[a] = dim[a] - 1;
            cid[3 * i + a] = q[a];
        }
        head[(q[2] * (long long)dim[1] + q[1]) * dim[0] + q[0] + 1]++;
    }
    for (long long cc = 0; cc < ncell; cc++) head[cc + 1] += head[cc];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * ncell);
    memcpy(fill, head, sizeof(int64_t) * ncell);
    for (int64_t i = 0; i < np; i++) {
        long long cc = ((long long)cid[3 * i + 2] * dim[1] + cid[3 * i + 1]) * dim[0] + cid[3 * i];
        order[fill[cc]++] = i;
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < np; i++) {
        double *ld = d2 + i * k;
        int64_t *li = idx + i * k;
        int cnt = 0;
        const int *q = cid + 3 * i;
        for (int r = 0;; r++) {
            /* every cell at Chebyshev ring distance r from q */
            for (int dz = -r; dz <= r; dz++)
                for (int dy = -r; dy <= r; dy++)
                    for (int dx = -r; dx <= r; dx++) {
                        if (abs(dx) != r && abs(dy) != r && abs(dz) != r) continue;
                        int cx = q[0] + dx, cy = q[1] + dy, cz = q[2] + dz;
                        if (cx < 0 || cy < 0 || cz < 0 || cx >= dim[0] || cy >= dim[1] || cz >= dim[2])
                            continue;
                        long long cc = ((long long)cz * dim[1] + cy) * dim[0] + cx;
                        for (int64_t t = head[cc]; t < head[cc + 1]; t++) {
                            int64_t j = order[t];
                            list_insert(ld, li, &cnt, k, dist2(x, y, z, i, j), j);
                        }
                    }
            /* particles outside ring r are at least r*cell away (minus the
             * offset inside the own cell); stop once the k-th is closer */
            if (cnt == k) {
                double rmin = (double)r * cell;
                /* conservative: subtract nothing extra, ring r+1 starts beyond r*cell
                 * from any point of the centre cell */
                if (ld[k - 1] < rmin * rmin) break;
            }
            if (r > dim[0] + dim[1] + dim[2]) break;
        }
    }
    free(fill);
    free(cid);
    free(order);
    free(head);
    return 0;
}

/* ------------------------------------------------------------ SPH density */
/* W4, nnost.c:536-555: float arguments, double constants */
static float W4(float dist, float h) {
    float twomr, r;
    r = dist / h;
    if (r < 1.) {
        return (float)((-0.2387324) * ((2. - r) * r * r - 1.333333) / (double)(h * h * h));
    } else if (r < 2.) {
        twomr = (float)((2. - r) / h);
        return (float)(0.07957747 * twomr * twomr * twomr);
    }
    return 0.f;
}

int or_sph_density(int64_t np, int k, const double *d2, float *dens) {
    for (int64_t i = 0; i < np; i++) {
        const double *l = d2 + i * k;
        /* Find_Near's maxr = sqrtf(maxdist2) (nnost.c:292,415), then h = maxr/2 */
        float neardist = sqrtf((float)l[k - 1]);
        float rho = 0.f;
        for (int j = 0; j < k; j++) {
            float dj = sqrtf((float)l[j]); /* nnost.c:620: dist2[j] = sqrtf(dist2[j]) */
            rho += W4(dj, (float)(neardist / 2.));
        }
        dens[i] = rho;
    }
    return 0;
}

/* starfindsphdensity's stellar density, nnost.c:687-703: for each particle,
 * over its k nearest stars in distance order (d2: their exact FP64 squared
 * distances; sidx: star indices into smass, the stars' masses as float),
 * W4(sqrtf(d2_j), r_k/2) * m_j summed in float, r_k = sqrtf of the last d2
 * (Find_Near's maxr).  cnt[i] < k where the halo has fewer than k stars. */
int or_star_density(int64_t np, int k, const double *d2, const int64_t *sidx, const int32_t *cnt,
                    const float *smass, float *dens) {
    for (int64_t i = 0; i < np; i++) {
        const double *l = d2 + i * k;
        const int64_t *s = sidx + i * k;
        const int res = cnt[i];
        float rho = 0.f;
        if (res > 0) {
            float neardist = sqrtf((float)l[res - 1]);
            for (int j = 0; j < res; j++) {
                float dj = sqrtf((float)l[j]);
                rho += W4(dj, (float)(neardist / 2.)) * smass[s[j]];
            }
        }
        dens[i] = rho;
    }
    return 0;
}

/* ---------------------------------------------------------------- potential */
/* Node record exported by libgf (gf_tree_export), preorder. */
typedef struct {
    double com[3];
    double open_r2;
    float mass, trq;
    float q[6];
    int32_t skip, lstart, lcount, count;
} or_bhnode;

/* FP64 evaluation of the walk of ost.c:226-251 on a given tree: the same
 * opening decisions as the tree's owner (|t - com|^2 < open_r2 evaluated
 * with the same separately rounded double operations), exact terms -m/r for
 * opened loose particles, and for accepted cells the monopole + quadrupole
 * expansion about the node's exported centre with mass and second moments
 * recomputed in FP64 from the node's particles.  (Cell term of
 * CELLPLUMPOTENT, ost.c:144-176, with exact kernels in place of the spline
 * tables.) */
int or_tree_potential(int32_t nnode, const void *nodes_v, int64_t nsrc, const float *sx,
                      const float *sy, const float *sz, const float *sm, int64_t ntgt,
                      const float *tx, const float *ty, const float *tz, const int32_t *troot,
                      const int32_t *trend, const int32_t *topen, double *phi) {
    const or_bhnode *nodes = (const or_bhnode *)nodes_v;
    double *M = (double *)malloc(sizeof(double) * (nnode > 0 ? nnode : 1));
    double *Q = (double *)malloc(sizeof(double) * 6 * (nnode > 0 ? nnode : 1));
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < nnode; i++) {
        const or_bhnode *nd = nodes + i;
        double m = 0, q[6] = {0, 0, 0, 0, 0, 0};
        for (int64_t j = nd->lstart; j < (int64_t)nd->lstart + nd->count; j++) {
            double dx = (double)sx[j] - nd->com[0], dy = (double)sy[j] - nd->com[1],
                   dz = (double)sz[j] - nd->com[2], w = sm[j];
            m += w;
            q[0] += w * dx * dx; q[1] += w * dy * dy; q[2] += w * dz * dz;
            q[3] += w * dx * dy; q[4] += w * dx * dz; q[5] += w * dy * dz;
        }
        M[i] = m;
        for (int a = 0; a < 6; a++) Q[6 * (int64_t)i + a] = q[a];
    }
    (void)nsrc;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t t = 0; t < ntgt; t++) {
        const double px = (double)tx[t], py = (double)ty[t], pz = (double)tz[t];
        double acc = 0.0;
        int32_t i = troot[t];
        const int32_t end = trend[t];
        while (i < end) {
            const or_bhnode *nd = nodes + i;
            const double dx = px - nd->com[0], dy = py - nd->com[1], dz = pz - nd->com[2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            if ((topen && topen[t]) || d2 < nd->open_r2) {
                for (int64_t j = nd->lstart; j < (int64_t)nd->lstart + nd->lcount; j++) {
                    double ex = px - sx[j], ey = py - sy[j], ez = pz - sz[j];
                    double r2 = ex * ex + ey * ey + ez * ez;
                    if (r2 > 0) acc += -(double)sm[j] / sqrt(r2);
                }
                i = i + 1;
            } else {
                const double *q = Q + 6 * (int64_t)i;
                const double r = sqrt(d2);
                const double qxy = q[0] * dx * dx + q[1] * dy * dy + q[2] * dz * dz +
                                   2. * (q[3] * dx * dy + q[4] * dx * dz + q[5] * dy * dz);
                acc += -M[i] / r + 0.5 * (q[0] + q[1] + q[2]) / (r * r * r) -
                       1.5 * qxy / (r * r * r * r * r);
                i = nd->skip;
            }
        }
        phi[t] = acc;
    }
    free(Q);
    free(M);
    return 0;
}

/* FP64 direct sum: phi_t = sum over sources at nonzero distance of -m/r. */
int or_direct_potential(int64_t nsrc, const float *sx, const float *sy, const float *sz,
                        const float *sm, int64_t ntgt, const float *tx, const float *ty,
                        const float *tz, double *phi) {
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < ntgt; t++) {
        double acc = 0.0;
        const double px = tx[t], py = ty[t], pz = tz[t];
        for (int64_t j = 0; j < nsrc; j++) {
            double ex = px - sx[j], ey = py - sy[j], ez = pz - sz[j];
            double r2 = ex * ex + ey * ey + ez * ez;
            if (r2 > 0) acc += -(double)sm[j] / sqrt(r2);
        }
        phi[t] = acc;
    }
    return 0;
}
