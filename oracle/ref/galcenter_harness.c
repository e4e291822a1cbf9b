/* Harness around GalCenter's centre search (GalCenter/find_centers.c, compiled
 * unmodified by oracle/Makefile into _ref/libgalcenter.so).  It defines the
 * box size global the search reads and exposes find_centers on plain arrays.
 * Test infrastructure only: the search-based centres that the GPU's
 * gradient-ascent refinement is compared with. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mpi.h>

#include "Memory.h"
#include "header.h"
#include "ramses.h"
#include "tree.h"
#include "defs.h"
#include "galcenter.h"

float size = 100.f; /* the periodic box (cMpc/h); renamed by defs.h */

static int g_ready = 0;

int gc_init(long long megabytes) {
    if (g_ready) return 0;
    if (!Make_Total_Memory(megabytes * 1024LL * 1024LL)) return -1;
    g_ready = 1;
    return 0;
}

/* find_centers (find_centers.c:106) on one galaxy's particles: out[0..3] the
 * stellar centre (x, y, z, R), out[4..7] the dark-matter one. */
int gc_find_centers(int np, const int *type, const double *x, const double *y, const double *z,
                    const double *mass, double *out) {
    if (!g_ready) return -1;
    FoFTPtlStruct *bp = (FoFTPtlStruct *)calloc((size_t)(np > 0 ? np : 1), sizeof(FoFTPtlStruct));
    for (int i = 0; i < np; i++) {
        bp[i].type = (unsigned)type[i];
        bp[i].x = x[i]; bp[i].y = y[i]; bp[i].z = z[i];
        bp[i].mass = mass[i];
    }
    GalCenter gal;
    memset(&gal, 0, sizeof(gal));
    find_centers(&gal, bp, np);
    out[0] = gal.gal.x; out[1] = gal.gal.y; out[2] = gal.gal.z; out[3] = gal.gal.R;
    out[4] = gal.dmhalo.x; out[5] = gal.dmhalo.y; out[6] = gal.dmhalo.z; out[7] = gal.dmhalo.R;
    free(bp);
    return 0;
}
