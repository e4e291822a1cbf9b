/* Test harness around the reference's FoF catalogue reader and GALFIND
 * writer helpers (NewGalFinder/gfind.c: FREAD :23-91, GetHaloInfo :557-617,
 * GetSubHaloInfo :618-689), compiled from the reference's own gfind.c with
 * the MPI stub.  Reports the reference build's record layouts (sizeof and
 * field offsets) so that the product's numpy record types can be pinned.
 * Test infrastructure only: built by oracle/Makefile into
 * oracle/_ref/libgfref_io.so; nothing here calls MPI or gfind.c's main. */
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "Memory.h"
#include "header.h"
#include "ramses.h"
#include "tree.h"
#include "defs.h"
#include "params.h"
/* defs.h renames some globals by macro (mpeak -> D_mpeak, den -> D_den); the
 * field `den` of GasType is not one of them */
#undef den

void FREAD(FoFTPtlStruct *p, HaloQ *haloq, FILE *fp, float omep);
HaloInfo GetHaloInfo(FoFTPtlStruct *bp, int np);
void GetSubHaloInfo(FoFTPtlStruct *bp, int np, lint *rptl2halonum, int id, SubInfo *shalo, size_t *asize,
                    void *subdata);
extern FoFTPtlStruct *rbuffer;
extern size_t nbuffer;
extern int mpeak;

static int g_ready = 0;

int io_init(long long megabytes) {
    if (g_ready) return 0;
    if (Make_Total_Memory(megabytes) == 0) return -1;
    g_ready = 1;
    return 0;
}

#define OFF(T, f) (long long)offsetof(T, f)
/* sizes and field offsets of the record types (see the Python side for the order) */
int io_layout(long long *out) {
    int k = 0;
    out[k++] = sizeof(HaloQ);
    out[k++] = OFF(HaloQ, np); out[k++] = OFF(HaloQ, npstar); out[k++] = OFF(HaloQ, npgas);
    out[k++] = OFF(HaloQ, npdm); out[k++] = OFF(HaloQ, npsink); out[k++] = OFF(HaloQ, x);
    out[k++] = OFF(HaloQ, mass); out[k++] = OFF(HaloQ, vx);
    out[k++] = sizeof(DmType);
    out[k++] = OFF(DmType, x); out[k++] = OFF(DmType, mass); out[k++] = OFF(DmType, id);
    out[k++] = OFF(DmType, levelp); out[k++] = OFF(DmType, family); out[k++] = OFF(DmType, tag);
    out[k++] = OFF(DmType, tp); out[k++] = OFF(DmType, zp); out[k++] = OFF(DmType, chem);
    out[k++] = OFF(DmType, mass0); out[k++] = OFF(DmType, birth_d); out[k++] = OFF(DmType, partp);
    out[k++] = sizeof(GasType);
    out[k++] = OFF(GasType, x); out[k++] = OFF(GasType, cellsize); out[k++] = OFF(GasType, vx);
    out[k++] = OFF(GasType, den); out[k++] = OFF(GasType, temp); out[k++] = OFF(GasType, metallicity);
    out[k++] = OFF(GasType, chem); out[k++] = OFF(GasType, mass); out[k++] = OFF(GasType, potent);
    out[k++] = sizeof(SinkType);
    out[k++] = OFF(SinkType, x); out[k++] = OFF(SinkType, mass); out[k++] = OFF(SinkType, tbirth);
    out[k++] = OFF(SinkType, Jx); out[k++] = OFF(SinkType, Sx); out[k++] = OFF(SinkType, dMsmbh);
    out[k++] = OFF(SinkType, Esave); out[k++] = OFF(SinkType, id);
    out[k++] = sizeof(StarType);
    out[k++] = sizeof(HaloInfo);
    out[k++] = OFF(HaloInfo, nsub); out[k++] = OFF(HaloInfo, totm); out[k++] = OFF(HaloInfo, x);
    out[k++] = sizeof(SubInfo);
    out[k++] = OFF(SubInfo, npdm); out[k++] = OFF(SubInfo, totm); out[k++] = OFF(SubInfo, x);
    return k;
}

/* Reads halo `index` (0-based) of a catalogue / member-file pair with the
 * reference's FREAD; the particles' type, x, y, z, vx, vy, vz, mass and
 * float link02 go to the output arrays (np entries).  Returns np, or -1. */
long long io_fread(const char *catfile, const char *memfile, long long index, float omep, int *type,
                   double *x, double *y, double *z, double *vx, double *vy, double *vz, double *mass,
                   float *link02, long long cap) {
    if (!g_ready) return -1;
    FILE *hf = fopen(catfile, "rb"), *mf = fopen(memfile, "rb");
    if (!hf || !mf) return -1;
    HaloQ q;
    long long np = -1;
    FoFTPtlStruct *p = NULL;
    for (long long h = 0; h <= index; h++) {
        if (fread(&q, sizeof(HaloQ), 1, hf) != 1) { np = -1; goto done; }
        if ((long long)q.np > cap) { np = -1; goto done; }
        if (!rbuffer) {
            nbuffer = 1024;
            rbuffer = (FoFTPtlStruct *)Malloc(sizeof(FoFTPtlStruct) * nbuffer, PPTR(rbuffer));
        }
        if (!p) p = (FoFTPtlStruct *)Malloc(sizeof(FoFTPtlStruct) * (size_t)cap, PPTR(p));
        FREAD(p, &q, mf, omep);
        np = (long long)q.np;
    }
    for (long long i = 0; i < np; i++) {
        type[i] = (int)p[i].type;
        x[i] = p[i].x; y[i] = p[i].y; z[i] = p[i].z;
        vx[i] = p[i].vx; vy[i] = p[i].vy; vz[i] = p[i].vz;
        mass[i] = p[i].mass; link02[i] = p[i].link02;
    }
done:
    if (p) Free(p);
    fclose(hf); fclose(mf);
    return np;
}

/* The records write_data (gfind.c:690-732) writes for one halo read from a
 * member file (halo `index`): the HaloInfo (nsub = nsub), then for each
 * sub-halo id in [0, nsub) its SubInfo and particle records, then the
 * background's (id NOT_HALO_MEMBER) SubInfo and records.  membership[i] is
 * each particle's sub-halo id.  Returns the number of bytes written to out
 * (up to cap), or -1. */
long long io_write_halo(const char *catfile, const char *memfile, long long index, float omep, int nsub,
                        const long long *membership, char *out, long long cap) {
    if (!g_ready) return -1;
    FILE *hf = fopen(catfile, "rb"), *mf = fopen(memfile, "rb");
    if (!hf || !mf) return -1;
    HaloQ q;
    FoFTPtlStruct *p = NULL;
    long long np = 0, size = 0;
    for (long long h = 0; h <= index; h++) {
        if (fread(&q, sizeof(HaloQ), 1, hf) != 1) { size = -1; goto done; }
        if (!rbuffer) {
            nbuffer = 1024;
            rbuffer = (FoFTPtlStruct *)Malloc(sizeof(FoFTPtlStruct) * nbuffer, PPTR(rbuffer));
        }
        if (p) { Free(p); p = NULL; }
        p = (FoFTPtlStruct *)Malloc(sizeof(FoFTPtlStruct) * (q.np > 0 ? q.np : 1), PPTR(p));
        FREAD(p, &q, mf, omep);
        np = (long long)q.np;
    }
    {
        lint *m = (lint *)malloc(sizeof(lint) * (size_t)(np > 0 ? np : 1));
        for (long long i = 0; i < np; i++) m[i] = (lint)membership[i];
        mpeak = nsub;
        HaloInfo hinfo = GetHaloInfo(p, (int)np);
        hinfo.nsub = nsub;
        if (size + (long long)sizeof(HaloInfo) > cap) { free(m); size = -1; goto done; }
        memcpy(out + size, &hinfo, sizeof(HaloInfo)); size += sizeof(HaloInfo);
        void *sub = malloc(sizeof(FoFTPtlStruct) * (size_t)(np > 0 ? np : 1));
        for (int i = -1; i < nsub; i++) {
            const int id = i < 0 ? NOT_HALO_MEMBER : i;  /* background last, as a separate file */
            if (i < 0) continue;
            SubInfo si; size_t sz = 0;
            GetSubHaloInfo(p, (int)np, m, id, &si, &sz, sub);
            if (size + (long long)(sizeof(SubInfo) + sz) > cap) { size = -1; break; }
            memcpy(out + size, &si, sizeof(SubInfo)); size += sizeof(SubInfo);
            memcpy(out + size, sub, sz); size += (long long)sz;
        }
        if (size >= 0) {
            SubInfo si; size_t sz = 0;
            GetSubHaloInfo(p, (int)np, m, NOT_HALO_MEMBER, &si, &sz, sub);
            if (size + (long long)(sizeof(SubInfo) + sz) > cap) size = -1;
            else {
                memcpy(out + size, &si, sizeof(SubInfo)); size += sizeof(SubInfo);
                memcpy(out + size, sub, sz); size += (long long)sz;
            }
        }
        free(sub);
        free(m);
    }
done:
    if (p) Free(p);
    fclose(hf); fclose(mf);
    return size;
}
