/* Data layouts of the reference's hot-path interfaces, restated so that the
 * drop-in entry points in gf.h take exactly the bytes the reference's callers
 * pass.  Field order, types and padding must match the reference (built with
 * -DXYZDBL and without -DDOUBLE_PRECISION, NewGalFinder/Makefile.in:29):
 *
 *   SimpleBasicParticleType  NewGalFinder/tree.h:155-162   88 bytes
 *   Vector3d                 NewGalFinder/subhaloden.mod6.c:70-72   24 bytes
 *   Coretype                 NewGalFinder/tree.h:204-213   56 bytes
 *   Kptype                   NewGalFinder/subhaloden.mod6.c:73-77   48 bytes
 *   Coresorttype             NewGalFinder/subhaloden.mod6.c:298-301 16 bytes
 *   TPtlStruct               NewGalFinder/tree.h:72-77     56 bytes
 *   TStruct                  NewGalFinder/tree.h:79-91     176 bytes
 *   particle                 NewGalFinder/tree.h:145-149   40 bytes
 *
 * TPtlStruct and TStruct are the threaded tree of the reference's kNN and
 * potential walks (nnost.c and ost.c both include tree.h, and both read the
 * node size from `dist`): a node's `daughter` points to its first offspring
 * (a node or a particle), every offspring's `sibling` to the next one, and the
 * last offspring's `sibling` to the node's own sibling; `type` tells nodes
 * (GF_TYPE_TREE) from particles (GF_TYPE_PTL).
 * Only the layout is shared; no reference code is included. */
#ifndef GF_REF_TYPES_H
#define GF_REF_TYPES_H

#ifdef __cplusplus
extern "C" {
#endif

/* Particle-type tags, NewGalFinder/tree.h:47-48 */
enum {
    GF_TYPE_TREE = 0, GF_TYPE_PTL = 1, GF_TYPE_STAR = 1, GF_TYPE_DM = 2,
    GF_TYPE_GAS = 3, GF_TYPE_SINK = 4, GF_TYPE_ALL = 5
};

typedef struct SimpleBasicParticleType {
    unsigned int type;
    double mass, x, y, z;
    double vx, vy, vz;
    double link02;
    int indx;                                /* idtype = int (ramses.h:6-10) */
    struct SimpleBasicParticleType *bp;      /* linked-list pointer, unused here */
} SimpleBasicParticleType;

typedef struct Vector3d {
    double x, y, z;
} Vector3d;

typedef struct Coretype {
    int peak;
    int nummem, numstar;
    float starmass;
    float coredensity;
    float cx, cy, cz;
    float cvx, cvy, cvz;
    float Rtidal, density;
    unsigned char flag;
} Coretype;

typedef struct Kptype {
    double x, y, z;
    float vx, vy, vz, mass;
    SimpleBasicParticleType *bp;
} Kptype;

typedef struct Coresorttype {
    int nmem;
    Coretype *core;
} Coresorttype;

typedef struct TPtlStruct {
    unsigned int type;
    void *sibling;
    double x, y, z;
    double mass;
    int indx;
} TPtlStruct;

typedef struct TStruct {
    unsigned int type;
    void *sibling;
    void *daughter;
    double L;
    double dist, dist2;        /* node size max|x - com| and its square */
    double x0, y0, z0;
    double mass;
    int Nparticle;
    double monox, monoy, monoz; /* centre of mass */
    double trQ;
    double quad[6];            /* xx, yy, zz, xy, xz, yz second moments about the COM */
    double dist_over_thetasq;
} TStruct;

typedef struct particle {
    double x, y, z;
    double link02;
    int indx;
} particle;

/* Bound flags of CheckSelfTE/CheckExternalTE (subhaloden.mod6.c:32-33) */
#define GF_BOUND 1
#define GF_UNBOUND 0

#ifdef __cplusplus
}
#endif
#endif
