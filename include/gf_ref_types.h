/* Data layouts of the reference's hot-path interfaces, restated so that the
 * drop-in entry points in gf.h take exactly the bytes the reference's callers
 * pass.  Field order, types and padding must match the reference (built with
 * -DXYZDBL and without -DDOUBLE_PRECISION, NewGalFinder/Makefile.in:29):
 *
 *   SimpleBasicParticleType  NewGalFinder/tree.h:155-162   88 bytes
 *   Vector3d                 NewGalFinder/subhaloden.mod6.c:70-72   24 bytes
 *   Coretype                 NewGalFinder/tree.h:204-213   56 bytes
 *
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

#ifdef __cplusplus
}
#endif
#endif
