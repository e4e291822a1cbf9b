// The TSC stencil of one particle: cells and weights of the reference's mass
// assignment (NewGalFinder/tsc_omp2.c:303-343) and interpolation (:51-94,
// :96-124), for the XYZDBL build (FP64 positions, float offsets).  Every
// operation is written with an explicitly rounded intrinsic in the order the
// reference evaluates it, so the weights and the interpolated sums are
// bit-identical to the reference's in any translation unit, whatever its
// floating-point contraction setting.
#pragma once

#include "gf_internal.cuh"

namespace gf {

struct TscStencil {
    int64_t i[3], j[3], k[3];  // near, near + sign, near - sign per axis
    float wx[3], wy[3], wz[3];
};

// Position -> mesh coordinate, nearest node and float offset (tsc_omp2.c:303-314).
__device__ __forceinline__ void tsc_axis_rn(double pos, double origin, double cellsize, int64_t &near1,
                                            int64_t &near2, int64_t &near3, float &d1) {
    const double xp = __ddiv_rn(__dsub_rn(pos, origin), cellsize);
    const double nr = rint(xp);
    const float rem = __double2float_rn(__dsub_rn(xp, nr));
    const int64_t sgn = (int64_t)copysignf(1.f, rem);
    near1 = (int64_t)nr;
    near2 = near1 + sgn;
    near3 = near1 - sgn;
    d1 = fabsf(rem);
}

__device__ __forceinline__ void tsc_cells(double x, double y, double z, const gf_mesh_desc &m, TscStencil &s,
                                          float &xd1, float &yd1, float &zd1) {
    tsc_axis_rn(x, m.xmin, m.cellsize, s.i[0], s.i[1], s.i[2], xd1);
    tsc_axis_rn(y, m.ymin, m.cellsize, s.j[0], s.j[1], s.j[2], yd1);
    tsc_axis_rn(z, m.zmin, m.cellsize, s.k[0], s.k[1], s.k[2], zd1);
}

// The stencil spans [near - 1, near + 1] on every axis.
__device__ __forceinline__ bool tsc_in_mesh(const TscStencil &s, const gf_mesh_desc &m) {
    return s.i[0] >= 1 && s.i[0] + 1 < m.nx && s.j[0] >= 1 && s.j[0] + 1 < m.ny && s.k[0] >= 1 &&
           s.k[0] + 1 < m.nz;
}

// 0.75 - d^2 (the centre weight)
__device__ __forceinline__ double tsc_w1(float d) { return __dsub_rn(0.75, (double)__fmul_rn(d, d)); }
// 0.25 + d (d - 1) (twice the outer weight)
__device__ __forceinline__ double tsc_w3x2(float d) {
    return __dadd_rn(0.25, __dmul_rn((double)d, __dsub_rn((double)d, 1.)));
}

// Deposit weights, tsc_omp2.c:335-343: the mass folded into the x weights,
// double intermediates rounded to float at each assignment.
__device__ __forceinline__ void tsc_deposit_weights(TscStencil &s, float xd1, float yd1, float zd1,
                                                    double pmas0) {
    const double p05 = __dmul_rn(pmas0, 0.5);
    s.wx[0] = __double2float_rn(__dmul_rn(tsc_w1(xd1), pmas0));
    s.wy[0] = __double2float_rn(tsc_w1(yd1));
    s.wz[0] = __double2float_rn(tsc_w1(zd1));
    s.wx[2] = __double2float_rn(__dmul_rn(p05, tsc_w3x2(xd1)));
    s.wx[1] = __double2float_rn(__dadd_rn((double)s.wx[2], __dmul_rn(pmas0, (double)xd1)));
    s.wy[2] = __double2float_rn(__dmul_rn(0.5, tsc_w3x2(yd1)));
    s.wy[1] = __fadd_rn(s.wy[2], yd1);
    s.wz[2] = __double2float_rn(__dmul_rn(0.5, tsc_w3x2(zd1)));
    s.wz[1] = __fadd_rn(s.wz[2], zd1);
}

// Interpolation weights, tsc_omp2.c:75-83.
__device__ __forceinline__ void tsc_interp_weights(TscStencil &s, float xd1, float yd1, float zd1) {
    s.wx[0] = __double2float_rn(tsc_w1(xd1));
    s.wy[0] = __double2float_rn(tsc_w1(yd1));
    s.wz[0] = __double2float_rn(tsc_w1(zd1));
    s.wx[2] = __double2float_rn(__dmul_rn(0.5, tsc_w3x2(xd1)));
    s.wx[1] = __fadd_rn(s.wx[2], xd1);
    s.wy[2] = __double2float_rn(__dmul_rn(0.5, tsc_w3x2(yd1)));
    s.wy[1] = __fadd_rn(s.wy[2], yd1);
    s.wz[2] = __double2float_rn(__dmul_rn(0.5, tsc_w3x2(zd1)));
    s.wz[1] = __fadd_rn(s.wz[2], zd1);
}

// Deposit of cell (a, b, c) of the stencil: (wx wy) wz, times volfold (1 or
// an exact power of two).
__device__ __forceinline__ float tsc_deposit_value(const TscStencil &s, int a, int b, int c, float volfold) {
    return __fmul_rn(__fmul_rn(__fmul_rn(s.wx[a], s.wy[b]), s.wz[c]), volfold);
}

// One term of the interpolation, tsc_omp2.c:96-124: density += (v wxwy) wz,
// summed over z planes c, y rows b, x cells a in that order.
__device__ __forceinline__ float tsc_interp_add(float density, float v, const TscStencil &s, int a, int b,
                                                int c) {
    return __fadd_rn(density, __fmul_rn(__fmul_rn(v, __fmul_rn(s.wx[a], s.wy[b])), s.wz[c]));
}

}  // namespace gf
