// TSC mass assignment and TSC-weighted mesh interpolation.
//
// This translation unit is compiled with --fmad=false: every float and
// double operation below is rounded separately, in the order the reference
// evaluates it, so the per-particle stencil weights are bit-identical to
// NewGalFinder/tsc_omp2.c:301-353 (deposit) and :51-94 (interpolation) for
// the same FP64 positions.  The only difference left in the deposited mesh
// is the order in which float atomics sum the contributions of different
// particles to one cell.
#include "gf_internal.cuh"

namespace gf {

namespace {

struct Stencil {
    int64_t i[3], j[3], k[3];
    float wx[3], wy[3], wz[3];
};

// Position -> mesh coordinate, nearest node and float offset, as
// tsc_omp2.c:303-314 (XYZDBL build: double xp, rint, float remainder).
__device__ __forceinline__ void tsc_axis(double pos, double origin, double cellsize,
                                         int64_t &near1, int64_t &near2, int64_t &near3,
                                         float &d1) {
    double xp = (pos - origin) / cellsize;
    double nr = rint(xp);
    float rem = (float)(xp - nr);
    int64_t sgn = (int64_t)copysignf(1.f, rem);
    near1 = (int64_t)nr;
    near2 = near1 + sgn;
    near3 = near1 - sgn;
    d1 = fabsf(rem);
}

__device__ __forceinline__ bool in_mesh(const Stencil &s, const gf_mesh_desc &m) {
    // the stencil spans [near-1, near+1] on every axis
    return s.i[0] >= 1 && s.i[0] + 1 < m.nx && s.j[0] >= 1 && s.j[0] + 1 < m.ny &&
           s.k[0] >= 1 && s.k[0] + 1 < m.nz;
}

__global__ void tsc_deposit_kernel(int64_t n, const double *__restrict__ x,
                                   const double *__restrict__ y, const double *__restrict__ z,
                                   const double *__restrict__ mass,
                                   const int32_t *__restrict__ type,
                                   const int32_t *__restrict__ hid,
                                   const gf_mesh_desc *__restrict__ mesh,
                                   float *__restrict__ den, float volfold, int *err,
                                   const int32_t *__restrict__ order) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        // with an order (the octree's permutation) a warp deposits spatial
        // neighbours, whose stencils share cache lines of the mesh
        const int64_t p = order ? (int64_t)order[t] : t;
        const gf_mesh_desc m = mesh[hid ? hid[p] : 0];
        if (m.ptype != GF_TYPE_ALL && (type ? type[p] : GF_TYPE_DM) != m.ptype) continue;
        Stencil s;
        float xd1, yd1, zd1;
        tsc_axis(x[p], m.xmin, m.cellsize, s.i[0], s.i[1], s.i[2], xd1);
        tsc_axis(y[p], m.ymin, m.cellsize, s.j[0], s.j[1], s.j[2], yd1);
        tsc_axis(z[p], m.zmin, m.cellsize, s.k[0], s.k[1], s.k[2], zd1);
        if (!in_mesh(s, m)) {
            atomicOr(err, GF_ERRBIT_RANGE);
            continue;
        }
        // tsc_omp2.c:335-343: mass folded into the x weights, double
        // intermediates rounded to float at each assignment.
        const double pmas0 = mass[p];
        const double p05 = pmas0 * 0.5;
        float wx1 = (float)((0.75 - (double)(xd1 * xd1)) * pmas0);
        float wy1 = (float)(0.75 - (double)(yd1 * yd1));
        float wz1 = (float)(0.75 - (double)(zd1 * zd1));
        float wx3 = (float)(p05 * (0.25 + (double)xd1 * ((double)xd1 - 1.)));
        float wx2 = (float)((double)wx3 + pmas0 * (double)xd1);
        float wy3 = (float)(0.5 * (0.25 + (double)yd1 * ((double)yd1 - 1.)));
        float wy2 = wy3 + yd1;
        float wz3 = (float)(0.5 * (0.25 + (double)zd1 * ((double)zd1 - 1.)));
        float wz2 = wz3 + zd1;
        s.wx[0] = wx1; s.wx[1] = wx2; s.wx[2] = wx3;
        s.wy[0] = wy1; s.wy[1] = wy2; s.wy[2] = wy3;
        s.wz[0] = wz1; s.wz[1] = wz2; s.wz[2] = wz3;
        const int64_t mx = 2 * (m.nx / 2 + 1);
        float *mesh_h = den + m.off;
#pragma unroll
        for (int c = 0; c < 3; c++) {
#pragma unroll
            for (int b = 0; b < 3; b++) {
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    float wxy = s.wx[a] * s.wy[b];
                    float w = wxy * s.wz[c];
                    // volfold is 1 or an exact power of two (see launch_tsc_deposit)
                    atomicAdd(mesh_h + s.i[a] + mx * (s.j[b] + (int64_t)m.ny * s.k[c]), w * volfold);
                }
            }
        }
    }
}

__global__ void find_den_kernel(int64_t n, const double *__restrict__ x,
                                const double *__restrict__ y, const double *__restrict__ z,
                                const int32_t *__restrict__ hid,
                                const gf_mesh_desc *__restrict__ mesh,
                                const float *__restrict__ den, float *__restrict__ densph,
                                int *err, const int32_t *__restrict__ order) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = order ? (int64_t)order[t] : t;  // octree order: shared stencil lines
        const gf_mesh_desc m = mesh[hid ? hid[p] : 0];
        Stencil s;
        float xd1, yd1, zd1;
        tsc_axis(x[p], m.xmin, m.cellsize, s.i[0], s.i[1], s.i[2], xd1);
        tsc_axis(y[p], m.ymin, m.cellsize, s.j[0], s.j[1], s.j[2], yd1);
        tsc_axis(z[p], m.zmin, m.cellsize, s.k[0], s.k[1], s.k[2], zd1);
        if (!in_mesh(s, m)) {
            atomicOr(err, GF_ERRBIT_RANGE);
            densph[p] = 0.f;
            continue;
        }
        // tsc_omp2.c:75-83
        s.wx[0] = (float)(0.75 - (double)(xd1 * xd1));
        s.wy[0] = (float)(0.75 - (double)(yd1 * yd1));
        s.wz[0] = (float)(0.75 - (double)(zd1 * zd1));
        s.wx[2] = (float)(0.5 * (0.25 + (double)xd1 * ((double)xd1 - 1.)));
        s.wx[1] = s.wx[2] + xd1;
        s.wy[2] = (float)(0.5 * (0.25 + (double)yd1 * ((double)yd1 - 1.)));
        s.wy[1] = s.wy[2] + yd1;
        s.wz[2] = (float)(0.5 * (0.25 + (double)zd1 * ((double)zd1 - 1.)));
        s.wz[1] = s.wz[2] + zd1;
        const int64_t mx = 2 * (m.nx / 2 + 1);
        const float *mesh_h = den + m.off;
        // tsc_omp2.c:96-124: for each z plane, y rows in order 1,2,3, x in
        // order 1,2,3; each term is (den * wxwy) * wz.
        float density = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) {
#pragma unroll
            for (int b = 0; b < 3; b++) {
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    float wxy = s.wx[a] * s.wy[b];
                    float v = __ldg(mesh_h + s.i[a] + mx * (s.j[b] + (int64_t)m.ny * s.k[c]));
                    density += (v * wxy) * s.wz[c];
                }
            }
        }
        densph[p] = density;
    }
}

__global__ void scale_kernel(float *__restrict__ den, int64_t n, double factor) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        den[p] = (float)(den[p] * factor);  // tsc_omp2.c:497 (float *= double)
}

inline int grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    const int64_t cap = (int64_t)sm_count() * 16;  // 16 resident blocks per SM at most
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

bool is_pow2_double(double v) {
    int e;
    double f = frexp(v, &e);
    return f == 0.5;
}

}  // namespace

double tsc_volfact() {
    // tsc_omp2.c:188, TSC_CELL_SIZE = 0.004 (params.h:92)
    const double r = 0.001 / 0.004;
    return r * r * r;
}

int launch_tsc_deposit(gf_ctx *ctx, int64_t n, const double *x, const double *y,
                       const double *z, const double *mass, const int32_t *type,
                       const int32_t *hid, const gf_mesh_desc *mesh, float *den,
                       double volfact, const int32_t *order) {
    if (n <= 0) return GF_OK;
    // A power-of-two volfact commutes with every float rounding, so folding
    // it into the weights gives the same bits as the reference's final
    // den *= volfact pass without a second sweep over the mesh.
    float fold = is_pow2_double(volfact) ? (float)volfact : 1.f;
    const int block = 256;
    tsc_deposit_kernel<<<grid_for(n, block), block, 0, ctx->stream>>>(
        n, x, y, z, mass, type, hid, mesh, den, fold, ctx->d_err, order);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

int launch_scale(gf_ctx *ctx, float *den, int64_t ncells, double factor) {
    const int block = 256;
    scale_kernel<<<grid_for(ncells, block), block, 0, ctx->stream>>>(den, ncells, factor);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

int launch_find_den(gf_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                    const int32_t *hid, const gf_mesh_desc *mesh, const float *den,
                    float *densph, const int32_t *order) {
    if (n <= 0) return GF_OK;
    const int block = 256;
    find_den_kernel<<<grid_for(n, block), block, 0, ctx->stream>>>(n, x, y, z, hid, mesh, den,
                                                                   densph, ctx->d_err, order);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

bool volfact_folds(double v) { return is_pow2_double(v); }

}  // namespace gf
