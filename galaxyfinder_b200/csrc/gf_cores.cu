// lagFindStellarCore (NewGalFinder/nnost.c:991-1548) as a drop-in: the mesh
// density, the mesh peak scan with its core particles and the all-particle
// kNN run on the GPU; the merging of nearby peaks stays the reference's own
// host C (MergingPeak, subhaloden.mod6.c:341) and the core array is resized
// with the reference's arena (Realloc, Memory2.c:217).
//
// Steps, in the reference's order:
//   1. mesh over the particles' FP64 bounding box (nnost.c:1036-1057):
//      xmax += (xmax - xmin) 1e-4, n = (xmax - xmin)/cell + NCELLBUFF,
//      origin = xmin - cell NCELLBUFF/2, cell = TSC_CELL_SIZE;
//   2. TSC deposit of the ptype particles, Gaussian smoothing with
//      Gaussian_Smoothing_Length, findDen at every particle (:1058-1096);
//   3. peaks: cells of the interior [NCELLBUFF/2, n - NCELLBUFF/2) above
//      PEAKTHRESHOLD that exceed all 26 neighbours and hold a ptype particle
//      (cell = rint((x - origin)/cell) per axis, :1120-1150); the core is the
//      particle of the cell with the largest findDen density, the highest
//      index among equal ones (the cell lists are built by prepending, and
//      the scan keeps the first strict maximum); a cell whose lowest particle
//      index is 0 yields no core (the scan tests the last particle it
//      visited, :1197, :1248); cores in scan order (k, j, i) (:1176-1268);
//   4. MergingPeak when there are more than 10 cores (:1288-1289), then
//      Realloc of the core array to the final count (:1290);
//   5. kNN (self included) of every particle on a unit-mass octree
//      (:1298-1535).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gf_tree.cuh"

extern "C" {
// Resolved when libgf is linked into the reference program; absent (NULL)
// when libgf is loaded on its own.
void *Realloc(void *a, long long size, void **src) __attribute__((weak));
int MergingPeak(SimpleBasicParticleType *bp, int np, Coretype *core, int numcore, int iflag)
    __attribute__((weak));
}

namespace gf {

namespace {

constexpr double kCell = 0.004;          // TSC_CELL_SIZE, params.h:92
constexpr float kRG = 0.008f;            // Gaussian_Smoothing_Length, params.h:104 (a float RG)
constexpr int kNbuff = 10;               // NCELLBUFF, params.h:115
constexpr float kPeakThreshold = 2000.f; // PEAKTHRESHOLD 2000.L, params.h:19 (exact in float)
constexpr int kMergeAbove = 10;          // nnost.c:1289

int grid_for(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sm_count() * 16));
}

__global__ void unit_pos_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                                const double *__restrict__ z, float4 *__restrict__ pos) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        pos[i] = make_float4((float)x[i], (float)y[i], (float)z[i], 1.f);
}

__device__ __forceinline__ unsigned int ordered_bits(float v) {
    const unsigned int b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Each ptype particle whose rint cell is a peak (peaks sorted by cell offset)
// offers (density, index) to that peak's maximum and its index to the peak's
// minimum (nnost.c:1120-1150, 1185-1200).
__global__ void core_assoc_kernel(int64_t n, const double *__restrict__ x,
                                  const double *__restrict__ y, const double *__restrict__ z,
                                  const int32_t *__restrict__ type, int ptype, gf_mesh_desc m,
                                  const int64_t *__restrict__ peak_cell, int64_t npeak,
                                  const float *__restrict__ densph,
                                  unsigned long long *__restrict__ best,
                                  unsigned int *__restrict__ lowest) {
    const int64_t mx = 2 * (m.nx / 2 + 1);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (ptype == GF_TYPE_STAR && type[i] != GF_TYPE_STAR) continue;
        const long long ir = (long long)rint((x[i] - m.xmin) / m.cellsize);
        const long long jr = (long long)rint((y[i] - m.ymin) / m.cellsize);
        const long long kr = (long long)rint((z[i] - m.zmin) / m.cellsize);
        const long long ioff = ir + mx * (jr + (long long)m.ny * kr);
        int64_t lo = 0, hi = npeak;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (peak_cell[mid] < ioff) lo = mid + 1; else hi = mid;
        }
        if (lo == npeak || peak_cell[lo] != ioff) continue;
        const unsigned long long key = ((unsigned long long)ordered_bits(densph[i]) << 32) |
                                       (unsigned long long)(unsigned int)i;
        atomicMax(best + lo, key);
        atomicMin(lowest + lo, (unsigned int)i);
    }
}

// Smoothed density at (x, y, z) and its gradient: the TSC-weighted 27-cell
// gather of findDen (tsc_omp2.c:40-163) with FP64 weights, accumulated in
// FP64 in the order c (z), b (y), a (x).
struct DenGrad {
    double rho, gx, gy, gz;
    bool ok;
};

__device__ DenGrad density_and_gradient(const gf_mesh_desc &m, const float *__restrict__ den, double x,
                                        double y, double z) {
    DenGrad o{0, 0, 0, 0, false};
    const Axis64 ax = tsc_axis64(x, m.xmin, m.cellsize);
    const Axis64 ay = tsc_axis64(y, m.ymin, m.cellsize);
    const Axis64 az = tsc_axis64(z, m.zmin, m.cellsize);
    if (!stencil_in(ax, ay, az, m)) return o;
    const int64_t mx = 2 * (m.nx / 2 + 1);
    const float *d = den + m.off;
    for (int c = 0; c < 3; c++) {
        for (int b = 0; b < 3; b++) {
            const float *row = d + ax.i0 + mx * ((ay.i0 + b) + (int64_t)m.ny * (az.i0 + c));
            const double wyz = ay.w[b] * az.w[c];
            const double dyz = ay.dw[b] * az.w[c];
            const double ydz = ay.w[b] * az.dw[c];
            for (int a = 0; a < 3; a++) {
                const double v = row[a];
                o.rho += v * ax.w[a] * wyz;
                o.gx += v * ax.dw[a] * wyz;
                o.gy += v * ax.w[a] * dyz;
                o.gz += v * ax.w[a] * ydz;
            }
        }
    }
    o.ok = true;
    return o;
}

// Gradient ascent of each centre on its halo's smoothed density: up to
// max_steps moves of length step (step_frac * the mesh's smoothing length)
// along the gradient; a move that does not raise the density is not taken
// and halves the step.  One thread per centre.
__global__ void centre_ascent_kernel(int ncentre, const int32_t *__restrict__ halo,
                                     const gf_mesh_desc *__restrict__ mesh,
                                     const float *__restrict__ den, double *__restrict__ cx,
                                     double *__restrict__ cy, double *__restrict__ cz, int max_steps,
                                     double step_frac, double *__restrict__ rho_out,
                                     int *__restrict__ moves_out, int *err) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncentre) return;
    const gf_mesh_desc m = mesh[halo ? halo[c] : 0];
    double x = cx[c], y = cy[c], z = cz[c];
    DenGrad e = density_and_gradient(m, den, x, y, z);
    if (!e.ok) {
        atomicOr(err, GF_ERRBIT_RANGE);
        rho_out[c] = 0.0;
        moves_out[c] = 0;
        return;
    }
    double step = step_frac * m.rg;
    int moves = 0;
    for (int it = 0; it < max_steps; it++) {
        const double gn = sqrt(e.gx * e.gx + e.gy * e.gy + e.gz * e.gz);
        if (!(gn > 0.0)) break;
        const double nx = x + step * (e.gx / gn);
        const double ny = y + step * (e.gy / gn);
        const double nz = z + step * (e.gz / gn);
        const DenGrad f = density_and_gradient(m, den, nx, ny, nz);
        if (f.ok && f.rho > e.rho) {
            x = nx;
            y = ny;
            z = nz;
            e = f;
            moves++;
        } else {
            step *= 0.5;
        }
    }
    cx[c] = x;
    cy[c] = y;
    cz[c] = z;
    rho_out[c] = e.rho;
    moves_out[c] = moves;
}

int do_lag_find_stellar_core(SimpleBasicParticleType *bp, int np, int numnear, float *densph,
                             Coretype **Core, int *NumCore, int maxnumcore, long long *nearindex,
                             int ptype) {
    if (np <= 0 || !bp || !densph || !Core || !*Core || !NumCore || !nearindex || numnear < 1 ||
        numnear > 32 || numnear > np || maxnumcore < 0 ||
        (ptype != GF_TYPE_STAR && ptype != GF_TYPE_ALL)) {
        set_status(GF_EINVAL, "lagFindStellarCore: invalid arguments (1 <= Numnear <= min(32, np))");
        return GF_EINVAL;
    }
    // 1. mesh (host FP64, the reference's formulas)
    double xmin = 1e20, ymin = 1e20, zmin = 1e20, xmax = -1e20, ymax = -1e20, zmax = -1e20;
    for (int i = 0; i < np; i++) {
        xmin = std::min(xmin, bp[i].x);
        ymin = std::min(ymin, bp[i].y);
        zmin = std::min(zmin, bp[i].z);
        xmax = std::max(xmax, bp[i].x);
        ymax = std::max(ymax, bp[i].y);
        zmax = std::max(zmax, bp[i].z);
    }
    xmax = xmax + (xmax - xmin) * 0.0001;
    ymax = ymax + (ymax - ymin) * 0.0001;
    zmax = zmax + (zmax - zmin) * 0.0001;
    gf_mesh_desc m{};
    m.nx = (int)((xmax - xmin) / kCell + kNbuff);
    m.ny = (int)((ymax - ymin) / kCell + kNbuff);
    m.nz = (int)((zmax - zmin) / kCell + kNbuff);
    m.xmin = xmin - kCell * kNbuff / 2.;
    m.ymin = ymin - kCell * kNbuff / 2.;
    m.zmin = zmin - kCell * kNbuff / 2.;
    m.cellsize = kCell;
    m.rg = kRG;
    m.ptype = ptype;
    m.off = 0;
    const int64_t cells = mesh_cells(m);

    gf_ctx *ctx = default_ctx();
    if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
    std::lock_guard<std::mutex> g(ctx->lock);
    const size_t n = (size_t)np;
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    // pinned staging: x, y, z, mass (FP64), type, pstart
    const size_t hbytes = al(4 * n * sizeof(double)) + al(n * sizeof(int32_t)) + 2 * sizeof(int64_t);
    GF_TRY(ctx->pin[0].reserve(hbytes));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    char *h = ctx->pin[0].as<char>();
    double *hx = reinterpret_cast<double *>(h);
    int32_t *ht = reinterpret_cast<int32_t *>(h + al(4 * n * sizeof(double)));
    int64_t *hp = reinterpret_cast<int64_t *>(h + al(4 * n * sizeof(double)) + al(n * sizeof(int32_t)));
    for (size_t i = 0; i < n; i++) {
        hx[i] = bp[i].x;
        hx[n + i] = bp[i].y;
        hx[2 * n + i] = bp[i].z;
        hx[3 * n + i] = bp[i].mass;
        ht[i] = (int32_t)bp[i].type;
    }
    hp[0] = 0;
    hp[1] = np;
    // device: staged inputs | float4 positions | densph | mesh desc
    size_t off = 0;
    const size_t o_in = off; off += al(hbytes);
    const size_t o_pos = off; off += al(n * sizeof(float4));
    const size_t o_dens = off; off += al(n * sizeof(float));
    const size_t o_mesh = off; off += al(sizeof(gf_mesh_desc));
    GF_TRY(ctx->particles.reserve(off));
    char *d = ctx->particles.as<char>();
    GF_CUDA_TRY(cudaMemcpyAsync(d + o_in, h, hbytes, cudaMemcpyHostToDevice, ctx->stream));
    GF_CUDA_TRY(cudaMemcpyAsync(d + o_mesh, &m, sizeof(m), cudaMemcpyHostToDevice, ctx->stream));
    const double *dx = reinterpret_cast<const double *>(d + o_in);
    const int32_t *dtype = reinterpret_cast<const int32_t *>(d + o_in + al(4 * n * sizeof(double)));
    const int64_t *dpstart = reinterpret_cast<const int64_t *>(d + o_in + al(4 * n * sizeof(double)) +
                                                               al(n * sizeof(int32_t)));
    float4 *dpos = reinterpret_cast<float4 *>(d + o_pos);
    float *ddens = reinterpret_cast<float *>(d + o_dens);
    const gf_mesh_desc *dmesh = reinterpret_cast<const gf_mesh_desc *>(d + o_mesh);

    // 2. TSC -> smoothing -> findDen
    GF_TRY(ctx->tmp[0].reserve(sizeof(float) * (size_t)cells));
    float *dden = ctx->tmp[0].as<float>();
    GF_CUDA_TRY(cudaMemsetAsync(dden, 0, sizeof(float) * (size_t)cells, ctx->stream));
    const double vf = tsc_volfact();
    // occupied box: the smoothing skips all-zero pencils (the whole mesh is
    // still smoothed: the peak scan reads all of it)
    GF_TRY(ctx->mesh_boxes.reserve(sizeof(int32_t) * kMeshBoxInts));
    int32_t *boxes = ctx->mesh_boxes.as<int32_t>();
    GF_TRY(launch_tsc_deposit(ctx, np, dx, dx + n, dx + 2 * n, dx + 3 * n, dtype, nullptr, dmesh, dden, vf,
                              nullptr, 1, boxes));
    if (!volfact_folds(vf)) GF_TRY(launch_scale(ctx, dden, cells, vf));
    MeshBoxes mb;
    mb.dev = boxes;
    GF_TRY(smooth_meshes(ctx, 1, &m, dmesh, dden, nullptr, &mb));
    GF_TRY(launch_find_den(ctx, np, dx, dx + n, dx + 2 * n, nullptr, dmesh, dden, ddens));

    // 3. peaks and their core particles
    const int64_t maxcell = (int64_t)m.nx * m.ny * m.nz;
    int64_t cap = 1 << 16;
    int64_t npeak = 0;
    for (int pass = 0; pass < 2; pass++) {
        const size_t pbytes = al((size_t)cap * sizeof(int32_t)) + al((size_t)cap * sizeof(int64_t)) +
                              al((size_t)cap * sizeof(float)) + 256;
        GF_TRY(ctx->tmp[3].reserve(pbytes));
        char *pb = ctx->tmp[3].as<char>();
        int32_t *ph = reinterpret_cast<int32_t *>(pb);
        int64_t *pc = reinterpret_cast<int64_t *>(pb + al((size_t)cap * sizeof(int32_t)));
        float *pv = reinterpret_cast<float *>(pb + al((size_t)cap * sizeof(int32_t)) +
                                              al((size_t)cap * sizeof(int64_t)));
        unsigned long long *dcount = reinterpret_cast<unsigned long long *>(pb + pbytes - 256);
        GF_TRY(launch_mesh_peaks(ctx, 1, maxcell, dmesh, dden, kNbuff / 2, kPeakThreshold, cap, ph, pc,
                                 pv, dcount));
        unsigned long long hc = 0;
        GF_CUDA_TRY(cudaMemcpyAsync(&hc, dcount, sizeof(hc), cudaMemcpyDeviceToHost, ctx->stream));
        GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        npeak = (int64_t)hc;
        if (npeak <= cap) break;
        cap = npeak;
    }
    std::vector<int64_t> peak_cell((size_t)npeak);
    std::vector<unsigned long long> best((size_t)npeak, 0ull);
    std::vector<unsigned int> lowest((size_t)npeak, 0xffffffffu);
    if (npeak > 0) {
        const char *pb = ctx->tmp[3].as<char>();
        const int64_t *pc = reinterpret_cast<const int64_t *>(pb + al((size_t)cap * sizeof(int32_t)));
        GF_CUDA_TRY(cudaMemcpyAsync(peak_cell.data(), pc, (size_t)npeak * sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, ctx->stream));
        GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        std::sort(peak_cell.begin(), peak_cell.end());  // scan order (k, j, i)
        const size_t abytes = al((size_t)npeak * sizeof(int64_t)) + al((size_t)npeak * 8) +
                              al((size_t)npeak * 4);
        GF_TRY(ctx->tmp[2].reserve(abytes));
        char *ab = ctx->tmp[2].as<char>();
        int64_t *dcell = reinterpret_cast<int64_t *>(ab);
        unsigned long long *dbest = reinterpret_cast<unsigned long long *>(ab + al((size_t)npeak * sizeof(int64_t)));
        unsigned int *dlow = reinterpret_cast<unsigned int *>(ab + al((size_t)npeak * sizeof(int64_t)) +
                                                              al((size_t)npeak * 8));
        GF_CUDA_TRY(cudaMemcpyAsync(dcell, peak_cell.data(), (size_t)npeak * sizeof(int64_t),
                                    cudaMemcpyHostToDevice, ctx->stream));
        GF_CUDA_TRY(cudaMemcpyAsync(dbest, best.data(), (size_t)npeak * 8, cudaMemcpyHostToDevice, ctx->stream));
        GF_CUDA_TRY(cudaMemcpyAsync(dlow, lowest.data(), (size_t)npeak * 4, cudaMemcpyHostToDevice, ctx->stream));
        core_assoc_kernel<<<grid_for(np), 256, 0, ctx->stream>>>(np, dx, dx + n, dx + 2 * n, dtype, ptype, m,
                                                                 dcell, npeak, ddens, dbest, dlow);
        GF_LAUNCH_CHECK();
        GF_CUDA_TRY(cudaMemcpyAsync(best.data(), dbest, (size_t)npeak * 8, cudaMemcpyDeviceToHost, ctx->stream));
        GF_CUDA_TRY(cudaMemcpyAsync(lowest.data(), dlow, (size_t)npeak * 4, cudaMemcpyDeviceToHost, ctx->stream));
    }
    GF_CUDA_TRY(cudaMemcpyAsync(densph, ddens, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    GF_TRY(check_device_errors(ctx));  // synchronises
    int numcore = 0;
    for (int64_t p = 0; p < npeak; p++)
        if (best[p] != 0ull && lowest[p] != 0u) numcore++;
    if (numcore > maxnumcore) {
        set_status(GF_ERANGE, "lagFindStellarCore: %d cores exceed maxnumcore = %d", numcore, maxnumcore);
        return GF_ERANGE;
    }
    Coretype *core = *Core;
    int c = 0;
    for (int64_t p = 0; p < npeak; p++) {
        if (best[p] == 0ull || lowest[p] == 0u) continue;
        const int jbp = (int)(best[p] & 0xffffffffull);
        core[c].peak = jbp;
        core[c].cx = (float)bp[jbp].x;
        core[c].cy = (float)bp[jbp].y;
        core[c].cz = (float)bp[jbp].z;
        core[c].density = densph[jbp];
        c++;
    }
    // 4. the reference's peak merging and arena resize
    if (numcore > kMergeAbove) {
        if (!MergingPeak) {
            set_status(GF_ENOTIMPL, "lagFindStellarCore: %d cores need the reference's MergingPeak "
                                    "(link libgf into the reference program)", numcore);
            return GF_ENOTIMPL;
        }
        numcore = MergingPeak(bp, np, core, numcore, 0);
    }
    if (Realloc) *Core = (Coretype *)Realloc(*Core, (long long)sizeof(Coretype) * numcore, (void **)Core);

    // 5. kNN of every particle (unit masses)
    unit_pos_kernel<<<grid_for(np), 256, 0, ctx->stream>>>(np, dx, dx + n, dx + 2 * n, dpos);
    GF_LAUNCH_CHECK();
    GF_TRY(build_tree(ctx, 1, np, dpstart, dpos, 0.5f, 0, &ctx->last_tree));
    GF_TRY(ctx->tmp[1].reserve(n * (size_t)numnear * sizeof(int32_t)));
    int32_t *near32 = ctx->tmp[1].as<int32_t>();
    GF_TRY(launch_knn(ctx, ctx->last_tree, dpstart, dpos, numnear, near32, nullptr));
    GF_TRY(ctx->pin[2].reserve(n * (size_t)numnear * sizeof(int32_t)));
    int32_t *hn = ctx->pin[2].as<int32_t>();
    GF_CUDA_TRY(cudaMemcpyAsync(hn, near32, n * (size_t)numnear * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                ctx->stream));
    GF_TRY(check_device_errors(ctx));
    for (size_t i = 0; i < n * (size_t)numnear; i++) nearindex[i] = hn[i];
    *NumCore = numcore;
    return GF_OK;
}

}  // namespace

}  // namespace gf

using namespace gf;

extern "C" {

int gf_refine_centres(gf_ctx *ctx, int32_t nhalo, const gf_mesh_desc *mesh_dev, const float *den,
                      int32_t ncentre, const int32_t *halo_dev, double *cx, double *cy, double *cz,
                      int max_steps, double step_frac, double *rho, int32_t *moves) {
    clear_status();
    if (!ctx || nhalo <= 0 || ncentre < 0 || max_steps < 0 || !(step_frac > 0) ||
        (ncentre > 0 && (!mesh_dev || !den || !cx || !cy || !cz || !rho || !moves ||
                         (nhalo > 1 && !halo_dev)))) {
        set_status(GF_EINVAL, "gf_refine_centres: invalid arguments");
        return GF_EINVAL;
    }
    if (ncentre == 0) return GF_OK;
    std::lock_guard<std::mutex> g(ctx->lock);
    centre_ascent_kernel<<<(ncentre + 127) / 128, 128, 0, ctx->stream>>>(
        ncentre, nhalo > 1 ? halo_dev : nullptr, mesh_dev, den, cx, cy, cz, max_steps, step_frac, rho,
        moves, ctx->d_err);
    GF_LAUNCH_CHECK();
    return check_device_errors(ctx);
}

void lagFindStellarCore(SimpleBasicParticleType *bp, int np, int Numnear, float *densph,
                        Coretype **Core, int *NumCore, int maxnumcore, long long *nearindex,
                        int ptype) {
    clear_status();
    dropin_exit_on_error(do_lag_find_stellar_core(bp, np, Numnear, densph, Core, NumCore, maxnumcore,
                                                  nearindex, ptype), "lagFindStellarCore");
}

}  // extern "C"
