// Context, status handling and the C-ABI entry points of libgf (gf.h).
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "gf_internal.cuh"

namespace gf {

std::atomic<uint64_t> g_launches{0};

int sm_count() {
    constexpr int kMaxDev = 64;
    static std::atomic<int> cache[kMaxDev];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) dev = -1;
    if (dev >= 0) {
        const int v = cache[dev].load(std::memory_order_relaxed);
        if (v > 0) return v;
    }
    int c = 0;
    if (dev < 0 || cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0)
        return 1;  // no usable device: the launch that follows reports the error
    cache[dev].store(c, std::memory_order_relaxed);
    return c;
}

namespace {
thread_local int t_status = GF_OK;
thread_local char t_msg[512] = "";
int g_device = -1;
std::mutex g_default_lock;
gf_ctx *g_default = nullptr;
gf_physics g_phys;
bool g_phys_ready = false;
}  // namespace

void set_status(int status, const char *fmt, ...) {
    t_status = status;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof(t_msg), fmt, ap);
    va_end(ap);
}

void clear_status() {
    t_status = GF_OK;
    t_msg[0] = 0;
}

int last_status() { return t_status; }

int DevBuf::reserve(size_t need) {
    if (need <= bytes && ptr) return GF_OK;
    release();
    size_t want = std::max<size_t>(need, 256);
    if (cudaMalloc(&ptr, want) != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        bytes = 0;
        set_status(GF_ENOMEM, "cudaMalloc(%zu) failed", want);
        return GF_ENOMEM;
    }
    bytes = want;
    return GF_OK;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

int HostPinned::reserve(size_t need) {
    if (need <= bytes && ptr) return GF_OK;
    release();
    size_t want = std::max<size_t>(need, 256);
    if (cudaMallocHost(&ptr, want) != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        bytes = 0;
        set_status(GF_ENOMEM, "cudaMallocHost(%zu) failed", want);
        return GF_ENOMEM;
    }
    bytes = want;
    return GF_OK;
}

void HostPinned::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

static int ctx_init(gf_ctx *c, int device, void *stream) {
    GF_CUDA_TRY(cudaSetDevice(device));
    c->device = device;
    if (stream) {
        c->stream = (cudaStream_t)stream;
        c->own_stream = false;
    } else {
        GF_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    GF_CUDA_TRY(cudaMalloc(&c->d_err, sizeof(int)));
    GF_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    return GF_OK;
}

gf_ctx *default_ctx() {
    std::lock_guard<std::mutex> g(g_default_lock);
    if (g_default) {
        cudaSetDevice(g_default->device);
        return g_default;
    }
    int dev = g_device;
    if (dev < 0) {
        const char *e = getenv("GF_DEVICE");
        dev = e ? atoi(e) : 0;
    }
    gf_ctx *c = new gf_ctx();
    if (ctx_init(c, dev, nullptr) != GF_OK) {
        delete c;
        return nullptr;
    }
    g_default = c;
    return c;
}

void dropin_exit_on_error(int status, const char *who) {
    if (status == GF_OK || t_status == GF_OK) return;
    const char *e = getenv("GF_NOEXIT");
    if (e && *e && strcmp(e, "0") != 0) return;
    fprintf(stderr, "%s: %s\n", who, t_msg[0] ? t_msg : "libgf error");
    fflush(stderr);
    exit(99);
}

int check_device_errors(gf_ctx *ctx) {
    int h = 0;
    GF_CUDA_TRY(cudaMemcpyAsync(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (h) {
        GF_CUDA_TRY(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
        if (h & GF_ERRBIT_PLAN) {
            set_status(GF_ESTALE, "the batch no longer fits the captured stage plan");
            return GF_ESTALE;
        }
        if (h & GF_ERRBIT_RANGE) {
            set_status(GF_ERANGE, "a particle's TSC stencil falls outside its mesh");
            return GF_ERANGE;
        }
        if (h & GF_ERRBIT_TREE) {
            set_status(GF_ENOMEM, "tree build exceeded its node capacity");
            return GF_ENOMEM;
        }
        if (h & GF_ERRBIT_KNN) {
            set_status(GF_EINVAL, "a kNN query found fewer neighbours than requested");
            return GF_EINVAL;
        }
        if (h & GF_ERRBIT_WAIT) {
            set_status(GF_ETIMEOUT, "an asynchronous copy did not complete within its wait bound");
            return GF_ETIMEOUT;
        }
        if (h & GF_ERRBIT_WALK) {
            set_status(GF_ETIMEOUT, "a tree walk exceeded its step bound");
            return GF_ETIMEOUT;
        }
        if (h & GF_ERRBIT_INDEX) {
            set_status(GF_EINVAL, "an index argument is out of range");
            return GF_EINVAL;
        }
        set_status(GF_EDEVICE, "device error word 0x%x", h);
        return GF_EDEVICE;
    }
    return GF_OK;
}

namespace {

__global__ void hid_kernel(int32_t nhalo, int64_t n, const int64_t *__restrict__ pstart,
                           int32_t *__restrict__ hid) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = nhalo;  // largest h with pstart[h] <= p
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (pstart[mid] <= p) lo = mid; else hi = mid;
        }
        hid[p] = lo;
    }
}

// gfind.c:842-890 (the second, effective block of physical_parameters)
void physics_from_cosmology(gf_physics &ph) {
    const double Mpc = 3.0857E24, Msun = 1.989E33, G = 6.672E-8;  // ramses.h:30-32, header.h:1
    float omepk = 1.f - ph.omep - ph.omeplam;
    float h0 = ph.hubble / 100.f;
    float Hsub = sqrt(ph.omep * pow(ph.amax / ph.a, 3) + ph.omeplam + omepk * pow(ph.amax / ph.a, 2));
    double com2real = 1.0 / h0 * ph.a / ph.amax * Mpc;
    double pntmass = Msun / h0;
    ph.potentfact = G * pntmass / com2real;
    ph.r1kineticfact = 100.E5 * Hsub * ph.a / ph.amax;
    ph.r2kineticfact = 1.E5;
}

void ensure_physics() {
    if (g_phys_ready) return;
    g_phys.amax = 1.f;
    g_phys.a = 1.f;
    g_phys.omep = 0.3f;
    g_phys.omeplam = 0.7f;
    g_phys.hubble = 70.f;
    physics_from_cosmology(g_phys);
    g_phys_ready = true;
}

}  // namespace

int compute_hid(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart, int32_t *hid) {
    if (n <= 0) return GF_OK;
    int64_t g = std::min<int64_t>((n + 255) / 256, sm_count() * 16);
    hid_kernel<<<(int)g, 256, 0, ctx->stream>>>(nhalo, n, pstart, hid);
    GF_LAUNCH_CHECK();
    return GF_OK;
}

const gf_physics &physics() {
    ensure_physics();
    return g_phys;
}

// NFW helpers of subhaloden.mod6.c:1059-1092 with the reference's operand
// types: amax, a and omep are float, the constants with an L suffix (RHOC,
// G, 1.L, ...) make their expressions long double (x87 extended precision on
// x86-64), the C library's double pow/log receive those values rounded to
// double, and every result is stored as double.  The casts below spell out
// exactly those conversions (C++ would otherwise pick the long double
// overloads of pow/log).
namespace {
constexpr long double kRhoc = 2.7755E11L;  // RHOC, subhaloden.mod6.c:1081
constexpr long double kG = 6.672E-8L;      // G, header.h:1

long double nfw_vv() {  // vv, subhaloden.mod6.c:1082
    const long double om1 = (long double)physics().omep - 1.0L;
    return 18.0L * (long double)M_PI * (long double)M_PI + 82.0L * om1 -
           39.0L * (long double)pow((double)om1, 2.0);
}
}  // namespace

double nfw_concentration(double mass) {  // get_concentration, :1059-1066
    const gf_physics &ph = physics();
    const double mstar = (double)1.3E13L;
    const double redshift = (double)((long double)(ph.amax / ph.a) - 1.0L);
    return (double)((long double)(14.5 * pow(mass / mstar, -0.15)) / (1.0L + redshift));
}

double nfw_alpha(double c, double s) {  // get_alpha, :1067-1074
    const double cs = c * s;
    const long double t = cs / (1.0L + cs);
    const double res = (double)(2.0L - t * t);
    return (double)(res / ((long double)log((double)(1.0L + cs)) - cs / (1.0L + cs)));
}

double nfw_gnfw(double c) {  // gnfw, :1083-1087
    return (double)(1. / ((long double)log((double)(1.0L + c)) - c / (1.0L + c)));
}

double nfw_rvir(double mvir) {  // GetRvir, :1088-1092
    return pow((double)(3. * mvir / (4.0L * (long double)M_PI * nfw_vv() * kRhoc)),
               (double)0.3333333333333L);
}

// GetBGpotent, subhaloden.mod6.c:1093-1101.
double bg_potent(double mvir) {
    const double c = nfw_concentration(mvir);
    const double gc = nfw_gnfw(c);
    const double rvir = nfw_rvir(mvir);
    const double vc2 = (double)(kG * mvir / rvir) * physics().potentfact;  // Get_Vc2, :1075-1079
    return vc2 * (1 - gc * log(1 + c));
}

}  // namespace gf

using namespace gf;

// =========================================================================
// generic C entry points
// =========================================================================
extern "C" {

const char *gf_status_string(int status) {
    switch (status) {
        case GF_OK: return "ok";
        case GF_EINVAL: return "invalid argument";
        case GF_ENOMEM: return "out of memory";
        case GF_EDEVICE: return "CUDA device error";
        case GF_ETIMEOUT: return "device wait timed out";
        case GF_ERANGE: return "particle outside mesh";
        case GF_ENOTIMPL: return "not implemented";
        case GF_ESTALE: return "stage graph plan no longer fits the batch";
        default: return "unknown status";
    }
}

int gf_last_status(void) { return t_status; }
const char *gf_last_error(void) { return t_msg; }

int gf_set_device(int device) {
    std::lock_guard<std::mutex> g(g_default_lock);
    if (g_default) {
        set_status(GF_EINVAL, "gf_set_device after the default context was created");
        return GF_EINVAL;
    }
    g_device = device;
    return GF_OK;
}

uint64_t gf_kernel_launch_count(void) { return g_launches.load(); }

int gf_tuning_value(const char *name, int64_t *value) {
    clear_status();
    static const struct {
        const char *name;
        int64_t value;
    } params[] = {{"GF_KNN_ALGO", GF_KNN_ALGO},       {"GF_KNNB_BLOCK", GF_KNNB_BLOCK},
                  {"GF_KNNB_ARITY", GF_KNNB_ARITY},   {"GF_KNNB_SEEDS", GF_KNNB_SEEDS},
                  {"GF_KNN_BLOCK", GF_KNN_BLOCK},
                  {"GF_KNN_MINB", GF_KNN_MINB},       {"GF_KNN_CHUNK", GF_KNN_CHUNK},
                  {"GF_BH_BLOCK", GF_BH_BLOCK},       {"GF_BH_MINB", GF_BH_MINB},
                  {"GF_FFT_PENCILS", GF_FFT_PENCILS}, {"GF_TREE_BLOCK", GF_TREE_BLOCK},
                  {"GF_KNNB_QUEUE", GF_KNNB_QUEUE},   {"GF_KNNB_LANECERT", GF_KNNB_LANECERT},
                  {"GF_BH_DYN", GF_BH_DYN},           {"GF_KNNB_DYN", GF_KNNB_DYN},
                  {"GF_BH_ACC", GF_BH_ACC},           {"GF_KNNB_WIN", GF_KNNB_WIN},
                  {"GF_KNNB_MINB", GF_KNNB_MINB},     {"GF_BH_TMA", GF_BH_TMA},
                  {"GF_KNNB_FILT", GF_KNNB_FILT},     {"GF_KNNB_HEAPF", GF_KNNB_HEAPF},
                  {"GF_BH_LEAF4", GF_BH_LEAF4},
                  {"GF_FFT_PENCILS_64", GF_FFT_PENCILS_64},
                  {"GF_FFT_PENCILS_128", GF_FFT_PENCILS_128}, {"GF_TSC_TILE", GF_TSC_TILE}};
    if (!name || !value) return GF_EINVAL;
    for (const auto &p : params)
        if (strcmp(p.name, name) == 0) {
            *value = p.value;
            return GF_OK;
        }
    set_status(GF_EINVAL, "unknown tuning parameter %s", name);
    return GF_EINVAL;
}

int gf_set_cosmology(float amax, float a, float omep, float omeplam, float hubble) {
    ensure_physics();
    g_phys.amax = amax;
    g_phys.a = a;
    g_phys.omep = omep;
    g_phys.omeplam = omeplam;
    g_phys.hubble = hubble;
    physics_from_cosmology(g_phys);
    return GF_OK;
}

int gf_get_physics(gf_physics *out) {
    if (!out) return GF_EINVAL;
    *out = physics();
    return GF_OK;
}

double gf_bg_potent(double mvir) { return bg_potent(mvir); }

int gf_ctx_create(gf_ctx **out, int device, void *stream) {
    clear_status();
    if (!out) return GF_EINVAL;
    gf_ctx *c = new gf_ctx();
    int s = ctx_init(c, device, stream);
    if (s != GF_OK) {
        delete c;
        return s;
    }
    *out = c;
    return GF_OK;
}

int gf_ctx_destroy(gf_ctx *c) {
    if (!c) return GF_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    c->hid.release();
    c->mesh.release();
    c->mesh_boxes.release();
    c->work.release();
    c->smooth_tables.release();
    c->particles.release();
    for (auto &b : c->tmp) b.release();
    for (auto &b : c->tree) b.release();
    for (auto &b : c->pin) b.release();
    if (c->d_err) cudaFree(c->d_err);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return GF_OK;
}

int gf_ctx_set_stream(gf_ctx *c, void *stream) {
    if (!c) return GF_EINVAL;
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    return GF_OK;
}

// ---------------------------------------------------------------- batched mesh API
int gf_tsc_deposit(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev,
                   const gf_mesh_desc *mesh_host, float *den) {
    clear_status();
    if (!ctx || !b || !mesh_dev || !mesh_host || !den) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    GF_TRY(ctx->hid.reserve(sizeof(int32_t) * std::max<int64_t>(b->nparticle, 1)));
    int32_t *hid = ctx->hid.as<int32_t>();
    GF_TRY(compute_hid(ctx, b->nhalo, b->nparticle, b->pstart, hid));
    int64_t cells = 0;
    for (int h = 0; h < b->nhalo; h++)
        cells = std::max<int64_t>(cells, mesh_host[h].off + mesh_cells(mesh_host[h]));
    GF_CUDA_TRY(cudaMemsetAsync(den, 0, sizeof(float) * cells, ctx->stream));
    const double vf = tsc_volfact();
    GF_TRY(launch_tsc_deposit(ctx, b->nparticle, b->x, b->y, b->z, b->mass, b->type, hid, mesh_dev,
                              den, vf));
    if (!volfact_folds(vf)) GF_TRY(launch_scale(ctx, den, cells, vf));
    return check_device_errors(ctx);
}

int gf_gaussian_smooth(gf_ctx *ctx, int32_t nhalo, const gf_mesh_desc *mesh_host,
                       const gf_mesh_desc *mesh_dev, float *den) {
    clear_status();
    if (!ctx || !mesh_host || !mesh_dev || !den) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    GF_TRY(smooth_meshes(ctx, nhalo, mesh_host, mesh_dev, den));
    return check_device_errors(ctx);
}

int gf_find_den(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev, const float *den,
                float *densph) {
    clear_status();
    if (!ctx || !b || !mesh_dev || !den || !densph) return GF_EINVAL;
    std::lock_guard<std::mutex> g(ctx->lock);
    GF_TRY(ctx->hid.reserve(sizeof(int32_t) * std::max<int64_t>(b->nparticle, 1)));
    int32_t *hid = ctx->hid.as<int32_t>();
    GF_TRY(compute_hid(ctx, b->nhalo, b->nparticle, b->pstart, hid));
    GF_TRY(launch_find_den(ctx, b->nparticle, b->x, b->y, b->z, hid, mesh_dev, den, densph));
    return check_device_errors(ctx);
}

int gf_mesh_stage(gf_ctx *ctx, const gf_batch *b, const gf_mesh_desc *mesh_dev,
                  const gf_mesh_desc *mesh_host, float *den, float *densph, int smooth) {
    int s = gf_tsc_deposit(ctx, b, mesh_dev, mesh_host, den);
    if (s != GF_OK || !smooth) return s;
    GF_TRY(gf_gaussian_smooth(ctx, b->nhalo, mesh_host, mesh_dev, den));
    return gf_find_den(ctx, b, mesh_dev, den, densph);
}

}  // extern "C"

// =========================================================================
// drop-in entry points (reference signatures, host buffers)
// =========================================================================
namespace {

// Copies bp's positions/masses/types into device SoA buffers of ctx.
struct DevParticles {
    double *x, *y, *z, *mass;
    int32_t *type;
};

int upload_bp(gf_ctx *ctx, const SimpleBasicParticleType *bp, int np, DevParticles &d) {
    const size_t n = (size_t)np;
    const size_t bytes = n * (4 * sizeof(double) + sizeof(int32_t));
    GF_TRY(ctx->pin[0].reserve(bytes));
    GF_TRY(ctx->particles.reserve(bytes));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // staging buffer reuse
    char *h = ctx->pin[0].as<char>();
    double *hx = (double *)h, *hy = hx + n, *hz = hy + n, *hm = hz + n;
    int32_t *ht = (int32_t *)(hm + n);
    for (size_t i = 0; i < n; i++) {
        hx[i] = bp[i].x;
        hy[i] = bp[i].y;
        hz[i] = bp[i].z;
        hm[i] = bp[i].mass;
        ht[i] = (int32_t)bp[i].type;
    }
    char *dv = ctx->particles.as<char>();
    GF_CUDA_TRY(cudaMemcpyAsync(dv, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
    d.x = (double *)dv;
    d.y = d.x + n;
    d.z = d.y + n;
    d.mass = d.z + n;
    d.type = (int32_t *)(d.mass + n);
    return GF_OK;
}

int upload_mesh_desc(gf_ctx *ctx, const gf_mesh_desc &m, gf_mesh_desc **dev) {
    GF_TRY(ctx->mesh.reserve(sizeof(gf_mesh_desc)));
    GF_CUDA_TRY(cudaMemcpyAsync(ctx->mesh.ptr, &m, sizeof(m), cudaMemcpyHostToDevice, ctx->stream));
    GF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // &m is a stack object
    *dev = ctx->mesh.as<gf_mesh_desc>();
    return GF_OK;
}

int do_assign_density_TSC(SimpleBasicParticleType *bp, int np, float *den, int nx, int ny, int nz,
                          double Xmin, double Ymin, double Zmin, double cellsize, int ptype) {
    if (np < 0 || !den || nx < 3 || ny < 3 || nz < 3 || !(cellsize > 0) || (np > 0 && !bp)) {
        set_status(GF_EINVAL, "assign_density_TSC: invalid arguments");
        return GF_EINVAL;
    }
    gf_ctx *ctx = default_ctx();
    if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
    std::lock_guard<std::mutex> g(ctx->lock);
    gf_mesh_desc m{};
    m.off = 0;
    m.nx = nx; m.ny = ny; m.nz = nz;
    m.ptype = ptype;
    m.xmin = Xmin; m.ymin = Ymin; m.zmin = Zmin;
    m.cellsize = cellsize;
    const int64_t cells = mesh_cells(m);
    DevParticles d{};
    if (np > 0) GF_TRY(upload_bp(ctx, bp, np, d));
    gf_mesh_desc *dm;
    GF_TRY(upload_mesh_desc(ctx, m, &dm));
    GF_TRY(ctx->tmp[0].reserve(sizeof(float) * cells));
    float *dden = ctx->tmp[0].as<float>();
    GF_CUDA_TRY(cudaMemsetAsync(dden, 0, sizeof(float) * cells, ctx->stream));
    const double vf = tsc_volfact();
    GF_TRY(launch_tsc_deposit(ctx, np, d.x, d.y, d.z, d.mass, d.type, nullptr, dm, dden, vf));
    if (!volfact_folds(vf)) GF_TRY(launch_scale(ctx, dden, cells, vf));
    GF_CUDA_TRY(cudaMemcpyAsync(den, dden, sizeof(float) * cells, cudaMemcpyDeviceToHost, ctx->stream));
    return check_device_errors(ctx);
}

int do_findDen(SimpleBasicParticleType *bp, int np, float *densph, double xmin, double ymin,
               double zmin, double cellsize, float *den, int nx, int ny, int nz) {
    if (np < 0 || !den || nx < 3 || ny < 3 || nz < 3 || !(cellsize > 0) ||
        (np > 0 && (!bp || !densph))) {
        set_status(GF_EINVAL, "findDen: invalid arguments");
        return GF_EINVAL;
    }
    if (np == 0) return GF_OK;
    gf_ctx *ctx = default_ctx();
    if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
    std::lock_guard<std::mutex> g(ctx->lock);
    gf_mesh_desc m{};
    m.nx = nx; m.ny = ny; m.nz = nz;
    m.ptype = GF_TYPE_ALL;
    m.xmin = xmin; m.ymin = ymin; m.zmin = zmin;
    m.cellsize = cellsize;
    const int64_t cells = mesh_cells(m);
    DevParticles d{};
    GF_TRY(upload_bp(ctx, bp, np, d));
    gf_mesh_desc *dm;
    GF_TRY(upload_mesh_desc(ctx, m, &dm));
    GF_TRY(ctx->tmp[0].reserve(sizeof(float) * cells));
    GF_TRY(ctx->tmp[1].reserve(sizeof(float) * (size_t)np));
    float *dden = ctx->tmp[0].as<float>();
    float *dout = ctx->tmp[1].as<float>();
    GF_CUDA_TRY(cudaMemcpyAsync(dden, den, sizeof(float) * cells, cudaMemcpyHostToDevice, ctx->stream));
    GF_TRY(launch_find_den(ctx, np, d.x, d.y, d.z, nullptr, dm, dden, dout));
    GF_CUDA_TRY(cudaMemcpyAsync(densph, dout, sizeof(float) * np, cudaMemcpyDeviceToHost, ctx->stream));
    return check_device_errors(ctx);
}

int do_gaussian_Smoothing(float *denGrid, int nx, int ny, int nz, double cellsize, float RG) {
    if (!denGrid || nx < 1 || ny < 1 || nz < 1 || !(cellsize > 0)) {
        set_status(GF_EINVAL, "gaussian_Smoothing: invalid arguments");
        return GF_EINVAL;
    }
    gf_ctx *ctx = default_ctx();
    if (!ctx) return last_status() ? last_status() : GF_EDEVICE;
    std::lock_guard<std::mutex> g(ctx->lock);
    gf_mesh_desc m{};
    m.nx = nx; m.ny = ny; m.nz = nz;
    m.ptype = GF_TYPE_ALL;
    m.cellsize = cellsize;
    m.rg = RG;  // gsmooth.c:67 divides the float RG by cellsize
    const int64_t cells = mesh_cells(m);
    gf_mesh_desc *dm;
    GF_TRY(upload_mesh_desc(ctx, m, &dm));
    GF_TRY(ctx->tmp[0].reserve(sizeof(float) * cells));
    float *dden = ctx->tmp[0].as<float>();
    GF_CUDA_TRY(cudaMemcpyAsync(dden, denGrid, sizeof(float) * cells, cudaMemcpyHostToDevice, ctx->stream));
    GF_TRY(smooth_meshes(ctx, 1, &m, dm, dden));
    GF_CUDA_TRY(cudaMemcpyAsync(denGrid, dden, sizeof(float) * cells, cudaMemcpyDeviceToHost, ctx->stream));
    return check_device_errors(ctx);
}

}  // namespace

extern "C" {

void assign_density_TSC(SimpleBasicParticleType *bp, int np, float *den, int nx, int ny, int nz,
                        double Xmin, double Ymin, double Zmin, double cellsize, int ptype) {
    clear_status();
    dropin_exit_on_error(do_assign_density_TSC(bp, np, den, nx, ny, nz, Xmin, Ymin, Zmin, cellsize, ptype), "assign_density_TSC");
}

void findDen(SimpleBasicParticleType *bp, int np, float *densph, double xmin, double ymin,
             double zmin, double cellsize, float *den, int nx, int ny, int nz) {
    clear_status();
    dropin_exit_on_error(do_findDen(bp, np, densph, xmin, ymin, zmin, cellsize, den, nx, ny, nz), "findDen");
}

void gaussian_Smoothing(float *denGrid, int nx, int ny, int nz, double cellsize, float RG) {
    clear_status();
    dropin_exit_on_error(do_gaussian_Smoothing(denGrid, nx, ny, nz, cellsize, RG), "gaussian_Smoothing");
}

void i_potent_spline(void) {
    clear_status();
    if (!default_ctx()) return;
}

}  // extern "C"

