// Gaussian smoothing for callers that cannot allocate device memory.
//
// gf_gaussian_smooth() and the gaussian_Smoothing() drop-in keep their twiddle
// tables, filter factors and tile lists in buffers that a gf_ctx allocates
// (and grows) with cudaMalloc/cudaMallocHost.  Some callers cannot do that:
// code that runs under a fixed device-memory budget handed out by another
// allocator (a framework's caching pool, a reservation that owns the whole
// GPU), code on a latency-critical path where an allocation's implicit device
// synchronisation is not acceptable, and host drivers that must not grow
// device memory behind their own accounting.  For them this entry point runs
// the same kernels on a caller-owned device mesh, with all of its scratch in
// one file-scope device array of fixed size; it calls no cudaMalloc,
// cudaFree, cudaMallocHost or other allocating routine.
#include <string.h>

#include <mutex>

#include "gf_internal.cuh"

namespace {

// Scratch: the single-mesh plan of smooth_single_build (mesh descriptor,
// three axis headers and tile lists, and the FP64-generated twiddle, filter
// or convolution tables of three axes of at most kNoAllocMaxAxis = 1024
// cells, i.e. at most 9 * 1024 floats).  64 KiB holds the largest plan.
constexpr size_t kScratchBytes = 64 * 1024;
static __device__ __align__(256) unsigned char g_smooth_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
// Device address of g_smooth_scratch on each device (host code cannot use the
// symbol itself as a device pointer).
unsigned char *g_scratch_addr[kMaxDevices];
// Host staging for the plan; guarded by g_lock until the copy has consumed it.
unsigned char g_host_blob[kScratchBytes];

}  // namespace

using namespace gf;

extern "C" int gf_gaussian_smooth_noalloc(float *den, int nx, int ny, int nz, double cellsize,
                                          float RG, void *stream) {
    clear_status();
    if (!den || nx < 1 || ny < 1 || nz < 1 || !(cellsize > 0)) {
        set_status(GF_EINVAL, "gf_gaussian_smooth_noalloc: invalid arguments");
        return GF_EINVAL;
    }
    if (nx > kNoAllocMaxAxis || ny > kNoAllocMaxAxis || nz > kNoAllocMaxAxis) {
        set_status(GF_EINVAL,
                   "gf_gaussian_smooth_noalloc: mesh %d x %d x %d exceeds the %d-cell axis limit of "
                   "its fixed scratch; use gf_gaussian_smooth", nx, ny, nz, kNoAllocMaxAxis);
        return GF_EINVAL;
    }
    int dev = 0;
    GF_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_status(GF_EINVAL, "gf_gaussian_smooth_noalloc: device %d out of range", dev);
        return GF_EINVAL;
    }
    std::lock_guard<std::mutex> g(g_lock);
    if (!g_scratch_addr[dev]) {
        // once per device, with that device current: the scratch's device address
        void *p = nullptr;
        GF_CUDA_TRY(cudaGetSymbolAddress(&p, g_smooth_scratch));
        g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    gf_mesh_desc m{};
    m.nx = nx;
    m.ny = ny;
    m.nz = nz;
    m.ptype = GF_TYPE_ALL;
    m.cellsize = cellsize;
    m.rg = RG;
    SingleMeshPlan plan;
    GF_TRY(smooth_single_build(m, g_host_blob, kScratchBytes, &plan));
    cudaStream_t s = (cudaStream_t)stream;
    // pageable source: the call returns once the plan has been staged, so the
    // host blob may be rewritten by the next call
    GF_CUDA_TRY(cudaMemcpyAsync(g_scratch_addr[dev], g_host_blob, plan.bytes,
                                cudaMemcpyHostToDevice, s));
    gf_ctx launch_ctx;  // carries the stream only; owns no memory
    launch_ctx.device = dev;
    launch_ctx.stream = s;
    return smooth_single_launch(&launch_ctx, den, g_scratch_addr[dev], plan);
}
