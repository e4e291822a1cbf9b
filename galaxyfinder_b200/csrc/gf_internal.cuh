// Internal declarations shared by the libgf CUDA translation units.
#pragma once

#include "gf_tuning.cuh"

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "gf.h"

namespace gf {

// ---------------------------------------------------------------- status
void set_status(int status, const char *fmt, ...);
void clear_status();
int last_status();

// Streaming multiprocessors of the current device (queried once per device);
// grid-stride launches size their grids as a multiple of it.
int sm_count();

// Counts every kernel launch issued through libgf.
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

#define GF_CUDA_TRY(call)                                                                     \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess) {                                                              \
            ::gf::set_status(GF_EDEVICE, "%s:%d %s: %s", __FILE__, __LINE__, #call,          \
                             cudaGetErrorString(_e));                                         \
            return GF_EDEVICE;                                                                \
        }                                                                                     \
    } while (0)

#define GF_LAUNCH_CHECK()                                                                     \
    do {                                                                                      \
        ::gf::count_launch();                                                                 \
        cudaError_t _e = cudaGetLastError();                                                  \
        if (_e != cudaSuccess) {                                                              \
            ::gf::set_status(GF_EDEVICE, "%s:%d launch failed: %s", __FILE__, __LINE__,      \
                             cudaGetErrorString(_e));                                         \
            return GF_EDEVICE;                                                                \
        }                                                                                     \
    } while (0)

#define GF_TRY(expr)                                                                          \
    do {                                                                                      \
        int _s = (expr);                                                                      \
        if (_s != GF_OK) return _s;                                                           \
    } while (0)

// Device error word bits (set by kernels with atomicOr, read back by the host).
enum : int {
    GF_ERRBIT_RANGE = 1,      // a particle's TSC stencil left its mesh
    GF_ERRBIT_TREE = 2,       // tree build ran out of node capacity
    GF_ERRBIT_KNN = 4,        // a kNN query found fewer than k neighbours
    GF_ERRBIT_WALK = 8,       // a tree walk exceeded its step bound
    GF_ERRBIT_INDEX = 16,     // an index argument (query, neighbour) is out of range
    GF_ERRBIT_PLAN = 32,      // the batch no longer fits a captured stage plan
    GF_ERRBIT_WAIT = 64,      // a bounded wait for an asynchronous copy ran out
};

// ---------------------------------------------------------------- workspace
// Grow-only device allocation owned by a context.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    int reserve(size_t need);
    void release();
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

struct HostPinned {
    void *ptr = nullptr;
    size_t bytes = 0;
    int reserve(size_t need);
    void release();
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// ---------------------------------------------------------------- octree
// Node of the kNN walk (preorder).  lo/hi is the exact FP32 bounding box of
// every particle in the subtree; loose particles are those of the node's
// octants that were not divided (fewer than 10 particles).
struct KnnNode {
    float lo[3], hi[3];
    int32_t skip;    // preorder index just past this subtree
    int32_t lstart;  // first loose particle (tree order)
    int32_t lcount;
    int32_t count;   // particles in the subtree: [lstart, lstart + count)
    int32_t parent;  // preorder index of the parent node, -1 for a halo root
    int32_t pad;
};

// Node of the potential walk (preorder): monopole + quadrupole about the
// centre of mass, opening radius^2 = dist2/theta2 (ost.c:72-83, 557-582).
// 80 bytes, 16-byte aligned: the walk reads it as five 16-byte loads.
struct __align__(16) BhNode {
    double com[3];
    double open_r2;
    float mass, trq;
    float q[6];  // xx, yy, zz, xy, xz, yz second moments about the COM
    int32_t skip, lstart, lcount, count;
};
static_assert(sizeof(BhNode) == 80 && alignof(BhNode) == 16, "BhNode is read as five 16-byte words");

struct TreeView {
    int32_t nhalo = 0, nnode = 0;
    int64_t n = 0;
    const float4 *pos = nullptr;   // tree order (x, y, z, mass)
    const int32_t *perm = nullptr; // tree order -> batch index
    const int32_t *root = nullptr; // [nhalo] preorder root of halo h
    const int32_t *rend = nullptr; // [nhalo] preorder end of halo h
    const KnnNode *knn = nullptr;
    const BhNode *bh = nullptr;
    const int32_t *phalo = nullptr; // tree order -> halo
    const int32_t *owner = nullptr; // tree order -> preorder node holding it as loose
};

}  // namespace gf

struct gf_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int *d_err = nullptr;  // device error word
    // scratch buffers, named by use
    gf::DevBuf hid, mesh, mesh_boxes, smooth_tables, particles, tmp[8];
    gf::DevBuf work;  // work counters of the kernels that take their items from a queue
    gf::DevBuf tree[16];
    gf::HostPinned pin[4];
    gf::TreeView last_tree;  // the most recent build_tree() on this context
    std::mutex lock;
};

namespace gf {

// The context used by the drop-in (reference-signature) entry points.
gf_ctx *default_ctx();

// Reads and clears the device error word; maps set bits to a status.
int check_device_errors(gf_ctx *ctx);

// Fill hid[i] = halo index of particle i from pstart (device).
int compute_hid(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart, int32_t *hid);

// Mesh helpers implemented in gf_smooth.cu / gf_tsc.cu.
//
// Occupied boxes: kMeshBoxInts ints per mesh, the cell ranges (x lo, x hi,
// y lo, y hi, z lo, z hi) of every TSC stencil deposited into the mesh, then
// the same ranges over the stencils of every particle of the halo (where
// findDen reads).  An empty range has lo > hi.  launch_tsc_deposit fills them
// when given `boxes`; the smoothing then skips the pencils whose input is
// all zero (exact: a zero pencil filters to zero) and, with `trim_last`, the
// last pass's pencils outside the evaluation box (the smoothed mesh is then
// valid only where findDen reads it).
constexpr int kMeshBoxInts = 12;
int launch_tsc_deposit(gf_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                       const double *mass, const int32_t *type, const int32_t *hid,
                       const gf_mesh_desc *mesh, float *den, double volfact,
                       const int32_t *order = nullptr, int32_t nhalo = 0, int32_t *boxes = nullptr);
// The stage's deposit (gf_tsc.cu): with GF_TSC_TILE > 0 and an octree
// order (order = tree order -> batch index, thalo = tree order -> halo; the
// halos' tree-order ranges are pstart's) through shared-memory tiles, else
// launch_tsc_deposit in batch order.  Fills the occupied boxes when given.
int launch_stage_deposit(gf_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                         const double *mass, const int32_t *type, const int32_t *hid, const int64_t *pstart,
                         const int32_t *order, const int32_t *thalo, int32_t nhalo, const gf_mesh_desc *mesh,
                         float *den, double volfact, int32_t *boxes);
int launch_find_den(gf_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                    const int32_t *hid, const gf_mesh_desc *mesh, const float *den, float *densph,
                    const int32_t *order = nullptr);
int launch_scale(gf_ctx *ctx, float *den, int64_t ncells, double factor);
// Halos whose whole mesh stage (TSC deposit, smoothing, findDen) runs on
// chip: meshes of kOnChipMesh^3 cells held in the distributed shared memory
// of one thread-block cluster, never written to device memory.  Their mesh
// descriptors carry ptype == kMeshOnChip, which the device-memory kernels skip.
constexpr int kOnChipMesh = 64;
constexpr int32_t kMeshOnChip = -1;
struct OnChipMeshes {
    int32_t nmesh = 0;
    const int32_t *halos_host = nullptr;  // [nmesh] halo ids (host; uploaded with the tables)
    int32_t ptype = GF_TYPE_ALL;          // particles deposited
    const int64_t *pstart = nullptr;      // device, batch halo starts
    const double *x = nullptr, *y = nullptr, *z = nullptr, *mass = nullptr;  // device, batch order
    const int32_t *type = nullptr;
    float volfold = 1.f;                  // 1 or the exact power-of-two volfact
    float *densph = nullptr;              // device, mesh density at every particle of these halos
};
struct MeshBoxes {
    const int32_t *dev = nullptr;  // kMeshBoxInts per mesh, from launch_tsc_deposit
    bool trim_last = false;        // last pass only over the evaluation box
};
int smooth_meshes(gf_ctx *ctx, int32_t nhalo, const gf_mesh_desc *mesh_host,
                  const gf_mesh_desc *mesh_dev, float *den, const OnChipMeshes *onchip = nullptr,
                  const MeshBoxes *boxes = nullptr);
// smooth_meshes in two steps: the host plan (axis tables, per-(axis, length)
// tile groups) in one blob, and the launches once the blob is in device
// memory at dbuf (a CUDA graph uploads it once and captures the launches).
struct SmoothGroup {
    int axis, n, pmax;
    size_t off_halos, off_starts;  // blob offsets: halo list, tile prefix
    int32_t ngroup;
    int64_t ntiles;
};
struct SmoothPlan {
    // [axes | tables | on-chip halos | per group: halos, starts | zeroed-plane prefix]
    std::vector<char> blob;
    size_t off_tab = 0, off_chip = 0, off_zero = 0;
    int32_t nchip = 0, nhalo = 0;
    bool box_ok = false;  // every group an FFT axis: the box-restricted passes apply
    std::vector<SmoothGroup> groups;
};
int smooth_plan(int32_t nhalo, const gf_mesh_desc *mesh_host, const OnChipMeshes *onchip, SmoothPlan *plan);
int smooth_launch(gf_ctx *ctx, const SmoothPlan &plan, const char *dbuf, const gf_mesh_desc *mesh_dev,
                  float *den, const OnChipMeshes *onchip = nullptr, const MeshBoxes *boxes = nullptr);
// Copies the plan's blob into ctx->smooth_tables (through pinned staging);
// *dbuf receives its device address.
int smooth_upload(gf_ctx *ctx, const SmoothPlan &plan, char **dbuf);
// The box-restricted mesh stage, for meshes that only findDen reads (the
// stage): launch_mesh_boxes fills the occupied boxes from the particles
// before any deposit; smooth_box_prepare counts the passes' tiles from the
// boxes (into the uploaded blob at dbuf) and zeroes only each mesh's deposit
// box (its evaluation box when nothing is deposited) — the rest of den is
// never read; after the deposit, smooth_box_launch runs the three passes over
// the boxes.  Needs plan.box_ok.
int launch_mesh_boxes(gf_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                      const int32_t *type, const int32_t *hid, int32_t nhalo, const gf_mesh_desc *mesh,
                      int32_t *boxes);
int smooth_box_prepare(gf_ctx *ctx, const SmoothPlan &plan, char *dbuf, const gf_mesh_desc *mesh_dev,
                       float *den, const int32_t *boxes);
int smooth_box_launch(gf_ctx *ctx, const SmoothPlan &plan, const char *dbuf, const gf_mesh_desc *mesh_dev,
                      float *den, const int32_t *boxes, const OnChipMeshes *onchip = nullptr);

// Single-mesh smoothing plan in one contiguous byte blob (see gf_smooth.cu):
// [mesh desc | 3 axis tables | per axis: halo list, tile prefix | tables].
constexpr int kNoAllocMaxAxis = 1024;
struct SingleMeshPlan {
    size_t bytes;
    size_t off_mesh, off_axes, off_tables;
    size_t off_halos[3], off_starts[3];
    int64_t ntiles[3];
    int n[3], pmax[3];
};
int smooth_single_build(const gf_mesh_desc &m, unsigned char *blob, size_t cap, SingleMeshPlan *plan);
int smooth_single_launch(gf_ctx *ctx, float *den, const unsigned char *dev_blob,
                         const SingleMeshPlan &plan);

inline int64_t mesh_cells(const gf_mesh_desc &m) {
    return (int64_t)(2 * (m.nx / 2 + 1)) * m.ny * m.nz;
}

// Halo frames (per axis: min and periodic-shift flag) and recentred extents.
int halo_frames(gf_ctx *ctx, const gf_batch *b, const int32_t *hid, double box,
                std::vector<double> &frame_host, std::vector<double> &extent_host);
// FP64 recentring (Dump2BP) -> double SoA + float4 (x, y, z, mass).
int recentre(gf_ctx *ctx, const gf_batch *b, const int32_t *hid, const double *frame_dev,
             double box, double *xr, double *yr, double *zr, float4 *pos);
__host__ __device__ gf_mesh_desc plan_one_mesh(const double ext[3], const gf_mesh_rule &r);
// Graph mode: frames and meshes computed on the device from the extents that
// the same pass found (ext: the extent kernel's keys, as halo_frames reads
// them).  Each mesh must keep the shape of `planned` (nx, ny, nz, the float
// rg/cellsize its smoothing tables were built for); otherwise the kernel sets
// GF_ERRBIT_PLAN.  Offsets and ptype come from `planned`.
int launch_frames_plan(gf_ctx *ctx, int32_t nhalo, double box, const gf_mesh_rule &rule, int do_mesh,
                       const gf_mesh_desc *planned, double *frame_dev, gf_mesh_desc *mesh_dev);
// The extent kernels alone (keys into ctx->tmp[6]), for graph mode.
int launch_extents(gf_ctx *ctx, const gf_batch *b, const int32_t *hid, double box);

// volfact of tsc_omp2.c:188 for the reference cell size 0.004 cMpc/h.
double tsc_volfact();

// FP64 TSC weights and their derivatives along one axis (adjoints, centre
// refinement): cells i0, i0+1, i0+2 with i0 = nearest - 1 and
// r = xp - nearest in [-1/2, 1/2]:
//   W = (1/2 - r)^2 / 2,  3/4 - r^2,  (1/2 + r)^2 / 2   (tsc_omp2.c:335-343)
struct Axis64 {
    int64_t i0;
    double w[3], dw[3];
};

__device__ __forceinline__ Axis64 tsc_axis64(double pos, double origin, double cell) {
    Axis64 a;
    const double xp = (pos - origin) / cell;
    const double nr = rint(xp);
    const double r = xp - nr;
    a.i0 = (int64_t)nr - 1;
    a.w[0] = 0.5 * (0.5 - r) * (0.5 - r);
    a.w[1] = 0.75 - r * r;
    a.w[2] = 0.5 * (0.5 + r) * (0.5 + r);
    a.dw[0] = (r - 0.5) / cell;
    a.dw[1] = -2.0 * r / cell;
    a.dw[2] = (0.5 + r) / cell;
    return a;
}

__device__ __forceinline__ bool stencil_in(const Axis64 &ax, const Axis64 &ay, const Axis64 &az,
                                           const gf_mesh_desc &m) {
    return ax.i0 >= 0 && ax.i0 + 2 < m.nx && ay.i0 >= 0 && ay.i0 + 2 < m.ny && az.i0 >= 0 &&
           az.i0 + 2 < m.nz;
}
// End of a void drop-in entry point: where the reference would print and
// exit(99), print the status message and exit unless GF_NOEXIT is set in the
// environment (the Python package sets it and raises instead).
void dropin_exit_on_error(int status, const char *who);
// True when volfact is folded into the deposit weights (exact power of two).
bool volfact_folds(double v);

}  // namespace gf
