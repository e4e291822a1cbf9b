// Compile-time launch parameters of the hot kernels.  galaxyfinder_b200/tune.py
// measures variants on the GPU and records the fastest in
// galaxyfinder_b200/tuned.json; build.py passes them as -D flags.  The values
// below are the defaults used when no tuned value is given.
#pragma once

#ifndef GF_KNN_BLOCK   // threads per block of knn_kernel
#define GF_KNN_BLOCK 256
#endif
#ifndef GF_KNN_MINB    // min resident blocks per SM (__launch_bounds__); caps registers
#define GF_KNN_MINB 1
#endif
#ifndef GF_KNN_CHUNK   // consecutive tree-order queries per warp task
#define GF_KNN_CHUNK 32
#endif
#ifndef GF_KNN_ALGO    // 1: bucket kNN (a warp walks once for 32 tree-order queries,
#define GF_KNN_ALGO 1  //    lane = query); 2: the same with float heap keys and an
#endif                 //    exact certification; 0: one warp per query
#ifndef GF_KNNB_BLOCK  // threads per block of knn_bucket_kernel (14.5 KB shared memory per warp)
#define GF_KNNB_BLOCK 32
#endif
#ifndef GF_KNNB_MINB
#define GF_KNNB_MINB 1
#endif
#ifndef GF_KNNB_SEEDS  // tree-order neighbours that seed each query's heap (float-key kernel)
#define GF_KNNB_SEEDS 64
#endif
#ifndef GF_KNNB_LANECERT  // float-key kernel: 1 = each lane certifies its own query, 0 = the warp, query by query
#define GF_KNNB_LANECERT 0
#endif
#ifndef GF_KNNB_QUEUE  // float-key kernel: survivors queued per lane (0: inserted at once)
#define GF_KNNB_QUEUE 0
#endif
#ifndef GF_KNNB_ARITY  // children per node of the bucket kernel's per-lane heaps (2 or 4)
#define GF_KNNB_ARITY 2
#endif
#ifndef GF_BH_BLOCK    // threads per block of bh_kernel
#define GF_BH_BLOCK 128
#endif
#ifndef GF_BH_DYN      // Barnes-Hut walk: 1 = warps take targets from a work counter, 0 = grid-stride
#define GF_BH_DYN 0
#endif
#ifndef GF_BH_TMA      // Barnes-Hut walk: 1 = opened leaves staged in shared memory by bulk copies
#define GF_BH_TMA 0
#endif
#ifndef GF_BH_ACC      // Barnes-Hut sums: 0 = FP32 with Kahan compensation, 1 = FP64
#define GF_BH_ACC 0
#endif
#ifndef GF_KNNB_WIN    // float-key kNN: nodes staged per warp in shared memory (0, 8, 16 or 32)
#define GF_KNNB_WIN 32
#endif
#ifndef GF_KNNB_DYN    // float-key kNN: 1 = warps take buckets from a work counter, 0 = grid-stride
#define GF_KNNB_DYN 0
#endif
#ifndef GF_KNNB_FILT   // float-key kNN tile filter: 1 = four independent chains over a sentinel-padded tile
#define GF_KNNB_FILT 0
#endif
#ifndef GF_KNNB_HEAPF  // float-key kNN heaps: 1 = ordered by the float part of the key only, 2 = also hole-first sift-down, 3 = also float admission test
#define GF_KNNB_HEAPF 0
#endif
#ifndef GF_BH_LEAF4    // Barnes-Hut walk: 1 = opened leaves loaded four particles at a time
#define GF_BH_LEAF4 0
#endif
#ifndef GF_BH_MINB
#define GF_BH_MINB 1
#endif
#ifndef GF_FFT_PENCILS // real pencils per shared-memory FFT tile (2 per complex pencil)
#define GF_FFT_PENCILS 32
#endif
#ifndef GF_FFT_PENCILS_64  // real pencils per tile of the 64-cell FFT axes
#define GF_FFT_PENCILS_64 32
#endif
#ifndef GF_FFT_PENCILS_128 // real pencils per tile of the 128-cell FFT axes
#define GF_FFT_PENCILS_128 32
#endif
#ifndef GF_TSC_TILE  // cells of the stage deposit's shared-memory tile (0: direct global atomics)
#define GF_TSC_TILE 0
#endif
#ifndef GF_TREE_BLOCK  // threads per block of the per-particle tree-build kernels
#define GF_TREE_BLOCK 256
#endif

static_assert(GF_KNN_BLOCK % 32 == 0 && GF_KNN_BLOCK <= 1024, "GF_KNN_BLOCK");
static_assert(GF_KNN_CHUNK >= 1, "GF_KNN_CHUNK");
static_assert(GF_KNNB_BLOCK % 32 == 0 && GF_KNNB_BLOCK <= 512, "GF_KNNB_BLOCK");
static_assert(GF_KNN_ALGO >= 0 && GF_KNN_ALGO <= 2, "GF_KNN_ALGO");
static_assert(GF_KNNB_ARITY == 2 || GF_KNNB_ARITY == 4, "GF_KNNB_ARITY");
static_assert(GF_KNNB_LANECERT == 0 || GF_KNNB_LANECERT == 1, "GF_KNNB_LANECERT");
static_assert(GF_KNNB_QUEUE >= 0 && GF_KNNB_QUEUE <= 16, "GF_KNNB_QUEUE");
static_assert(GF_KNNB_SEEDS >= 32 && GF_KNNB_SEEDS % 2 == 0, "GF_KNNB_SEEDS");
static_assert(GF_BH_BLOCK % 32 == 0 && GF_BH_BLOCK <= 1024, "GF_BH_BLOCK");
static_assert(GF_BH_DYN == 0 || GF_BH_DYN == 1, "GF_BH_DYN");
static_assert(GF_KNNB_DYN == 0 || GF_KNNB_DYN == 1, "GF_KNNB_DYN");
static_assert(GF_KNNB_WIN == 0 || GF_KNNB_WIN == 8 || GF_KNNB_WIN == 16 || GF_KNNB_WIN == 32, "GF_KNNB_WIN");
static_assert(GF_BH_ACC == 0 || GF_BH_ACC == 1, "GF_BH_ACC");
static_assert(GF_BH_TMA == 0 || GF_BH_TMA == 1, "GF_BH_TMA");
static_assert(GF_KNNB_FILT == 0 || GF_KNNB_FILT == 1, "GF_KNNB_FILT");
static_assert(GF_KNNB_HEAPF >= 0 && GF_KNNB_HEAPF <= 3, "GF_KNNB_HEAPF");
static_assert(GF_BH_LEAF4 == 0 || GF_BH_LEAF4 == 1, "GF_BH_LEAF4");
static_assert(GF_FFT_PENCILS % 2 == 0 && (GF_FFT_PENCILS / 2) * 512 / 8 <= 1024, "GF_FFT_PENCILS");
static_assert(GF_FFT_PENCILS_64 >= 32 && GF_FFT_PENCILS_64 <= 128 &&
                  (GF_FFT_PENCILS_64 & (GF_FFT_PENCILS_64 - 1)) == 0, "GF_FFT_PENCILS_64");
static_assert(GF_FFT_PENCILS_128 >= 32 && GF_FFT_PENCILS_128 <= 64 &&
                  (GF_FFT_PENCILS_128 & (GF_FFT_PENCILS_128 - 1)) == 0, "GF_FFT_PENCILS_128");
static_assert(GF_TSC_TILE == 0 || (GF_TSC_TILE >= 1024 && GF_TSC_TILE <= 12288), "GF_TSC_TILE");
static_assert(GF_TREE_BLOCK % 32 == 0 && GF_TREE_BLOCK >= 128 && GF_TREE_BLOCK <= 1024, "GF_TREE_BLOCK");
