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
#ifndef GF_BH_BLOCK    // threads per block of bh_kernel
#define GF_BH_BLOCK 128
#endif
#ifndef GF_BH_MINB
#define GF_BH_MINB 1
#endif
#ifndef GF_FFT_PENCILS // real pencils per shared-memory FFT tile (2 per complex pencil)
#define GF_FFT_PENCILS 32
#endif
#ifndef GF_TREE_BLOCK  // threads per block of the per-particle tree-build kernels
#define GF_TREE_BLOCK 256
#endif

static_assert(GF_KNN_BLOCK % 32 == 0 && GF_KNN_BLOCK <= 1024, "GF_KNN_BLOCK");
static_assert(GF_KNN_CHUNK >= 1, "GF_KNN_CHUNK");
static_assert(GF_BH_BLOCK % 32 == 0 && GF_BH_BLOCK <= 1024, "GF_BH_BLOCK");
static_assert(GF_FFT_PENCILS % 2 == 0 && (GF_FFT_PENCILS / 2) * 512 / 8 <= 1024, "GF_FFT_PENCILS");
static_assert(GF_TREE_BLOCK % 32 == 0 && GF_TREE_BLOCK >= 128 && GF_TREE_BLOCK <= 1024, "GF_TREE_BLOCK");
