// Centre-of-mass octree shared by the kNN search and the Barnes-Hut potential.
#pragma once

#include "gf_internal.cuh"

namespace gf {

// Node of the kNN walk (preorder).  lo/hi is the exact FP32 bounding box of
// every particle in the subtree; loose particles are those of the node's
// octants that were not divided (fewer than 10 particles).
struct KnnNode {
    float lo[3], hi[3];
    int32_t skip;    // preorder index just past this subtree
    int32_t lstart;  // first loose particle (tree order)
    int32_t lcount;
    int32_t pad;
};

// Node of the potential walk (preorder): monopole + quadrupole about the
// centre of mass, opening radius^2 = dist2/theta2 (ost.c:72-83, 557-582).
struct BhNode {
    double com[3];
    double open_r2;
    float mass, trq;
    float q[6];  // xx, yy, zz, xy, xz, yz second moments about the COM
    int32_t skip, lstart, lcount, pad;
};

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
};

// Builds the octree of every halo of a batch.  pos (batch order, halo h is
// [pstart[h], pstart[h+1])) holds recentred FP32 positions and masses.
// theta2 fills BhNode::open_r2; q5_asbuilt reproduces ost.c:571 (m*y*x in
// place of m*y*z).  Buffers live in ctx->tree[]; the view stays valid until
// the next build on ctx.
int build_tree(gf_ctx *ctx, int32_t nhalo, int64_t n, const int64_t *pstart_dev,
               const float4 *pos, float theta2, int q5_asbuilt, TreeView *out);

// Copies the preorder node arrays and particle order to the host (tests).
int export_tree(gf_ctx *ctx, const TreeView &t, void *knn_host, void *bh_host, float4 *pos_host,
                int32_t *perm_host, int32_t *root_host, int32_t *rend_host);

}  // namespace gf
