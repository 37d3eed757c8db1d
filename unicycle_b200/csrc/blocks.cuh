// Dense blocks of K for the hierarchical approximation (hmatrix.cu): the
// per-source records of one patch family on the device and the block
// assembly entry point (assemble.cu).
#pragma once
#include <vector>
#include "ucg_internal.cuh"
#include "okada92.cuh"
#include "nikkhoo15.cuh"

namespace ucg {

struct BlockSources {
    int family = 0;          // 0 rectangles, 1 triangles
    int okada_mode = UCG_OKADA_FP64;
    double *src = nullptr;   // SoA source records on the device
    int ns = 0;
    OkMed med{};
    NwConst cst{};
};

// records of the context's single patch family and the receiver table (c->rcv);
// UCG_E_UNSUPPORTED for volumes or mixed rectangles and triangles
int block_sources_build(ucg_ctx *c, int okada_mode, BlockSources *bs);
void block_sources_free(BlockSources *bs);
// K rows of receivers ridx[0..nrb) by columns of sources sidx[0..nsb) (device
// element-id arrays) into out, row-major (3 nrb) x (2 nsb); enqueued on c->stream
void assemble_block(ucg_ctx *c, const BlockSources &bs, const int *ridx, int nrb, const int *sidx, int nsb,
                    double *out);
// bounding box (lo, hi) and centre of every patch, in K's element order
void element_boxes(const ucg_ctx *c, std::vector<double> &box, std::vector<double> &ctr);

}  // namespace ucg
