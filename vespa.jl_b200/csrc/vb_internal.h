// vb_internal.h -- host-side internals shared by the C-ABI implementation
// files (vb_api.cu, vb_batch.cu).  Not part of the public ABI.
#pragma once

#include <string>

#include "../../include/vespa_b200.h"
#include "vb_launch.h"

struct vb_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t launches = 0;
    void *scratch = nullptr;  // vb_hllc_faces staging (device)
    size_t scratch_bytes = 0;
    cudaEvent_t marks[16] = {};
};

namespace vb {
namespace detail {

// record the calling thread's error message and return `code`
int fail(int code, const std::string &msg);
// make ctx's device current
int use(vb_ctx *ctx);
// geometry of a validated descriptor (VB_EINVAL on a bad one)
int make_geom(const vb_problem_desc *d, Geom *g);
// TMA descriptors of a state buffer for the tiled kernels
int encode_maps(TiledMaps *m, const double *base, const Geom &g);
// box-table entry and item count of a tiled grid
BoxDesc make_box(const TiledMaps &mU, const TiledMaps &mU1, const Geom &g, double *U, double *U1,
                 Ctrl *ctrl, int kz, int item0);
int64_t box_items(const Geom &g, int kz);
// default z-chunk of a tiled grid
int default_kz(const Geom &g);

}  // namespace detail
}  // namespace vb

#define VB_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return vb::detail::fail(e_ == cudaErrorMemoryAllocation ? VB_ENOMEM : VB_ECUDA, \
                                    std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

#define VB_CHECK_LAUNCH(ctx, n)                                                            \
    do {                                                                                   \
        int n_ = (n);                                                                      \
        if (n_ < 0) return vb::detail::fail(VB_EINVAL, "invalid launch configuration");   \
        (ctx)->launches += n_;                                                             \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess)                                                             \
            return vb::detail::fail(VB_ECUDA,                                              \
                                    std::string("kernel launch: ") + cudaGetErrorString(e_)); \
    } while (0)
