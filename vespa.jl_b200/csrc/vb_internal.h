// vb_internal.h -- host-side internals shared by the C-ABI implementation
// files (vb_api.cu, vb_batch.cu).  Not part of the public ABI.
#pragma once

#include <string>

#include <nvtx3/nvToolsExt.h>

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

struct vb_gravity;  // self-gravity state of a grid (vb_gravity.cu)

struct vb_grid {
    vb_ctx *ctx = nullptr;
    vb::Geom g{};
    int precision = VB_FP64;
    double *U = nullptr;   // state (and u0: the stage-2 update runs in place)
    double *U1 = nullptr;  // stage-1 state
    vb::Ctrl *ctrl = nullptr;   // device control block
    vb::Ctrl *hctrl = nullptr;  // pinned host mirror
    double *partials = nullptr;
    double *totals = nullptr;
    double *htot = nullptr;     // pinned
    double *bflux = nullptr;            // outer planes, then (interior) the [axis][5][ncell] block
    int64_t bflux_n = 0;                // doubles allocated
    int64_t bflux_outer_n = 0;          // doubles of the outer planes
    bool bflux_on = false;
    bool bflux_interior = false;        // the register also records interior faces
    bool invdt_valid = false;   // ctrl->invdt_bits holds the CFL max of the current state
    bool tiled = false;         // the tiled 3D kernels apply to this grid
    int kz = 64;                // z planes per tiled work item
    vb::TiledMaps maps_U{}, maps_U1{};  // TMA descriptors of the two stage inputs
    vb::BoxDesc box{};                  // the tiled kernels' box descriptor (passed by value)
    int box_kz = 0;                     // kz the descriptor was written with
    int taper = -1;                     // tapered z chunks: -1 auto, 0 off, 1 on
    int taper_tuned = -1;               // auto: the autotuner's choice (-1: none, VB_MIXED tapers)
    int box_taper = -1;                 // taper the descriptor was written with
    // CUDA graph of GRAPH_STEPS steps (finalize + RK2), replayed by the step loop
    cudaGraphExec_t gexec = nullptr;
    uint64_t gkey = 0;                  // kernel configuration it was captured for
    int64_t glaunches = 0;              // kernels per replay
    bool warmed = false;                // one direct step ran (launch setup done)
    vb_gravity *grav = nullptr;         // self-gravity (a solve per step; source in the stages)
    bool slab = false;                  // a z window is set (vb_grid_set_zwindow): tiled kernels only
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
                 Ctrl *ctrl, int kz, int item0, bool taper = false);
int64_t box_items(const Geom &g, int kz, bool taper = false);
// default z-chunk of a tiled box (batches)
int default_kz(const Geom &g);
// automatic kernel choice and default chunk of a single grid
bool tiled_auto(const Geom &g);
int grid_default_kz(const Geom &g);

// Context-owned device staging buffer of at least `bytes` (grown with
// cudaMalloc; reused across calls on the context's stream).
int ctx_scratch(vb_ctx *ctx, size_t bytes, void **out);

// Grid stepping helpers shared with the adjoint (vb_api.cu).
int grid_ensure_cfl(vb_grid *gr);   // CFL max of the current state, if stale
int grid_rk2(vb_grid *gr);          // one RK2 step with dt already in the control block
int grid_pull_ctrl(vb_grid *gr);    // device control block -> gr->hctrl (synchronous)
int grid_push_ctrl(vb_grid *gr);    // gr->hctrl -> device control block (synchronous)

// Self-gravity (vb_gravity.cu): solve_poisson! for the current density and
// refresh the field g the stages add; free a grid's gravity state.
int gravity_solve(vb_grid *gr, int64_t *iters, double *relres);
void gravity_free(vb_gravity *gv);

// NVTX range over a host API call, named after it: Nsight Systems shows the
// calls (and the launches they enqueue) on the host timeline; without an
// attached tool a push/pop costs a few nanoseconds.
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

}  // namespace detail
}  // namespace vb

#define VB_RANGE(name) vb::detail::Range vb_range_(name)

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
