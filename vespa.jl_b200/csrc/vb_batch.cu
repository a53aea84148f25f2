// vb_batch.cu -- batches of independent uniform 3D problems stepped together.
//
// Each box owns its state buffers, control block (clock, CFL dt, flags) and
// TMA descriptors, gathered in a device box table.  A step is four launches
// for the whole batch: per-box dt finalisation, the stage-1 and stage-2
// persistent tiled kernels pulling (box, column tile, z chunk) items from one
// queue, and the per-box clock advance.  Items are numbered largest box first
// so the tail of each stage is made of small items.  A run of nsteps steps is
// captured once as a CUDA graph and replayed.  vb_batch_autotune picks the
// work items' depth: a cap on the z chunk of every box, timed over the whole
// batch.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <numeric>
#include <vector>

#include "vb_internal.h"

using vb::detail::fail;
using vb::detail::use;

struct vb_batch {
    vb_ctx *ctx = nullptr;
    int nbox = 0;
    int precision = VB_FP64;
    std::vector<vb::Geom> geom;
    std::vector<double *> U, U1;
    vb::Ctrl *ctrl = nullptr;   // device, one per box
    vb::Ctrl *hctrl = nullptr;  // pinned mirror
    vb::BoxDesc *boxes = nullptr;
    int *item_box = nullptr;
    int nitems = 0;
    int kz_cap = 0;                          // chunk cap of the item layout (0: default chunks)
    std::vector<vb::TiledMaps> mU, mU1;      // per-box TMA descriptors
    std::vector<int> order;                  // boxes, largest first
    unsigned int *work = nullptr;  // the two stage cursors
    double *partials = nullptr, *totals = nullptr, *htot = nullptr;
    bool invdt_valid = false;
    std::map<int64_t, cudaGraphExec_t> graphs;  // nsteps -> instantiated graph
};

namespace {

int pull(vb_batch *b)
{
    VB_CUDA(cudaMemcpyAsync(b->hctrl, b->ctrl, sizeof(vb::Ctrl) * b->nbox, cudaMemcpyDeviceToHost,
                            b->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(b->ctx->stream));
    return VB_OK;
}

int push(vb_batch *b)
{
    VB_CUDA(cudaMemcpyAsync(b->ctrl, b->hctrl, sizeof(vb::Ctrl) * b->nbox, cudaMemcpyHostToDevice,
                            b->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(b->ctx->stream));
    return VB_OK;
}

int cfl_all(vb_batch *b)
{
    if (b->invdt_valid) return VB_OK;
    for (int i = 0; i < b->nbox; ++i)
        VB_CHECK_LAUNCH(b->ctx, vb::launch_cfl(b->geom[i], b->U[i], b->ctrl + i, b->ctx->stream));
    b->invdt_valid = true;
    return VB_OK;
}

int queue(vb_batch *b, int64_t nsteps)
{
    cudaStream_t s = b->ctx->stream;
    for (int64_t k = 0; k < nsteps; ++k) {
        VB_CHECK_LAUNCH(b->ctx, vb::launch_finalize_boxes(b->boxes, b->nbox, b->work, s));
        for (int st = 1; st <= 2; ++st)
            VB_CHECK_LAUNCH(b->ctx, b->precision == VB_MIXED
                                        ? vb::launch_stage_tiled3d_mixed(nullptr, b->boxes,
                                                                         b->item_box, b->nitems,
                                                                         b->work, st, s)
                                        : vb::launch_stage_tiled3d_fp64(nullptr, b->boxes,
                                                                        b->item_box, b->nitems,
                                                                        b->work, st, s));
        VB_CHECK_LAUNCH(b->ctx, vb::launch_advance_boxes(b->boxes, b->nbox, s));
    }
    return VB_OK;
}

// Work items for chunk cap `cap` (0: each box's default chunk): box
// descriptors and the item -> box table, uploaded on the stream.  Captured
// graphs hold the old item count, so they are dropped.
int set_layout(vb_batch *b, int cap)
{
    std::vector<vb::BoxDesc> hb(b->nbox);
    std::vector<int> item_box;
    for (int i : b->order) {
        const vb::Geom &g = b->geom[i];
        const int nz = (int)g.n[2];
        const int kz = cap > 0 ? (cap < nz ? cap : nz) : vb::detail::default_kz(g);
        const int64_t n = vb::detail::box_items(g, kz);
        if ((int64_t)item_box.size() + n > INT_MAX) return fail(VB_ENOTSUP, "too many work items");
        hb[i] = vb::detail::make_box(b->mU[i], b->mU1[i], g, b->U[i], b->U1[i], b->ctrl + i, kz,
                                     (int)item_box.size());
        item_box.insert(item_box.end(), (size_t)n, i);
    }
    VB_CUDA(cudaStreamSynchronize(b->ctx->stream));  // no step still reads the old tables
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    if ((int)item_box.size() > b->nitems || !b->item_box) {
        cudaFree(b->item_box);
        b->item_box = nullptr;
        VB_CUDA(cudaMalloc(&b->item_box, sizeof(int) * item_box.size()));
    }
    b->nitems = (int)item_box.size();
    VB_CUDA(cudaMemcpyAsync(b->boxes, hb.data(), sizeof(vb::BoxDesc) * b->nbox,
                            cudaMemcpyHostToDevice, b->ctx->stream));
    VB_CUDA(cudaMemcpyAsync(b->item_box, item_box.data(), sizeof(int) * item_box.size(),
                            cudaMemcpyHostToDevice, b->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(b->ctx->stream));
    b->kz_cap = cap;
    return VB_OK;
}

// Replay (capturing on first use) a graph of nsteps steps.
int run_graph(vb_batch *b, int64_t nsteps)
{
    auto it = b->graphs.find(nsteps);
    cudaGraphExec_t exec = nullptr;
    if (it != b->graphs.end()) {
        exec = it->second;
    } else {
        cudaStream_t s = b->ctx->stream;
        VB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int64_t before = b->ctx->launches;
        int rc = queue(b, nsteps);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return fail(VB_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(VB_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        b->ctx->launches = before;  // counted per replay below
        b->graphs[nsteps] = exec;
    }
    VB_CUDA(cudaGraphLaunch(exec, b->ctx->stream));
    b->ctx->launches += nsteps * 4;
    return VB_OK;
}

}  // namespace

extern "C" {

int vb_batch_create(vb_ctx *ctx, int nbox, const vb_problem_desc *descs, int precision,
                    vb_batch **out)
{
    if (!out) return fail(VB_EINVAL, "null output pointer");
    *out = nullptr;
    int rc = use(ctx);
    if (rc) return rc;
    if (nbox < 1 || !descs) return fail(VB_EINVAL, "need at least one box");
    if (precision != VB_FP64 && precision != VB_MIXED) return fail(VB_EINVAL, "unknown precision");
    std::vector<vb::Geom> geom(nbox);
    for (int i = 0; i < nbox; ++i) {
        rc = vb::detail::make_geom(&descs[i], &geom[i]);
        if (rc) return rc;
        if (!vb::tiled3d_supported(geom[i]))
            return fail(VB_ENOTSUP, "batch box " + std::to_string(i) +
                                        ": needs a 3D grid with nx, ny multiples of 16 and nz >= 2");
    }
    // make sure the persistent kernels' one-time set-up is done outside any capture
    vb::launch_stage_tiled3d_fp64(nullptr, nullptr, nullptr, 0, nullptr, 1, ctx->stream);
    vb::launch_stage_tiled3d_mixed(nullptr, nullptr, nullptr, 0, nullptr, 1, ctx->stream);

    vb_batch *b = new (std::nothrow) vb_batch();
    if (!b) return fail(VB_ENOMEM, "host allocation failed");
    b->ctx = ctx;
    b->nbox = nbox;
    b->precision = precision;
    b->geom = geom;
    b->U.assign(nbox, nullptr);
    b->U1.assign(nbox, nullptr);
    auto bail = [&](int code, const std::string &msg) {
        std::string m = msg;
        vb_batch_destroy(b);
        return fail(code, m);
    };
    cudaError_t e;
    for (int i = 0; i < nbox; ++i) {
        const size_t bytes = sizeof(double) * 5 * (size_t)geom[i].ncell;
        if ((e = cudaMalloc(&b->U[i], bytes)) != cudaSuccess ||
            (e = cudaMalloc(&b->U1[i], bytes)) != cudaSuccess)
            return bail(VB_ENOMEM, std::string("batch state allocation: ") + cudaGetErrorString(e));
        cudaMemsetAsync(b->U[i], 0, bytes, ctx->stream);
        cudaMemsetAsync(b->U1[i], 0, bytes, ctx->stream);
    }
    if ((e = cudaMalloc(&b->ctrl, sizeof(vb::Ctrl) * nbox)) != cudaSuccess ||
        (e = cudaMallocHost(&b->hctrl, sizeof(vb::Ctrl) * nbox)) != cudaSuccess ||
        (e = cudaMalloc(&b->boxes, sizeof(vb::BoxDesc) * nbox)) != cudaSuccess ||
        (e = cudaMalloc(&b->work, 2 * sizeof(unsigned int))) != cudaSuccess ||
        (e = cudaMalloc(&b->partials, sizeof(double) * 5 * vb::TOTALS_PARTS)) != cudaSuccess ||
        (e = cudaMalloc(&b->totals, sizeof(double) * 5)) != cudaSuccess ||
        (e = cudaMallocHost(&b->htot, sizeof(double) * 5)) != cudaSuccess)
        return bail(VB_ENOMEM, std::string("batch allocation: ") + cudaGetErrorString(e));
    std::memset(b->hctrl, 0, sizeof(vb::Ctrl) * nbox);
    for (int i = 0; i < nbox; ++i) {
        b->hctrl[i].tfinal = INFINITY;
        b->hctrl[i].step_limit = LLONG_MAX;
    }
    rc = push(b);
    if (rc) return bail(rc, "batch control upload failed");

    // work items: largest boxes first, chunk-major within a box
    b->order.resize(nbox);
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](int a, int c) { return geom[a].ncell > geom[c].ncell; });
    b->mU.resize(nbox);
    b->mU1.resize(nbox);
    for (int i = 0; i < nbox; ++i) {
        rc = vb::detail::encode_maps(&b->mU[i], b->U[i], geom[i]);
        if (!rc) rc = vb::detail::encode_maps(&b->mU1[i], b->U1[i], geom[i]);
        if (rc) return bail(rc, "batch tensor maps failed");
    }
    rc = set_layout(b, 0);
    if (rc) {
        char msg[256];
        vb_last_error(msg, sizeof msg);
        return bail(rc, std::string("batch work items: ") + msg);
    }
    *out = b;
    return VB_OK;
}

int vb_batch_destroy(vb_batch *b)
{
    if (!b) return VB_OK;
    if (b->ctx) {
        cudaSetDevice(b->ctx->device);
        cudaStreamSynchronize(b->ctx->stream);
    }
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    for (double *p : b->U) cudaFree(p);
    for (double *p : b->U1) cudaFree(p);
    cudaFree(b->ctrl);
    cudaFreeHost(b->hctrl);
    cudaFree(b->boxes);
    cudaFree(b->item_box);
    cudaFree(b->work);
    cudaFree(b->partials);
    cudaFree(b->totals);
    cudaFreeHost(b->htot);
    delete b;
    return VB_OK;
}

int vb_batch_ncell(const vb_batch *b, int box, int64_t *n)
{
    if (!b || !n) return fail(VB_EINVAL, "null argument");
    if (box == -1) {
        int64_t s = 0;
        for (const auto &g : b->geom) s += g.ncell;
        *n = s;
        return VB_OK;
    }
    if (box < 0 || box >= b->nbox) return fail(VB_EINVAL, "box index out of range");
    *n = b->geom[box].ncell;
    return VB_OK;
}

int vb_batch_upload(vb_batch *b, int box, const double *U)
{
    if (!b || !U) return fail(VB_EINVAL, "null argument");
    if (box < 0 || box >= b->nbox) return fail(VB_EINVAL, "box index out of range");
    int rc = use(b->ctx);
    if (rc) return rc;
    VB_CUDA(cudaMemcpyAsync(b->U[box], U, sizeof(double) * 5 * (size_t)b->geom[box].ncell,
                            cudaMemcpyHostToDevice, b->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(b->ctx->stream));
    b->invdt_valid = false;
    return VB_OK;
}

int vb_batch_download(vb_batch *b, int box, double *U)
{
    if (!b || !U) return fail(VB_EINVAL, "null argument");
    if (box < 0 || box >= b->nbox) return fail(VB_EINVAL, "box index out of range");
    int rc = use(b->ctx);
    if (rc) return rc;
    VB_CUDA(cudaMemcpyAsync(U, b->U[box], sizeof(double) * 5 * (size_t)b->geom[box].ncell,
                            cudaMemcpyDeviceToHost, b->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(b->ctx->stream));
    return VB_OK;
}

int vb_batch_run_steps_async(vb_batch *b, int64_t nsteps)
{
    VB_RANGE("vb_batch_run_steps_async");
    if (!b) return fail(VB_EINVAL, "null batch");
    if (nsteps < 0) return fail(VB_EINVAL, "nsteps < 0");
    if (nsteps == 0) return VB_OK;
    int rc = use(b->ctx);
    if (rc) return rc;
    rc = cfl_all(b);
    if (rc) return rc;
    return run_graph(b, nsteps);
}

int vb_batch_run_steps(vb_batch *b, int64_t nsteps)
{
    VB_RANGE("vb_batch_run_steps");
    int rc = vb_batch_run_steps_async(b, nsteps);
    if (rc) return rc;
    rc = pull(b);
    if (rc) return rc;
    for (int i = 0; i < b->nbox; ++i) {
        if (b->hctrl[i].flags & vb::CTRL_F_NONFINITE)
            return fail(VB_ENONFINITE, "box " + std::to_string(i) + ": non-finite dt");
        if (b->hctrl[i].flags & vb::CTRL_F_TIMEOUT)
            return fail(VB_ETIMEOUT, "box " + std::to_string(i) + ": a bounded device wait gave up");
    }
    return VB_OK;
}

int vb_batch_autotune(vb_batch *b, int nsteps, int64_t *best_cap, double *best_ms)
{
    VB_RANGE("vb_batch_autotune");
    if (!b || nsteps < 1) return fail(VB_EINVAL, "bad argument");
    int rc = use(b->ctx);
    if (rc) return rc;
    cudaStream_t s = b->ctx->stream;
    // scratch copies of every box's state and of the control blocks: the
    // candidates' steps are undone afterwards
    std::vector<double *> save(b->nbox, nullptr);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&]() {  // stream-ordered: no device-wide synchronisation
        for (double *p : save)
            if (p) cudaFreeAsync(p, s);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
    for (int i = 0; i < b->nbox && !rc; ++i) {
        const size_t bytes = sizeof(double) * 5 * (size_t)b->geom[i].ncell;
        if (cudaMallocAsync(&save[i], bytes, s) != cudaSuccess ||
            cudaMemcpyAsync(save[i], b->U[i], bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            rc = fail(VB_ENOMEM, "autotune: no room for a copy of the batch state");
    }
    if (!rc) rc = pull(b);
    if (rc) {
        cleanup();
        return rc;
    }
    const std::vector<vb::Ctrl> ctrl0(b->hctrl, b->hctrl + b->nbox);
    const bool valid0 = b->invdt_valid;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cleanup();
        return fail(VB_ECUDA, "autotune events");
    }
    // candidates: the default chunks (0) and caps on every box's chunk
    const int cand[] = {0, 16, 24, 32, 48, 64, 96, 128};
    int best = b->kz_cap;
    float best_t = INFINITY;
    for (int c : cand) {
        rc = set_layout(b, c);
        if (!rc) rc = cfl_all(b);
        if (!rc) rc = queue(b, 1);               // warm-up
        if (!rc) rc = run_graph(b, nsteps);      // capture outside the timed region
        if (rc) break;
        cudaEventRecord(e0, s);
        rc = run_graph(b, nsteps);
        cudaEventRecord(e1, s);
        if (rc) break;
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = fail(VB_ECUDA, "autotune timing failed");
            break;
        }
        if (ms < best_t) {
            best_t = ms;
            best = c;
        }
    }
    // restore states, clocks and the best layout, whatever happened
    for (int i = 0; i < b->nbox; ++i)
        cudaMemcpyAsync(b->U[i], save[i], sizeof(double) * 5 * (size_t)b->geom[i].ncell,
                        cudaMemcpyDeviceToDevice, s);
    std::copy(ctrl0.begin(), ctrl0.end(), b->hctrl);
    int rc2 = push(b);
    b->invdt_valid = valid0;  // the restored control blocks hold the saved states' CFL maxima
    int rc3 = set_layout(b, best);
    cleanup();
    if (rc) return rc;
    if (rc2) return rc2;
    if (rc3) return rc3;
    if (best_cap) *best_cap = best;
    if (best_ms) *best_ms = best_t / nsteps;
    return VB_OK;
}

int vb_batch_get_time(vb_batch *b, int box, double *t, int64_t *step)
{
    if (!b) return fail(VB_EINVAL, "null batch");
    if (box < 0 || box >= b->nbox) return fail(VB_EINVAL, "box index out of range");
    int rc = use(b->ctx);
    if (!rc) rc = pull(b);
    if (rc) return rc;
    if (t) *t = b->hctrl[box].t;
    if (step) *step = b->hctrl[box].step;
    return VB_OK;
}

int vb_batch_conserved_totals(vb_batch *b, int box, double out[5])
{
    if (!b || !out) return fail(VB_EINVAL, "null argument");
    if (box < 0 || box >= b->nbox) return fail(VB_EINVAL, "box index out of range");
    int rc = use(b->ctx);
    if (rc) return rc;
    VB_CHECK_LAUNCH(b->ctx, vb::launch_totals(b->geom[box], b->U[box], b->partials,
                                              vb::TOTALS_PARTS, b->totals, b->ctx->stream));
    VB_CUDA(cudaMemcpyAsync(b->htot, b->totals, sizeof(double) * 5, cudaMemcpyDeviceToHost,
                            b->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(b->ctx->stream));
    std::memcpy(out, b->htot, sizeof(double) * 5);
    return VB_OK;
}

}  // extern "C"
