// vb_amr.cu -- the extern "C" AMR API: a composite leaf-only mesh over a base
// grid (lib/HGBackend/src/HGBackend.jl), its regrid (src/driver.jl:400-462)
// and the single-rate and subcycled drivers (src/driver.jl:483-605,
// src/reflux.jl:51-103).
//
// Everything that touches leaves runs on the device: the stage kernels
// (vb_amr_kern.cu) and the topology work of a regrid -- tags, 2:1 balance,
// in-place children, the leaf hash, neighbour kinds, faces in emission order
// and the per-leaf CSR (vb_amr_regrid.cu).  The host keeps the counts, the
// clock and the driver loops; it reads a few words back per regrid.
//
// Choices where the reference defers to HierarchicalGrids.jl (absent here):
// the base grid is a forest of roots in column-major order, children are
// ordered x fastest (x + 2y + 4z), the representative of a face with finer
// leaves is the first of them in that order, and balance is across faces.
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <utility>
#include <vector>

#include "vb_amr.h"
#include "vb_internal.h"

using vb::detail::fail;
using vb::detail::use;

namespace {
constexpr int CBITS = 20;  // bits per integer coordinate in a leaf key
}  // namespace

struct vb_amr {
    vb_ctx *ctx = nullptr;
    vb::Geom g{};  // base geometry: nd, bcs, gamma, cfl, aexp (cells per axis = base)
    int nd = 1;
    int64_t base[3] = {1, 1, 1};
    double w0[3] = {1, 1, 1};
    double t = 0.0;
    int64_t step = 0;
    int n = 0;          // leaves
    int maxlev = 0;     // deepest leaf level
    int nface = 0, nent = 0;
    // leaf-indexed device buffers (stride cap)
    int64_t cap = 0;
    double *U = nullptr, *U1 = nullptr, *reg = nullptr;
    int *lev = nullptr, *cx = nullptr;          // level, [3][cap] coordinates
    double *U2 = nullptr;                       // refinement targets, swapped in
    int *lev2 = nullptr, *cx2 = nullptr;
    int *rep = nullptr, *faceid = nullptr;      // [6][cap]
    int8_t *kind = nullptr;                     // [6][cap]
    int *off = nullptr, *fbase = nullptr;       // cap + 1
    int *cnt = nullptr, *fcnt = nullptr, *ecnt = nullptr;
    int *bsum = nullptr;                        // scan block sums
    uint8_t *tag = nullptr;
    // face-indexed (stride fcap) and CSR
    int64_t fcap = 0, ecap = 0;
    double *F = nullptr, *farea = nullptr;
    int *fL = nullptr, *fR = nullptr, *ent = nullptr;
    int8_t *fax = nullptr;
    // hash of (level, coordinates) -> leaf
    int64_t hcap = 0;
    uint64_t *hkey = nullptr;
    int *hval = nullptr;
    // small device words: [0] error bits, [1] unused, [2] max level, [3] scan total (faces
    // in a table build), [4] tags, [5] entries of a table build, [8, 8 + BAL_GROUP) marks
    // changed by each balance pass of a group
    int *word = nullptr, *hword = nullptr;
    vb::Ctrl *ctrl = nullptr, *hctrl = nullptr;
    double *partials = nullptr, *totals = nullptr, *htot = nullptr;
    vb::AmrDev dev{};
    vb::AmrAreas areas{};
    double ms_regrid = 0.0;
    // device-driven subcycling: per-level loop state, error bits, and the
    // graph of one root step (nested WHILE nodes, one per level), valid for
    // the table version and deepest level it was built for
    vb::AmrSubLevel *sub = nullptr;
    int *suberr = nullptr;
    cudaGraphExec_t sg_exec = nullptr;
    int64_t sg_version = -1;
    int64_t table_version = 0;
    int sg_launches = 0;
};

namespace {

double level_width(const vb_amr *a, int l, int d) { return a->w0[d] * std::ldexp(1.0, -l); }

void release(vb_amr *a)
{
    if (a->sg_exec) cudaGraphExecDestroy(a->sg_exec);
    cudaFree(a->sub);
    cudaFree(a->suberr);
    void *p[] = {a->U, a->U1, a->U2, a->lev2, a->cx2, a->reg, a->lev, a->cx, a->rep, a->faceid, a->kind, a->off,
                 a->fbase, a->cnt, a->fcnt, a->ecnt, a->bsum, a->tag, a->F, a->farea,
                 a->fL, a->fR, a->ent, a->fax, a->hkey, a->hval, a->word, a->ctrl,
                 a->partials, a->totals};
    for (void *q : p) cudaFree(q);
    cudaFreeHost(a->hword);
    cudaFreeHost(a->hctrl);
    cudaFreeHost(a->htot);
}

// Stream-ordered (re)allocation from the device's memory pool: a regrid that
// grows its tables neither synchronises the device (as cudaFree does) nor
// maps fresh memory once the pool holds enough (the pool keeps what is freed,
// see vb_ctx_create).
template <typename T>
int realloc_dev(T **p, int64_t count, cudaStream_t s)
{
    if (*p) VB_CUDA(cudaFreeAsync(*p, s));
    *p = nullptr;
    VB_CUDA(cudaMallocAsync((void **)p, sizeof(T) * (size_t)(count > 0 ? count : 1), s));
    return VB_OK;
}

// Leaf buffers other than U, lev and cx (which a refinement replaces itself).
int alloc_leaf_buffers(vb_amr *a, int64_t c)
{
    int rc = realloc_dev(&a->U1, 5 * c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->U2, 5 * c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->lev2, c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->cx2, 3 * c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->reg, 5 * c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->rep, 6 * c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->faceid, 6 * c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->kind, 6 * c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->off, c + 1, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->fbase, c + 1, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->cnt, c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->fcnt, c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->ecnt, c, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->bsum, c / 1024 + 2, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->tag, c, a->ctx->stream);
    if (rc) return rc;
    VB_CUDA(cudaMemsetAsync(a->reg, 0, sizeof(double) * 5 * c, a->ctx->stream));
    a->cap = c;
    return VB_OK;
}

constexpr int NWORD = 16;     // device words per mesh (see vb_amr::word)
constexpr int BAL_GROUP = 4;  // balance passes queued per host read

int sync_words(vb_amr *a)
{
    VB_CUDA(cudaMemcpyAsync(a->hword, a->word, sizeof(int) * NWORD, cudaMemcpyDeviceToHost,
                            a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

vb::AmrTopo topo(const vb_amr *a)
{
    vb::AmrTopo t{};
    t.nd = a->nd;
    for (int d = 0; d < 3; ++d) {
        t.base[d] = a->base[d];
        t.bc_lo[d] = a->g.bc_lo[d];
        t.bc_hi[d] = a->g.bc_hi[d];
    }
    t.n = a->n;
    t.cap = a->cap;
    t.lev = a->lev;
    t.cx = a->cx;
    t.hkey = a->hkey;
    t.hval = a->hval;
    t.hmask = (uint64_t)a->hcap - 1;
    return t;
}

// Rebuild the hash and every table from (lev, cx) of the current leaves.
int build_tables(vb_amr *a)
{
    cudaStream_t s = a->ctx->stream;
    int64_t hc = 1024;
    while (hc < 2 * (int64_t)a->n) hc *= 2;
    if (hc != a->hcap) {
        int rc = realloc_dev(&a->hkey, hc, a->ctx->stream);
        if (!rc) rc = realloc_dev(&a->hval, hc, a->ctx->stream);
        if (rc) return rc;
        a->hcap = hc;
    }
    // Face and entry arrays sized for the most these leaves can have (a leaf
    // emits at most its hi and lo face per axis; its CSR holds those and at
    // most 2^(nd-1) finer faces per side), so the whole build queues behind
    // one read of the totals and the error bits.
    const int64_t nf_max = 2ll * a->nd * a->n;
    const int64_t ne_max = nf_max * (1 + (1 << (a->nd - 1)));
    int rc = VB_OK;
    if (nf_max > a->fcap) {
        int64_t c = a->fcap ? a->fcap : 4096;
        while (c < nf_max) c *= 2;
        rc = realloc_dev(&a->fL, c, a->ctx->stream);
        if (!rc) rc = realloc_dev(&a->fR, c, a->ctx->stream);
        if (!rc) rc = realloc_dev(&a->fax, c, a->ctx->stream);
        if (!rc) rc = realloc_dev(&a->farea, c, a->ctx->stream);
        if (!rc) rc = realloc_dev(&a->F, 5 * c, a->ctx->stream);
        if (rc) return rc;
        a->fcap = c;
    }
    if (ne_max > a->ecap) {
        int64_t c = a->ecap ? a->ecap : 8192;
        while (c < ne_max) c *= 2;
        rc = realloc_dev(&a->ent, c, a->ctx->stream);
        if (rc) return rc;
        a->ecap = c;
    }
    VB_CUDA(cudaMemsetAsync(a->word, 0, sizeof(int) * NWORD, s));
    vb::AmrTopo t = topo(a);
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_hash_build(t, a->hkey, a->hval, a->word, s));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_kinds(t, a->kind, a->rep, a->fcnt, s));
    VB_CHECK_LAUNCH(a->ctx, vb::amr_scan(a->fcnt, a->n, a->fbase, a->bsum, a->word + 3, s));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_csr_count(t, a->kind, a->fcnt, a->ecnt, s));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_faces(t, a->kind, a->rep, a->fbase, a->areas, a->fL,
                                                 a->fR, a->fax, a->farea, a->faceid, s));
    VB_CHECK_LAUNCH(a->ctx, vb::amr_scan(a->ecnt, a->n, a->off, a->bsum, a->word + 5, s));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_csr_fill(t, a->kind, a->rep, a->faceid, a->off,
                                                    a->ent, a->word, s));
    rc = sync_words(a);
    if (rc) return rc;
    const int nf = a->hword[3];
    const int ne = a->hword[5];
    if (a->hword[0]) return fail(VB_ECUDA, "AMR table build failed (hash or CSR overflow)");
    if (nf > a->fcap || ne > a->ecap) return fail(VB_ECUDA, "AMR table build: face count out of range");
    a->nface = nf;
    a->nent = ne;
    vb::AmrDev &m = a->dev;
    m.nd = a->nd;
    for (int d = 0; d < 3; ++d) {
        m.bc_lo[d] = a->g.bc_lo[d];
        m.bc_hi[d] = a->g.bc_hi[d];
    }
    m.gamma = a->g.gamma;
    m.aexp = a->g.aexp;
    m.cap = a->cap;
    m.fcap = a->fcap;
    m.nleaf = a->n;
    m.nface = nf;
    m.nent = ne;
    m.lev = a->lev;
    m.rep = a->rep;
    m.fL = a->fL;
    m.fR = a->fR;
    m.fax = a->fax;
    m.farea = a->farea;
    m.off = a->off;
    m.ent = a->ent;
    m.reg = a->reg;
    ++a->table_version;  // kernels capture the tables by value: graphs are stale
    return VB_OK;
}

// Refine the leaves marked in a->tag (with 2:1 balance), remap the state and
// rebuild the tables.  Balance passes queue in groups of BAL_GROUP, each pass
// gated on the previous one having changed a mark (the group's first pass on
// `gate`, the tag count, when given), and the leaf count is queued behind the
// group: one host read settles both unless the group's last pass still
// changed marks (then another group runs and the count is redone).
int refine_marked(vb_amr *a, const int *gate = nullptr, int64_t *ntag = nullptr)
{
    cudaStream_t s = a->ctx->stream;
    vb::AmrTopo t = topo(a);
    int *flags = a->word + 8;
    for (int group = 0;; ++group) {
        if (group * BAL_GROUP > 2 * vb::AMR_MAX_LEVEL + 4)
            return fail(VB_ECUDA, "AMR balance did not converge");
        VB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * BAL_GROUP, s));
        for (int p = 0; p < BAL_GROUP; ++p) {
            const int *g = p > 0 ? flags + p - 1 : (group == 0 ? gate : nullptr);
            VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_balance(t, a->tag, flags + p, g, s));
        }
        VB_CUDA(cudaMemsetAsync(a->word + 2, 0, sizeof(int), s));
        VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_count_children(t, a->tag, a->cnt, a->word + 2, s));
        VB_CHECK_LAUNCH(a->ctx, vb::amr_scan(a->cnt, a->n, a->fbase, a->bsum, a->word + 3, s));
        int rc = sync_words(a);
        if (rc) return rc;
        if (group == 0 && ntag) *ntag = a->hword[4];
        if (!a->hword[8 + BAL_GROUP - 1]) break;  // a pass of the group changed nothing
    }
    const int64_t n_new = a->hword[3];
    const int maxlev = a->hword[2];
    if (n_new == a->n) return VB_OK;  // nothing refined
    if (maxlev > vb::AMR_MAX_LEVEL) return fail(VB_ENOTSUP, "refinement beyond the supported depth");
    for (int d = 0; d < a->nd; ++d)
        if ((a->base[d] << maxlev) >= (1LL << CBITS))
            return fail(VB_ENOTSUP, "refinement beyond the supported coordinate range");
    if (n_new > INT_MAX / 8) return fail(VB_ENOTSUP, "too many leaves");
    int64_t cap_new = a->cap;
    while (cap_new < n_new) cap_new *= 2;
    if (cap_new > a->cap) {
        // grow: fresh targets of the new capacity; the other leaf buffers follow
        double *Unew = nullptr;
        int *lev_new = nullptr, *cx_new = nullptr;
        cudaError_t e = cudaMallocAsync(&Unew, sizeof(double) * 5 * cap_new, s);
        if (e == cudaSuccess) e = cudaMallocAsync(&lev_new, sizeof(int) * cap_new, s);
        if (e == cudaSuccess) e = cudaMallocAsync(&cx_new, sizeof(int) * 3 * cap_new, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(cx_new, 0, sizeof(int) * 3 * cap_new, s);
        if (e != cudaSuccess) {
            if (Unew) cudaFreeAsync(Unew, s);
            if (lev_new) cudaFreeAsync(lev_new, s);
            if (cx_new) cudaFreeAsync(cx_new, s);
            return fail(VB_ENOMEM, std::string("regrid buffers: ") + cudaGetErrorString(e));
        }
        VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_emit(t, a->tag, a->fbase, lev_new, cx_new, cap_new,
                                                    a->U, Unew, s));
        // stream order: the frees follow the emit that reads the old buffers
        VB_CUDA(cudaFreeAsync(a->U, s));
        VB_CUDA(cudaFreeAsync(a->lev, s));
        VB_CUDA(cudaFreeAsync(a->cx, s));
        a->U = Unew;
        a->lev = lev_new;
        a->cx = cx_new;
        const int rc = alloc_leaf_buffers(a, cap_new);
        if (rc) return rc;
    } else {
        // same capacity: emit into the spare buffers and swap
        VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_emit(t, a->tag, a->fbase, a->lev2, a->cx2, a->cap,
                                                    a->U, a->U2, s));
        std::swap(a->U, a->U2);
        std::swap(a->lev, a->lev2);
        std::swap(a->cx, a->cx2);
    }
    a->n = (int)n_new;
    a->maxlev = maxlev;
    return build_tables(a);
}

int pull_ctrl(vb_amr *a)
{
    VB_CUDA(cudaMemcpyAsync(a->hctrl, a->ctrl, sizeof(vb::Ctrl), cudaMemcpyDeviceToHost,
                            a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

int push_ctrl(vb_amr *a)
{
    VB_CUDA(cudaMemcpyAsync(a->ctrl, a->hctrl, sizeof(vb::Ctrl), cudaMemcpyHostToDevice,
                            a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

int compute_dt_level(vb_amr *a, int level, double *dt)
{
    cudaStream_t s = a->ctx->stream;
    VB_CUDA(cudaMemsetAsync(&a->ctrl->invdt_bits, 0, sizeof(unsigned long long), s));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_cfl(a->dev, a->U, level, a->ctrl, s));
    int rc = pull_ctrl(a);
    if (rc) return rc;
    double invdt;
    std::memcpy(&invdt, &a->hctrl->invdt_bits, sizeof invdt);
    if (std::isnan(invdt)) return fail(VB_ENONFINITE, "non-finite or negative density/pressure");
    *dt = invdt == 0.0 ? INFINITY : a->g.cfl / invdt;
    return VB_OK;
}

// step!(sim, dt; level) / step_level! with the given registers (host dt)
int step_level(vb_amr *a, double dt, int level, int nreg, const int *rl, const double *rsc)
{
    vb::AmrStageArgs s{};
    s.dt = dt;
    s.level = level;
    s.nreg = nreg;
    for (int r = 0; r < nreg; ++r) {
        s.reg_level[r] = rl[r];
        s.reg_scale[r] = rsc[r];
    }
    s.cfl_all = 0;
    cudaStream_t st = a->ctx->stream;
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 1, a->U, a->U, a->U1, a->F, s, a->ctrl, st));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 2, a->U1, a->U, a->U, a->F, s, a->ctrl, st));
    return VB_OK;
}

inline double jmin(double x, double y)
{
    if (x != x || y != y) return x + y;
    return y < x ? y : x;
}

// ---- device-driven subcycling: evolve_level! as nested CUDA-graph loops ----
//
// One root step is one graph.  Level l contributes, in the graph of its
// parent's substep body (the root graph for level 0): its CFL maximum, a plan
// node (substep count and dt from that maximum and the dt target: the
// parent's substep dt), and a WHILE node whose body is one substep -- zero the
// level's flux registers when a finer level exists, the two stages with the
// substep dt read on the device, then (with a finer level) that level's own
// CFL / plan / WHILE nodes and the reflux, and finally a node that counts the
// substep and sets the loop condition.  Every loop is bounded
// (AMR_MAX_SUBSTEPS) and stops on the first error bit, so the graph always
// ends.  The kernels and their order are those of the host recursion below,
// with the same dt values, so the results are the same bits.

struct SubBody {
    cudaGraph_t graph;
    int level;
    cudaGraphConditionalHandle handle;
};

// In the graph being captured on `s`: level l's CFL maximum, plan and WHILE
// node; the node's (empty) body goes to `todo`.
int emit_level_head(vb_amr *a, cudaStream_t s, int l, std::vector<SubBody> &todo)
{
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    VB_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps));
    if (st != cudaStreamCaptureStatusActive || !g) return fail(VB_ECUDA, "subcycle graph: no capture");
    cudaGraphConditionalHandle h;
    VB_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_cfl_bits(a->dev, a->U, l, &a->sub[l].invdt_bits, s));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_sub_plan(a->sub, l, a->g.cfl,
                                                    l > 0 ? &a->sub[l - 1].dt_sub : nullptr, h,
                                                    a->suberr, s));
    VB_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    VB_CUDA(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
    VB_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    todo.push_back({cp.conditional.phGraph_out[0], l, h});
    return VB_OK;
}

// Capture one substep of level b.level into its WHILE body (b by value: the
// nested head appends to `todo`).
int fill_level_body(vb_amr *a, cudaStream_t s, SubBody b, std::vector<SubBody> &todo)
{
    const int l = b.level;
    const bool has_finer = l < a->maxlev;
    VB_CUDA(cudaStreamBeginCaptureToGraph(s, b.graph, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
    int rc = VB_OK;
    auto body = [&]() -> int {
        if (has_finer) VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_zero_reg(a->dev, l, s));
        vb::AmrStageArgs sa{};
        sa.dt = 0.0;
        sa.level = l;
        sa.dt_dev = &a->sub[l].dt_sub;
        int nr = 0;
        if (l > 0) { sa.reg_level[nr] = l - 1; sa.reg_scale[nr] = 1.0; ++nr; }
        if (has_finer) { sa.reg_level[nr] = l; sa.reg_scale[nr] = -1.0; ++nr; }
        sa.nreg = nr;
        sa.cfl_all = 0;
        VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 1, a->U, a->U, a->U1, a->F, sa, a->ctrl, s));
        VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 2, a->U1, a->U, a->U, a->F, sa, a->ctrl, s));
        if (has_finer) {
            int r = emit_level_head(a, s, l + 1, todo);
            if (r) return r;
            VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_reflux(a->dev, a->U, l, s));
        }
        VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_sub_next(a->sub, l, b.handle, a->suberr, s));
        return VB_OK;
    };
    rc = body();
    cudaGraph_t out = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &out);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(VB_ECUDA, std::string("subcycle body capture: ") + cudaGetErrorString(e));
    return VB_OK;
}

// The graph of one root step for the current tables (rebuilt after a regrid).
int build_subcycle_graph(vb_amr *a)
{
    if (a->sg_exec) {
        cudaGraphExecDestroy(a->sg_exec);
        a->sg_exec = nullptr;
    }
    if (!a->sub) {
        VB_CUDA(cudaMalloc(&a->sub, sizeof(vb::AmrSubLevel) * (vb::AMR_MAX_LEVEL + 1)));
        VB_CUDA(cudaMalloc(&a->suberr, sizeof(int)));
    }
    cudaStream_t s = a->ctx->stream;
    const int64_t launches0 = a->ctx->launches;
    cudaGraph_t root = nullptr;
    VB_CUDA(cudaGraphCreate(&root, 0));
    std::vector<SubBody> todo;
    int rc = VB_OK;
    cudaError_t e = cudaStreamBeginCaptureToGraph(s, root, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) rc = fail(VB_ECUDA, std::string("subcycle capture: ") + cudaGetErrorString(e));
    if (!rc) {
        rc = emit_level_head(a, s, 0, todo);
        cudaGraph_t out = nullptr;
        e = cudaStreamEndCapture(s, &out);
        if (!rc && e != cudaSuccess)
            rc = fail(VB_ECUDA, std::string("subcycle capture: ") + cudaGetErrorString(e));
    }
    for (size_t i = 0; i < todo.size() && !rc; ++i) rc = fill_level_body(a, s, todo[i], todo);
    if (!rc) {
        e = cudaGraphInstantiate(&a->sg_exec, root, 0);
        if (e != cudaSuccess) {
            a->sg_exec = nullptr;
            rc = fail(VB_ECUDA, std::string("subcycle graph instantiate: ") + cudaGetErrorString(e));
        }
    }
    cudaGraphDestroy(root);
    a->sg_launches = (int)(a->ctx->launches - launches0);
    a->ctx->launches = launches0;  // counted when the graph runs
    if (rc) {
        cudaGetLastError();
        return rc;
    }
    a->sg_version = a->table_version;
    return VB_OK;
}

// One subcycled root step of dt_root on the device (evolve_level!(sim, 0,
// dt_root)); the host reads the error bits back with the next control-block
// read.
int root_step_graph(vb_amr *a, double dt_root)
{
    cudaStream_t s = a->ctx->stream;
    VB_CUDA(cudaMemsetAsync(a->sub, 0, sizeof(vb::AmrSubLevel) * (vb::AMR_MAX_LEVEL + 1), s));
    VB_CUDA(cudaMemsetAsync(a->suberr, 0, sizeof(int), s));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_sub_target(a->sub, dt_root, s));
    VB_CUDA(cudaGraphLaunch(a->sg_exec, s));
    a->ctx->launches += a->sg_launches;  // nodes of one pass (loops repeat some)
    return VB_OK;
}

int regrid(vb_amr *a, double above, int maxl, int64_t *ntag)
{
    cudaStream_t st = a->ctx->stream;
    VB_CUDA(cudaMemsetAsync(a->word + 4, 0, sizeof(int), st));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_tag(a->dev, a->U, above, maxl, a->tag, nullptr,
                                               a->word + 4, st));
    // no host read of the tag count: with none tagged the balance passes skip
    // and the leaf count comes back unchanged
    return refine_marked(a, a->word + 4, ntag);
}

}  // namespace

extern "C" {

int vb_amr_create(vb_ctx *ctx, const vb_problem_desc *d, vb_amr **out)
{
    if (!ctx || !d || !out) return fail(VB_EINVAL, "null argument");
    *out = nullptr;
    vb::Geom g{};
    int rc = vb::detail::make_geom(d, &g);
    if (rc) return rc;
    for (int k = 0; k < g.nd; ++k)
        if (g.n[k] >= (1LL << CBITS)) return fail(VB_EINVAL, "base grid too large for AMR keys");
    rc = use(ctx);
    if (rc) return rc;
    vb_amr *a = new (std::nothrow) vb_amr;
    if (!a) return fail(VB_ENOMEM, "host allocation failed");
    a->ctx = ctx;
    a->g = g;
    a->nd = g.nd;
    for (int k = 0; k < 3; ++k) {
        a->base[k] = k < g.nd ? g.n[k] : 1;
        a->w0[k] = k < g.nd ? g.w[k] : 1.0;
    }
    for (int l = 0; l <= vb::AMR_MAX_LEVEL; ++l) {
        double v = 1.0;
        for (int d = 0; d < 3; ++d) {
            double ar = 1.0;
            for (int e2 = 0; e2 < a->nd; ++e2)
                if (e2 != d) ar = ar * level_width(a, l, e2);
            a->areas.area[l][d] = ar;
            a->dev.w[l][d] = d < a->nd ? level_width(a, l, d) : 1.0;
        }
        for (int d = 0; d < a->nd; ++d) v = v * a->dev.w[l][d];
        a->dev.vol[l] = v;
    }
    const int64_t n = a->base[0] * a->base[1] * a->base[2];
    if (n > INT_MAX / 8) {
        delete a;
        return fail(VB_EINVAL, "base grid too large");
    }
    std::vector<int> lev0((size_t)n, 0), cx0;
    cudaError_t e = cudaMalloc(&a->ctrl, sizeof(vb::Ctrl));
    if (e == cudaSuccess) e = cudaMallocHost(&a->hctrl, sizeof(vb::Ctrl));
    if (e == cudaSuccess) e = cudaMalloc(&a->partials, sizeof(double) * 5 * vb::TOTALS_PARTS);
    if (e == cudaSuccess) e = cudaMalloc(&a->totals, sizeof(double) * 5);
    if (e == cudaSuccess) e = cudaMallocHost(&a->htot, sizeof(double) * 5);
    if (e != cudaSuccess) {
        release(a);
        delete a;
        return fail(VB_ENOMEM, std::string("AMR buffers: ") + cudaGetErrorString(e));
    }
    std::memset(a->hctrl, 0, sizeof(vb::Ctrl));
    a->hctrl->tfinal = INFINITY;
    a->hctrl->step_limit = LLONG_MAX;
    e = cudaMalloc(&a->word, sizeof(int) * NWORD);
    if (e == cudaSuccess) e = cudaMallocHost(&a->hword, sizeof(int) * NWORD);
    if (e != cudaSuccess) {
        release(a);
        delete a;
        return fail(VB_ENOMEM, std::string("AMR buffers: ") + cudaGetErrorString(e));
    }
    int64_t cap = 1024;
    while (cap < n) cap *= 2;
    // base leaves: level 0, column-major
    cx0.assign((size_t)(3 * cap), 0);
    for (int64_t i = 0; i < n; ++i) {
        cx0[i] = (int)(i % a->base[0]);
        cx0[cap + i] = (int)((i / a->base[0]) % a->base[1]);
        cx0[2 * cap + i] = (int)(i / (a->base[0] * a->base[1]));
    }
    rc = realloc_dev(&a->U, 5 * cap, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->lev, cap, a->ctx->stream);
    if (!rc) rc = realloc_dev(&a->cx, 3 * cap, a->ctx->stream);
    if (!rc) rc = alloc_leaf_buffers(a, cap);
    if (!rc && (cudaMemcpy(a->lev, lev0.data(), sizeof(int) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(a->cx, cx0.data(), sizeof(int) * 3 * cap, cudaMemcpyHostToDevice) != cudaSuccess))
        rc = fail(VB_ECUDA, "AMR base upload failed");
    a->n = (int)n;
    a->maxlev = 0;
    if (!rc) rc = push_ctrl(a);
    if (!rc) rc = build_tables(a);
    if (!rc) {
        VB_CUDA(cudaMemsetAsync(a->U, 0, sizeof(double) * 5 * a->cap, ctx->stream));
        VB_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    if (rc) {
        release(a);
        delete a;
        return rc;
    }
    *out = a;
    return VB_OK;
}

int vb_amr_destroy(vb_amr *a)
{
    if (!a) return VB_OK;
    cudaSetDevice(a->ctx->device);
    cudaStreamSynchronize(a->ctx->stream);
    release(a);
    delete a;
    return VB_OK;
}

int vb_amr_nleaf(const vb_amr *a, int64_t *n)
{
    if (!a || !n) return fail(VB_EINVAL, "null argument");
    *n = a->n;
    return VB_OK;
}

int vb_amr_leaves(const vb_amr *a, int32_t *level, int64_t *coords)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    const int64_t n = a->n;
    std::vector<int> lev((size_t)n), cx((size_t)(3 * n));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    VB_CUDA(cudaMemcpy(lev.data(), a->lev, sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (int d = 0; d < 3; ++d)
        VB_CUDA(cudaMemcpy(cx.data() + d * n, a->cx + d * a->cap, sizeof(int) * n,
                           cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; ++i) {
        if (level) level[i] = lev[i];
        if (coords)
            for (int d = 0; d < 3; ++d) coords[3 * i + d] = cx[d * n + i];
    }
    return VB_OK;
}

int vb_amr_nface(const vb_amr *a, int64_t *n)
{
    if (!a || !n) return fail(VB_EINVAL, "null argument");
    *n = a->nface;
    return VB_OK;
}

int vb_amr_max_level(const vb_amr *a, int32_t *level)
{
    if (!a || !level) return fail(VB_EINVAL, "null argument");
    *level = a->maxlev;
    return VB_OK;
}

int vb_amr_upload(vb_amr *a, const double *U)
{
    if (!a || !U) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    const int64_t n = a->n;
    VB_CUDA(cudaMemcpy2DAsync(a->U, sizeof(double) * a->cap, U, sizeof(double) * n,
                              sizeof(double) * n, 5, cudaMemcpyHostToDevice, a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

int vb_amr_download(vb_amr *a, double *U)
{
    if (!a || !U) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    const int64_t n = a->n;
    VB_CUDA(cudaMemcpy2DAsync(U, sizeof(double) * n, a->U, sizeof(double) * a->cap,
                              sizeof(double) * n, 5, cudaMemcpyDeviceToHost, a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

int vb_amr_set_time(vb_amr *a, double t, int64_t step)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    a->t = t;
    a->step = step;
    return VB_OK;
}

int vb_amr_get_time(const vb_amr *a, double *t, int64_t *step)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    if (t) *t = a->t;
    if (step) *step = a->step;
    return VB_OK;
}

int vb_amr_refine(vb_amr *a, const int64_t *leaves, int64_t n)
{
    VB_RANGE("vb_amr_refine");
    if (!a || (n > 0 && !leaves)) return fail(VB_EINVAL, "null argument");
    const int64_t nl = a->n;
    std::vector<uint8_t> mark((size_t)nl, 0);
    for (int64_t k = 0; k < n; ++k) {
        if (leaves[k] < 0 || leaves[k] >= nl) return fail(VB_EINVAL, "leaf index out of range");
        mark[(size_t)leaves[k]] = 1;
    }
    int rc = use(a->ctx);
    if (rc) return rc;
    if (n == 0) return VB_OK;
    VB_CUDA(cudaMemcpy(a->tag, mark.data(), (size_t)nl, cudaMemcpyHostToDevice));
    return refine_marked(a);
}

int vb_amr_indicator(vb_amr *a, double *out)
{
    if (!a || !out) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    const int64_t n = a->n;
    double *d = nullptr;
    VB_CUDA(cudaMallocAsync(&d, sizeof(double) * (n > 0 ? n : 1), a->ctx->stream));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_tag(a->dev, a->U, INFINITY, 0, a->tag, d, nullptr,
                                               a->ctx->stream));
    cudaError_t e = cudaMemcpyAsync(out, d, sizeof(double) * n, cudaMemcpyDeviceToHost, a->ctx->stream);
    cudaFreeAsync(d, a->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(a->ctx->stream);
    if (e != cudaSuccess) return fail(VB_ECUDA, cudaGetErrorString(e));
    return VB_OK;
}

int vb_amr_regrid(vb_amr *a, double refine_above, int max_level_, int64_t *ntagged)
{
    VB_RANGE("vb_amr_regrid");
    if (!a) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    return regrid(a, refine_above, max_level_, ntagged);
}

int vb_amr_compute_dt(vb_amr *a, int level, double *dt)
{
    VB_RANGE("vb_amr_compute_dt");
    if (!a || !dt) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    return compute_dt_level(a, level, dt);
}

int vb_amr_step(vb_amr *a, double dt)
{
    VB_RANGE("vb_amr_step");
    if (!a) return fail(VB_EINVAL, "null argument");
    if (!std::isfinite(dt)) return fail(VB_EINVAL, "dt must be finite");
    int rc = use(a->ctx);
    if (rc) return rc;
    rc = step_level(a, dt, -1, 0, nullptr, nullptr);
    if (rc) return rc;
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    a->t += dt;
    a->step += 1;
    return VB_OK;
}

int vb_amr_step_level(vb_amr *a, double dt, int level)
{
    VB_RANGE("vb_amr_step_level");
    if (!a) return fail(VB_EINVAL, "null argument");
    if (!std::isfinite(dt)) return fail(VB_EINVAL, "dt must be finite");
    int rc = use(a->ctx);
    if (rc) return rc;
    rc = step_level(a, dt, level, 0, nullptr, nullptr);
    if (rc) return rc;
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

int vb_amr_evolve(vb_amr *a, double tfinal, int64_t max_steps, double refine_above,
                  int max_level_, int every, int subcycle, double *t_out, int64_t *nsteps)
{
    VB_RANGE("vb_amr_evolve");
    if (!a) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    cudaStream_t st = a->ctx->stream;
    int64_t done = 0;
    a->ms_regrid = 0.0;
    auto do_regrid = [&]() -> int {
        if (every > 0 && a->step % every == 0) {
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, st);
            int r = regrid(a, refine_above, max_level_, nullptr);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            a->ms_regrid += ms;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return r;
        }
        return VB_OK;
    };
    if (subcycle) {
        // each root step runs as one graph: the recursion over the levels,
        // their substep counts and dts all on the device
        int errbits = 0;
        while (a->t < tfinal * (1 - 1e-12)) {
            if (max_steps >= 0 && done >= max_steps) break;
            rc = do_regrid();
            if (rc) return rc;
            double dt0;
            rc = compute_dt_level(a, 0, &dt0);  // also synchronises the previous root step
            if (rc) return rc;
            if (a->sub) {
                VB_CUDA(cudaMemcpy(&errbits, a->suberr, sizeof(int), cudaMemcpyDeviceToHost));
                if (errbits) break;
            }
            const double dt_root = jmin(dt0, tfinal - a->t);
            if (a->sg_version != a->table_version) {
                rc = build_subcycle_graph(a);
                if (rc) return rc;
            }
            rc = root_step_graph(a, dt_root);
            if (rc) return rc;
            a->t += dt_root;
            a->step += 1;
            ++done;
        }
        if (!errbits && a->sub) {
            VB_CUDA(cudaStreamSynchronize(st));
            VB_CUDA(cudaMemcpy(&errbits, a->suberr, sizeof(int), cudaMemcpyDeviceToHost));
        }
        if (errbits & vb::AMR_SUB_NONFINITE)
            return fail(VB_ENONFINITE, "non-finite dt: NaN or negative density/pressure");
        if (errbits & vb::AMR_SUB_TOO_MANY)
            return fail(VB_ENONFINITE, "a level needed more than 2^20 substeps");
    } else {
        // single rate: dt, stages and clock on the device between regrids
        vb::Geom gq = a->g;  // finalize kernel reads cfl (its invV is unused here)
        while (a->t < tfinal * (1 - 1e-12)) {
            if (max_steps >= 0 && done >= max_steps) break;
            rc = do_regrid();
            if (rc) return rc;
            int64_t chunk = every > 0 ? every - a->step % every : 64;
            if (max_steps >= 0 && chunk > max_steps - done) chunk = max_steps - done;
            a->hctrl->t = a->t;
            a->hctrl->step = a->step;
            a->hctrl->tfinal = tfinal;
            a->hctrl->step_limit = a->step + chunk;
            a->hctrl->active = 1;
            a->hctrl->flags = 0;
            // queued, not awaited: the host writes hctrl again only after the
            // pull below has synchronised the stream
            VB_CUDA(cudaMemcpyAsync(a->ctrl, a->hctrl, sizeof(vb::Ctrl), cudaMemcpyHostToDevice, st));
            VB_CUDA(cudaMemsetAsync(&a->ctrl->invdt_bits, 0, sizeof(unsigned long long), st));
            VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_cfl(a->dev, a->U, -1, a->ctrl, st));
            vb::AmrStageArgs s{};
            s.level = -1;
            s.cfl_all = 1;
            s.dt = -1.0;  // read from the control block
            for (int64_t k = 0; k < chunk; ++k) {
                VB_CHECK_LAUNCH(a->ctx, vb::launch_finalize_cfl(gq, a->ctrl, st));
                VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 1, a->U, a->U, a->U1, a->F, s, a->ctrl, st));
                VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 2, a->U1, a->U, a->U, a->F, s, a->ctrl, st));
                VB_CHECK_LAUNCH(a->ctx, vb::launch_advance(a->ctrl, st));
            }
            rc = pull_ctrl(a);
            if (rc) return rc;
            if (a->hctrl->flags & vb::CTRL_F_NONFINITE)
                return fail(VB_ENONFINITE, "non-finite dt: NaN or negative density/pressure");
            done += a->hctrl->step - a->step;
            a->t = a->hctrl->t;
            a->step = a->hctrl->step;
            if (!a->hctrl->active && a->step < a->hctrl->step_limit) break;  // reached tfinal
        }
    }
    if (t_out) *t_out = a->t;
    if (nsteps) *nsteps = done;
    return VB_OK;
}

int vb_amr_regrid_ms(const vb_amr *a, double *ms)
{
    if (!a || !ms) return fail(VB_EINVAL, "null argument");
    *ms = a->ms_regrid;
    return VB_OK;
}

int vb_amr_conserved_totals(vb_amr *a, double out[5])
{
    VB_RANGE("vb_amr_conserved_totals");
    if (!a || !out) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_totals(a->dev, a->U, a->partials, vb::TOTALS_PARTS,
                                                  a->totals, a->ctx->stream));
    VB_CUDA(cudaMemcpyAsync(a->htot, a->totals, sizeof(double) * 5, cudaMemcpyDeviceToHost,
                            a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    std::memcpy(out, a->htot, sizeof(double) * 5);
    return VB_OK;
}

}  // extern "C"
