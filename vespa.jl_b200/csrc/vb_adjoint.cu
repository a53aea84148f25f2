// vb_adjoint.cu -- the extern "C" adjoint API: checkpointed forward runs,
// the reverse sweep with recompute, and the single-step adjoint.
//
// Forward (vb_adjoint_forward): the grid's own CFL-limited stepping path
// (tiled or cell-centric, unchanged), plus a copy of the state at the start
// of every checkpoint segment and the dt of every step, recorded on the
// device.  The adjoint differentiates the map with this dt sequence frozen.
//
// Reverse (vb_adjoint_backward), segment by segment from the last: recompute
// the segment from its checkpoint with the same float64 stage kernels and the
// recorded dts (bit-identical to the forward), keeping the state at the start
// of each step and its stage-1 state; then walk the steps backwards, two
// adjoint stages per step.  With a checkpoint every step the forward run
// also keeps each step's stage-1 state (a tape of 2 states per step in HBM:
// 4.2 GB for 200 steps of a 512^2 grid) and the reverse sweep recomputes
// nothing.  The adjoint stages are:
//   lam1 = 0.5*lam - invV * (dD/dU)^T(U^1) (0.5*lam)
//   lam  = 0.5*lam + lam1 - invV * (dD/dU)^T(U^n) lam1
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "vb_internal.h"

using vb::detail::fail;
using vb::detail::use;

struct vb_adjoint {
    vb_grid *grid = nullptr;   // not touched by vb_adjoint_destroy
    int device = 0;
    int64_t max_steps = 0;
    int64_t every = 0;
    int64_t nseg = 0;
    size_t state_bytes = 0;
    double *ckpt = nullptr;    // nseg states: U at steps 0, every, 2*every, ...
    double *segU = nullptr;    // every states: U^n within the segment being reversed
    double *segU1 = nullptr;   // every states: stage-1 states within that segment
    double *tape1 = nullptr;   // every == 1: the stage-1 state of every step (forward run)
    double *lam = nullptr;     // adjoint state
    double *lam1 = nullptr;    // adjoint of the stage-1 state
    double *gL = nullptr, *gR = nullptr;  // face adjoints, 5*nd*ncell each
    uint16_t *code = nullptr;  // minmod branch codes, nd*ncell
    double *dts = nullptr;     // device: dt of each recorded step
    std::vector<double> hdts;  // host copy of dts[0..nsteps)
    int64_t nsteps = 0;        // steps recorded by the last forward run
    vb::Ctrl *ctrl = nullptr;  // control block of the recompute stages
    cudaEvent_t ev[2] = {};
    double ms[3] = {0, 0, 0};  // forward, recompute, adjoint stages (last runs)
};

namespace {

double *state_at(const vb_adjoint *a, double *base, int64_t k)
{
    return base + (size_t)k * 5 * (size_t)a->grid->g.ncell;
}

void release(vb_adjoint *a)
{
    cudaFree(a->ckpt);
    cudaFree(a->segU);
    cudaFree(a->segU1);
    cudaFree(a->tape1);
    cudaFree(a->lam);
    cudaFree(a->lam1);
    cudaFree(a->gL);
    cudaFree(a->gR);
    cudaFree(a->code);
    cudaFree(a->dts);
    cudaFree(a->ctrl);
    for (auto &e : a->ev)
        if (e) cudaEventDestroy(e);
}

int check_grid(const vb_grid *gr)
{
    if (gr->precision != VB_FP64)
        return fail(VB_ENOTSUP, "the adjoint differentiates the VB_FP64 step; create the grid with VB_FP64");
    for (int a = 0; a < gr->g.nd; ++a)
        if (gr->g.bc_lo[a] != vb::BC_PERIODIC || gr->g.bc_hi[a] != vb::BC_PERIODIC)
            return fail(VB_ENOTSUP, "the adjoint supports periodic boundaries only");
    if (gr->grav) return fail(VB_ENOTSUP, "the adjoint does not differentiate the gravity source");
    return VB_OK;
}

float elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float m = 0.f;
    cudaEventElapsedTime(&m, a, b);
    return m;
}

// Stage 1 (and stage 2 unless `last`) of step n of the recompute.
int recompute_step(vb_adjoint *a, const double *Un, double *U1, double *Unext, double dt)
{
    vb_grid *gr = a->grid;
    cudaStream_t s = gr->ctx->stream;
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_set_dt(gr->g, a->ctrl, dt, s));
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_stage_fp64(gr->g, 1, Un, Un, U1, a->ctrl, nullptr, s));
    if (Unext)
        VB_CHECK_LAUNCH(gr->ctx,
                        vb::launch_stage_fp64(gr->g, 2, U1, Un, Unext, a->ctrl, nullptr, s));
    return VB_OK;
}

// Both adjoint stages of one step: a->lam <- (dU^{n+1}/dU^n)^T a->lam.
int adjoint_step(vb_adjoint *a, const double *Un, const double *U1, double dt)
{
    vb_grid *gr = a->grid;
    cudaStream_t s = gr->ctx->stream;
    const double invV = dt / (gr->g.aexp * gr->g.vol);
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_adj_stage(gr->g, U1, a->lam, nullptr, invV, a->gL, a->gR,
                                                  a->code, a->lam1, s));
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_adj_stage(gr->g, Un, a->lam, a->lam1, invV, a->gL, a->gR,
                                                  a->code, a->lam, s));
    return VB_OK;
}

}  // namespace

extern "C" {

int vb_adjoint_create(vb_grid *gr, int64_t max_steps, int64_t checkpoint_every, vb_adjoint **out)
{
    if (!gr || !out) return fail(VB_EINVAL, "null argument");
    *out = nullptr;
    if (max_steps < 1 || checkpoint_every < 1) return fail(VB_EINVAL, "max_steps and checkpoint_every must be >= 1");
    int rc = check_grid(gr);
    if (rc) return rc;
    rc = use(gr->ctx);
    if (rc) return rc;
    vb_adjoint *a = new (std::nothrow) vb_adjoint;
    if (!a) return fail(VB_ENOMEM, "host allocation failed");
    a->grid = gr;
    a->device = gr->ctx->device;
    a->max_steps = max_steps;
    a->every = checkpoint_every < max_steps ? checkpoint_every : max_steps;
    a->nseg = (max_steps + a->every - 1) / a->every;
    const size_t nc = (size_t)gr->g.ncell, nd = (size_t)gr->g.nd;
    a->state_bytes = 5 * nc * sizeof(double);
    cudaError_t e = cudaSuccess;
    auto get = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    get((void **)&a->ckpt, a->state_bytes * (size_t)a->nseg);
    get((void **)&a->segU, a->state_bytes * (size_t)a->every);
    get((void **)&a->segU1, a->state_bytes * (size_t)a->every);
    if (a->every == 1) get((void **)&a->tape1, a->state_bytes * (size_t)max_steps);
    get((void **)&a->lam, a->state_bytes);
    get((void **)&a->lam1, a->state_bytes);
    get((void **)&a->gL, a->state_bytes * nd);
    get((void **)&a->gR, a->state_bytes * nd);
    get((void **)&a->code, sizeof(uint16_t) * nc * nd);
    get((void **)&a->dts, sizeof(double) * (size_t)max_steps);
    get((void **)&a->ctrl, sizeof(vb::Ctrl));
    if (e == cudaSuccess) e = cudaEventCreate(&a->ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&a->ev[1]);
    if (e == cudaSuccess) e = cudaMemset(a->ctrl, 0, sizeof(vb::Ctrl));
    if (e != cudaSuccess) {
        release(a);
        delete a;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? VB_ENOMEM : VB_ECUDA,
                    std::string("adjoint buffers: ") + cudaGetErrorString(e));
    }
    *out = a;
    return VB_OK;
}

int vb_adjoint_destroy(vb_adjoint *a)
{
    if (!a) return VB_OK;
    // the grid and its context may already be gone: touch neither
    cudaSetDevice(a->device);
    cudaDeviceSynchronize();
    release(a);
    delete a;
    return VB_OK;
}

int vb_adjoint_forward(vb_adjoint *a, double tfinal, int64_t max_steps, double *t, int64_t *nsteps)
{
    VB_RANGE("vb_adjoint_forward");
    if (!a) return fail(VB_EINVAL, "null adjoint");
    vb_grid *gr = a->grid;
    if (max_steps < 0 || max_steps > a->max_steps) max_steps = a->max_steps;
    int rc = check_grid(gr);  // gravity may have been enabled since creation
    if (rc) return rc;
    rc = use(gr->ctx);
    if (rc) return rc;
    cudaStream_t s = gr->ctx->stream;
    rc = vb::detail::grid_pull_ctrl(gr);
    if (rc) return rc;
    const long long step0 = gr->hctrl->step;
    gr->hctrl->tfinal = tfinal;
    gr->hctrl->step_limit = step0 + max_steps;
    gr->hctrl->flags = 0;
    gr->hctrl->active = 1;
    rc = vb::detail::grid_push_ctrl(gr);
    if (rc) return rc;
    a->nsteps = 0;
    VB_CUDA(cudaEventRecord(a->ev[0], s));
    rc = vb::detail::grid_ensure_cfl(gr);
    int status = VB_OK;
    // the host looks at the control block about every 20 steps (steps queued
    // past the end are no-ops: the stage kernels check the active flag)
    const int64_t look = a->every >= 20 ? 1 : (20 + a->every - 1) / a->every;
    for (int64_t seg = 0; seg < a->nseg && rc == VB_OK; ++seg) {
        VB_CUDA(cudaMemcpyAsync(state_at(a, a->ckpt, seg), gr->U, a->state_bytes,
                                cudaMemcpyDeviceToDevice, s));
        for (int64_t i = 0; i < a->every && rc == VB_OK; ++i) {
            VB_CHECK_LAUNCH(gr->ctx, vb::launch_finalize_cfl(gr->g, gr->ctrl, s));
            VB_CHECK_LAUNCH(gr->ctx, vb::launch_record_dt(gr->ctrl, a->dts, step0, a->max_steps, s));
            rc = vb::detail::grid_rk2(gr);
            if (!rc && a->tape1)
                VB_CUDA(cudaMemcpyAsync(state_at(a, a->tape1, seg), gr->U1, a->state_bytes,
                                        cudaMemcpyDeviceToDevice, s));
        }
        if (rc) break;
        if ((seg + 1) % look != 0 && seg + 1 < a->nseg) continue;
        rc = vb::detail::grid_pull_ctrl(gr);
        if (rc) break;
        if (gr->hctrl->flags & vb::CTRL_F_NONFINITE) {
            status = fail(VB_ENONFINITE, "non-finite dt: NaN or negative density/pressure");
            break;
        }
        if (gr->hctrl->flags & vb::CTRL_F_TIMEOUT) {
            status = fail(VB_ETIMEOUT, "a bounded device wait (TMA stage load) gave up");
            break;
        }
        if (!gr->hctrl->active) break;
    }
    VB_CUDA(cudaEventRecord(a->ev[1], s));
    if (rc) return rc;
    rc = vb::detail::grid_pull_ctrl(gr);
    if (rc) return rc;
    a->ms[0] = elapsed(a->ev[0], a->ev[1]);
    const int64_t done = gr->hctrl->step - step0;
    a->nsteps = done;
    a->hdts.assign((size_t)done, 0.0);
    if (done > 0)
        VB_CUDA(cudaMemcpy(a->hdts.data(), a->dts, sizeof(double) * (size_t)done,
                           cudaMemcpyDeviceToHost));
    if (t) *t = gr->hctrl->t;
    if (nsteps) *nsteps = done;
    gr->hctrl->tfinal = INFINITY;
    gr->hctrl->step_limit = LLONG_MAX;
    gr->hctrl->active = 0;
    rc = vb::detail::grid_push_ctrl(gr);
    return status ? status : rc;
}

int vb_adjoint_steps(const vb_adjoint *a, int64_t *nsteps)
{
    if (!a || !nsteps) return fail(VB_EINVAL, "null argument");
    *nsteps = a->nsteps;
    return VB_OK;
}

int vb_adjoint_dts(const vb_adjoint *a, double *dts, int64_t n)
{
    if (!a || (!dts && n > 0)) return fail(VB_EINVAL, "null argument");
    if (n != a->nsteps) return fail(VB_EINVAL, "n must equal the recorded step count");
    if (n > 0) std::memcpy(dts, a->hdts.data(), sizeof(double) * (size_t)n);
    return VB_OK;
}

int vb_adjoint_backward(vb_adjoint *a, const double *lam_final, double *lam_init)
{
    VB_RANGE("vb_adjoint_backward");
    if (!a || !lam_final || !lam_init) return fail(VB_EINVAL, "null argument");
    if (a->nsteps <= 0) return fail(VB_EINVAL, "no recorded forward run (vb_adjoint_forward)");
    vb_grid *gr = a->grid;
    int rc = use(gr->ctx);
    if (rc) return rc;
    cudaStream_t s = gr->ctx->stream;
    VB_CUDA(cudaMemcpyAsync(a->lam, lam_final, a->state_bytes, cudaMemcpyHostToDevice, s));
    double ms_re = 0.0, ms_adj = 0.0;
    if (a->tape1) {  // every step's two states were kept: no recompute
        VB_CUDA(cudaEventRecord(a->ev[0], s));
        for (int64_t i = a->nsteps - 1; i >= 0; --i) {
            rc = adjoint_step(a, state_at(a, a->ckpt, i), state_at(a, a->tape1, i),
                              a->hdts[(size_t)i]);
            if (rc) return rc;
        }
        VB_CUDA(cudaEventRecord(a->ev[1], s));
        VB_CUDA(cudaMemcpyAsync(lam_init, a->lam, a->state_bytes, cudaMemcpyDeviceToHost, s));
        VB_CUDA(cudaStreamSynchronize(s));
        a->ms[1] = 0.0;
        a->ms[2] = elapsed(a->ev[0], a->ev[1]);
        return VB_OK;
    }
    const int64_t nseg = (a->nsteps + a->every - 1) / a->every;
    for (int64_t seg = nseg - 1; seg >= 0; --seg) {
        const int64_t s0 = seg * a->every;
        const int64_t s1 = (s0 + a->every < a->nsteps) ? s0 + a->every : a->nsteps;
        const int64_t m = s1 - s0;
        // recompute: segU[0] aliases the checkpoint
        VB_CUDA(cudaEventRecord(a->ev[0], s));
        for (int64_t i = 0; i < m; ++i) {
            const double *Un = i == 0 ? state_at(a, a->ckpt, seg) : state_at(a, a->segU, i);
            double *Unext = (i + 1 < m) ? state_at(a, a->segU, i + 1) : nullptr;
            rc = recompute_step(a, Un, state_at(a, a->segU1, i), Unext, a->hdts[(size_t)(s0 + i)]);
            if (rc) return rc;
        }
        VB_CUDA(cudaEventRecord(a->ev[1], s));
        VB_CUDA(cudaEventSynchronize(a->ev[1]));
        ms_re += elapsed(a->ev[0], a->ev[1]);
        VB_CUDA(cudaEventRecord(a->ev[0], s));
        for (int64_t i = m - 1; i >= 0; --i) {
            const double *Un = i == 0 ? state_at(a, a->ckpt, seg) : state_at(a, a->segU, i);
            rc = adjoint_step(a, Un, state_at(a, a->segU1, i), a->hdts[(size_t)(s0 + i)]);
            if (rc) return rc;
        }
        VB_CUDA(cudaEventRecord(a->ev[1], s));
        VB_CUDA(cudaEventSynchronize(a->ev[1]));
        ms_adj += elapsed(a->ev[0], a->ev[1]);
    }
    VB_CUDA(cudaMemcpyAsync(lam_init, a->lam, a->state_bytes, cudaMemcpyDeviceToHost, s));
    VB_CUDA(cudaStreamSynchronize(s));
    a->ms[1] = ms_re;
    a->ms[2] = ms_adj;
    return VB_OK;
}

int vb_adjoint_step(vb_adjoint *a, double dt, const double *lam_out, double *lam_in)
{
    VB_RANGE("vb_adjoint_step");
    if (!a || !lam_out || !lam_in) return fail(VB_EINVAL, "null argument");
    if (!std::isfinite(dt)) return fail(VB_EINVAL, "dt must be finite");
    vb_grid *gr = a->grid;
    int rc = use(gr->ctx);
    if (rc) return rc;
    cudaStream_t s = gr->ctx->stream;
    VB_CUDA(cudaMemcpyAsync(a->lam, lam_out, a->state_bytes, cudaMemcpyHostToDevice, s));
    double *U1 = state_at(a, a->segU1, 0);
    rc = recompute_step(a, gr->U, U1, nullptr, dt);
    if (rc) return rc;
    rc = adjoint_step(a, gr->U, U1, dt);
    if (rc) return rc;
    VB_CUDA(cudaMemcpyAsync(lam_in, a->lam, a->state_bytes, cudaMemcpyDeviceToHost, s));
    VB_CUDA(cudaStreamSynchronize(s));
    return VB_OK;
}

int vb_adjoint_timing(const vb_adjoint *a, double ms[3])
{
    if (!a || !ms) return fail(VB_EINVAL, "null argument");
    for (int k = 0; k < 3; ++k) ms[k] = a->ms[k];
    return VB_OK;
}

}  // extern "C"
