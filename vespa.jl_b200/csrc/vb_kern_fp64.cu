// vb_kern_fp64.cu -- float64 kernels of libvespa_b200, compiled with
// -fmad=false so every product and sum is rounded separately, in the
// reference's order (bit-identical to a serial float64 evaluation).
//
//   - RK2 stage kernels (VB_FP64 precision)
//   - CFL reduction, dt finalisation and set-dt kernels
//   - deterministic conserved-totals reduction
//   - batched HLLC face kernel (the compute_face_fluxes! drop-in)
#include "vb_launch.h"
#include "vb_stage_generic.cuh"
#include "vb_stage_tiled3d.cuh"
#include "vb_stage_tiled3d_f64.cuh"
#include "vb_stage_tiled2d.cuh"

namespace vb {

namespace {

template <int ND, int STAGE>
int launch_generic(const Geom &g, const double *Uin, const double *U0, double *Uout, Ctrl *ctrl,
                   double *bflux, double *bflux_int, cudaStream_t s)
{
    const int bs = 256;
    const int64_t nb = (g.ncell + bs - 1) / bs;
    if (nb <= 0 || nb > 0x7fffffffLL) return -1;
    k_stage_generic<double, ND, STAGE><<<(unsigned)nb, bs, 0, s>>>(g, Uin, U0, Uout, ctrl, bflux,
                                                                   bflux_int);
    return 1;
}

// compute_dt's per-cell term folded into the running max, src/driver.jl:169-199
__global__ void __launch_bounds__(256) k_cfl(Geom g, const double *__restrict__ U, Ctrl *ctrl)
{
    __shared__ double red[32];
    double m = 0.0;
    for (int64_t lin = g.act0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; lin < g.act1;
         lin += (int64_t)gridDim.x * blockDim.x) {
        double u[5], W[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) u[k] = __ldg(U + k * g.ncell + lin);
        cons2prim(u, g.gamma, W);
        const double c = sound_speed(W, g.gamma);
        for (int d = 0; d < g.nd; ++d) m = nan_max(m, (fabs(W[1 + d]) + c) / g.w[d]);
        if (g.grav_g) m = nan_max(m, gravity_invdt(g.grav_G, W[0]));
    }
    block_max_to(&ctrl->invdt_bits, m, red);
}

__global__ void k_reset_cfl(Ctrl *ctrl) { ctrl->invdt_bits = 0ull; }

// evolve!'s loop head, src/driver.jl:493-499: stop once t >= tfinal*(1-1e-12)
// (or the step budget is spent); else dt = min(cfl/invdt, tfinal - t).
__global__ void k_finalize_cfl(Geom g, Ctrl *ctrl)
{
    const double t = ctrl->t;
    if (!(t < ctrl->tfinal * (1.0 - 1e-12)) || ctrl->step >= ctrl->step_limit) {
        ctrl->active = 0;
        return;
    }
    const double invdt = __longlong_as_double((long long)ctrl->invdt_bits);
    double dt = (invdt == 0.0) ? (double)INFINITY : g.cfl / invdt;
    dt = fmin(dt, ctrl->tfinal - t);
    if (invdt != invdt || !(dt < (double)INFINITY)) {
        ctrl->flags |= CTRL_F_NONFINITE;
        ctrl->active = 0;
        return;
    }
    ctrl->dt = dt;
    ctrl->invV = dt / (g.aexp * g.vol);
    ctrl->active = 1;
    ctrl->invdt_bits = 0ull;
    ctrl->work[0] = ctrl->work[1] = 0u;
}

// step!(sim, dt) with a caller-chosen dt.
__global__ void k_set_dt(Geom g, Ctrl *ctrl, double dt)
{
    ctrl->dt = dt;
    ctrl->invV = dt / (g.aexp * g.vol);
    ctrl->active = 1;
    ctrl->invdt_bits = 0ull;
    ctrl->work[0] = ctrl->work[1] = 0u;
}

// conserved_totals (src/diagnostics.jl:16-31): fixed grid of TOTALS_PARTS
// blocks, each summing a fixed strided subset, then one block folding the
// partials in index order.  The order is fixed, so the result is identical
// from run to run (it differs from the serial sum by rounding only).
__global__ void __launch_bounds__(256) k_totals_part(Geom g, const double *__restrict__ U,
                                                     double *partials)
{
    __shared__ double red[5][8];
    double s[5] = {0, 0, 0, 0, 0};
    for (int64_t lin = g.act0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; lin < g.act1;
         lin += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 5; ++k) s[k] += __ldg(U + k * g.ncell + lin) * g.vol;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double v = warp_sum(s[k]);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += red[threadIdx.x][w];
        partials[blockIdx.x * 5 + threadIdx.x] = v;
    }
}

__global__ void k_totals_final(const double *partials, int npart, double *out)
{
    __shared__ double red[5][32];
    const int lane = threadIdx.x;  // 32 threads
    double s[5] = {0, 0, 0, 0, 0};
    for (int p = lane; p < npart; p += 32)
        for (int k = 0; k < 5; ++k) s[k] += partials[p * 5 + k];
    for (int k = 0; k < 5; ++k) red[k][lane] = s[k];
    __syncwarp();
    if (lane < 5) {
        double v = 0.0;
        for (int i = 0; i < 32; ++i) v += red[lane][i];
        out[lane] = v;
    }
}

// compute_face_fluxes! batch: one thread per face (ext/VespaKAFluxExt.jl:23-35)
__global__ void __launch_bounds__(256) k_hllc_faces(int64_t nf, const double *__restrict__ WL,
                                                    const double *__restrict__ WR,
                                                    const int32_t *__restrict__ axis,
                                                    double gamma, double *__restrict__ F)
{
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < nf;
         f += (int64_t)gridDim.x * blockDim.x) {
        double wl[5], wr[5], fl[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            wl[k] = __ldg(WL + 5 * f + k);
            wr[k] = __ldg(WR + 5 * f + k);
        }
        hllc_flux_axis<double>(wl, wr, gamma, __ldg(axis + f), fl);
#pragma unroll
        for (int k = 0; k < 5; ++k) F[5 * f + k] = fl[k];
    }
}

}  // namespace

int launch_stage_fp64(const Geom &g, int stage, const double *Uin, const double *U0,
                      double *Uout, Ctrl *ctrl, double *bflux, cudaStream_t s, double *bflux_int)
{
    switch (g.nd * 10 + stage) {
    case 11: return launch_generic<1, 1>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 12: return launch_generic<1, 2>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 21: return launch_generic<2, 1>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 22: return launch_generic<2, 2>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 31: return launch_generic<3, 1>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 32: return launch_generic<3, 2>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    default: return -1;
    }
}

int launch_stage_tiled2d_fp64(const BoxDesc *hbox, int nitems, unsigned int *work, int stage,
                              cudaStream_t s, bool bf)
{
    return launch_tiled2d<false, 2>(hbox, nitems, work, stage, s, bf);
}

int launch_stage_tiled3d_fp64(const BoxDesc *hbox, const BoxDesc *boxes, const int *item_box,
                              int nitems, unsigned int *work, int stage, cudaStream_t s, bool grav,
                              bool bf)
{
    return launch_tiled3d_f64<2>(hbox, boxes, item_box, nitems, work, stage, s, grav, bf);
}

namespace {

// evolve!'s loop head for every box of a table (one thread per box); thread 0
// of block 0 also rewinds the shared work cursors.
__global__ void k_finalize_boxes(const BoxDesc *boxes, int nbox, unsigned int *work)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b == 0) work[0] = work[1] = 0u;
    if (b >= nbox) return;
    const Geom &g = boxes[b].g;
    Ctrl *ctrl = boxes[b].ctrl;
    const double t = ctrl->t;
    if (!(t < ctrl->tfinal * (1.0 - 1e-12)) || ctrl->step >= ctrl->step_limit) {
        ctrl->active = 0;
        return;
    }
    const double invdt = __longlong_as_double((long long)ctrl->invdt_bits);
    double dt = (invdt == 0.0) ? (double)INFINITY : g.cfl / invdt;
    dt = fmin(dt, ctrl->tfinal - t);
    if (invdt != invdt || !(dt < (double)INFINITY)) {
        ctrl->flags |= CTRL_F_NONFINITE;
        ctrl->active = 0;
        return;
    }
    ctrl->dt = dt;
    ctrl->invV = dt / (g.aexp * g.vol);
    ctrl->active = 1;
    ctrl->invdt_bits = 0ull;
    ctrl->work[0] = ctrl->work[1] = 0u;
}

// step!'s clock advance (src/driver.jl:353-356) after stage 2.
__global__ void k_advance_boxes(const BoxDesc *boxes, int nbox)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    Ctrl *ctrl = boxes[b].ctrl;
    if (ctrl->active) {
        ctrl->t = ctrl->t + ctrl->dt;
        ctrl->step = ctrl->step + 1;
    }
}

__global__ void k_advance(Ctrl *ctrl)
{
    if (ctrl->active) {
        ctrl->t = ctrl->t + ctrl->dt;
        ctrl->step = ctrl->step + 1;
    }
}

// The running CFL maximum of a slab <-> a device word the ranks all-reduce
// (max over int64: non-negative doubles order like their bit patterns; a NaN
// with the sign bit set is stored as the positive quiet NaN, so that it still
// wins the max).
__global__ void k_cfl_bits(Ctrl *ctrl, unsigned long long *dev, int put)
{
    if (put) {
        ctrl->invdt_bits = *dev;
    } else {
        const unsigned long long b = ctrl->invdt_bits;
        *dev = (b >> 63) ? 0x7FF8000000000000ull : b;
    }
}

// Failure-path self-test: the tiled kernels' bounded stage wait on an
// mbarrier that nothing will ever complete (no copy is issued, so nothing is
// in flight), then the same block-uniform decision and abandon path as a
// stage kernel whose TMA load never arrived.  Touches no state.
__global__ void k_wait_selftest(Ctrl *ctrl, uint64_t limit_ns)
{
    __shared__ uint64_t bar;
    __shared__ int stall_sh;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        stall_sh = 0;
    }
    __syncthreads();
    if (!mbar_wait(&bar, 0, limit_ns)) stall_sh = 1;  // phase 0 never completes
    __syncthreads();
    if (stall_sh) stage_abandon<1>(&bar, 0, 0, 0, ctrl);  // no stage planes in flight
}

}  // namespace

int launch_cfl_bits(Ctrl *ctrl, unsigned long long *dev, int put, cudaStream_t s)
{
    if (!ctrl || !dev) return -1;
    k_cfl_bits<<<1, 1, 0, s>>>(ctrl, dev, put);
    return 1;
}

int launch_wait_selftest(Ctrl *ctrl, uint64_t limit_ns, cudaStream_t s)
{
    if (!ctrl || limit_ns == 0) return -1;
    k_wait_selftest<<<1, 64, 0, s>>>(ctrl, limit_ns);
    return 1;
}

int launch_finalize_boxes(const BoxDesc *boxes, int nbox, unsigned int *work, cudaStream_t s)
{
    if (nbox <= 0) return -1;
    k_finalize_boxes<<<(nbox + 127) / 128, 128, 0, s>>>(boxes, nbox, work);
    return 1;
}

int launch_advance_boxes(const BoxDesc *boxes, int nbox, cudaStream_t s)
{
    if (nbox <= 0) return -1;
    k_advance_boxes<<<(nbox + 127) / 128, 128, 0, s>>>(boxes, nbox);
    return 1;
}

int launch_advance(Ctrl *ctrl, cudaStream_t s)
{
    k_advance<<<1, 1, 0, s>>>(ctrl);
    return 1;
}

static unsigned grid_for(int64_t n, int bs, int maxb)
{
    int64_t nb = (n + bs - 1) / bs;
    if (nb < 1) nb = 1;
    if (nb > maxb) nb = maxb;
    return (unsigned)nb;
}

int launch_cfl(const Geom &g, const double *U, Ctrl *ctrl, cudaStream_t s)
{
    k_reset_cfl<<<1, 1, 0, s>>>(ctrl);
    k_cfl<<<grid_for(g.ncell, 256, 148 * 16), 256, 0, s>>>(g, U, ctrl);
    return 2;
}

int launch_finalize_cfl(const Geom &g, Ctrl *ctrl, cudaStream_t s)
{
    k_finalize_cfl<<<1, 1, 0, s>>>(g, ctrl);
    return 1;
}

int launch_set_dt(const Geom &g, Ctrl *ctrl, double dt, cudaStream_t s)
{
    k_set_dt<<<1, 1, 0, s>>>(g, ctrl, dt);
    return 1;
}

int launch_totals(const Geom &g, const double *U, double *partials, int npart, double *out,
                  cudaStream_t s)
{
    k_totals_part<<<npart, 256, 0, s>>>(g, U, partials);
    k_totals_final<<<1, 32, 0, s>>>(partials, npart, out);
    return 2;
}

int launch_totals_final(const double *partials, int npart, double *out, cudaStream_t s)
{
    k_totals_final<<<1, 32, 0, s>>>(partials, npart, out);
    return 1;
}

int launch_hllc_faces(int64_t nf, const double *WL, const double *WR, const int32_t *axis,
                      double gamma, double *F, cudaStream_t s)
{
    if (nf <= 0) return 0;
    k_hllc_faces<<<grid_for(nf, 256, 148 * 32), 256, 0, s>>>(nf, WL, WR, axis, gamma, F);
    return 1;
}

}  // namespace vb
