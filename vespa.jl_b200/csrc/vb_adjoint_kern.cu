// vb_adjoint_kern.cu -- adjoint (reverse-mode) kernels of one SSP-RK2 stage
// on a periodic uniform mesh, float64, built with -fmad=false so the
// recomputed forward quantities (and hence every frozen branch) are the
// forward step's own bits.
//
// A stage is Uout = base - invV * D(U) with D(U)_i = sum over the faces of
// cell i of +-area * F(WL, WR) (src/driver.jl:236-281, 297-321).  Its
// transpose applied to an adjoint mu is, face by face,
//   Fb = area * (mu_L - mu_R)  ->  HLLC reverse  ->  WLb, WRb
// then through the PLM face values WL = W_i + s_i/2, WR = W_{i+1} - s_{i+1}/2
// (src/driver.jl:227-233) and minmod slopes into the cell primitives, and
// through cons2prim into the conserved adjoint.
//
// Two passes, no atomics (the result does not depend on scheduling):
//   k_adj_face: one thread per (cell i, axis): face i+1/2 of that axis; writes
//     WLb, WRb of the face and the minmod branch codes of s_i.
//   k_adj_cell: one thread per cell: gathers the face adjoints that depend on
//     its primitives, applies the cons2prim reverse and the RK2 combination.
#include "vb_adjoint.cuh"
#include "vb_launch.h"
#include "vb_stage_generic.cuh"

namespace vb {

namespace {

// the cell `off` cells away along ax (periodic); the modulo only at the wrap
__device__ __forceinline__ int64_t wrap_lin(const Geom &g, int ax, int64_t lin, int64_t c, int off)
{
    const int64_t n = g.n[ax];
    int64_t j = c + off;
    if (j < 0 || j >= n) {
        j %= n;
        if (j < 0) j += n;
    }
    return lin + (j - c) * g.stride[ax];
}

__device__ __forceinline__ int64_t coord(const Geom &g, int ax, int64_t lin)
{
    int64_t cc[3];
    cell_coords(g, lin, cc);
    return cc[ax];
}

template <int AX>
__device__ __forceinline__ void adj_face_axis(const Geom &g, const double *__restrict__ U,
                                              const double *__restrict__ M, double ms, int64_t lin,
                                              double *__restrict__ gL, double *__restrict__ gR,
                                              uint16_t *__restrict__ code)
{
    const int64_t nc = g.ncell;
    const int64_t c = coord(g, AX, lin);
    const int64_t lm1 = wrap_lin(g, AX, lin, c, -1);
    const int64_t lp1 = wrap_lin(g, AX, lin, c, 1);
    const int64_t lp2 = wrap_lin(g, AX, lin, c, 2);
    double Wm1[5], W0[5], Wp1[5], Wp2[5];
    load_prim<double>(g, U, lm1, Wm1);
    load_prim<double>(g, U, lin, W0);
    load_prim<double>(g, U, lp1, Wp1);
    load_prim<double>(g, U, lp2, Wp2);
    double WL[5], WR[5], Fb[5];
    unsigned cd = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const double a0 = W0[k] - Wm1[k], b0 = Wp1[k] - W0[k];
        cd |= minmod_code(a0, b0) << (2 * k);
        WL[k] = face_val(W0[k], 0.5, minmod<double>(a0, b0));
        WR[k] = face_val(Wp1[k], -0.5, limited_slope<double>(W0[k], Wp1[k], Wp2[k]));
        Fb[k] = g.area[AX] * (ms * __ldg(M + k * nc + lin) - ms * __ldg(M + k * nc + lp1));
    }
    double WLb[5] = {0, 0, 0, 0, 0}, WRb[5] = {0, 0, 0, 0, 0};
    hllc_vjp<AX + 1>(WL, WR, g.gamma, Fb, WLb, WRb);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        gL[(AX * 5 + k) * nc + lin] = WLb[k];
        gR[(AX * 5 + k) * nc + lin] = WRb[k];
    }
    code[AX * nc + lin] = (uint16_t)cd;
}

template <int ND>
__global__ void __launch_bounds__(128)
k_adj_face(Geom g, const double *__restrict__ U, const double *__restrict__ M, double ms,
           double *__restrict__ gL, double *__restrict__ gR, uint16_t *__restrict__ code)
{
    const int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lin >= g.ncell) return;
    const int ax = blockIdx.y;
    if (ax == 0) adj_face_axis<0>(g, U, M, ms, lin, gL, gR, code);
    if constexpr (ND > 1) if (ax == 1) adj_face_axis<1>(g, U, M, ms, lin, gL, gR, code);
    if constexpr (ND > 2) if (ax == 2) adj_face_axis<2>(g, U, M, ms, lin, gL, gR, code);
}

// out = 0.5*lam + (M ? M : 0) - invV * (dD/dU)^T mu   (per cell)
template <int ND>
__global__ void __launch_bounds__(256)
k_adj_cell(Geom g, const double *__restrict__ U, const double *__restrict__ gL,
           const double *__restrict__ gR, const uint16_t *__restrict__ code,
           const double *lam, const double *M, double invV, double *out)
{
    const int64_t nc = g.ncell;
    const int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lin >= nc) return;
    double Wb[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int ax = 0; ax < ND; ++ax) {
        const int64_t c = coord(g, ax, lin);
        const int64_t km1 = wrap_lin(g, ax, lin, c, -1);
        const int64_t km2 = wrap_lin(g, ax, lin, c, -2);
        const int64_t kp1 = wrap_lin(g, ax, lin, c, 1);
        const unsigned ck = code[ax * nc + lin];
        const unsigned cp = code[ax * nc + kp1];
        const unsigned cm = code[ax * nc + km1];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const int64_t o = (int64_t)(ax * 5 + k) * nc;
            const double fl = gL[o + lin], fr = gR[o + km1];
            // own value in both faces' states
            double w = fl + fr;
            // own slope s_k (hi face +1/2, lo face -1/2)
            const double sb = 0.5 * fl - 0.5 * fr;
            const unsigned bk = (ck >> (2 * k)) & 3u;
            if (bk == 1u) w += sb;
            else if (bk == 2u) w -= sb;
            // s_{k+1} = W_{k+1} - W_k when its branch is the left difference
            if (((cp >> (2 * k)) & 3u) == 1u) w -= 0.5 * gL[o + kp1] - 0.5 * gR[o + lin];
            // s_{k-1} = W_k - W_{k-1} when its branch is the right difference
            if (((cm >> (2 * k)) & 3u) == 2u) w += 0.5 * gL[o + km1] - 0.5 * gR[o + km2];
            Wb[k] += w;
        }
    }
    double u[5], Ub[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) u[k] = __ldg(U + k * nc + lin);
    cons2prim_vjp(u, g.gamma, Wb, Ub);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int64_t i = k * nc + lin;
        double v = 0.5 * lam[i];
        if (M) v = v + M[i];
        out[i] = v - invV * Ub[k];
    }
}

__global__ void k_record_dt(const Ctrl *ctrl, double *dts, long long step0, long long cap)
{
    if (!ctrl->active) return;
    const long long i = ctrl->step - step0;
    if (i >= 0 && i < cap) dts[i] = ctrl->dt;
}

}  // namespace

int launch_adj_stage(const Geom &g, const double *U, const double *lam, const double *M,
                     double invV, double *gL, double *gR, uint16_t *code, double *out,
                     cudaStream_t s)
{
    const int64_t nb_f = (g.ncell + 127) / 128;
    if (g.ncell <= 0 || nb_f > 0x7fffffffLL) return -1;
    // mu = 0.5*lam (adjoint of stage 2) or M (adjoint of stage 1)
    const double *mu = M ? M : lam;
    const double ms = M ? 1.0 : 0.5;
    const dim3 gf((unsigned)nb_f, (unsigned)g.nd);
    const unsigned gc = (unsigned)((g.ncell + 255) / 256);
    switch (g.nd) {
    case 1:
        k_adj_face<1><<<gf, 128, 0, s>>>(g, U, mu, ms, gL, gR, code);
        k_adj_cell<1><<<gc, 256, 0, s>>>(g, U, gL, gR, code, lam, M, invV, out);
        break;
    case 2:
        k_adj_face<2><<<gf, 128, 0, s>>>(g, U, mu, ms, gL, gR, code);
        k_adj_cell<2><<<gc, 256, 0, s>>>(g, U, gL, gR, code, lam, M, invV, out);
        break;
    case 3:
        k_adj_face<3><<<gf, 128, 0, s>>>(g, U, mu, ms, gL, gR, code);
        k_adj_cell<3><<<gc, 256, 0, s>>>(g, U, gL, gR, code, lam, M, invV, out);
        break;
    default: return -1;
    }
    return 2;
}

int launch_record_dt(const Ctrl *ctrl, double *dts, int64_t step0, int64_t cap, cudaStream_t s)
{
    k_record_dt<<<1, 1, 0, s>>>(ctrl, dts, (long long)step0, (long long)cap);
    return 1;
}

}  // namespace vb
