// vb_amr_kern.cu -- device kernels of the composite AMR mesh (float64, built
// with -fmad=false: bit-identical to a serial evaluation in the reference's
// order).
//
// The mesh is a table set rebuilt on the host after every regrid:
//   - leaves in depth-first order with their level; per-level widths/volumes
//   - rep[2*axis+side][leaf]: the representative face neighbour (PLM stencil
//     and refinement indicator), -1 at a domain boundary
//   - faces in the reference's emission order (HGBackend.jl:220-276):
//     left leaf, right leaf (-1 = boundary ghost side), axis, area
//   - per-leaf CSR of (face, sign) in emission order, so each leaf sums its
//     flux contributions in exactly the reference's order
// One RK2 stage is two launches: k_amr_faces (one thread per face: PLM face
// states, HLLC) and k_amr_cells (one thread per leaf: ordered flux
// divergence, flux-register capture, stage update, CFL maximum).
#include "vb_amr.h"
#include "vb_physics.cuh"

namespace vb {

namespace {

__device__ __forceinline__ void amr_prim(const AmrDev &m, const double *__restrict__ U, int i,
                                         double W[5])
{
    double u[5] = {1.0, 0.0, 0.0, 0.0, 1.0};
    if (VB_DCHECK(i >= 0 && i < m.nleaf))  // check build only
#pragma unroll
        for (int k = 0; k < 5; ++k) u[k] = U[(int64_t)k * m.cap + i];
    cons2prim(u, m.gamma, W);
}

// _face_value(sim, i, axis, side) with the slope from representatives
__device__ __forceinline__ void amr_face_value(const AmrDev &m, const double *__restrict__ U, int i,
                                               int ax, bool hi, double out[5])
{
    double Wc[5], Wl[5], Wr[5];
    amr_prim(m, U, i, Wc);
    if (!VB_DCHECK(i >= 0 && i < m.nleaf)) i = 0;  // check build only (amr_prim flagged it)
    const int jl = m.rep[(2 * ax) * m.cap + i];
    const int jr = m.rep[(2 * ax + 1) * m.cap + i];
    if (jl >= 0) amr_prim(m, U, jl, Wl); else ghost_state<double>(Wc, m.bc_lo[ax], ax, Wl);
    if (jr >= 0) amr_prim(m, U, jr, Wr); else ghost_state<double>(Wc, m.bc_hi[ax], ax, Wr);
    const double h = hi ? 0.5 : -0.5;
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = face_val(Wc[k], h, limited_slope<double>(Wl[k], Wc[k], Wr[k]));
}

template <int DIM>
__device__ __forceinline__ void amr_face(const AmrDev &m, const double *__restrict__ U, int f,
                                         double *__restrict__ F)
{
    const int L = m.fL[f], R = m.fR[f];
    if (!VB_DCHECK(L < m.nleaf && R < m.nleaf && (L >= 0 || R >= 0))) return;  // check build only
    constexpr int ax = DIM - 1;
    double WL[5], WR[5], out[5];
    if (L >= 0 && R >= 0) {
        amr_face_value(m, U, L, ax, true, WL);
        amr_face_value(m, U, R, ax, false, WR);
    } else if (R < 0) {
        amr_face_value(m, U, L, ax, true, WL);
        ghost_state<double>(WL, m.bc_hi[ax], ax, WR);
    } else {
        amr_face_value(m, U, R, ax, false, WR);
        ghost_state<double>(WR, m.bc_lo[ax], ax, WL);
    }
    hllc_flux<double, DIM>(WL, WR, m.gamma, out);
#pragma unroll
    for (int k = 0; k < 5; ++k) F[(int64_t)k * m.fcap + f] = out[k];
}

__global__ void __launch_bounds__(256) k_amr_faces(AmrDev m, const double *__restrict__ U,
                                                   double *__restrict__ F, const Ctrl *gate)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nface) return;
    if (gate && !gate->active) return;
    switch (m.fax[f]) {
    case 0: amr_face<1>(m, U, f, F); break;
    case 1: amr_face<2>(m, U, f, F); break;
    default: amr_face<3>(m, U, f, F); break;
    }
}

// One stage over the leaves.  `level` < 0 updates every leaf; otherwise only
// that level (step!(sim, dt; level)), and stage 1 copies the other leaves into
// Uout so stage 2 reads one consistent state.  Registers: up to two active
// (coarse level, scale) pairs; a leaf at a register's coarse level adds
// scale*F*area (sign by side) for each face to a leaf one level finer.
template <int STAGE>
__global__ void __launch_bounds__(256)
k_amr_cells(AmrDev m, const double *__restrict__ Uin, const double *U0, double *Uout,
            const double *__restrict__ F, AmrStageArgs a, Ctrl *ctrl)
{
    __shared__ double red[32];
    // a.dt < 0: dt from the control block, and nothing to do once inactive;
    // a.dt_dev: a subcycled level's substep dt
    double dt = a.dt;
    if (a.dt_dev) {
        dt = *a.dt_dev;
    } else if (dt < 0.0) {
        if (!ctrl->active) return;
        dt = ctrl->dt;
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double invdt = 0.0;
    if (i < m.nleaf) {
        const int li = m.lev[i];
        const bool upd = a.level < 0 || li == a.level;
        int rslot = -1;
        for (int r = 0; r < a.nreg; ++r)
            if (a.reg_level[r] == li) rslot = r;
        if (upd || rslot >= 0) {
            double acc[5] = {0, 0, 0, 0, 0}, rg[5];
            const double rs = rslot < 0 ? 0.0
                              : a.dt_dev ? a.reg_scale[rslot] * (0.5 * dt)
                                         : a.reg_scale[rslot];
            if (rslot >= 0)
#pragma unroll
                for (int k = 0; k < 5; ++k) rg[k] = m.reg[(int64_t)k * m.cap + i];
            const int e0 = m.off[i], e1 = m.off[i + 1];
            for (int e = e0; e < e1; ++e) {
                if (!VB_DCHECK(e >= 0 && e < m.nent)) break;  // check build only
                const int code = m.ent[e];
                const int f = code >> 1;
                if (!VB_DCHECK(f >= 0 && f < m.nface)) continue;
                const bool neg = code & 1;
                const double ar = m.farea[f];
                double Fk[5];
#pragma unroll
                for (int k = 0; k < 5; ++k) Fk[k] = F[(int64_t)k * m.fcap + f];
                const double s = neg ? -ar : ar;
#pragma unroll
                for (int k = 0; k < 5; ++k) acc[k] = acc[k] + s * Fk[k];
                if (rslot >= 0) {
                    const int other = neg ? m.fL[f] : m.fR[f];
                    if (other >= 0 && VB_DCHECK(other < m.nleaf) && m.lev[other] == li + 1) {
                        const double ss = neg ? -rs : rs;
#pragma unroll
                        for (int k = 0; k < 5; ++k) rg[k] = rg[k] + ss * Fk[k] * ar;
                    }
                }
            }
            if (rslot >= 0)
#pragma unroll
                for (int k = 0; k < 5; ++k) m.reg[(int64_t)k * m.cap + i] = rg[k];
            if (upd) {
                const double invV = dt / (m.aexp * m.vol[li]);
                double un[5];
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    const int64_t o = (int64_t)k * m.cap + i;
                    if constexpr (STAGE == 1)
                        un[k] = U0[o] - invV * acc[k];
                    else
                        un[k] = 0.5 * U0[o] + 0.5 * (Uin[o] - invV * acc[k]);
                    Uout[o] = un[k];
                }
                if constexpr (STAGE == 2) {
                    double W[5];
                    cons2prim(un, m.gamma, W);
                    const double c = sqrt(m.gamma * W[4] / W[0]);
                    for (int d = 0; d < m.nd; ++d)
                        invdt = nan_max(invdt, (fabs(W[1 + d]) + c) / m.w[li][d]);
                }
            }
        }
        if constexpr (STAGE == 1) {
            if (!upd)
#pragma unroll
                for (int k = 0; k < 5; ++k) Uout[(int64_t)k * m.cap + i] = Uin[(int64_t)k * m.cap + i];
        }
    }
    if constexpr (STAGE == 2)
        if (a.cfl_all) block_max_to(&ctrl->invdt_bits, invdt, red);
}

// compute_dt(sim; level) maximum; level < 0: every leaf
__global__ void __launch_bounds__(256) k_amr_cfl(AmrDev m, const double *__restrict__ U, int level,
                                                 Ctrl *ctrl)
{
    __shared__ double red[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double invdt = 0.0;
    if (i < m.nleaf && (level < 0 || m.lev[i] == level)) {
        double W[5];
        amr_prim(m, U, i, W);
        const double c = sqrt(m.gamma * W[4] / W[0]);
        for (int d = 0; d < m.nd; ++d)
            invdt = nan_max(invdt, (fabs(W[1 + d]) + c) / m.w[m.lev[i]][d]);
    }
    block_max_to(&ctrl->invdt_bits, invdt, red);
}

// the same maximum into a given word
__global__ void __launch_bounds__(256) k_amr_cfl_bits(AmrDev m, const double *__restrict__ U,
                                                      int level, unsigned long long *bits)
{
    __shared__ double red[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double invdt = 0.0;
    if (i < m.nleaf && (level < 0 || m.lev[i] == level)) {
        double W[5];
        amr_prim(m, U, i, W);
        const double c = sqrt(m.gamma * W[4] / W[0]);
        for (int d = 0; d < m.nd; ++d)
            invdt = nan_max(invdt, (fabs(W[1 + d]) + c) / m.w[m.lev[i]][d]);
    }
    block_max_to(bits, invdt, red);
}

// evolve_level!'s head (src/driver.jl:555-560) on the device: dt_stable from
// the level's CFL maximum, n = max(1, ceil(target / dt_stable * (1 - 1e-12)))
// substeps of target / n; no substeps when dt_stable is not finite (a level
// at rest or without leaves).  The maximum word is reset for its next use.
__global__ void k_amr_sub_plan(AmrSubLevel *sub, int level, double cfl, const double *target_src,
                               cudaGraphConditionalHandle h, int *err)
{
    AmrSubLevel &L = sub[level];
    const double target = target_src ? *target_src : L.dt_target;
    L.dt_target = target;
    const double invdt = __longlong_as_double((long long)L.invdt_bits);
    L.invdt_bits = 0ull;
    L.left = 0;
    L.iters = 0;
    if (invdt != invdt || *err) {
        atomicOr(err, invdt != invdt ? AMR_SUB_NONFINITE : 0);
        cudaGraphSetConditional(h, 0);
        return;
    }
    const double dt_stable = invdt == 0.0 ? (double)INFINITY : cfl / invdt;
    if (!(dt_stable < (double)INFINITY)) {
        cudaGraphSetConditional(h, 0);
        return;
    }
    const double q = ceil(target / dt_stable * (1 - 1e-12));
    if (!(q <= (double)AMR_MAX_SUBSTEPS)) {
        atomicOr(err, AMR_SUB_TOO_MANY);
        cudaGraphSetConditional(h, 0);
        return;
    }
    const long long n = q < 1.0 ? 1 : (long long)q;
    L.dt_sub = target / (double)n;
    L.left = n;
    cudaGraphSetConditional(h, 1);
}

// end of one substep of the level's loop: the condition for another
__global__ void k_amr_sub_next(AmrSubLevel *sub, int level, cudaGraphConditionalHandle h, int *err)
{
    AmrSubLevel &L = sub[level];
    L.left -= 1;
    L.iters += 1;
    bool more = L.left > 0 && *err == 0;
    if (L.iters >= AMR_MAX_SUBSTEPS) {
        atomicOr(err, AMR_SUB_TOO_MANY);
        more = false;
    }
    cudaGraphSetConditional(h, more ? 1 : 0);
}

__global__ void k_amr_sub_target(AmrSubLevel *sub, double dt) { sub[0].dt_target = dt; }

// density_gradient_indicator (src/driver.jl:406-420) and the regrid! tag
__global__ void __launch_bounds__(256) k_amr_tag(AmrDev m, const double *__restrict__ U,
                                                 double above, int max_level, uint8_t *tag,
                                                 double *ind, int *ntag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nleaf) return;
    double W[5], Wn[5];
    amr_prim(m, U, i, W);
    const double rc = W[0];
    double g = 0.0;
    for (int s = 0; s < 2 * m.nd; ++s) {
        const int j = m.rep[s * m.cap + i];
        if (j < 0) continue;
        amr_prim(m, U, j, Wn);
        const double rn = Wn[0];
        g = fmax(g, fabs(rn - rc) / fmax(fmax(rc, rn), 2.220446049250313e-16));
    }
    if (ind) ind[i] = g;
    const bool on = m.lev[i] < max_level && g > above;
    tag[i] = on ? 1 : 0;
    if (on && ntag) atomicAdd(ntag, 1);
}

// _reflux_apply! (src/reflux.jl:91-101) for the leaves of one level
__global__ void k_amr_reflux(AmrDev m, double *U, int level)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nleaf || m.lev[i] != level) return;
    const double invV = 1.0 / m.vol[level];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int64_t o = (int64_t)k * m.cap + i;
        U[o] = U[o] - invV * m.reg[o];
        m.reg[o] = 0.0;
    }
}

__global__ void k_amr_zero_reg(AmrDev m, int level)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nleaf || m.lev[i] != level) return;
#pragma unroll
    for (int k = 0; k < 5; ++k) m.reg[(int64_t)k * m.cap + i] = 0.0;
}

// conserved_totals: fixed partition (deterministic), then one folding block
__global__ void __launch_bounds__(256) k_amr_totals_part(AmrDev m, const double *__restrict__ U,
                                                         double *partials)
{
    __shared__ double red[5][8];
    double s[5] = {0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nleaf; i += gridDim.x * blockDim.x) {
        const double v = m.vol[m.lev[i]];
#pragma unroll
        for (int k = 0; k < 5; ++k) s[k] += U[(int64_t)k * m.cap + i] * v;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const double v = warp_sum(s[k]);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += red[threadIdx.x][w];
        partials[blockIdx.x * 5 + threadIdx.x] = v;
    }
}

}  // namespace

static unsigned blocks(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs > 0 ? (n + bs - 1) / bs : 1); }

int launch_amr_stage(const AmrDev &m, int stage, const double *Uin, const double *U0,
                     double *Uout, double *F, const AmrStageArgs &a, Ctrl *ctrl, cudaStream_t s)
{
    if (m.nface > 0)
        k_amr_faces<<<blocks(m.nface, 256), 256, 0, s>>>(m, Uin, F,
                                                         (a.dt < 0.0 && !a.dt_dev) ? ctrl : nullptr);
    if (stage == 1)
        k_amr_cells<1><<<blocks(m.nleaf, 256), 256, 0, s>>>(m, Uin, U0, Uout, F, a, ctrl);
    else
        k_amr_cells<2><<<blocks(m.nleaf, 256), 256, 0, s>>>(m, Uin, U0, Uout, F, a, ctrl);
    return m.nface > 0 ? 2 : 1;
}

int launch_amr_cfl(const AmrDev &m, const double *U, int level, Ctrl *ctrl, cudaStream_t s)
{
    k_amr_cfl<<<blocks(m.nleaf, 256), 256, 0, s>>>(m, U, level, ctrl);
    return 1;
}

int launch_amr_cfl_bits(const AmrDev &m, const double *U, int level, unsigned long long *bits,
                        cudaStream_t s)
{
    k_amr_cfl_bits<<<blocks(m.nleaf, 256), 256, 0, s>>>(m, U, level, bits);
    return 1;
}

int launch_amr_sub_plan(AmrSubLevel *sub, int level, double cfl, const double *target_src,
                        cudaGraphConditionalHandle h, int *err, cudaStream_t s)
{
    k_amr_sub_plan<<<1, 1, 0, s>>>(sub, level, cfl, target_src, h, err);
    return 1;
}

int launch_amr_sub_next(AmrSubLevel *sub, int level, cudaGraphConditionalHandle h, int *err,
                        cudaStream_t s)
{
    k_amr_sub_next<<<1, 1, 0, s>>>(sub, level, h, err);
    return 1;
}

int launch_amr_sub_target(AmrSubLevel *sub, double dt, cudaStream_t s)
{
    k_amr_sub_target<<<1, 1, 0, s>>>(sub, dt);
    return 1;
}

int launch_amr_tag(const AmrDev &m, const double *U, double above, int max_level, uint8_t *tag,
                   double *ind, int *ntag, cudaStream_t s)
{
    k_amr_tag<<<blocks(m.nleaf, 256), 256, 0, s>>>(m, U, above, max_level, tag, ind, ntag);
    return 1;
}

int launch_amr_reflux(const AmrDev &m, double *U, int level, cudaStream_t s)
{
    k_amr_reflux<<<blocks(m.nleaf, 256), 256, 0, s>>>(m, U, level);
    return 1;
}

int launch_amr_zero_reg(const AmrDev &m, int level, cudaStream_t s)
{
    k_amr_zero_reg<<<blocks(m.nleaf, 256), 256, 0, s>>>(m, level);
    return 1;
}

int launch_amr_totals(const AmrDev &m, const double *U, double *partials, int npart, double *out,
                      cudaStream_t s)
{
    k_amr_totals_part<<<npart, 256, 0, s>>>(m, U, partials);
    return 1 + launch_totals_final(partials, npart, out, s);
}

}  // namespace vb
