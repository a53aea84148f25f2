// vb_stage_generic.cuh -- cell-centric fused RK2 stage kernel for uniform
// meshes of rank 1-3 with any mix of Outflow / Periodic / Reflecting sides.
//
// One thread owns one cell.  It evaluates cons2prim on its star stencil
// (+-2 cells per axis), the minmod slopes of itself and its two neighbours per
// axis, the HLLC flux of both of its faces per axis, and sums the flux
// divergence in exactly the order the reference's face enumeration
// (lib/RefMesh/src/RefMesh.jl:187-197 driving src/driver.jl:236-281) adds
// contributions into that cell.  The stage epilogue (_euler_apply!,
// src/driver.jl:297-307, or _rk2_combine!, 310-321) follows, and stage 2 folds
// the next step's CFL maximum (compute_dt, 169-199) over the new state.
//
// This kernel evaluates every interior face twice (once per adjacent cell).
// It is the general path: the tiled kernels in vb_stage_tiled.cuh take the
// common large periodic / outflow cases.
#pragma once

#include "vb_physics.cuh"

namespace vb {

// Order class of a cell's lo-face contribution relative to its own faces.
// The reference enumerates cells in column-major order and emits every
// interior face from its lower cell's hi query; a lo-side domain-boundary face
// is emitted by the cell itself right after its hi face on the same axis.
//   LO_BEFORE: emitted by the lower neighbour (linear index < this cell)
//   LO_SELF:   emitted by this cell (domain boundary, or a 1-cell periodic axis)
//   LO_AFTER:  emitted by a periodic partner on the far edge (index > this cell)
enum { LO_BEFORE = 0, LO_SELF = 1, LO_AFTER = 2 };

// Neighbour across the (AX, side) face: linear index, or -1 at a domain
// boundary (lib/RefMesh/src/RefMesh.jl:147-161, periodic wraps).
__device__ __forceinline__ int64_t nb_lin(const Geom &g, int64_t lin, int64_t c, int ax, bool hi)
{
    const int64_t n = g.n[ax];
    const int64_t j = hi ? c + 1 : c - 1;
    if (j >= 0 && j < n) return hi ? lin + g.stride[ax] : lin - g.stride[ax];
    const int bc = hi ? g.bc_hi[ax] : g.bc_lo[ax];
    if (bc == BC_PERIODIC) return lin + ((j < 0 ? n - 1 : 0) - c) * g.stride[ax];
    return -1;
}

// _W(sim, cell) (src/driver.jl:137): cons2prim in float64, then rounded to T.
template <typename T>
__device__ __forceinline__ void load_prim(const Geom &g, const double *__restrict__ U, int64_t lin,
                                          T W[5])
{
    double u[5] = {1.0, 0.0, 0.0, 0.0, 1.0}, w[5];
    if (VB_DCHECK(lin >= 0 && lin < g.ncell))
#pragma unroll
        for (int k = 0; k < 5; ++k) u[k] = __ldg(U + k * g.ncell + lin);
    cons2prim(u, g.gamma, w);
#pragma unroll
    for (int k = 0; k < 5; ++k) W[k] = T(w[k]);
}

template <typename T>
struct AxisFlux {
    T hi[5];    // flux through the cell's hi face (+axis normal leaves the cell)
    T lo[5];    // flux through the cell's lo face (+axis normal enters the cell)
    int cat;    // LO_* order class of the lo contribution
    bool hi_bnd, lo_bnd;
};

// Both face fluxes of cell `lin` (coordinate c on axis AX); Wc is its primitive.
template <typename T, int AX>
__device__ __forceinline__ void axis_faces(const Geom &g, const double *__restrict__ U, int64_t lin,
                                           int64_t c, const T Wc[5], AxisFlux<T> &out)
{
    const int64_t n = g.n[AX];
    const int64_t nlo = nb_lin(g, lin, c, AX, false);
    const int64_t nhi = nb_lin(g, lin, c, AX, true);
    T Wlo[5], Whi[5];
    if (nlo >= 0) load_prim<T>(g, U, nlo, Wlo); else ghost_state<T>(Wc, g.bc_lo[AX], AX, Wlo);
    if (nhi >= 0) load_prim<T>(g, U, nhi, Whi); else ghost_state<T>(Wc, g.bc_hi[AX], AX, Whi);

    // _face_value(cell, axis, :hi/:lo), src/driver.jl:227-233
    T fhi[5], flo[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const T s = limited_slope<T>(Wlo[k], Wc[k], Whi[k]);
        fhi[k] = face_val(Wc[k], T(0.5), s);
        flo[k] = face_val(Wc[k], T(-0.5), s);
    }

    // hi face: (cell, hi neighbour) or the hi domain boundary
    if (nhi >= 0) {
        const int64_t chi = (c + 1 < n) ? c + 1 : 0;
        const int64_t nhi2 = nb_lin(g, nhi, chi, AX, true);
        T Whi2[5];
        if (nhi2 >= 0) load_prim<T>(g, U, nhi2, Whi2); else ghost_state<T>(Whi, g.bc_hi[AX], AX, Whi2);
        T WR[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) WR[k] = face_val(Whi[k], T(-0.5), limited_slope<T>(Wc[k], Whi[k], Whi2[k]));
        hllc_face<T, AX + 1>(fhi, WR, g.gamma, out.hi);
        out.hi_bnd = false;
    } else {
        T Wg[5];
        ghost_state<T>(fhi, g.bc_hi[AX], AX, Wg);
        hllc_face<T, AX + 1>(fhi, Wg, g.gamma, out.hi);
        out.hi_bnd = true;
    }

    // lo face: (lo neighbour, cell) or the lo domain boundary
    if (nlo >= 0) {
        const int64_t clo = (c > 0) ? c - 1 : n - 1;
        const int64_t nlo2 = nb_lin(g, nlo, clo, AX, false);
        T Wlo2[5];
        if (nlo2 >= 0) load_prim<T>(g, U, nlo2, Wlo2); else ghost_state<T>(Wlo, g.bc_lo[AX], AX, Wlo2);
        T WL[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) WL[k] = face_val(Wlo[k], T(0.5), limited_slope<T>(Wlo2[k], Wlo[k], Wc[k]));
        hllc_face<T, AX + 1>(WL, flo, g.gamma, out.lo);
        out.cat = nlo < lin ? LO_BEFORE : (nlo == lin ? LO_SELF : LO_AFTER);
        out.lo_bnd = false;
    } else {
        T Wg[5];
        ghost_state<T>(flo, g.bc_lo[AX], AX, Wg);
        hllc_face<T, AX + 1>(Wg, flo, g.gamma, out.lo);
        out.cat = LO_SELF;
        out.lo_bnd = true;
    }
}

// Offset of the bflux plane entry for (axis, side) of cell `lin`.
__device__ __forceinline__ int64_t bflux_offset(const Geom &g, int ax, int side, const int64_t *cc)
{
    int64_t off = 0;
    for (int e = 0; e < ax; ++e) off += 2 * 5 * (g.ncell / g.n[e]);
    off += (int64_t)side * 5 * (g.ncell / g.n[ax]);
    int64_t idx = 0, mul = 1;
    for (int e = 0; e < g.nd; ++e) {
        if (e == ax) continue;
        idx += cc[e] * mul;
        mul *= g.n[e];
    }
    return off + idx;
}

// One SSP-RK2 stage.  STAGE 1: Uout = U0 - invV*acc(Uin), with U0 == Uin.
// STAGE 2: Uout = 0.5*U0 + 0.5*(Uin - invV*acc(Uin)); Uout may alias U0.
template <typename T, int ND, int STAGE>
__global__ void __launch_bounds__(256)
k_stage_generic(Geom g, const double *__restrict__ Uin, const double *U0, double *Uout,
                Ctrl *ctrl, double *bflux, double *bflux_int)
{
    __shared__ double red[32];
    if (!ctrl->active) return;
    const int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double invdt = 0.0;
    if (lin < g.ncell) {
        int64_t cc[3];
        cell_coords(g, lin, cc);
        T Wc[5];
        load_prim<T>(g, Uin, lin, Wc);
        AxisFlux<T> af[ND];
        axis_faces<T, 0>(g, Uin, lin, cc[0], Wc, af[0]);
        if constexpr (ND > 1) axis_faces<T, 1>(g, Uin, lin, cc[1], Wc, af[1]);
        if constexpr (ND > 2) axis_faces<T, 2>(g, Uin, lin, cc[2], Wc, af[2]);

        // flux divergence in the reference's per-cell accumulation order
        double acc[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            double a = 0.0;
#pragma unroll
            for (int d = ND - 1; d >= 0; --d)
                if (af[d].cat == LO_BEFORE) a += (-g.area[d]) * double(af[d].lo[k]);
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                a += g.area[d] * double(af[d].hi[k]);
                if (af[d].cat == LO_SELF) a += (-g.area[d]) * double(af[d].lo[k]);
            }
#pragma unroll
            for (int d = 0; d < ND; ++d)
                if (af[d].cat == LO_AFTER) a += (-g.area[d]) * double(af[d].lo[k]);
            acc[k] = a;
        }
        if (g.grav_g) {  // gravity source from the stage state, after the fluxes
            double u[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) u[k] = Uin[k * g.ncell + lin];
            gravity_source<ND>(g, lin, u, acc);
        }

        const double invV = ctrl->invV;
        double un[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const int64_t i = k * g.ncell + lin;
            if constexpr (STAGE == 1) {
                un[k] = U0[i] - invV * acc[k];
            } else {
                un[k] = 0.5 * U0[i] + 0.5 * (Uin[i] - invV * acc[k]);
            }
            Uout[i] = un[k];
        }

        // interior faces (src/reflux.jl:138-146, _flux_face! src/driver.jl:251):
        // the cell's hi face on each axis when the hi neighbour is a cell
        // (periodic wrap included), keyed by this lo cell: [axis][5][ncell]
        if (bflux_int) {
            const double scale = 0.5 * ctrl->dt;
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                if (af[d].hi_bnd) continue;
                double *o = bflux_int + (int64_t)d * 5 * g.ncell + lin;
                for (int k = 0; k < 5; ++k) o[k * g.ncell] += scale * double(af[d].hi[k]) * g.area[d];
            }
        }

        // boundary-flux register capture, src/reflux.jl:125-132
        if (bflux) {
            const double scale = 0.5 * ctrl->dt;
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                if (af[d].lo_bnd) {
                    const int64_t o = bflux_offset(g, d, 0, cc);
                    const int64_t P = g.ncell / g.n[d];
                    for (int k = 0; k < 5; ++k)
                        bflux[o + k * P] += scale * double(af[d].lo[k]) * g.area[d];
                }
                if (af[d].hi_bnd) {
                    const int64_t o = bflux_offset(g, d, 1, cc);
                    const int64_t P = g.ncell / g.n[d];
                    for (int k = 0; k < 5; ++k)
                        bflux[o + k * P] += scale * double(af[d].hi[k]) * g.area[d];
                }
            }
        }

        if constexpr (STAGE == 2) {
            // next step's CFL term on the new state, src/driver.jl:178-185
            double W[5];
            cons2prim(un, g.gamma, W);
            const double cs = sound_speed(W, g.gamma);
#pragma unroll
            for (int d = 0; d < ND; ++d) invdt = nan_max(invdt, (fabs(W[1 + d]) + cs) / g.w[d]);
            if (g.grav_g) invdt = nan_max(invdt, gravity_invdt(g.grav_G, W[0]));
        }
    }
    if constexpr (STAGE == 2) block_max_to(&ctrl->invdt_bits, invdt, red);
}

}  // namespace vb
