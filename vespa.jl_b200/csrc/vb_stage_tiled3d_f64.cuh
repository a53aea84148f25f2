// vb_stage_tiled3d_f64.cuh -- VB_FP64 tiled 3D stage kernel.
//
// The exact-float64 counterpart of k_stage_tiled3d_mixed (same tiling, TMA
// pipeline, persistent queue and plane structure; see that file): a ring of
// three float64 primitive planes with mirror ghosts at walls; each thread
// rebuilds the states of its own lo x and lo y faces from the four cells
// across each and solves them with the reference's HLLC (src/riemann.jl) one
// after the other; warps 6 and 7 add the tile's hi-edge y and x faces; the z
// face runs down the thread's column, before the first barrier in warps 4..7
// and after it in warps 0..3; two barriers per plane.  Every operation is the
// reference's, rounded separately (-fmad=false), in the reference's per-cell
// accumulation order, so the result is bit-identical to the cell-centric
// kernel and to the oracle.
#pragma once

#include "vb_stage_tiled3d_mixed.cuh"

namespace vb {

namespace t3d {

using t3::NH;
using t3::NT;
using t3::TX;
using t3::TY;
using t3m::PC;
using t3m::PSLOT;
using t3m::wrow;
using t3m::wxs;

template <int NS>
struct Smem {
    double u[NS][t3::UPLANE];     // TMA stage buffers (raw conserved state)
    double w[3][PSLOT];           // primitive ring (t3m layout, float64)
    double gx[5][TY * (TX + 1)];  // x-face area * flux
    double gy[5][(TY + 1) * TX];  // y-face area * flux
    uint64_t bar[NS];
};

// Left / right states of one face along axis AX (0 x, 1 y) from the four cells
// across it (ring offsets o[0..3]): the hi face value of the cell behind and
// the lo face value of the cell ahead (_face_value, src/driver.jl:227-233).
__device__ __forceinline__ void face_states(const double *wk, const int o[4], double L[5],
                                            double R[5])
{
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        const double *p = wk + f * PC;
        const double a0 = p[o[0]], a1 = p[o[1]], a2 = p[o[2]], a3 = p[o[3]];
        L[f] = face_val(a1, 0.5, limited_slope<double>(a0, a1, a2));
        R[f] = face_val(a2, -0.5, limited_slope<double>(a1, a2, a3));
    }
}

}  // namespace t3d

template <int NS, int STAGE, bool BATCH, bool GRAV = false, bool BF = false>
__global__ void __launch_bounds__(256, 2)
k_stage_tiled3d_f64(const __grid_constant__ BoxDesc box0, const BoxDesc *__restrict__ boxes,
                    const int *__restrict__ item_box, int nitems, unsigned int *work)
{
    using namespace t3;
    using namespace t3d;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // check build only: TMA destinations need a 128-byte aligned base (uniform)
    if (!VB_DCHECK(((uintptr_t)smem_raw & 127) == 0)) return;
    t3d::Smem<NS> &S = *reinterpret_cast<t3d::Smem<NS> *>(smem_raw);
    __shared__ double red[32];
    __shared__ int item_sh;
    __shared__ int stall_sh;  // a stage load's bounded wait gave up

    const int t = threadIdx.x;
    const int tx = t & (TX - 1), ty = t >> 4;
    const int warp = t >> 5, lane = t & 31;
    const int o_c = wrow(tx, ty);
    const int ox[4] = {tx >= 2 ? o_c - 2 : wxs(tx - 2, ty), tx >= 1 ? o_c - 1 : wxs(-1, ty), o_c,
                       tx <= TX - 2 ? o_c + 1 : wxs(TX, ty)};
    const int oy[4] = {o_c - 32, o_c - 16, o_c, o_c + 16};
    const int h_u = halo_uoff(t < NH ? t : 0, 0);
    const int h_w = t < 32   ? wxs(-2 + (t & 1), t >> 1)
                    : t < 64 ? wxs(TX + (t & 1), (t - 32) >> 1)
                    : t < 96 ? wrow((t - 64) & 15, -2 + ((t - 64) >> 4))
                             : wrow((t - 96) & 15, TY + ((t - 96) >> 4));
    const bool z_early = warp >= 4;

    if (t == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&S.bar[s], 1);
        fence_mbar_init();
        stall_sh = 0;
    }
    __syncthreads();

    int qb = 0;
    for (;;) {
    if (t == 0) item_sh = (int)atomicAdd(&work[STAGE - 1], 1u);
    __syncthreads();
    const int item = item_sh;
    if (item >= nitems) break;
    const BoxDesc &B = box_of<BATCH>(box0, boxes, item_box, item);
    Ctrl *ctrl = B.ctrl;
    if (!ctrl->active) {  // uniform: the box is not stepping
        __syncthreads();  // everyone has read item_sh before thread 0 rewrites it
        continue;
    }
    const Geom &g = B.g;
    const CUtensorMap *tm = B.map[STAGE - 1];
    if (!VB_DCHECK(((uintptr_t)tm & 63) == 0)) return;  // check build only (uniform)
    const double *__restrict__ Uin = STAGE == 1 ? B.U : B.U1;
    const double *U0 = B.U;
    double *Uout = STAGE == 1 ? B.U1 : B.U;
    const int kz = B.kz, ntx = B.ntx, ntiles = B.ntiles;
    const int nx = (int)g.n[0], ny = (int)g.n[1], nz = (int)g.n[2];
    const bool perx = g.bc_lo[0] == BC_PERIODIC, pery = g.bc_lo[1] == BC_PERIODIC;
    const bool perz = g.bc_lo[2] == BC_PERIODIC;
    const double gamma = g.gamma;
    const double invV = ctrl->invV;
    const double bscale = BF ? 0.5 * ctrl->dt : 0.0;  // boundary-flux stage weight
    const double ax = g.area[0], ay = g.area[1], az = g.area[2];
    const int bx_lo = g.bc_lo[0], bx_hi = g.bc_hi[0], by_lo = g.bc_lo[1], by_hi = g.bc_hi[1];
    const int bz_lo = g.bc_lo[2], bz_hi = g.bc_hi[2];
    double invdt = 0.0;
    const int local = item - B.item0;
    const int tile = local % ntiles;
    const int x0 = (tile % ntx) * TX, y0 = (tile / ntx) * TY;
    int k0, k1;
    chunk_span(nz, kz, B.nchu, local / ntiles, k0, k1);
    const int nplanes = (k1 - k0) + 4;
    const bool xlo_bnd = !perx && x0 == 0, xhi_bnd = !perx && x0 + TX == nx;
    const bool ylo_bnd = !pery && y0 == 0, yhi_bnd = !pery && y0 + TY == ny;
    const bool h_ghost = t < 32 ? xlo_bnd : (t < 64 ? xhi_bnd : (t < 96 ? ylo_bnd : yhi_bnd));

    auto issue = [&](int q) {
        const int p = k0 - 2 + q;
        // periodic wrap of the planes k0 - 2 .. k1 + 1 (a modulo only when nz < 3)
        int z = p;
        if (perz) {
            z = p < 0 ? p + nz : (p >= nz ? p - nz : p);
            if (z < 0 || z >= nz) z = ((p % nz) + nz) % nz;
        }
        double *dst = S.u[(qb + q) % NS];
        uint64_t *bar = &S.bar[(qb + q) % NS];
        const int xl = (perx && x0 == 0) ? nx - 2 : x0 - 2;
        const int xh = (perx && x0 + TX == nx) ? 0 : x0 + TX;
        const int yl = (pery && y0 == 0) ? ny - 2 : y0 - 2;
        const int yh = (pery && y0 + TY == ny) ? 0 : y0 + TY;
        mbar_expect_tx(bar, PLANE_BYTES);
        tma_load_4d(dst, &tm[0], x0, y0, z, 0, bar);
        tma_load_4d(dst + U_XLO, &tm[1], xl, y0, z, 0, bar);
        tma_load_4d(dst + U_XHI, &tm[1], xh, y0, z, 0, bar);
        tma_load_4d(dst + U_YLO, &tm[2], x0, yl, z, 0, bar);
        tma_load_4d(dst + U_YHI, &tm[2], x0, yh, z, 0, bar);
    };
    // the stage loads are issued by one thread of warp 5, whose share of the
    // plane's second phase is the smallest
    if (t == TMA_ISSUER) {
        fence_proxy_async_smem();
        for (int q = 0; q < NS && q < nplanes; ++q) issue(q);
    }
    // Halo strips of staged plane q into ring slot q % 3 (threads t < NH).
    auto halo_c2p = [&](int q) {
        if (t < NH && !h_ghost) {
            const double *u = S.u[(qb + q) % NS];
            double *ws = S.w[q % 3];
            double uu[5], w[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) uu[f] = u[h_u + f * (2 * TY)];
            cons2prim(uu, gamma, w);
#pragma unroll
            for (int f = 0; f < 5; ++f) ws[h_w + f * PC] = w[f];
        }
    };
    // Wait for staged plane q and convert the own cell into Wn.  keep = 0:
    // registers only; 1: also into ring slot q % 3 with the mirror ghosts and
    // the halo strips; 2: as 1 without the halo strips (halo_c2p follows).
    auto consume = [&](int q, double Wn[5], int keep) {
        const int b = (qb + q) % NS;
        if (!mbar_wait(&S.bar[b], ((qb + q) / NS) & 1, WAIT_LIMIT_NS)) stall_sh = 1;
        const double *u = S.u[b];
        {
            double uu[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) uu[f] = u[f * NT + t];
            cons2prim(uu, gamma, Wn);
        }
        if (!keep) return;
        double *ws = S.w[q % 3];
#pragma unroll
        for (int f = 0; f < 5; ++f) ws[f * PC + o_c] = Wn[f];
        if (xlo_bnd && tx < 2) {
            double *d = ws + wxs(-1 - tx, ty);
#pragma unroll
            for (int f = 0; f < 5; ++f) d[f * PC] = (bx_lo == BC_REFLECTING && f == 1) ? -Wn[f] : Wn[f];
        }
        if (xhi_bnd && tx >= TX - 2) {
            double *d = ws + wxs(2 * TX - 1 - tx, ty);
#pragma unroll
            for (int f = 0; f < 5; ++f) d[f * PC] = (bx_hi == BC_REFLECTING && f == 1) ? -Wn[f] : Wn[f];
        }
        if (ylo_bnd && ty < 2) {
            double *d = ws + wrow(tx, -1 - ty);
#pragma unroll
            for (int f = 0; f < 5; ++f) d[f * PC] = (by_lo == BC_REFLECTING && f == 2) ? -Wn[f] : Wn[f];
        }
        if (yhi_bnd && ty >= TY - 2) {
            double *d = ws + wrow(tx, 2 * TY - 1 - ty);
#pragma unroll
            for (int f = 0; f < 5; ++f) d[f * PC] = (by_hi == BC_REFLECTING && f == 2) ? -Wn[f] : Wn[f];
        }
        if (keep == 1) halo_c2p(q);
    };
    auto release = [&](int q) {
        if (t == TMA_ISSUER && q + NS < nplanes) {
            fence_proxy_async_smem();
            issue(q + NS);
        }
    };
    // after the barrier that follows consume(q): uniform across the block
    auto stalled = [&](int q) -> bool {
        if (!stall_sh) return false;
        stage_abandon<NS>(S.bar, qb, q, nplanes, ctrl);
        return true;
    };

    double Wa[5], Wb[5], Wc[5], Wd[5];
    consume(0, Wa, 0);
    __syncthreads();
    if (stalled(0)) return;
    release(0);
    consume(1, Wb, 0);
    __syncthreads();
    if (stalled(1)) return;
    release(1);
    consume(2, Wc, 1);
    __syncthreads();
    if (stalled(2)) return;
    release(2);
    consume(3, Wd, 1);
    __syncthreads();
    if (stalled(3)) return;
    release(3);

    // z state entering plane k0: hi face value of k0 and the flux through k0-1/2
    double hz[5], Fzlo[5];
    {
        const bool gl = !perz && k0 == 0;
        const bool gh = !perz && k0 + 1 >= nz;
        double loz[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const double wl = gl ? ((bz_lo == BC_REFLECTING && f == 3) ? -Wc[f] : Wc[f]) : Wb[f];
            const double wr = gh ? ((bz_hi == BC_REFLECTING && f == 3) ? -Wc[f] : Wc[f]) : Wd[f];
            const double s = limited_slope<double>(wl, Wc[f], wr);
            hz[f] = face_val(Wc[f], 0.5, s);
            loz[f] = face_val(Wc[f], -0.5, s);
        }
        if (gl) {
            double gst[5];
            ghost_state<double>(loz, bz_lo, 2, gst);
            tiled_hllc<3>(gst, loz, gamma, Fzlo);
            if constexpr (BF)  // z-lo domain face of cell (x, y, 0)
                bflux_add(g, B.bflux, 2, 0, (int64_t)(x0 + tx) + (int64_t)nx * (y0 + ty), bscale, az, Fzlo);
        } else {
            const bool gll = !perz && k0 - 2 < 0;
            double hzm[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const double wl = gll ? ((bz_lo == BC_REFLECTING && f == 3) ? -Wb[f] : Wb[f]) : Wa[f];
                hzm[f] = face_val(Wb[f], 0.5, limited_slope<double>(wl, Wb[f], Wc[f]));
            }
            tiled_hllc<3>(hzm, loz, gamma, Fzlo);
        }
    }

    // flux through k+1/2 from planes k, k+1 (ring) and k+2 (W2) of the own
    // column; advances hz
    auto zsolve = [&](int k, const double *w0, const double *w1, const double W2[5], double Fzhi[5]) {
        double zr[5], hz1[5];
        if (perz || k + 1 < nz) {
            const bool gh = !perz && k + 2 >= nz;
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const double c = w1[f * PC];
                const double r = gh ? ((bz_hi == BC_REFLECTING && f == 3) ? -c : c) : W2[f];
                const double s = limited_slope<double>(w0[f * PC], c, r);
                zr[f] = face_val(c, -0.5, s);
                hz1[f] = face_val(c, 0.5, s);
            }
        } else {
            ghost_state<double>(hz, bz_hi, 2, zr);
#pragma unroll
            for (int f = 0; f < 5; ++f) hz1[f] = hz[f];
        }
        tiled_hllc<3>(hz, zr, gamma, Fzhi);
        if constexpr (BF) {
            if (!perz && k + 1 >= nz)  // z-hi domain face of cell (x, y, nz-1)
                bflux_add(g, B.bflux, 2, 1, (int64_t)(x0 + tx) + (int64_t)nx * (y0 + ty), bscale, az, Fzhi);
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) hz[f] = hz1[f];
    };
    // the own lo x face and lo y face of plane k (ring slot w0)
    auto xy_faces = [&](const double *w0, int k) {
        double L[5], R[5], F[5];
        face_states(w0, ox, L, R);
        tiled_hllc<1>(L, R, gamma, F);
#pragma unroll
        for (int f = 0; f < 5; ++f) S.gx[f][ty * (TX + 1) + tx] = ax * F[f];
        if constexpr (BF) {
            if (xlo_bnd && tx == 0)  // x-lo domain face of cell (0, y, k)
                bflux_add(g, B.bflux, 0, 0, (int64_t)(y0 + ty) + (int64_t)ny * k, bscale, ax, F);
        }
        face_states(w0, oy, L, R);
        tiled_hllc<2>(L, R, gamma, F);
#pragma unroll
        for (int f = 0; f < 5; ++f) S.gy[f][ty * TX + tx] = ay * F[f];
        if constexpr (BF) {
            if (ylo_bnd && ty == 0)  // y-lo domain face of cell (x, 0, k)
                bflux_add(g, B.bflux, 1, 0, (int64_t)(x0 + tx) + (int64_t)nx * k, bscale, ay, F);
        }
    };
    // the hi-edge faces: x at fx = TX (warp 7) or y at fy = TY (warp 6), lanes < 16
    auto edge_face = [&](const double *w0, int k) {
        const int j = lane;
        double L[5], R[5], F[5];
        if (warp == 7) {
            const int ex[4] = {wrow(TX - 2, j), wrow(TX - 1, j), wxs(TX, j), wxs(TX + 1, j)};
            face_states(w0, ex, L, R);
            tiled_hllc<1>(L, R, gamma, F);
#pragma unroll
            for (int f = 0; f < 5; ++f) S.gx[f][j * (TX + 1) + TX] = ax * F[f];
            if constexpr (BF) {
                if (xhi_bnd)  // x-hi domain face of cell (nx-1, y0+j, k)
                    bflux_add(g, B.bflux, 0, 1, (int64_t)(y0 + j) + (int64_t)ny * k, bscale, ax, F);
            }
        } else {
            const int ey[4] = {wrow(j, TY - 2), wrow(j, TY - 1), wrow(j, TY), wrow(j, TY + 1)};
            face_states(w0, ey, L, R);
            tiled_hllc<2>(L, R, gamma, F);
#pragma unroll
            for (int f = 0; f < 5; ++f) S.gy[f][TY * TX + j] = ay * F[f];
            if constexpr (BF) {
                if (yhi_bnd)  // y-hi domain face of cell (x0+j, ny-1, k)
                    bflux_add(g, B.bflux, 1, 1, (int64_t)(x0 + j) + (int64_t)nx * k, bscale, ay, F);
            }
        }
    };

    const int gx = x0 + tx, gy = y0 + ty;
    const int cx = lo_class(gx, nx, perx), cy = lo_class(gy, ny, pery);
    // previous plane's new state: its CFL term is folded one plane later (the
    // initial value is a finite placeholder whose term is discarded)
    double unp[5] = {1.0, 0.0, 0.0, 0.0, 1.0};
    const int64_t plane_cells = (int64_t)nx * ny;
    int64_t lin = (int64_t)gx + (int64_t)nx * ((int64_t)gy + (int64_t)ny * k0);

    for (int k = k0; k < k1; ++k) {
        const int q = k - k0 + 4;
        const double *w0 = S.w[(q - 2) % 3], *w1 = S.w[(q - 1) % 3], *w2 = S.w[q % 3];
        if (tx == 0) {  // one 128-byte row per field: warm L1 for the epilogue's loads
            const double *pa = Uin + lin, *pb = U0 + lin;
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                prefetch_l1(pa);
                if constexpr (STAGE == 2) prefetch_l1(pb);
                pa += g.ncell;
                pb += g.ncell;
            }
        }
        // ---- phase 1: plane k+2 to primitives; the CFL term of plane k-1; the
        //      z face (warps 4..7) or the halo strips (warps 0..3) ----
        double Fzhi[5];
        {
            double Wn[5];
            consume(q, Wn, 2);
            double cf = 0.0;
            if constexpr (STAGE == 2) cf = cfl_term_exact<GRAV>(unp, g, invdt);
            if (z_early) zsolve(k, w0 + o_c, w1 + o_c, Wn, Fzhi);
            else halo_c2p(q);
            if constexpr (STAGE == 2)
                if (k > k0 && k > g.zw0 && k <= g.zw1) invdt = cf;  // plane k-1, if the slab's own
        }
        __syncthreads();  // (1) plane k+2 converted
        if (stalled(q)) return;
        release(q);
        // ---- phase 2: the own lo x / lo y faces; the z face (warps 0..3) or
        //      a hi-edge face (warps 6, 7) ----
        if (z_early) {
            xy_faces(w0, k);
            if (warp >= 6 && lane < 16) edge_face(w0, k);
        } else {
            double W2[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) W2[f] = w2[o_c + f * PC];
            zsolve(k, w0 + o_c, w1 + o_c, W2, Fzhi);
            xy_faces(w0, k);
        }
        __syncthreads();  // (2) fluxes ready

        // ---- flux divergence in the reference's order, then the stage update ----
        const int cz = (k == g.zw0 && g.zcls0 >= 0) ? g.zcls0 : lo_class(k, nz, perz);
        const bool interior = cx == LO_BEFORE && cy == LO_BEFORE && cz == LO_BEFORE;
        double un[5];
        const bool inb = VB_DCHECK(lin >= 0 && lin < g.ncell);  // check build only
        const double *pin = Uin + lin, *p0 = U0 + lin;
        double *po = Uout + lin;
        double acc[5];  // GRAV: the flux sums, completed by the gravity source
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const double gxl = S.gx[f][ty * (TX + 1) + tx];
            const double gxh = S.gx[f][ty * (TX + 1) + tx + 1];
            const double gyl = S.gy[f][ty * TX + tx];
            const double gyh = S.gy[f][(ty + 1) * TX + tx];
            const double gzl = az * Fzlo[f], gzh = az * Fzhi[f];
            double a = 0.0;
            if (interior) {
                a = a - gzl - gyl - gxl + gxh + gyh + gzh;
            } else {
                if (cz == LO_BEFORE) a -= gzl;
                if (cy == LO_BEFORE) a -= gyl;
                if (cx == LO_BEFORE) a -= gxl;
                a += gxh;
                if (cx == LO_SELF) a -= gxl;
                a += gyh;
                if (cy == LO_SELF) a -= gyl;
                a += gzh;
                if (cz == LO_SELF) a -= gzl;
                if (cx == LO_AFTER) a -= gxl;
                if (cy == LO_AFTER) a -= gyl;
                if (cz == LO_AFTER) a -= gzl;
            }
            Fzlo[f] = Fzhi[f];
            if constexpr (GRAV) {
                acc[f] = a;
                continue;
            }
            const double uin = inb ? __ldg(pin) : 0.0;
            if constexpr (STAGE == 1) {
                un[f] = uin - invV * a;
            } else {
                un[f] = 0.5 * (inb ? *p0 : 0.0) + 0.5 * (uin - invV * a);
            }
            if (inb) *po = un[f];
            pin += g.ncell;
            p0 += g.ncell;
            po += g.ncell;
        }
        if constexpr (GRAV) {  // the source from the stage state, after the fluxes
            double u[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) u[f] = inb ? __ldg(pin + f * g.ncell) : 0.0;
            if (inb) gravity_source<3>(g, lin, u, acc);
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                if constexpr (STAGE == 1) un[f] = u[f] - invV * acc[f];
                else un[f] = 0.5 * (inb ? p0[f * g.ncell] : 0.0) + 0.5 * (u[f] - invV * acc[f]);
                if (inb) po[f * g.ncell] = un[f];
            }
        }
        lin += plane_cells;
        if constexpr (STAGE == 2) {
#pragma unroll
            for (int f = 0; f < 5; ++f) unp[f] = un[f];
        }
    }
    if constexpr (STAGE == 2)  // the item's last plane, when it is one of the slab's own
        if (k1 - 1 >= g.zw0 && k1 - 1 < g.zw1) invdt = cfl_term_exact<GRAV>(unp, g, invdt);
    qb += nplanes;
    if constexpr (STAGE == 2) block_max_to(&ctrl->invdt_bits, invdt, red);  // this box's CFL max
    }  // work items
}

template <int NS>
int launch_tiled3d_f64(const BoxDesc *hbox, const BoxDesc *boxes, const int *item_box,
                       int nitems, unsigned int *work, int stage, cudaStream_t s, bool grav,
                       bool bf)
{
    const size_t smem = sizeof(t3d::Smem<NS>);
    static int res1 = 0, resb = 0, resg = 0, resf = 0;
    if (!res1) res1 = persistent_blocks(k_stage_tiled3d_f64<NS, 1, false>,
                                        k_stage_tiled3d_f64<NS, 2, false>, smem);
    if (!resb) resb = persistent_blocks(k_stage_tiled3d_f64<NS, 1, true>,
                                        k_stage_tiled3d_f64<NS, 2, true>, smem);
    if (!resg) resg = persistent_blocks(k_stage_tiled3d_f64<NS, 1, false, true>,
                                        k_stage_tiled3d_f64<NS, 2, false, true>, smem);
    if (!resf) resf = persistent_blocks(k_stage_tiled3d_f64<NS, 1, false, false, true>,
                                        k_stage_tiled3d_f64<NS, 2, false, false, true>, smem);
    if ((grav || bf) && !hbox) return -1;  // gravity, boundary fluxes: single boxes only
    if (grav && bf) return -1;
    if (bf && !hbox->bflux) return -1;
    const int resident = grav ? resg : bf ? resf : hbox ? res1 : resb;
    if (resident <= 0 || nitems <= 0) return -1;
    const unsigned grid = (unsigned)(nitems < resident ? nitems : resident);
    BoxDesc box0;
    if (hbox) box0 = *hbox;
    else std::memset(&box0, 0, sizeof box0);
    if (grav && stage == 1)
        k_stage_tiled3d_f64<NS, 1, false, true><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (grav)
        k_stage_tiled3d_f64<NS, 2, false, true><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (bf && stage == 1)
        k_stage_tiled3d_f64<NS, 1, false, false, true><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (bf)
        k_stage_tiled3d_f64<NS, 2, false, false, true><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (hbox && stage == 1)
        k_stage_tiled3d_f64<NS, 1, false><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (hbox)
        k_stage_tiled3d_f64<NS, 2, false><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (stage == 1)
        k_stage_tiled3d_f64<NS, 1, true><<<grid, t3::NT, smem, s>>>(box0, boxes, item_box, nitems, work);
    else
        k_stage_tiled3d_f64<NS, 2, true><<<grid, t3::NT, smem, s>>>(box0, boxes, item_box, nitems, work);
    return 1;
}

}  // namespace vb
