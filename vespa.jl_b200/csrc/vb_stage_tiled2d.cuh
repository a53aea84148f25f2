// vb_stage_tiled2d.cuh -- tiled, y-marching fused RK2 stage kernel for 2D
// uniform meshes (the 4096^2 throughput configuration).
//
// A block owns a 256-cell row segment (one cell per thread) and marches along
// y through a chunk of rows.  For every row, one thread issues three TMA loads
// (4-D tensor map x, y, z = 0, field) of the segment and its two 2-cell x halos
// into a stage buffer, NS rows ahead of use.  Each loaded cell is converted to
// primitives once; its x slope and x face values go through shared memory;
// its y slope and the y face r+1/2 run in registers down the thread's column;
// every face flux is evaluated once.  The flux divergence of a cell is summed
// in the reference's per-cell order (LO_* classes, src/driver.jl:236-281 over
// lib/RefMesh/src/RefMesh.jl:187-197) and the stage epilogue writes the new
// state; stage 2 also folds the next step's CFL maximum over x and y.
//
// MIXED = false: the reference's float64 algebra (compiled with -fmad=false,
// bit-identical to the cell-centric kernel and the CPU restatement).
// MIXED = true: float64 state, cons2prim and accumulation; float32 slopes,
// face values and HLLC, the cell's x face and y face solved as one packed
// float32x2 HLLC.
//
// Requirements (checked on the host): nx % 256 == 0, ny >= 2, a periodic
// axis periodic on both sides, no boundary-flux capture.
#pragma once

#include <type_traits>

#include "vb_hllc_x2.cuh"
#include "vb_stage_tiled3d_mixed.cuh"

namespace vb {

namespace t2 {

constexpr int TX = 256, NT = 256;
// A staged row: interior [5][TX], then the two [5][2] x halos, each region on
// a 128-byte boundary (a TMA destination in shared memory must be 128-byte
// aligned), the row itself padded to a multiple of 128 bytes.
constexpr int U_XLO = TX * 5;            // [5][2] halo x = x0-2, x0-1
constexpr int U_XHI = U_XLO + 16;        // [5][2] halo x = x0+TX, x0+TX+1
constexpr int UROW = U_XHI + 16;         // float64 values per staged row (padded)
constexpr uint32_t ROW_BYTES = (TX * 5 + 2 * 2 * 5) * 8;  // bytes the three copies deliver
static_assert((U_XLO * 8) % 128 == 0 && (U_XHI * 8) % 128 == 0 && (UROW * 8) % 128 == 0,
              "TMA destinations must be 128-byte aligned");

template <typename T, int NS>
struct Smem {
    alignas(128) double u[NS][UROW];  // TMA stage buffers (raw conserved state)
    double ep[2][5][NT];   // own-cell epilogue inputs (Uin, U0), fetched by cp.async
    T w[5][NT];            // primitives of the current row
    T wh[3][5][4];         // halo primitives by row (ring of 3): x0-2, x0-1, x0+TX, x0+TX+1
    T fl[5][NT], fh[5][NT];  // lo / hi x face values of the row's cells
    T hf[2][5];            // hi face value of x0-1, lo face value of x0+TX
    double gx[5][TX + 1];  // x-face area * flux; face i between cells i-1 and i
    uint64_t bar[NS];
};

}  // namespace t2

// Mixed precision runs 3 CTAs per SM (80 registers, 67.5 KB of shared memory
// each): the step is 8 % faster than at 2 CTAs with 102 registers; float64
// keeps 2 (128 registers).
template <bool MIXED, int NS, int STAGE, bool BF = false>
__global__ void __launch_bounds__(256, MIXED ? 3 : 2)
k_stage_tiled2d(const __grid_constant__ BoxDesc B, int nitems, unsigned int *work)
{
    using namespace t2;
    using T = typename std::conditional<MIXED, float, double>::type;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // check build only: TMA destinations need a 128-byte aligned base (uniform)
    if (!VB_DCHECK(((uintptr_t)smem_raw & 127) == 0)) return;
    t2::Smem<T, NS> &S = *reinterpret_cast<t2::Smem<T, NS> *>(smem_raw);
    __shared__ double red[32];
    __shared__ int item_sh;
    __shared__ int stall_sh;  // a stage load's bounded wait gave up
    const int t = threadIdx.x;

    if (t == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&S.bar[s], 1);
        fence_mbar_init();
        stall_sh = 0;
    }
    __syncthreads();

    const Geom &g = B.g;
    Ctrl *ctrl = B.ctrl;
    const CUtensorMap *tm = B.map[STAGE - 1];
    if (!VB_DCHECK(((uintptr_t)tm & 63) == 0)) return;  // check build only (uniform)
    const double *__restrict__ Uin = STAGE == 1 ? B.U : B.U1;
    const double *U0 = B.U;
    double *Uout = STAGE == 1 ? B.U1 : B.U;
    const int ky = B.kz, ntx = B.ntx;
    const int nx = (int)g.n[0], ny = (int)g.n[1];
    const bool perx = g.bc_lo[0] == BC_PERIODIC, pery = g.bc_lo[1] == BC_PERIODIC;
    const int bx_lo = g.bc_lo[0], bx_hi = g.bc_hi[0], by_lo = g.bc_lo[1], by_hi = g.bc_hi[1];
    const double gamma = g.gamma;
    const float gf = (float)gamma, ig1 = 1.0f / ((float)gamma - 1.0f);
    const double ax = g.area[0], ay = g.area[1];
    const T half = T(0.5), mhalf = T(-0.5);
    const double bscale = BF ? 0.5 * ctrl->dt : 0.0;  // boundary-flux stage weight
    // boundary-flux capture of a solved domain face (axis d, side, plane entry)
    auto capture = [&](int d, int side, int64_t idx, const T F[5]) {
        const double Fd[5] = {(double)F[0], (double)F[1], (double)F[2], (double)F[3], (double)F[4]};
        bflux_add(g, B.bflux, d, side, idx, bscale, g.area[d], Fd);
    };

    // float32 slopes use the clamp form of minmod (t3m::mm), float64 the reference's
    auto slope = [](T l, T c, T r) -> T {
        if constexpr (MIXED) return t3m::mm(l, c, r);
        else return limited_slope<T>(l, c, r);
    };
    auto to_prim = [&](const double uu[5], T W[5]) {
        if constexpr (MIXED) {
            t3m::cons2prim_mixed(uu, gamma, W);
        } else {
            cons2prim(uu, gamma, W);
        }
    };
    // ghost value of component f across an x (ax = 0) or y (ax = 1) boundary
    auto ghostc = [](T w, int f, int bc, int axis) -> T {
        return (bc == BC_REFLECTING && f == 1 + axis) ? -w : w;
    };

    int qb = 0;
    double invdt = 0.0;
    for (;;) {
    if (t == 0) item_sh = (int)atomicAdd(&work[STAGE - 1], 1u);
    __syncthreads();
    const int item = item_sh;
    if (item >= nitems) break;
    if (!ctrl->active) {  // uniform: the grid is not stepping
        __syncthreads();
        continue;
    }
    const int x0 = (item % ntx) * TX;
    const int r0 = (item / ntx) * ky;
    const int r1 = min(ny, r0 + ky);
    const int nrows = (r1 - r0) + 4;  // rows r0-2 .. r1+1
    const bool xlo_bnd = !perx && x0 == 0, xhi_bnd = !perx && x0 + TX == nx;

    auto issue = [&](int q) {
        const int p = r0 - 2 + q;
        const int y = pery ? ((p % ny) + ny) % ny : p;  // out-of-range rows read the zero fill
        double *dst = S.u[(unsigned)(qb + q) % NS];
        uint64_t *bar = &S.bar[(unsigned)(qb + q) % NS];
        const int xl = (perx && x0 == 0) ? nx - 2 : x0 - 2;
        const int xh = (perx && x0 + TX == nx) ? 0 : x0 + TX;
        mbar_expect_tx(bar, ROW_BYTES);
        tma_load_4d(dst, &tm[0], x0, y, 0, 0, bar);
        tma_load_4d(dst + U_XLO, &tm[1], xl, y, 0, 0, bar);
        tma_load_4d(dst + U_XHI, &tm[1], xh, y, 0, 0, bar);
    };
    if (t == 0) {
        fence_proxy_async_smem();
        for (int q = 0; q < NS && q < nrows; ++q) issue(q);
    }
    auto consume = [&](int q, T Wown[5], bool halo) {
        const int b = (unsigned)(qb + q) % NS;
        if (!mbar_wait(&S.bar[b], ((unsigned)(qb + q) / NS) & 1, WAIT_LIMIT_NS)) stall_sh = 1;
        const double *u = S.u[b];
        double uu[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) uu[f] = u[f * TX + t];
        to_prim(uu, Wown);
        if (halo && t < 4) {
            T w[5];
            const int base = t < 2 ? U_XLO + t : U_XHI + (t - 2);
#pragma unroll
            for (int f = 0; f < 5; ++f) uu[f] = u[base + 2 * f];
            to_prim(uu, w);
#pragma unroll
            for (int f = 0; f < 5; ++f) S.wh[q % 3][f][t] = w[f];
        }
    };
    auto release = [&](int q) {
        if (t == 0 && q + NS < nrows) {
            fence_proxy_async_smem();
            issue(q + NS);
        }
    };
    // after the barrier that follows consume(q): uniform across the block
    auto stalled = [&](int q) -> bool {
        if (!stall_sh) return false;
        stage_abandon<NS>(S.bar, qb, q, nrows, ctrl);
        return true;
    };

    T Wa[5], Wb[5], Wy0[5], Wy1[5], Wy2[5];
    consume(0, Wa, false);
    __syncthreads();
    if (stalled(0)) return;
    release(0);
    consume(1, Wb, false);
    __syncthreads();
    if (stalled(1)) return;
    release(1);
    consume(2, Wy0, true);
    __syncthreads();
    if (stalled(2)) return;
    release(2);
    consume(3, Wy1, true);
    __syncthreads();
    if (stalled(3)) return;
    release(3);

    // y state entering row r0: hi face value of r0 and the flux through r0-1/2
    T hy[5], Fylo[5];
    {
        const bool gl = !pery && r0 == 0;
        const bool gh = !pery && r0 + 1 >= ny;
        T loy[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const T wl = gl ? ghostc(Wy0[f], f, by_lo, 1) : Wb[f];
            const T wr = gh ? ghostc(Wy0[f], f, by_hi, 1) : Wy1[f];
            const T s = slope(wl, Wy0[f], wr);
            hy[f] = face_val(Wy0[f], half, s);
            loy[f] = face_val(Wy0[f], mhalf, s);
        }
        T yl[5];  // left state of the face r0-1/2
        if (gl) {
            ghost_state<T>(loy, by_lo, 1, yl);
        } else {
            const bool gll = !pery && r0 - 2 < 0;
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const T wl = gll ? ghostc(Wb[f], f, by_lo, 1) : Wa[f];
                yl[f] = face_val(Wb[f], half, slope(wl, Wb[f], Wy0[f]));
            }
        }
        if constexpr (MIXED) {
            // the y lane of the packed solver, as the chunk below solved this
            // face in its last row: both sides of the face get the same bits
            const Face2 L{f2::splat(yl[0]), f2::splat(yl[2]), f2::splat(yl[1]), f2::splat(yl[3]),
                          f2::splat(yl[4])};
            const Face2 R{f2::splat(loy[0]), f2::splat(loy[2]), f2::splat(loy[1]),
                          f2::splat(loy[3]), f2::splat(loy[4])};
            f2 F[5];
            hllc_x2(L, R, gf, ig1, F);
            Fylo[0] = F[0].v.y;
            Fylo[1] = F[2].v.y;
            Fylo[2] = F[1].v.y;
            Fylo[3] = F[3].v.y;
            Fylo[4] = F[4].v.y;
        } else {
            hllc_flux<double, 2>(yl, loy, gamma, Fylo);
        }
        if constexpr (BF) {
            if (gl) capture(1, 0, x0 + t, Fylo);  // y-lo domain face of cell (x, 0)
        }
    }

    const int gxc = x0 + t;
    const int cx = lo_class(gxc, nx, perx);
    const double invV = ctrl->invV;
    double unp[5];

    for (int r = r0; r < r1; ++r) {
        const int q = r - r0 + 4;
        const int slot = (q - 2) % 3;  // ring slot of row r's halo
        const int64_t lin = (int64_t)gxc + (int64_t)nx * r;
        const bool inb = VB_DCHECK(lin >= 0 && lin < g.ncell);  // check build only
        if (inb)
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                cp_async8(&S.ep[0][f][t], Uin + (int64_t)f * g.ncell + lin);
                if constexpr (STAGE == 2) cp_async8(&S.ep[1][f][t], U0 + (int64_t)f * g.ncell + lin);
            }
        cp_async_commit();
        consume(q, Wy2, true);
        if constexpr (STAGE == 2) {
            if (r > r0) {
                if constexpr (MIXED) invdt = t3m::cfl_term2d(unp, g, invdt);
                else invdt = cfl_term2d_exact(unp, g, invdt);
            }
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) S.w[f][t] = Wy0[f];
        __syncthreads();  // (1) row r primitives complete
        if (stalled(q)) return;
        release(q);

        // ---- x slope and x face values of the own cell ----
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const T wc = Wy0[f];
            const T l = t > 0 ? S.w[f][t - 1]
                              : (xlo_bnd ? ghostc(wc, f, bx_lo, 0) : S.wh[slot][f][1]);
            const T rr = t < TX - 1 ? S.w[f][t + 1]
                                    : (xhi_bnd ? ghostc(wc, f, bx_hi, 0) : S.wh[slot][f][2]);
            const T s = slope(l, wc, rr);
            S.fl[f][t] = face_val(wc, mhalf, s);
            S.fh[f][t] = face_val(wc, half, s);
        }
        // face values of the cells just outside the segment
        if (t == 32 && !xlo_bnd) {
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const T c = S.wh[slot][f][1];
                S.hf[0][f] = face_val(c, half, slope(S.wh[slot][f][0], c, S.w[f][0]));
            }
        }
        if (t == 64 && !xhi_bnd) {
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const T c = S.wh[slot][f][2];
                S.hf[1][f] = face_val(c, mhalf, slope(S.w[f][TX - 1], c, S.wh[slot][f][3]));
            }
        }
        __syncthreads();  // (2) face values ready

        // ---- y face r+1/2 down the own column ----
        T yr[5], hy1[5];
        {
            const bool row_r1 = pery || r + 1 < ny;
            if (row_r1) {
                const bool gh = !pery && r + 2 >= ny;
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    const T wr = gh ? ghostc(Wy1[f], f, by_hi, 1) : Wy2[f];
                    const T s = slope(Wy0[f], Wy1[f], wr);
                    yr[f] = face_val(Wy1[f], mhalf, s);
                    hy1[f] = face_val(Wy1[f], half, s);
                }
            } else {
                ghost_state<T>(hy, by_hi, 1, yr);
#pragma unroll
                for (int f = 0; f < 5; ++f) hy1[f] = hy[f];
            }
        }
        // ---- x face t (between cells t-1 and t) and the y face ----
        T Lx[5], Rx[5], Fx[5], Fyhi[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) Rx[f] = S.fl[f][t];
        if (t > 0) {
#pragma unroll
            for (int f = 0; f < 5; ++f) Lx[f] = S.fh[f][t - 1];
        } else if (xlo_bnd) {
            ghost_state<T>(Rx, bx_lo, 0, Lx);
        } else {
#pragma unroll
            for (int f = 0; f < 5; ++f) Lx[f] = S.hf[0][f];
        }
        if constexpr (MIXED) {
            // x face in (rho, vx, vy, vz, p), y face rotated to (rho, vy, vx, vz, p)
            const Face2 L{f2(Lx[0], hy[0]), f2(Lx[1], hy[2]), f2(Lx[2], hy[1]), f2(Lx[3], hy[3]),
                          f2(Lx[4], hy[4])};
            const Face2 R{f2(Rx[0], yr[0]), f2(Rx[1], yr[2]), f2(Rx[2], yr[1]), f2(Rx[3], yr[3]),
                          f2(Rx[4], yr[4])};
            f2 F[5];
            hllc_x2(L, R, gf, ig1, F);
            Fx[0] = F[0].v.x; Fyhi[0] = F[0].v.y;
            Fx[1] = F[1].v.x; Fyhi[2] = F[1].v.y;
            Fx[2] = F[2].v.x; Fyhi[1] = F[2].v.y;
            Fx[3] = F[3].v.x; Fyhi[3] = F[3].v.y;
            Fx[4] = F[4].v.x; Fyhi[4] = F[4].v.y;
        } else {
            hllc_flux<double, 1>(Lx, Rx, gamma, Fx);
            hllc_flux<double, 2>(hy, yr, gamma, Fyhi);
        }
        if constexpr (BF) {
            if (t == 0 && xlo_bnd) capture(0, 0, r, Fx);                // x-lo face of (0, r)
            if (!pery && r + 1 >= ny) capture(1, 1, x0 + t, Fyhi);     // y-hi face of (x, ny-1)
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) S.gx[f][t] = ax * (double)Fx[f];
        if (t == TX - 1) {  // the segment's right edge face
            T L2[5], R2[5], F2[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) L2[f] = S.fh[f][TX - 1];
            if (xhi_bnd) {
                ghost_state<T>(L2, bx_hi, 0, R2);
            } else {
#pragma unroll
                for (int f = 0; f < 5; ++f) R2[f] = S.hf[1][f];
            }
            if constexpr (MIXED) {
                // the x lane of the packed solver, as the neighbouring segment's
                // thread 0 solves this face: both sides get the same bits
                const Face2 L{f2::splat(L2[0]), f2::splat(L2[1]), f2::splat(L2[2]),
                              f2::splat(L2[3]), f2::splat(L2[4])};
                const Face2 R{f2::splat(R2[0]), f2::splat(R2[1]), f2::splat(R2[2]),
                              f2::splat(R2[3]), f2::splat(R2[4])};
                f2 F[5];
                hllc_x2(L, R, gf, ig1, F);
#pragma unroll
                for (int f = 0; f < 5; ++f) F2[f] = F[f].v.x;
            } else {
                hllc_flux<double, 1>(L2, R2, gamma, F2);
            }
#pragma unroll
            for (int f = 0; f < 5; ++f) S.gx[f][TX] = ax * (double)F2[f];
            if constexpr (BF) {
                if (xhi_bnd) capture(0, 1, r, F2);  // x-hi face of (nx-1, r)
            }
        }
        __syncthreads();  // (3) x fluxes ready

        // ---- flux divergence (float64, reference order) and the stage update ----
        const int cy = lo_class(r, ny, pery);
        double un[5];
        cp_async_wait_all();
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const double gxl = S.gx[f][t], gxh = S.gx[f][t + 1];
            double gyl, gyh;
            if constexpr (MIXED) {
                gyl = __dmul_rn(ay, (double)Fylo[f]);
                gyh = __dmul_rn(ay, (double)Fyhi[f]);
            } else {
                gyl = ay * Fylo[f];
                gyh = ay * Fyhi[f];
            }
            double a = 0.0;
            if (cy == LO_BEFORE) a -= gyl;
            if (cx == LO_BEFORE) a -= gxl;
            a += gxh;
            if (cx == LO_SELF) a -= gxl;
            a += gyh;
            if (cy == LO_SELF) a -= gyl;
            if (cx == LO_AFTER) a -= gxl;
            if (cy == LO_AFTER) a -= gyl;
            if constexpr (MIXED) {
                if constexpr (STAGE == 1)
                    un[f] = __fma_rn(-invV, a, S.ep[0][f][t]);
                else
                    un[f] = __fma_rn(0.5, S.ep[1][f][t],
                                     __dmul_rn(0.5, __fma_rn(-invV, a, S.ep[0][f][t])));
            } else {
                if constexpr (STAGE == 1)
                    un[f] = S.ep[0][f][t] - invV * a;
                else
                    un[f] = 0.5 * S.ep[1][f][t] + 0.5 * (S.ep[0][f][t] - invV * a);
            }
            if (inb) Uout[(int64_t)f * g.ncell + lin] = un[f];
        }
        if constexpr (STAGE == 2) {
#pragma unroll
            for (int f = 0; f < 5; ++f) unp[f] = un[f];
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            Wy0[f] = Wy1[f];
            Wy1[f] = Wy2[f];
            hy[f] = hy1[f];
            Fylo[f] = Fyhi[f];
        }
    }
    if constexpr (STAGE == 2) {
        if constexpr (MIXED) invdt = t3m::cfl_term2d(unp, g, invdt);
        else invdt = cfl_term2d_exact(unp, g, invdt);
    }
    qb += nrows;
    }  // work items
    if constexpr (STAGE == 2) block_max_to(&ctrl->invdt_bits, invdt, red);
}

template <bool MIXED, int NS>
int launch_tiled2d(const BoxDesc *hbox, int nitems, unsigned int *work, int stage, cudaStream_t s,
                   bool bf)
{
    using T = typename std::conditional<MIXED, float, double>::type;
    const size_t smem = sizeof(t2::Smem<T, NS>);
    static int res = 0, resf = 0;
    if (!res) res = persistent_blocks(k_stage_tiled2d<MIXED, NS, 1>, k_stage_tiled2d<MIXED, NS, 2>, smem);
    if (!resf) resf = persistent_blocks(k_stage_tiled2d<MIXED, NS, 1, true>,
                                        k_stage_tiled2d<MIXED, NS, 2, true>, smem);
    if (!hbox || (bf && !hbox->bflux)) return -1;
    const int resident = bf ? resf : res;
    if (resident <= 0 || nitems <= 0) return -1;
    const unsigned grid = (unsigned)(nitems < resident ? nitems : resident);
    if (bf && stage == 1)
        k_stage_tiled2d<MIXED, NS, 1, true><<<grid, t2::NT, smem, s>>>(*hbox, nitems, work);
    else if (bf)
        k_stage_tiled2d<MIXED, NS, 2, true><<<grid, t2::NT, smem, s>>>(*hbox, nitems, work);
    else if (stage == 1)
        k_stage_tiled2d<MIXED, NS, 1><<<grid, t2::NT, smem, s>>>(*hbox, nitems, work);
    else
        k_stage_tiled2d<MIXED, NS, 2><<<grid, t2::NT, smem, s>>>(*hbox, nitems, work);
    return 1;
}

}  // namespace vb
