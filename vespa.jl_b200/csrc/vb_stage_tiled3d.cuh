// vb_stage_tiled3d.cuh -- tiled, z-marching fused RK2 stage kernel for 3D
// uniform meshes (the hot path of the 256^3 benchmark).
//
// A block owns a 16 x 16 column tile of cells and marches along z through a
// chunk of planes.  For every plane, one thread issues TMA loads (4-D tensor
// map over x, y, z and the five conserved fields) of the tile interior and of
// its four 2-cell halo strips into a shared-memory stage buffer, NS planes
// ahead of use.  Each loaded cell is converted to primitives exactly once; the
// x/y minmod slopes of each cell are computed once into shared memory; every
// face flux is evaluated exactly once (x and y faces from shared memory, the z
// face in registers from the thread's own column); the flux divergence of a
// cell is summed in the reference's per-cell order (same LO_* classes as the
// cell-centric kernel) and the stage epilogue writes the new state.  Stage 2
// also folds the next step's CFL maximum.
//
// Requirements (checked on the host): nx % 16 == 0, ny % 16 == 0, nz >= 2, and
// a periodic axis is periodic on both sides.  Boundary-flux capture is not
// done here (the cell-centric kernel handles grids with bflux enabled).
#pragma once

#include <cstring>

#include "vb_launch.h"
#include "vb_stage_generic.cuh"

namespace vb {

namespace t3 {

constexpr int TX = 16, TY = 16, NT = TX * TY;
constexpr int NH = 4 * TY + 4 * TX;  // halo cells: two 2-wide x strips, two 2-high y strips
constexpr int UPLANE = (NT + NH) * 5;  // float64 values per staged plane
// TMA box regions inside a staged plane (float64 offsets), each [5][..] field-major
constexpr int U_XLO = NT * 5;
constexpr int U_XHI = U_XLO + 2 * TY * 5;
constexpr int U_YLO = U_XHI + 2 * TY * 5;
constexpr int U_YHI = U_YLO + 2 * TX * 5;
constexpr uint32_t PLANE_BYTES = UPLANE * 8;
// every TMA destination in shared memory is 128-byte aligned
static_assert((U_XLO * 8) % 128 == 0 && (U_XHI * 8) % 128 == 0 && (U_YLO * 8) % 128 == 0 &&
                  (U_YHI * 8) % 128 == 0 && (UPLANE * 8) % 128 == 0,
              "TMA destinations must be 128-byte aligned");

// halo index -> staged-plane offset of field 0 (add f * region field stride)
__device__ __forceinline__ int halo_uoff(int h, int f)
{
    if (h < 32) return U_XLO + f * (2 * TY) + (h >> 1) * 2 + (h & 1);
    if (h < 64) { h -= 32; return U_XHI + f * (2 * TY) + (h >> 1) * 2 + (h & 1); }
    if (h < 96) { h -= 64; return U_YLO + f * (2 * TX) + (h >> 4) * TX + (h & 15); }
    h -= 96;
    return U_YHI + f * (2 * TX) + (h >> 4) * TX + (h & 15);
}
// halo index of local cell (lx, ly) outside the interior (star stencil only)
__device__ __forceinline__ int halo_idx(int lx, int ly)
{
    if (lx < 0) return ly * 2 + (lx + 2);
    if (lx >= TX) return 32 + ly * 2 + (lx - TX);
    if (ly < 0) return 64 + (ly + 2) * TX + lx;
    return 96 + (ly - TY) * TX + lx;
}

template <typename T, int NS>
struct Smem {
    double u[NS][UPLANE];     // TMA stage buffers (raw conserved state)
    T wi[5][NT];              // primitives of the current plane's interior
    T wh[3][5][NH];           // primitives of the halo strips, by plane (ring of 3)
    T sx[5][NT], sy[5][NT];   // x / y slopes of the interior cells
    T sxh[5][2 * TY];         // x slopes of the cells just outside x (lx = -1, TX)
    T syh[5][2 * TX];         // y slopes of the cells just outside y (ly = -1, TY)
    double fx[5][TY * (TX + 1)];  // x-face area * flux, face fx between lx = fx-1 and fx
    double fy[5][(TY + 1) * TX];  // y-face area * flux
    uint64_t bar[NS];
};

}  // namespace t3

// Precision policy: T = double runs the reference's exact float64 algebra;
// T = float runs the fast float32 Riemann solver.
template <typename T, int DIM>
__device__ __forceinline__ void tiled_hllc(const T WL[5], const T WR[5], double gamma, T F[5])
{
    if constexpr (sizeof(T) == 4)
        hllc_flux_fast<DIM>(WL, WR, (float)gamma, 1.0f / ((float)gamma - 1.0f), F);
    else
        hllc_flux<T, DIM>(WL, WR, gamma, F);
}

__device__ __forceinline__ int lo_class(int64_t c, int64_t n, bool periodic)
{
    if (c > 0) return LO_BEFORE;
    return (periodic && n > 1) ? LO_AFTER : LO_SELF;
}

__device__ __forceinline__ void prefetch_l1(const void *p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// compute_dt's per-cell term of a new state, exactly as src/driver.jl:178-185
__device__ __forceinline__ double cfl_term_exact(const double un[5], const Geom &g, double m)
{
    double W[5];
    cons2prim(un, g.gamma, W);
    const double cs = sound_speed(W, g.gamma);
    m = nan_max(m, (fabs(W[1]) + cs) / g.w[0]);
    m = nan_max(m, (fabs(W[2]) + cs) / g.w[1]);
    return nan_max(m, (fabs(W[3]) + cs) / g.w[2]);
}

// The same over x and y only (2D grids: compute_dt loops d in 1:N)
__device__ __forceinline__ double cfl_term2d_exact(const double un[5], const Geom &g, double m)
{
    double W[5];
    cons2prim(un, g.gamma, W);
    const double cs = sound_speed(W, g.gamma);
    m = nan_max(m, (fabs(W[1]) + cs) / g.w[0]);
    return nan_max(m, (fabs(W[2]) + cs) / g.w[1]);
}

// Persistent: a grid of (2 x SMs) blocks pulls work items from work[STAGE-1].
// An item is a column tile and a z chunk of one box (within a box, item =
// chunk * ntiles + tile, so concurrently processed items are spatial
// neighbours and share halo planes in L2).
//
// BATCH = false: one box, passed by value as a kernel parameter (its geometry
// and tensor maps are then read from the constant bank); BATCH = true: the box
// of each item is looked up in the device table.
template <bool BATCH>
__device__ __forceinline__ const BoxDesc &box_of(const BoxDesc &box0, const BoxDesc *boxes,
                                                 const int *item_box, int item)
{
    if constexpr (BATCH)
        return boxes[item_box[item]];
    else
        return box0;
}

template <typename T, int NS, int STAGE, bool BATCH>
__global__ void __launch_bounds__(256, 2)
k_stage_tiled3d(const __grid_constant__ BoxDesc box0, const BoxDesc *__restrict__ boxes,
                const int *__restrict__ item_box, int nitems, unsigned int *work)
{
    using namespace t3;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    t3::Smem<T, NS> &S = *reinterpret_cast<t3::Smem<T, NS> *>(smem_raw);
    __shared__ double red[32];
    __shared__ int item_sh;

    const int t = threadIdx.x;
    const int tx = t & (TX - 1), ty = t >> 4;

    if (t == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&S.bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    bool timed_out = false;
    int qb = 0;  // staged planes this block consumed before the current item
    for (;;) {
    if (t == 0) item_sh = (int)atomicAdd(&work[STAGE - 1], 1u);
    __syncthreads();
    const int item = item_sh;  // rewritten only after this item's barriers
    if (item >= nitems) break;
    const BoxDesc &B = box_of<BATCH>(box0, boxes, item_box, item);
    Ctrl *ctrl = B.ctrl;
    if (!ctrl->active) {  // uniform: the box is not stepping
        __syncthreads();  // everyone has read item_sh before thread 0 rewrites it
        continue;
    }
    const Geom &g = B.g;
    const CUtensorMap *tm = B.map[STAGE - 1];
    const double *__restrict__ Uin = STAGE == 1 ? B.U : B.U1;
    const double *U0 = B.U;
    double *Uout = STAGE == 1 ? B.U1 : B.U;
    const int kz = B.kz, ntx = B.ntx, ntiles = B.ntiles;
    const int nx = (int)g.n[0], ny = (int)g.n[1], nz = (int)g.n[2];
    const bool perx = g.bc_lo[0] == BC_PERIODIC, pery = g.bc_lo[1] == BC_PERIODIC;
    const bool perz = g.bc_lo[2] == BC_PERIODIC;
    const double gamma = g.gamma;
    const double invV = ctrl->invV;
    double invdt = 0.0;
    const int local = item - B.item0;
    const int tile = local % ntiles;
    const int x0 = (tile % ntx) * TX, y0 = (tile / ntx) * TY;
    const int k0 = (local / ntiles) * kz;
    const int k1 = min(nz, k0 + kz);
    const int nplanes = (k1 - k0) + 4;  // planes k0-2 .. k1+1
    // tile edges that are domain boundaries (ghost states instead of halo data)
    const bool xlo_bnd = !perx && x0 == 0, xhi_bnd = !perx && x0 + TX == nx;
    const bool ylo_bnd = !pery && y0 == 0, yhi_bnd = !pery && y0 + TY == ny;

    auto issue = [&](int q) {  // load staged plane q (plane k0 - 2 + q) of this item
        const int p = k0 - 2 + q;
        const int z = perz ? ((p % nz) + nz) % nz : p;  // out-of-range z reads the zero fill
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
    if (t == 0) {
        fence_proxy_async_smem();  // the previous item read these buffers
        for (int q = 0; q < NS && q < nplanes; ++q) issue(q);
    }

    // Wait for staged plane q, convert the own cell (and optionally the halo
    // strips into ring slot q % 3), then release the buffer for plane q + NS.
    auto consume = [&](int q, T Wown[5], bool halo) {
        const int b = (qb + q) % NS;
        if (!mbar_wait(&S.bar[b], ((qb + q) / NS) & 1, WAIT_LIMIT_NS)) timed_out = true;
        const double *u = S.u[b];
        {
            double uu[5], w[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) uu[f] = u[f * NT + t];
            cons2prim(uu, gamma, w);
#pragma unroll
            for (int f = 0; f < 5; ++f) Wown[f] = T(w[f]);
        }
        if (halo && t < NH) {
            double uu[5], w[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) uu[f] = u[halo_uoff(t, f)];
            cons2prim(uu, gamma, w);
#pragma unroll
            for (int f = 0; f < 5; ++f) S.wh[q % 3][f][t] = T(w[f]);
        }
    };
    auto release = [&](int q) {
        if (t == 0 && q + NS < nplanes) {
            fence_proxy_async_smem();
            issue(q + NS);
        }
    };

    // ---- prologue: planes k0-2 .. k0+1
    T Wa[5], Wb[5], Wz0[5], Wz1[5], Wz2[5];
    consume(0, Wa, false);
    __syncthreads();
    release(0);
    consume(1, Wb, false);
    __syncthreads();
    release(1);
    consume(2, Wz0, true);
    __syncthreads();
    release(2);
    consume(3, Wz1, true);
    __syncthreads();
    release(3);

    const int bz_lo = g.bc_lo[2], bz_hi = g.bc_hi[2];
    const T half = T(0.5), mhalf = T(-0.5);
    T hz[5], Fzlo[5];
    {
        // slope_z(k0) from W(k0-1), W(k0), W(k0+1)
        const bool gl = !perz && k0 == 0;          // W(k0-1) is a ghost
        const bool gh = !perz && k0 + 1 >= nz;     // W(k0+1) is a ghost
        T loz[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const T wl = gl ? ((bz_lo == BC_REFLECTING && f == 3) ? -Wz0[f] : Wz0[f]) : Wb[f];
            const T wr = gh ? ((bz_hi == BC_REFLECTING && f == 3) ? -Wz0[f] : Wz0[f]) : Wz1[f];
            const T s = limited_slope<T>(wl, Wz0[f], wr);
            hz[f] = face_val(Wz0[f], half, s);
            loz[f] = face_val(Wz0[f], mhalf, s);
        }
        if (gl) {
            T gst[5];
            ghost_state<T>(loz, bz_lo, 2, gst);
            tiled_hllc<T, 3>(gst, loz, gamma, Fzlo);
        } else {
            // hi face value of plane k0-1: slope from W(k0-2), W(k0-1), W(k0)
            const bool gll = !perz && k0 - 2 < 0;
            T hzm[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const T wl = gll ? ((bz_lo == BC_REFLECTING && f == 3) ? -Wb[f] : Wb[f]) : Wa[f];
                hzm[f] = face_val(Wb[f], half, limited_slope<T>(wl, Wb[f], Wz0[f]));
            }
            tiled_hllc<T, 3>(hzm, loz, gamma, Fzlo);
        }
    }

    const double ax = g.area[0], ay = g.area[1], az = g.area[2];
    const int gx = x0 + tx, gy = y0 + ty;
    const int cx = lo_class(gx, nx, perx), cy = lo_class(gy, ny, pery);
    const int bx_lo = g.bc_lo[0], bx_hi = g.bc_hi[0], by_lo = g.bc_lo[1], by_hi = g.bc_hi[1];
    double unp[5];  // previous plane's new state: its CFL term is folded one plane later

    for (int k = k0; k < k1; ++k) {
        const int q = k - k0 + 4;        // staged index of plane k + 2
        const int slot = (q - 2) % 3;    // ring slot of plane k's halo
        const int64_t lin = (int64_t)gx + (int64_t)nx * ((int64_t)gy + (int64_t)ny * k);
        if (tx == 0) {  // one 128-byte row per field: warm L1 for the epilogue's loads
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                prefetch_l1(Uin + (int64_t)f * g.ncell + lin);
                if constexpr (STAGE == 2) prefetch_l1(U0 + (int64_t)f * g.ncell + lin);
            }
        }
        consume(q, Wz2, true);
        if constexpr (STAGE == 2)
            if (k > k0) invdt = cfl_term_exact(unp, g, invdt);  // overlaps the cons2prim chain
#pragma unroll
        for (int f = 0; f < 5; ++f) S.wi[f][t] = Wz0[f];
        __syncthreads();  // (1) plane k primitives complete; stage buffer q consumed
        release(q);

        // ---- slopes of the interior cells (x and y) ----
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const T wc = Wz0[f];
            T wl, wr;
            if (tx > 0) wl = S.wi[f][t - 1];
            else if (xlo_bnd) wl = (bx_lo == BC_REFLECTING && f == 1) ? -wc : wc;
            else wl = S.wh[slot][f][halo_idx(-1, ty)];
            if (tx < TX - 1) wr = S.wi[f][t + 1];
            else if (xhi_bnd) wr = (bx_hi == BC_REFLECTING && f == 1) ? -wc : wc;
            else wr = S.wh[slot][f][halo_idx(TX, ty)];
            S.sx[f][t] = limited_slope<T>(wl, wc, wr);
            if (ty > 0) wl = S.wi[f][t - TX];
            else if (ylo_bnd) wl = (by_lo == BC_REFLECTING && f == 2) ? -wc : wc;
            else wl = S.wh[slot][f][halo_idx(tx, -1)];
            if (ty < TY - 1) wr = S.wi[f][t + TX];
            else if (yhi_bnd) wr = (by_hi == BC_REFLECTING && f == 2) ? -wc : wc;
            else wr = S.wh[slot][f][halo_idx(tx, TY)];
            S.sy[f][t] = limited_slope<T>(wl, wc, wr);
        }
        // ---- slopes of the cells just outside the tile (never domain ghosts) ----
        if (t >= 160 && t < 224) {
            const int j = t - 160;
            const int side = (j >> 4) & 1, i = j & 15;
            if (j < 32) {  // x slope at lx = -1 (side 0) or lx = TX (side 1), row i
                if (!(side ? xhi_bnd : xlo_bnd)) {
                    const int lx = side ? TX : -1;
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const T wc = S.wh[slot][f][halo_idx(lx, i)];
                        const T wl = side ? S.wi[f][i * TX + TX - 1] : S.wh[slot][f][halo_idx(-2, i)];
                        const T wr = side ? S.wh[slot][f][halo_idx(TX + 1, i)] : S.wi[f][i * TX];
                        S.sxh[f][j] = limited_slope<T>(wl, wc, wr);
                    }
                }
            } else {       // y slope at ly = -1 (side 0) or ly = TY (side 1), column i
                if (!(side ? yhi_bnd : ylo_bnd)) {
                    const int ly = side ? TY : -1;
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const T wc = S.wh[slot][f][halo_idx(i, ly)];
                        const T wl = side ? S.wi[f][(TY - 1) * TX + i] : S.wh[slot][f][halo_idx(i, -2)];
                        const T wr = side ? S.wh[slot][f][halo_idx(i, TY + 1)] : S.wi[f][i];
                        S.syh[f][j - 32] = limited_slope<T>(wl, wc, wr);
                    }
                }
            }
        }
        __syncthreads();  // (2) slopes ready

        // ---- z face k+1/2 from the own column (registers), in the same phase
        //      as the x/y faces so the independent solves can overlap ----
        T Fzhi[5], hz1[5];
        {
            T zr[5];  // right state of the z face
            const bool plane_k1 = perz || k + 1 < nz;   // plane k+1 exists
            if (plane_k1) {
                const bool gh = !perz && k + 2 >= nz;
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    const T wr = gh ? ((bz_hi == BC_REFLECTING && f == 3) ? -Wz1[f] : Wz1[f]) : Wz2[f];
                    const T s = limited_slope<T>(Wz0[f], Wz1[f], wr);
                    zr[f] = face_val(Wz1[f], mhalf, s);
                    hz1[f] = face_val(Wz1[f], half, s);
                }
            } else {
                ghost_state<T>(hz, bz_hi, 2, zr);
#pragma unroll
                for (int f = 0; f < 5; ++f) hz1[f] = hz[f];
            }
            tiled_hllc<T, 3>(hz, zr, gamma, Fzhi);
        }

        // ---- x and y faces: each thread its lo faces; 32 threads the hi edges ----
        {
            // x face fx = tx in row ty: between lx = tx-1 and tx
            T WL[5], WR[5], F[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) WR[f] = face_val(S.wi[f][t], mhalf, S.sx[f][t]);
            if (tx > 0) {
#pragma unroll
                for (int f = 0; f < 5; ++f) WL[f] = face_val(S.wi[f][t - 1], half, S.sx[f][t - 1]);
            } else if (xlo_bnd) {
                ghost_state<T>(WR, bx_lo, 0, WL);
            } else {
#pragma unroll
                for (int f = 0; f < 5; ++f)
                    WL[f] = face_val(S.wh[slot][f][halo_idx(-1, ty)], half, S.sxh[f][ty]);
            }
            tiled_hllc<T, 1>(WL, WR, gamma, F);
#pragma unroll
            for (int f = 0; f < 5; ++f) S.fx[f][ty * (TX + 1) + tx] = ax * double(F[f]);
            // y face fy = ty in column tx: between ly = ty-1 and ty
#pragma unroll
            for (int f = 0; f < 5; ++f) WR[f] = face_val(S.wi[f][t], mhalf, S.sy[f][t]);
            if (ty > 0) {
#pragma unroll
                for (int f = 0; f < 5; ++f) WL[f] = face_val(S.wi[f][t - TX], half, S.sy[f][t - TX]);
            } else if (ylo_bnd) {
                ghost_state<T>(WR, by_lo, 1, WL);
            } else {
#pragma unroll
                for (int f = 0; f < 5; ++f)
                    WL[f] = face_val(S.wh[slot][f][halo_idx(tx, -1)], half, S.syh[f][tx]);
            }
            tiled_hllc<T, 2>(WL, WR, gamma, F);
#pragma unroll
            for (int f = 0; f < 5; ++f) S.fy[f][ty * TX + tx] = ay * double(F[f]);
        }
        if (t >= 224) {
            const int j = t - 224;
            T WL[5], WR[5], F[5];
            if (j < 16) {  // x face fx = TX in row j
                const int c = j * TX + TX - 1;
#pragma unroll
                for (int f = 0; f < 5; ++f) WL[f] = face_val(S.wi[f][c], half, S.sx[f][c]);
                if (xhi_bnd) {
                    ghost_state<T>(WL, bx_hi, 0, WR);
                } else {
#pragma unroll
                    for (int f = 0; f < 5; ++f)
                        WR[f] = face_val(S.wh[slot][f][halo_idx(TX, j)], mhalf, S.sxh[f][16 + j]);
                }
                tiled_hllc<T, 1>(WL, WR, gamma, F);
#pragma unroll
                for (int f = 0; f < 5; ++f) S.fx[f][j * (TX + 1) + TX] = ax * double(F[f]);
            } else {       // y face fy = TY in column i
                const int i = j - 16;
                const int c = (TY - 1) * TX + i;
#pragma unroll
                for (int f = 0; f < 5; ++f) WL[f] = face_val(S.wi[f][c], half, S.sy[f][c]);
                if (yhi_bnd) {
                    ghost_state<T>(WL, by_hi, 1, WR);
                } else {
#pragma unroll
                    for (int f = 0; f < 5; ++f)
                        WR[f] = face_val(S.wh[slot][f][halo_idx(i, TY)], mhalf, S.syh[f][16 + i]);
                }
                tiled_hllc<T, 2>(WL, WR, gamma, F);
#pragma unroll
                for (int f = 0; f < 5; ++f) S.fy[f][TY * TX + i] = ay * double(F[f]);
            }
        }
        __syncthreads();  // (3) fluxes ready

        // ---- flux divergence in the reference's order, then the stage update ----
        const int cz = lo_class(k, nz, perz);
        const bool interior = cx == LO_BEFORE && cy == LO_BEFORE && cz == LO_BEFORE;
        double un[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            // area * flux per face; a lo contribution adds (-area) * F, which is
            // exactly -(area * F)
            const double gxl = S.fx[f][ty * (TX + 1) + tx];
            const double gxh = S.fx[f][ty * (TX + 1) + tx + 1];
            const double gyl = S.fy[f][ty * TX + tx];
            const double gyh = S.fy[f][(ty + 1) * TX + tx];
            const double gzl = az * double(Fzlo[f]), gzh = az * double(Fzhi[f]);
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
            const int64_t i = (int64_t)f * g.ncell + lin;
            if constexpr (STAGE == 1) {
                un[f] = __ldg(Uin + i) - invV * a;
            } else {
                un[f] = 0.5 * U0[i] + 0.5 * (__ldg(Uin + i) - invV * a);
            }
            Uout[i] = un[f];
        }
        if constexpr (STAGE == 2) {
#pragma unroll
            for (int f = 0; f < 5; ++f) unp[f] = un[f];
        }
        // ---- advance the column registers ----
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            Wz0[f] = Wz1[f];
            Wz1[f] = Wz2[f];
            hz[f] = hz1[f];
            Fzlo[f] = Fzhi[f];
        }
    }
    if constexpr (STAGE == 2) invdt = cfl_term_exact(unp, g, invdt);  // the item's last plane
    qb += nplanes;
    if (timed_out && t == 0) atomicOr(&ctrl->flags, CTRL_F_TIMEOUT);
    if constexpr (STAGE == 2) block_max_to(&ctrl->invdt_bits, invdt, red);  // this box's CFL max
    }  // work items
}

}  // namespace vb

namespace vb {

// Resident blocks of a persistent kernel on the current device (all SMs), with
// its dynamic shared memory opted in once.
template <typename K>
int persistent_blocks(K kernel1, K kernel2, size_t smem)
{
    if (cudaFuncSetAttribute(kernel1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(kernel2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
        return -1;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel2, t3::NT, smem) != cudaSuccess ||
        per_sm < 1)
        return -1;
    return sms * per_sm;
}

// Host-side launch of the persistent tiled 3D stage kernel: as many blocks as
// can be resident, pulling (box, tile, z-chunk) items.  hbox (host) set: one
// box passed by value; else the device table `boxes` with `item_box`.
template <typename T, int NS>
int launch_tiled3d(const BoxDesc *hbox, const BoxDesc *boxes, const int *item_box, int nitems,
                   unsigned int *work, int stage, cudaStream_t s)
{
    const size_t smem = sizeof(t3::Smem<T, NS>);
    static int res1 = 0, resb = 0;
    if (!res1) res1 = persistent_blocks(k_stage_tiled3d<T, NS, 1, false>,
                                        k_stage_tiled3d<T, NS, 2, false>, smem);
    if (!resb) resb = persistent_blocks(k_stage_tiled3d<T, NS, 1, true>,
                                        k_stage_tiled3d<T, NS, 2, true>, smem);
    const int resident = hbox ? res1 : resb;
    if (resident <= 0 || nitems <= 0) return -1;
    const unsigned grid = (unsigned)(nitems < resident ? nitems : resident);
    BoxDesc box0;
    if (hbox) box0 = *hbox;
    else std::memset(&box0, 0, sizeof box0);
    if (hbox && stage == 1)
        k_stage_tiled3d<T, NS, 1, false><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (hbox)
        k_stage_tiled3d<T, NS, 2, false><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (stage == 1)
        k_stage_tiled3d<T, NS, 1, true><<<grid, t3::NT, smem, s>>>(box0, boxes, item_box, nitems, work);
    else
        k_stage_tiled3d<T, NS, 2, true><<<grid, t3::NT, smem, s>>>(box0, boxes, item_box, nitems, work);
    return 1;
}

}  // namespace vb
