// vb_stage_tiled3d_mixed.cuh -- VB_MIXED tiled 3D stage kernel.
//
// 16 x 16 column tiles marching z with a TMA stage pipeline and a persistent
// work queue (vb_stage_tiled3d.cuh), specialised for float32 reconstruction
// and Riemann solves with float64 state:
//   - primitives live in a ring of three float32 planes (k, k+1, k+2) whose
//     layout puts the x/y halo and, at a non-periodic boundary, mirror ghost
//     cells beside the interior, so every slope and face formula is the
//     interior one;
//   - every thread reconstructs both states of its own lo x face and lo y face
//     from the four cells across each (the neighbour's slope is recomputed
//     rather than exchanged, which saves a barrier per plane) and solves the
//     pair as one packed float32x2 HLLC (vb_hllc_x2.cuh, faces rotated into
//     their normal frame); warp 7 adds the tile's hi-edge faces;
//   - the z face runs in registers down the thread's column, solved before
//     the plane's first barrier by warps 4..7 and after it by warps 0..3, so
//     that it balances the halo conversions (warps 0..3) and the edge faces
//     (warp 7) across the two phases;
//   - x/y face fluxes are stored once in float32 and multiplied by the face
//     area in float64 where the divergence reads them;
//     the flux divergence and the stage update stay in float64.
// Two barriers per plane: (1) plane k+2 converted, (2) fluxes of plane k ready.
#pragma once

#include "vb_hllc_x2.cuh"
#include "vb_stage_tiled3d.cuh"

namespace vb {

namespace t3m {

using t3::NH;
using t3::NT;
using t3::TX;
using t3::TY;

// Primitive planes in shared memory: a ring of three planes (k, k+1, k+2).
// Per plane and field, 384 floats: rows ly = -2..17 of columns lx = 0..15
// (row-major, 16 wide, so a warp's two rows never share a bank), then the
// x halo columns lx = -2, -1, 16, 17 of rows 0..15 (4 per row).  At a
// non-periodic boundary the halo holds mirror ghosts (the boundary cells
// reflected by ghost_state), which makes every face and slope formula the
// same as in the interior.
constexpr int PC = 384;          // floats per field
constexpr int PSLOT = 5 * PC;    // floats per plane
constexpr int XS = 320;          // first x halo column entry
__host__ __device__ constexpr int wrow(int lx, int ly) { return (ly + 2) * 16 + lx; }
__host__ __device__ constexpr int wxs(int lx, int ly)
{
    return XS + ly * 4 + (lx < 0 ? lx + 2 : lx - 14);
}

template <int NS>
struct Smem {
    double u[NS][t3::UPLANE];  // TMA stage buffers (raw conserved state)
    double ep[2][5][NT];       // own-cell epilogue inputs (Uin, U0), fetched by cp.async
    float w[3][PSLOT];         // primitive ring
    float gx[5][TY * (TX + 1)];  // x-face flux (float32; times the area in the epilogue)
    float gy[5][(TY + 1) * TX];  // y-face flux
    uint64_t bar[NS];
};

// minmod slope of (l, c, r) (limited_slope, src/reconstruct.jl:6-16) as a
// clamp: minmod(a, b) = a clamped to [min(0, b), max(0, b)].  Four min/max
// instead of a product, two compares and two selects; the value equals the
// reference's except where a * b underflows to zero in float32 (then the
// reference gives 0 and the clamp the smaller difference, both below 1e-22).
__device__ __forceinline__ float mm(float l, float c, float r)
{
    const float a = c - l, b = r - c;
    return fminf(fmaxf(a, fminf(0.f, b)), fmaxf(0.f, b));
}

// cons2prim for VB_MIXED (src/eos.jl:8-25): velocities and the
// total-energy-minus-kinetic pressure recovery in float64, results rounded
// to float32.  1/rho comes from the float64 approximate-reciprocal
// instruction refined by two Newton-Raphson steps x <- x (2 - rho x)
// (quadratic convergence: the seed's relative error e becomes e^4, far below
// float64 rounding) instead of a float64 division.
__device__ __forceinline__ void cons2prim_mixed(const double U[5], double g, float W[5])
{
    const double rho = U[0];
    double inv;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(inv) : "d"(rho));
    inv = inv * (2.0 - rho * inv);
    inv = inv * (2.0 - rho * inv);
    const double vx = U[1] * inv, vy = U[2] * inv, vz = U[3] * inv;
    const double kinetic = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
    const double p = (g - 1.0) * (U[4] - kinetic);
    W[0] = (float)rho;
    W[1] = (float)vx;
    W[2] = (float)vy;
    W[3] = (float)vz;
    W[4] = (float)fmax(p, 1e-12 * kinetic);
}

// VB_MIXED CFL term of a new float64 state: compute_dt's (|v_d| + c) / w_d
// (src/driver.jl:178-185) from the mixed primitives, wave speeds in float32
// (a dt estimate within float32 rounding of the float64 one).  The running
// maximum m stays in float32 (the conversion to float64 is exact and
// monotonic, so the maximum is the same); NaN wins, as in nan_max.
__device__ __forceinline__ float cfl_term(const double un[5], double gamma, float gf, float iw0,
                                          float iw1, float iw2, float m)
{
    float W[5];
    cons2prim_mixed(un, gamma, W);
    const float cs = sqrt_approx(gf * W[4] * rcp_approx(W[0]));
    const float t = fmaxf(fmaxf((fabsf(W[1]) + cs) * iw0, (fabsf(W[2]) + cs) * iw1),
                          (fabsf(W[3]) + cs) * iw2);
    return (t > m || t != t) ? t : m;
}

// cfl_term and, GRAV, the cell's free-fall rate (src/gravity.jl:439-441,
// float64, folded into the float32 maximum)
template <bool GRAV>
__device__ __forceinline__ float cfl_mixed(const double un[5], const Geom &g, float gf, float iw0,
                                           float iw1, float iw2, float m)
{
    float r = cfl_term(un, g.gamma, gf, iw0, iw1, iw2, m);
    if constexpr (GRAV) {
        const float t = (float)gravity_invdt(g.grav_G, un[0]);
        r = (t > r || t != t) ? t : r;
    }
    return r;
}

// the same over x and y only (2D grids)
__device__ __forceinline__ double cfl_term2d(const double un[5], const Geom &g, double m)
{
    float W[5];
    cons2prim_mixed(un, g.gamma, W);
    const float cs = sqrt_approx((float)g.gamma * W[4] * rcp_approx(W[0]));
    const float t = fmaxf((fabsf(W[1]) + cs) * (float)g.invw[0], (fabsf(W[2]) + cs) * (float)g.invw[1]);
    return nan_max(m, (double)t);
}

}  // namespace t3m

namespace t3m {

// Left / right states of a packed face pair, lane x an x face and lane y a y
// face, each reconstructed from the four cells across it (ring offsets o[0..3]
// along the face normal: two cells behind the face, two ahead).  Components
// come out in the face-normal frame (rho, u_n, u_t1, u_t2, p).
__device__ __forceinline__ void face_pair(const float *wk, const int ox[4], const int oy[4],
                                          Face2 &L, Face2 &R)
{
    f2 l[5], r[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        const int fx = j, fy = j == 1 ? 2 : (j == 2 ? 1 : j);
        const float *px = wk + fx * PC, *py = wk + fy * PC;
        const f2 a0(px[ox[0]], py[oy[0]]), a1(px[ox[1]], py[oy[1]]);
        const f2 a2(px[ox[2]], py[oy[2]]), a3(px[ox[3]], py[oy[3]]);
        // the slopes of the cells behind and ahead of the face share the
        // difference across it, so they share the clamp bounds (see mm)
        const f2 d1 = a1 - a0, d2 = a2 - a1, d3 = a3 - a2;
        const float lox = fminf(0.f, d2.v.x), hix = fmaxf(0.f, d2.v.x);
        const float loy = fminf(0.f, d2.v.y), hiy = fmaxf(0.f, d2.v.y);
        const f2 sl(fminf(fmaxf(d1.v.x, lox), hix), fminf(fmaxf(d1.v.y, loy), hiy));
        const f2 sc(fminf(fmaxf(d3.v.x, lox), hix), fminf(fmaxf(d3.v.y, loy), hiy));
        l[j] = fma2(f2::splat(0.5f), sl, a1);
        r[j] = fma2(f2::splat(-0.5f), sc, a2);
    }
    L = Face2{l[0], l[1], l[2], l[3], l[4]};
    R = Face2{r[0], r[1], r[2], r[3], r[4]};
}

// flux of a packed face pair into the x / y face arrays (un-rotating the y
// face's momentum components); the epilogue multiplies by the face area
__device__ __forceinline__ void store_pair(float (*gx)[TY * (TX + 1)], float (*gy)[(TY + 1) * TX],
                                           int ix, int iy, const f2 F[5])
{
    gx[0][ix] = F[0].v.x;  gy[0][iy] = F[0].v.y;
    gx[1][ix] = F[1].v.x;  gy[2][iy] = F[1].v.y;
    gx[2][ix] = F[2].v.x;  gy[1][iy] = F[2].v.y;
    gx[3][ix] = F[3].v.x;  gy[3][iy] = F[3].v.y;
    gx[4][ix] = F[4].v.x;  gy[4][iy] = F[4].v.y;
}

}  // namespace t3m

template <int NS, int STAGE, bool BATCH, bool GRAV = false, bool BF = false>
__global__ void __launch_bounds__(256, 2)
k_stage_tiled3d_mixed(const __grid_constant__ BoxDesc box0, const BoxDesc *__restrict__ boxes,
                      const int *__restrict__ item_box, int nitems, unsigned int *work)
{
    using namespace t3;
    using namespace t3m;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // check build only: TMA destinations need a 128-byte aligned base (uniform)
    if (!VB_DCHECK(((uintptr_t)smem_raw & 127) == 0)) return;
    t3m::Smem<NS> &S = *reinterpret_cast<t3m::Smem<NS> *>(smem_raw);
    __shared__ double red[32];
    __shared__ int item_sh;
    __shared__ int stall_sh;  // a stage load's bounded wait gave up

    const int t = threadIdx.x;
    const int tx = t & (TX - 1), ty = t >> 4;
    const int warp = t >> 5, lane = t & 31;
    // ring offsets of the own cell and of the cells across the own lo x / lo y faces
    const int o_c = wrow(tx, ty);
    const int ox[4] = {tx >= 2 ? o_c - 2 : wxs(tx - 2, ty), tx >= 1 ? o_c - 1 : wxs(-1, ty), o_c,
                       tx <= TX - 2 ? o_c + 1 : wxs(TX, ty)};
    const int oy[4] = {o_c - 32, o_c - 16, o_c, o_c + 16};
    // halo cell h = t (t < NH): staged-plane offset and ring offset
    const int h_u = halo_uoff(t < NH ? t : 0, 0);
    const int h_w = t < 32   ? wxs(-2 + (t & 1), t >> 1)
                    : t < 64 ? wxs(TX + (t & 1), (t - 32) >> 1)
                    : t < 96 ? wrow((t - 64) & 15, -2 + ((t - 64) >> 4))
                             : wrow((t - 96) & 15, TY + ((t - 96) >> 4));
    // the z face is solved before barrier (1) by warps 4..7 (balancing the
    // halo conversions of warps 0..3) and after it by warps 0..3 (balancing
    // the tile's hi-edge faces, solved by warp 7)
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
    const float gf = (float)gamma, ig1 = 1.0f / ((float)gamma - 1.0f);
    const double invV = ctrl->invV;
    const double bscale = BF ? 0.5 * ctrl->dt : 0.0;  // boundary-flux stage weight
    const double ax = g.area[0], ay = g.area[1], az = g.area[2];
    const int bx_lo = g.bc_lo[0], bx_hi = g.bc_hi[0], by_lo = g.bc_lo[1], by_hi = g.bc_hi[1];
    const int bz_lo = g.bc_lo[2], bz_hi = g.bc_hi[2];
    double invdt = 0.0;
    float invdtf = 0.f;  // running CFL maximum of this item
    const float iw0 = (float)g.invw[0], iw1 = (float)g.invw[1], iw2 = (float)g.invw[2];
    const int local = item - B.item0;
    const int tile = local % ntiles;
    const int x0 = (tile % ntx) * TX, y0 = (tile / ntx) * TY;
    int k0, k1;
    chunk_span(nz, kz, B.nchu, local / ntiles, k0, k1);
    const int nplanes = (k1 - k0) + 4;
    const bool xlo_bnd = !perx && x0 == 0, xhi_bnd = !perx && x0 + TX == nx;
    const bool ylo_bnd = !pery && y0 == 0, yhi_bnd = !pery && y0 + TY == ny;
    // this thread's halo strip lies outside the domain: mirror ghosts replace it
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
    // Halo strips of staged plane q into ring slot q % 3 (threads t < NH; a
    // strip outside a non-periodic boundary is left to the mirror ghosts).
    auto halo_c2p = [&](int q, float *ws) {
        if (t < NH && !h_ghost) {
            const double *u = S.u[(qb + q) % NS];
            double uu[5];
            float w[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) uu[f] = u[h_u + f * (2 * TY)];
            cons2prim_mixed(uu, gamma, w);
#pragma unroll
            for (int f = 0; f < 5; ++f) ws[h_w + f * PC] = w[f];
        }
    };
    // Wait for staged plane q and convert the own cell into Wn.  keep = 0:
    // registers only; 1: also into ring slot q % 3 with the mirror ghosts and
    // the halo strips; 2: as 1 without the halo strips (halo_c2p follows).
    auto consume = [&](int q, float Wn[5], int keep, float *ws) {
        const int b = (qb + q) % NS;
        if (!mbar_wait(&S.bar[b], ((qb + q) / NS) & 1, WAIT_LIMIT_NS)) stall_sh = 1;
        const double *u = S.u[b];
        {
            double uu[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) uu[f] = u[f * NT + t];
            cons2prim_mixed(uu, gamma, Wn);
        }
        if (!keep) return;
#pragma unroll
        for (int f = 0; f < 5; ++f) ws[f * PC + o_c] = Wn[f];
        if (xlo_bnd && tx < 2) {
            float *d = ws + wxs(-1 - tx, ty);
#pragma unroll
            for (int f = 0; f < 5; ++f) d[f * PC] = (bx_lo == BC_REFLECTING && f == 1) ? -Wn[f] : Wn[f];
        }
        if (xhi_bnd && tx >= TX - 2) {
            float *d = ws + wxs(2 * TX - 1 - tx, ty);
#pragma unroll
            for (int f = 0; f < 5; ++f) d[f * PC] = (bx_hi == BC_REFLECTING && f == 1) ? -Wn[f] : Wn[f];
        }
        if (ylo_bnd && ty < 2) {
            float *d = ws + wrow(tx, -1 - ty);
#pragma unroll
            for (int f = 0; f < 5; ++f) d[f * PC] = (by_lo == BC_REFLECTING && f == 2) ? -Wn[f] : Wn[f];
        }
        if (yhi_bnd && ty >= TY - 2) {
            float *d = ws + wrow(tx, 2 * TY - 1 - ty);
#pragma unroll
            for (int f = 0; f < 5; ++f) d[f * PC] = (by_hi == BC_REFLECTING && f == 2) ? -Wn[f] : Wn[f];
        }
        if (keep == 1) halo_c2p(q, ws);
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

    float Wa[5], Wb[5], Wc[5], Wd[5];
    consume(0, Wa, 0, nullptr);
    __syncthreads();
    if (stalled(0)) return;
    release(0);
    consume(1, Wb, 0, nullptr);
    __syncthreads();
    if (stalled(1)) return;
    release(1);
    consume(2, Wc, 1, S.w[2]);
    __syncthreads();
    if (stalled(2)) return;
    release(2);
    consume(3, Wd, 1, S.w[0]);
    __syncthreads();
    if (stalled(3)) return;
    release(3);

    // z state entering plane k0: hi face value of k0 and the flux through k0-1/2
    float hz[5];
    float fzl[5];
    {
        const bool gl = !perz && k0 == 0;
        const bool gh = !perz && k0 + 1 >= nz;
        float loz[5], Fzlo[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const float wl = gl ? ((bz_lo == BC_REFLECTING && f == 3) ? -Wc[f] : Wc[f]) : Wb[f];
            const float wr = gh ? ((bz_hi == BC_REFLECTING && f == 3) ? -Wc[f] : Wc[f]) : Wd[f];
            const float s = mm(wl, Wc[f], wr);
            hz[f] = fmaf(0.5f, s, Wc[f]);
            loz[f] = fmaf(-0.5f, s, Wc[f]);
        }
        if (gl) {
            float gst[5];
            ghost_state<float>(loz, bz_lo, 2, gst);
            hllc_flux_fast_bf<3>(gst, loz, gf, ig1, Fzlo);
            if constexpr (BF) {  // z-lo domain face of cell (x, y, 0)
                const double Fd[5] = {Fzlo[0], Fzlo[1], Fzlo[2], Fzlo[3], Fzlo[4]};
                bflux_add(g, B.bflux, 2, 0, (int64_t)(x0 + tx) + (int64_t)nx * (y0 + ty), bscale, az, Fd);
            }
        } else {
            const bool gll = !perz && k0 - 2 < 0;
            float hzm[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const float wl = gll ? ((bz_lo == BC_REFLECTING && f == 3) ? -Wb[f] : Wb[f]) : Wa[f];
                hzm[f] = fmaf(0.5f, mm(wl, Wb[f], Wc[f]), Wb[f]);
            }
            hllc_flux_fast_bf<3>(hzm, loz, gf, ig1, Fzlo);
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) fzl[f] = Fzlo[f];
    }

    // flux through k+1/2 from planes k, k+1 (ring) and k+2 (W2) of the own
    // column; advances hz
    auto zsolve = [&](int k, const float *w0, const float *w1, const float W2[5], float Fzhi[5]) {
        float zr[5], hz1[5];
        if (perz || k + 1 < nz) {
            const bool gh = !perz && k + 2 >= nz;
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const float c = w1[f * PC];
                const float r = gh ? ((bz_hi == BC_REFLECTING && f == 3) ? -c : c) : W2[f];
                const float s = mm(w0[f * PC], c, r);
                zr[f] = fmaf(-0.5f, s, c);
                hz1[f] = fmaf(0.5f, s, c);
            }
        } else {
            ghost_state<float>(hz, bz_hi, 2, zr);
#pragma unroll
            for (int f = 0; f < 5; ++f) hz1[f] = hz[f];
        }
        hllc_flux_fast_bf<3>(hz, zr, gf, ig1, Fzhi);
        if constexpr (BF) {
            if (!perz && k + 1 >= nz) {  // z-hi domain face of cell (x, y, nz-1)
                const double Fd[5] = {Fzhi[0], Fzhi[1], Fzhi[2], Fzhi[3], Fzhi[4]};
                bflux_add(g, B.bflux, 2, 1, (int64_t)(x0 + tx) + (int64_t)nx * (y0 + ty), bscale, az, Fd);
            }
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) hz[f] = hz1[f];
    };
    // the own lo x face and lo y face of plane k (ring slot w0), one packed solve
    auto xy_faces = [&](const float *w0, int k) {
        Face2 L, R;
        face_pair(w0, ox, oy, L, R);
        f2 F[5];
        hllc_x2(L, R, gf, ig1, F);
        store_pair(S.gx, S.gy, ty * (TX + 1) + tx, ty * TX + tx, F);
        if constexpr (BF) {
            if (xlo_bnd && tx == 0) {  // x-lo domain face of cell (0, y, k)
                const double Fd[5] = {F[0].v.x, F[1].v.x, F[2].v.x, F[3].v.x, F[4].v.x};
                bflux_add(g, B.bflux, 0, 0, (int64_t)(y0 + ty) + (int64_t)ny * k, bscale, ax, Fd);
            }
            if (ylo_bnd && ty == 0) {  // y-lo domain face of cell (x, 0, k), un-rotated
                const double Fd[5] = {F[0].v.y, F[2].v.y, F[1].v.y, F[3].v.y, F[4].v.y};
                bflux_add(g, B.bflux, 1, 0, (int64_t)(x0 + tx) + (int64_t)nx * k, bscale, ay, Fd);
            }
        }
    };
    // the hi-edge faces (x at fx = TX, y at fy = TY), one pair per lane < 16
    auto edge_faces = [&](const float *w0, int k) {
        const int j = lane;
        const int ex[4] = {wrow(TX - 2, j), wrow(TX - 1, j), wxs(TX, j), wxs(TX + 1, j)};
        const int ey[4] = {wrow(j, TY - 2), wrow(j, TY - 1), wrow(j, TY), wrow(j, TY + 1)};
        Face2 L, R;
        face_pair(w0, ex, ey, L, R);
        f2 F[5];
        hllc_x2(L, R, gf, ig1, F);
        store_pair(S.gx, S.gy, j * (TX + 1) + TX, TY * TX + j, F);
        if constexpr (BF) {
            if (xhi_bnd) {  // x-hi domain face of cell (nx-1, y0+j, k)
                const double Fd[5] = {F[0].v.x, F[1].v.x, F[2].v.x, F[3].v.x, F[4].v.x};
                bflux_add(g, B.bflux, 0, 1, (int64_t)(y0 + j) + (int64_t)ny * k, bscale, ax, Fd);
            }
            if (yhi_bnd) {  // y-hi domain face of cell (x0+j, ny-1, k)
                const double Fd[5] = {F[0].v.y, F[2].v.y, F[1].v.y, F[3].v.y, F[4].v.y};
                bflux_add(g, B.bflux, 1, 1, (int64_t)(x0 + j) + (int64_t)nx * k, bscale, ay, Fd);
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

    float *r0 = S.w[2], *r1 = S.w[0], *r2 = S.w[1];  // ring slots of planes k, k+1, k+2
    for (int k = k0; k < k1; ++k) {
        const int q = k - k0 + 4;
        const float *w0 = r0, *w1 = r1, *w2 = r2;
        const bool inb = VB_DCHECK(lin >= 0 && lin < g.ncell);  // check build only
        if (inb) {
            const double *pa = Uin + lin, *pb = U0 + lin;
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                cp_async8(&S.ep[0][f][t], pa);
                if constexpr (STAGE == 2) cp_async8(&S.ep[1][f][t], pb);
                pa += g.ncell;
                pb += g.ncell;
            }
        }
        cp_async_commit();
        // ---- phase 1: plane k+2 to primitives; the CFL term of plane k-1; the
        //      z face (warps 4..7) or the halo strips (warps 0..3) ----
        float Fzhi[5];
        {
            float Wn[5];
            consume(q, Wn, 2, r2);
            float cf = 0.f;
            if constexpr (STAGE == 2) cf = cfl_mixed<GRAV>(unp, g, gf, iw0, iw1, iw2, invdtf);
            if (z_early) {
                zsolve(k, w0 + o_c, w1 + o_c, Wn, Fzhi);
            } else {
                halo_c2p(q, r2);
            }
            if constexpr (STAGE == 2)
                if (k > k0 && k > g.zw0 && k <= g.zw1) invdtf = cf;  // plane k-1, if the slab's own
        }
        __syncthreads();  // (1) plane k+2 converted
        if (stalled(q)) return;
        release(q);
        // ---- phase 2: the own lo x / lo y face pair; the z face (warps 0..3)
        //      or the tile's hi-edge faces (warp 7) ----
        if (z_early) {
            xy_faces(w0, k);
            if (warp == 7 && lane < 16) edge_faces(w0, k);
        } else {
            float W2[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) W2[f] = w2[o_c + f * PC];
            zsolve(k, w0 + o_c, w1 + o_c, W2, Fzhi);
            xy_faces(w0, k);
        }
        __syncthreads();  // (2) fluxes ready

        // ---- flux divergence (float64, reference order) and the stage update ----
        const int cz = (k == g.zw0 && g.zcls0 >= 0) ? g.zcls0 : lo_class(k, nz, perz);
        const bool interior = cx == LO_BEFORE && cy == LO_BEFORE && cz == LO_BEFORE;
        double un[5];
        double *po = Uout + lin;
        double acc[5];  // GRAV: the flux sums, completed by the gravity source
        cp_async_wait_all();  // this thread's own epilogue inputs have landed
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const double gxl = __dmul_rn(ax, (double)S.gx[f][ty * (TX + 1) + tx]);
            const double gxh = __dmul_rn(ax, (double)S.gx[f][ty * (TX + 1) + tx + 1]);
            const double gyl = __dmul_rn(ay, (double)S.gy[f][ty * TX + tx]);
            const double gyh = __dmul_rn(ay, (double)S.gy[f][(ty + 1) * TX + tx]);
            // explicit roundings: the result must not depend on how the compiler
            // contracts this code in each kernel instantiation
            const double gzh = __dmul_rn(az, (double)Fzhi[f]);
            const double gz0 = __dmul_rn(az, (double)fzl[f]);
            double a = 0.0;
            if (interior) {
                a = a - gz0 - gyl - gxl + gxh + gyh + gzh;
            } else {
                if (cz == LO_BEFORE) a -= gz0;
                if (cy == LO_BEFORE) a -= gyl;
                if (cx == LO_BEFORE) a -= gxl;
                a += gxh;
                if (cx == LO_SELF) a -= gxl;
                a += gyh;
                if (cy == LO_SELF) a -= gyl;
                a += gzh;
                if (cz == LO_SELF) a -= gz0;
                if (cx == LO_AFTER) a -= gxl;
                if (cy == LO_AFTER) a -= gyl;
                if (cz == LO_AFTER) a -= gz0;
            }
            fzl[f] = Fzhi[f];
            if constexpr (GRAV) {
                acc[f] = a;
                continue;
            }
            if constexpr (STAGE == 1) {
                un[f] = __fma_rn(-invV, a, S.ep[0][f][t]);
            } else {
                un[f] = __fma_rn(0.5, S.ep[1][f][t],
                                 __dmul_rn(0.5, __fma_rn(-invV, a, S.ep[0][f][t])));
            }
            if (inb) *po = un[f];
            po += g.ncell;
        }
        if constexpr (GRAV) {  // the source from the stage state, after the fluxes
            double u[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) u[f] = S.ep[0][f][t];
            if (inb) gravity_source<3>(g, lin, u, acc);
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                if constexpr (STAGE == 1) un[f] = __fma_rn(-invV, acc[f], u[f]);
                else un[f] = __fma_rn(0.5, S.ep[1][f][t], __dmul_rn(0.5, __fma_rn(-invV, acc[f], u[f])));
                if (inb) po[f * g.ncell] = un[f];
            }
        }
        lin += plane_cells;
        if constexpr (STAGE == 2) {
#pragma unroll
            for (int f = 0; f < 5; ++f) unp[f] = un[f];
        }
        float *rt = r0;
        r0 = r1;
        r1 = r2;
        r2 = rt;
    }
    if constexpr (STAGE == 2)  // the item's last plane
        invdt = (k1 - 1 >= g.zw0 && k1 - 1 < g.zw1)
                    ? (double)cfl_mixed<GRAV>(unp, g, gf, iw0, iw1, iw2, invdtf)
                    : (double)invdtf;
    qb += nplanes;
    if constexpr (STAGE == 2) block_max_to(&ctrl->invdt_bits, invdt, red);  // this box's CFL max
    }  // work items
}

template <int NS>
int launch_tiled3d_mixed(const BoxDesc *hbox, const BoxDesc *boxes, const int *item_box,
                         int nitems, unsigned int *work, int stage, cudaStream_t s, bool grav,
                         bool bf)
{
    const size_t smem = sizeof(t3m::Smem<NS>);
    static int res1 = 0, resb = 0, resg = 0, resf = 0;
    if (!res1) res1 = persistent_blocks(k_stage_tiled3d_mixed<NS, 1, false>,
                                        k_stage_tiled3d_mixed<NS, 2, false>, smem);
    if (!resb) resb = persistent_blocks(k_stage_tiled3d_mixed<NS, 1, true>,
                                        k_stage_tiled3d_mixed<NS, 2, true>, smem);
    if (!resg) resg = persistent_blocks(k_stage_tiled3d_mixed<NS, 1, false, true>,
                                        k_stage_tiled3d_mixed<NS, 2, false, true>, smem);
    if (!resf) resf = persistent_blocks(k_stage_tiled3d_mixed<NS, 1, false, false, true>,
                                        k_stage_tiled3d_mixed<NS, 2, false, false, true>, smem);
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
        k_stage_tiled3d_mixed<NS, 1, false, true><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (grav)
        k_stage_tiled3d_mixed<NS, 2, false, true><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (bf && stage == 1)
        k_stage_tiled3d_mixed<NS, 1, false, false, true><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (bf)
        k_stage_tiled3d_mixed<NS, 2, false, false, true><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (hbox && stage == 1)
        k_stage_tiled3d_mixed<NS, 1, false><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (hbox)
        k_stage_tiled3d_mixed<NS, 2, false><<<grid, t3::NT, smem, s>>>(box0, nullptr, nullptr, nitems, work);
    else if (stage == 1)
        k_stage_tiled3d_mixed<NS, 1, true><<<grid, t3::NT, smem, s>>>(box0, boxes, item_box, nitems, work);
    else
        k_stage_tiled3d_mixed<NS, 2, true><<<grid, t3::NT, smem, s>>>(box0, boxes, item_box, nitems, work);
    return 1;
}

}  // namespace vb
