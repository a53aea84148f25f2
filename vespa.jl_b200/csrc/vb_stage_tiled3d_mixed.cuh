// vb_stage_tiled3d_mixed.cuh -- VB_MIXED tiled 3D stage kernel.
//
// Same tiling, TMA pipeline and persistent work queue as k_stage_tiled3d
// (16 x 16 column tiles marching z; see vb_stage_tiled3d.cuh), specialised
// for float32 reconstruction and Riemann solves with float64 state:
//   - each cell's four x/y face values (lo/hi per axis) are computed once from
//     packed (x, y) minmod slopes and stored as float4 + float records, so a
//     face reads both of its states with four shared-memory loads;
//   - every thread solves its x face and its y face together as one packed
//     float32x2 HLLC (vb_hllc_x2.cuh, faces rotated into their normal frame);
//     the z face runs in registers down the thread's column;
//   - face fluxes are stored once, multiplied by the face area, in float64;
//     the flux divergence and the stage update stay in float64.
#pragma once

#include "vb_hllc_x2.cuh"
#include "vb_stage_tiled3d.cuh"

namespace vb {

namespace t3m {

using t3::NH;
using t3::NT;
using t3::TX;
using t3::TY;

enum { XLO = 0, XHI = 1, YLO = 2, YHI = 3 };

// primitives in one buffer: the current plane's interior [5][NT], then the
// halo strips of the three planes in flight [3][5][NH]; one index space makes
// every neighbour fetch a branch-free load
constexpr int HB = 5 * NT;

template <int NS>
struct Smem {
    double u[NS][t3::UPLANE];  // TMA stage buffers (raw conserved state)
    double ep[2][5][NT];       // own-cell epilogue inputs (Uin, U0), fetched by cp.async
    float w[5 * NT + 3 * 5 * NH];
    float4 fv4[4][NT];         // face values of interior cells: comps 0..3 of set XLO..YHI
    float fv1[4][NT];          //   ... comp 4
    float4 hv4[4][16];         // face values of the cells just outside the tile:
    float hv1[4][16];          //   XHI of lx=-1, XLO of lx=TX, YHI of ly=-1, YLO of ly=TY
    double gx[5][TY * (TX + 1)];  // x-face area * flux
    double gy[5][(TY + 1) * TX];  // y-face area * flux
    uint64_t bar[NS];
};

__device__ __forceinline__ void put5(float4 *a4, float *a1, int i, const float v[5])
{
    a4[i] = make_float4(v[0], v[1], v[2], v[3]);
    a1[i] = v[4];
}
__device__ __forceinline__ void get5(const float4 *a4, const float *a1, int i, float v[5])
{
    const float4 q = a4[i];
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    v[4] = a1[i];
}

// minmod slope of (l, c, r), scalar
__device__ __forceinline__ float mm(float l, float c, float r)
{
    const float a = c - l, b = r - c;
    if (a * b <= 0.f) return 0.f;
    return fabsf(a) < fabsf(b) ? a : b;
}

// cons2prim for VB_MIXED (src/eos.jl:8-25): velocities and the
// total-energy-minus-kinetic pressure recovery in float64, results rounded
// to float32.  1/rho comes from a float32 reciprocal refined by two float64
// Newton steps (relative error ~1e-16) instead of a float64 division.
__device__ __forceinline__ void cons2prim_mixed(const double U[5], double g, float W[5])
{
    const double rho = U[0];
    double inv = (double)rcp_approx((float)rho);
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
// (a dt estimate within float32 rounding of the float64 one), max in float64.
__device__ __forceinline__ double cfl_term(const double un[5], const Geom &g, double m)
{
    float W[5];
    cons2prim_mixed(un, g.gamma, W);
    const float cs = sqrt_approx((float)g.gamma * W[4] * rcp_approx(W[0]));
    const float t = fmaxf(fmaxf((fabsf(W[1]) + cs) * (float)g.invw[0],
                                (fabsf(W[2]) + cs) * (float)g.invw[1]),
                          (fabsf(W[3]) + cs) * (float)g.invw[2]);
    return nan_max(m, (double)t);
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

template <int NS, int STAGE, bool BATCH>
__global__ void __launch_bounds__(256, 2)
k_stage_tiled3d_mixed(const __grid_constant__ BoxDesc box0, const BoxDesc *__restrict__ boxes,
                      const int *__restrict__ item_box, int nitems, unsigned int *work)
{
    using namespace t3;
    using namespace t3m;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    t3m::Smem<NS> &S = *reinterpret_cast<t3m::Smem<NS> *>(smem_raw);
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
    const double ax = g.area[0], ay = g.area[1], az = g.area[2];
    const int bx_lo = g.bc_lo[0], bx_hi = g.bc_hi[0], by_lo = g.bc_lo[1], by_hi = g.bc_hi[1];
    const int bz_lo = g.bc_lo[2], bz_hi = g.bc_hi[2];
    double invdt = 0.0;
    const int local = item - B.item0;
    const int tile = local % ntiles;
    const int x0 = (tile % ntx) * TX, y0 = (tile / ntx) * TY;
    const int k0 = (local / ntiles) * kz;
    const int k1 = min(nz, k0 + kz);
    const int nplanes = (k1 - k0) + 4;
    const bool xlo_bnd = !perx && x0 == 0, xhi_bnd = !perx && x0 + TX == nx;
    const bool ylo_bnd = !pery && y0 == 0, yhi_bnd = !pery && y0 + TY == ny;

    auto issue = [&](int q) {
        const int p = k0 - 2 + q;
        const int z = perz ? ((p % nz) + nz) % nz : p;
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
        fence_proxy_async_smem();
        for (int q = 0; q < NS && q < nplanes; ++q) issue(q);
    }
    auto consume = [&](int q, float Wown[5], bool halo) {
        const int b = (qb + q) % NS;
        if (!mbar_wait(&S.bar[b], ((qb + q) / NS) & 1, WAIT_LIMIT_NS)) timed_out = true;
        const double *u = S.u[b];
        {
            double uu[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) uu[f] = u[f * NT + t];
            cons2prim_mixed(uu, gamma, Wown);
        }
        if (halo && t < NH) {
            double uu[5];
            float w[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) uu[f] = u[halo_uoff(t, f)];
            cons2prim_mixed(uu, gamma, w);
#pragma unroll
            for (int f = 0; f < 5; ++f) S.w[HB + ((q % 3) * 5 + f) * NH + t] = w[f];
        }
    };
    auto release = [&](int q) {
        if (t == 0 && q + NS < nplanes) {
            fence_proxy_async_smem();
            issue(q + NS);
        }
    };

    float Wa[5], Wb[5], Wz0[5], Wz1[5], Wz2[5];
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

    // z state entering plane k0: hi face value of k0 and the flux through k0-1/2
    float hz[5], Fzlo[5];
    {
        const bool gl = !perz && k0 == 0;
        const bool gh = !perz && k0 + 1 >= nz;
        float loz[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const float wl = gl ? ((bz_lo == BC_REFLECTING && f == 3) ? -Wz0[f] : Wz0[f]) : Wb[f];
            const float wr = gh ? ((bz_hi == BC_REFLECTING && f == 3) ? -Wz0[f] : Wz0[f]) : Wz1[f];
            const float s = mm(wl, Wz0[f], wr);
            hz[f] = fmaf(0.5f, s, Wz0[f]);
            loz[f] = fmaf(-0.5f, s, Wz0[f]);
        }
        if (gl) {
            float gst[5];
            ghost_state<float>(loz, bz_lo, 2, gst);
            hllc_flux_fast<3>(gst, loz, gf, ig1, Fzlo);
        } else {
            const bool gll = !perz && k0 - 2 < 0;
            float hzm[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const float wl = gll ? ((bz_lo == BC_REFLECTING && f == 3) ? -Wb[f] : Wb[f]) : Wa[f];
                hzm[f] = fmaf(0.5f, mm(wl, Wb[f], Wz0[f]), Wb[f]);
            }
            hllc_flux_fast<3>(hzm, loz, gf, ig1, Fzlo);
        }
    }

    const int gx = x0 + tx, gy = y0 + ty;
    const int cx = lo_class(gx, nx, perx), cy = lo_class(gy, ny, pery);
    double unp[5];  // previous plane's new state: its CFL term is folded one plane later

    for (int k = k0; k < k1; ++k) {
        const int q = k - k0 + 4;
        const int slot = (q - 2) % 3;
        const int64_t lin = (int64_t)gx + (int64_t)nx * ((int64_t)gy + (int64_t)ny * k);
        // own-cell epilogue inputs, fetched asynchronously into shared memory
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            cp_async8(&S.ep[0][f][t], Uin + (int64_t)f * g.ncell + lin);
            if constexpr (STAGE == 2) cp_async8(&S.ep[1][f][t], U0 + (int64_t)f * g.ncell + lin);
        }
        cp_async_commit();
        consume(q, Wz2, true);
        if constexpr (STAGE == 2)
            if (k > k0) invdt = cfl_term(unp, g, invdt);  // overlaps the cons2prim chain
#pragma unroll
        for (int f = 0; f < 5; ++f) S.w[f * NT + t] = Wz0[f];
        __syncthreads();  // (1)
        release(q);

        // primitive of local cell (lx, ly) of plane k, interior or halo strip
        const int hb = HB + slot * 5 * NH;
        auto W = [&](int f, int lx, int ly) -> float {
            return (lx >= 0 && lx < TX && ly >= 0 && ly < TY) ? S.w[f * NT + ly * TX + lx]
                                                              : S.w[hb + f * NH + halo_idx(lx, ly)];
        };

        // ---- face values of the interior cells from packed (x, y) slopes ----
        {
            // neighbour offsets and field strides, branch-free per component
            const int oxl = tx > 0 ? t - 1 : hb + halo_idx(-1, ty);
            const int oxr = tx < TX - 1 ? t + 1 : hb + halo_idx(TX, ty);
            const int oyl = ty > 0 ? t - TX : hb + halo_idx(tx, -1);
            const int oyr = ty < TY - 1 ? t + TX : hb + halo_idx(tx, TY);
            const int sxl = tx > 0 ? NT : NH, sxr = tx < TX - 1 ? NT : NH;
            const int syl = ty > 0 ? NT : NH, syr = ty < TY - 1 ? NT : NH;
            const bool gxl = tx == 0 && xlo_bnd, gxr = tx == TX - 1 && xhi_bnd;
            const bool gyl = ty == 0 && ylo_bnd, gyr = ty == TY - 1 && yhi_bnd;
            float xl[5], xh[5], yl[5], yh[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const float wc = Wz0[f];
                float l = S.w[oxl + f * sxl], r = S.w[oxr + f * sxr];
                float d = S.w[oyl + f * syl], e = S.w[oyr + f * syr];
                if (gxl) l = (bx_lo == BC_REFLECTING && f == 1) ? -wc : wc;
                if (gxr) r = (bx_hi == BC_REFLECTING && f == 1) ? -wc : wc;
                if (gyl) d = (by_lo == BC_REFLECTING && f == 2) ? -wc : wc;
                if (gyr) e = (by_hi == BC_REFLECTING && f == 2) ? -wc : wc;
                const f2 wc2 = f2::splat(wc);
                const f2 a = wc2 - f2(l, d), b = f2(r, e) - wc2;
                const f2 pr = a * b;
                const float sx = pr.v.x <= 0.f ? 0.f : (fabsf(a.v.x) < fabsf(b.v.x) ? a.v.x : b.v.x);
                const float sy = pr.v.y <= 0.f ? 0.f : (fabsf(a.v.y) < fabsf(b.v.y) ? a.v.y : b.v.y);
                const f2 s = f2(sx, sy);
                const f2 lo = fma2(f2::splat(-0.5f), s, wc2), hi = fma2(f2::splat(0.5f), s, wc2);
                xl[f] = lo.v.x; yl[f] = lo.v.y;
                xh[f] = hi.v.x; yh[f] = hi.v.y;
            }
            put5(S.fv4[XLO], S.fv1[XLO], t, xl);
            put5(S.fv4[XHI], S.fv1[XHI], t, xh);
            put5(S.fv4[YLO], S.fv1[YLO], t, yl);
            put5(S.fv4[YHI], S.fv1[YHI], t, yh);
        }
        // ---- face values of the cells just outside the tile ----
        if (t >= 160 && t < 224) {
            const int j = t - 160;
            const int set = j >> 4, i = j & 15;
            float v[5];
            bool need;
            if (set == 0) {  // XHI of lx = -1, row i
                need = !xlo_bnd;
                if (need)
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const float c = W(f, -1, i);
                        v[f] = fmaf(0.5f, mm(W(f, -2, i), c, W(f, 0, i)), c);
                    }
            } else if (set == 1) {  // XLO of lx = TX, row i
                need = !xhi_bnd;
                if (need)
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const float c = W(f, TX, i);
                        v[f] = fmaf(-0.5f, mm(W(f, TX - 1, i), c, W(f, TX + 1, i)), c);
                    }
            } else if (set == 2) {  // YHI of ly = -1, column i
                need = !ylo_bnd;
                if (need)
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const float c = W(f, i, -1);
                        v[f] = fmaf(0.5f, mm(W(f, i, -2), c, W(f, i, 0)), c);
                    }
            } else {  // YLO of ly = TY, column i
                need = !yhi_bnd;
                if (need)
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const float c = W(f, i, TY);
                        v[f] = fmaf(-0.5f, mm(W(f, i, TY - 1), c, W(f, i, TY + 1)), c);
                    }
            }
            if (need) put5(S.hv4[set], S.hv1[set], i, v);
        }
        __syncthreads();  // (2) face values ready

        // ---- own lo x face and lo y face (one packed solve) and the z face
        //      k+1/2 down the own column: independent chains, one phase ----
        float Fzhi[5], hz1[5];
        {
            float zr[5];  // right state of the z face
            const bool plane_k1 = perz || k + 1 < nz;
            if (plane_k1) {
                const bool gh = !perz && k + 2 >= nz;
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    const float wr = gh ? ((bz_hi == BC_REFLECTING && f == 3) ? -Wz1[f] : Wz1[f]) : Wz2[f];
                    const float s = mm(Wz0[f], Wz1[f], wr);
                    zr[f] = fmaf(-0.5f, s, Wz1[f]);
                    hz1[f] = fmaf(0.5f, s, Wz1[f]);
                }
            } else {
                ghost_state<float>(hz, bz_hi, 2, zr);
#pragma unroll
                for (int f = 0; f < 5; ++f) hz1[f] = hz[f];
            }
            hllc_flux_fast<3>(hz, zr, gf, ig1, Fzhi);
        }
        {
            float Lx[5], Rx[5], Ly[5], Ry[5];
            get5(S.fv4[XLO], S.fv1[XLO], t, Rx);
            get5(S.fv4[YLO], S.fv1[YLO], t, Ry);
            if (tx > 0) get5(S.fv4[XHI], S.fv1[XHI], t - 1, Lx);
            else if (xlo_bnd) ghost_state<float>(Rx, bx_lo, 0, Lx);
            else get5(S.hv4[0], S.hv1[0], ty, Lx);
            if (ty > 0) get5(S.fv4[YHI], S.fv1[YHI], t - TX, Ly);
            else if (ylo_bnd) ghost_state<float>(Ry, by_lo, 1, Ly);
            else get5(S.hv4[2], S.hv1[2], tx, Ly);
            const Face2 L{f2(Lx[0], Ly[0]), f2(Lx[1], Ly[2]), f2(Lx[2], Ly[1]), f2(Lx[3], Ly[3]),
                          f2(Lx[4], Ly[4])};
            const Face2 R{f2(Rx[0], Ry[0]), f2(Rx[1], Ry[2]), f2(Rx[2], Ry[1]), f2(Rx[3], Ry[3]),
                          f2(Rx[4], Ry[4])};
            f2 F[5];
            hllc_x2(L, R, gf, ig1, F);
            const int ix = ty * (TX + 1) + tx, iy = ty * TX + tx;
            S.gx[0][ix] = ax * (double)F[0].v.x;  S.gy[0][iy] = ay * (double)F[0].v.y;
            S.gx[1][ix] = ax * (double)F[1].v.x;  S.gy[2][iy] = ay * (double)F[1].v.y;
            S.gx[2][ix] = ax * (double)F[2].v.x;  S.gy[1][iy] = ay * (double)F[2].v.y;
            S.gx[3][ix] = ax * (double)F[3].v.x;  S.gy[3][iy] = ay * (double)F[3].v.y;
            S.gx[4][ix] = ax * (double)F[4].v.x;  S.gy[4][iy] = ay * (double)F[4].v.y;
        }
        // ---- the hi-edge faces (x at fx = TX, y at fy = TY), one pair per lane ----
        if (t >= 224 && t < 240) {
            const int j = t - 224;
            float Lx[5], Rx[5], Ly[5], Ry[5];
            get5(S.fv4[XHI], S.fv1[XHI], j * TX + TX - 1, Lx);
            if (xhi_bnd) ghost_state<float>(Lx, bx_hi, 0, Rx);
            else get5(S.hv4[1], S.hv1[1], j, Rx);
            get5(S.fv4[YHI], S.fv1[YHI], (TY - 1) * TX + j, Ly);
            if (yhi_bnd) ghost_state<float>(Ly, by_hi, 1, Ry);
            else get5(S.hv4[3], S.hv1[3], j, Ry);
            const Face2 L{f2(Lx[0], Ly[0]), f2(Lx[1], Ly[2]), f2(Lx[2], Ly[1]), f2(Lx[3], Ly[3]),
                          f2(Lx[4], Ly[4])};
            const Face2 R{f2(Rx[0], Ry[0]), f2(Rx[1], Ry[2]), f2(Rx[2], Ry[1]), f2(Rx[3], Ry[3]),
                          f2(Rx[4], Ry[4])};
            f2 F[5];
            hllc_x2(L, R, gf, ig1, F);
            const int ix = j * (TX + 1) + TX, iy = TY * TX + j;
            S.gx[0][ix] = ax * (double)F[0].v.x;  S.gy[0][iy] = ay * (double)F[0].v.y;
            S.gx[1][ix] = ax * (double)F[1].v.x;  S.gy[2][iy] = ay * (double)F[1].v.y;
            S.gx[2][ix] = ax * (double)F[2].v.x;  S.gy[1][iy] = ay * (double)F[2].v.y;
            S.gx[3][ix] = ax * (double)F[3].v.x;  S.gy[3][iy] = ay * (double)F[3].v.y;
            S.gx[4][ix] = ax * (double)F[4].v.x;  S.gy[4][iy] = ay * (double)F[4].v.y;
        }
        __syncthreads();  // (3) fluxes ready

        // ---- flux divergence (float64, reference order) and the stage update ----
        const int cz = lo_class(k, nz, perz);
        const bool interior = cx == LO_BEFORE && cy == LO_BEFORE && cz == LO_BEFORE;
        double un[5];
        cp_async_wait_all();  // this thread's own epilogue inputs have landed
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const double gxl = S.gx[f][ty * (TX + 1) + tx];
            const double gxh = S.gx[f][ty * (TX + 1) + tx + 1];
            const double gyl = S.gy[f][ty * TX + tx];
            const double gyh = S.gy[f][(ty + 1) * TX + tx];
            // explicit roundings: the result must not depend on how the compiler
            // contracts this code in each kernel instantiation
            const double gzl = __dmul_rn(az, (double)Fzlo[f]);
            const double gzh = __dmul_rn(az, (double)Fzhi[f]);
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
                un[f] = __fma_rn(-invV, a, S.ep[0][f][t]);
            } else {
                un[f] = __fma_rn(0.5, S.ep[1][f][t],
                                 __dmul_rn(0.5, __fma_rn(-invV, a, S.ep[0][f][t])));
            }
            Uout[i] = un[f];
        }
        if constexpr (STAGE == 2) {
#pragma unroll
            for (int f = 0; f < 5; ++f) unp[f] = un[f];
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            Wz0[f] = Wz1[f];
            Wz1[f] = Wz2[f];
            hz[f] = hz1[f];
            Fzlo[f] = Fzhi[f];
        }
    }
    if constexpr (STAGE == 2) invdt = cfl_term(unp, g, invdt);  // the item's last plane
    qb += nplanes;
    if (timed_out && t == 0) atomicOr(&ctrl->flags, CTRL_F_TIMEOUT);
    if constexpr (STAGE == 2) block_max_to(&ctrl->invdt_bits, invdt, red);  // this box's CFL max
    }  // work items
}

template <int NS>
int launch_tiled3d_mixed(const BoxDesc *hbox, const BoxDesc *boxes, const int *item_box,
                         int nitems, unsigned int *work, int stage, cudaStream_t s)
{
    const size_t smem = sizeof(t3m::Smem<NS>);
    static int res1 = 0, resb = 0;
    if (!res1) res1 = persistent_blocks(k_stage_tiled3d_mixed<NS, 1, false>,
                                        k_stage_tiled3d_mixed<NS, 2, false>, smem);
    if (!resb) resb = persistent_blocks(k_stage_tiled3d_mixed<NS, 1, true>,
                                        k_stage_tiled3d_mixed<NS, 2, true>, smem);
    const int resident = hbox ? res1 : resb;
    if (resident <= 0 || nitems <= 0) return -1;
    const unsigned grid = (unsigned)(nitems < resident ? nitems : resident);
    BoxDesc box0;
    if (hbox) box0 = *hbox;
    else std::memset(&box0, 0, sizeof box0);
    if (hbox && stage == 1)
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
