// vb_hllc_x2.cuh -- two HLLC Riemann solves at once in packed float32x2
// arithmetic (sm_100 FFMA2/FADD2/FMUL2), for the VB_MIXED tiled kernel.
//
// Both faces are expressed in their own face-normal frame: (rho, u_n, u_t1,
// u_t2, p), so the two halves of every packed operation run the same
// algebra (hllc_flux, src/riemann.jl:33-88: Davis wave speeds, contact speed
// S*, star flux F + SK (U* - U)) whatever their normal axes are.  The branch
// on the wave pattern becomes per-half selects; the star correction is always
// computed and masked.  Reciprocals and square roots are per half
// (rcp.approx / sqrt.approx).
#pragma once

#include "vb_tma.cuh"

namespace vb {

struct f2 {
    float2 v;
    __device__ __forceinline__ f2() {}
    __device__ __forceinline__ f2(float a, float b) : v(make_float2(a, b)) {}
    __device__ __forceinline__ explicit f2(float2 x) : v(x) {}
    __device__ __forceinline__ static f2 splat(float a) { return f2(a, a); }
};
__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return f2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ f2 operator-(f2 a, f2 b)
{
    return f2(__fadd2_rn(a.v, make_float2(-b.v.x, -b.v.y)));
}
__device__ __forceinline__ f2 operator*(f2 a, f2 b) { return f2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return f2(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ f2 rcp2(f2 a) { return f2(rcp_approx(a.v.x), rcp_approx(a.v.y)); }
__device__ __forceinline__ f2 sqrt2(f2 a) { return f2(sqrt_approx(a.v.x), sqrt_approx(a.v.y)); }
__device__ __forceinline__ f2 min2(f2 a, f2 b) { return f2(fminf(a.v.x, b.v.x), fminf(a.v.y, b.v.y)); }
__device__ __forceinline__ f2 max2(f2 a, f2 b) { return f2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y)); }
__device__ __forceinline__ f2 sel2(bool cx, bool cy, f2 a, f2 b)
{
    return f2(cx ? a.v.x : b.v.x, cy ? a.v.y : b.v.y);
}

// A face state in its face-normal frame, two faces per value.
struct Face2 {
    f2 rho, un, ut1, ut2, p;
};

// F receives (mass, normal momentum, tangential 1, tangential 2, energy).
__device__ __forceinline__ void hllc_x2(const Face2 &L, const Face2 &R, float g, float ig1,
                                        f2 F[5])
{
    const f2 irL = rcp2(L.rho), irR = rcp2(R.rho);
    const f2 gg = f2::splat(g);
    const f2 cL = sqrt2(gg * L.p * irL), cR = sqrt2(gg * R.p * irR);
    const f2 SL = min2(L.un - cL, R.un - cR);
    const f2 SR = max2(L.un + cL, R.un + cR);
    const f2 aL = L.rho * (SL - L.un), aR = R.rho * (SR - R.un);
    const f2 Ss = (R.p - L.p + L.un * aL - R.un * aR) * rcp2(aL - aR);
    // wave pattern per half: supersonic left (FL), supersonic right (FR), or star
    const bool supL_x = SL.v.x >= 0.f, supL_y = SL.v.y >= 0.f;
    const bool supR_x = SR.v.x <= 0.f, supR_y = SR.v.y <= 0.f;
    const bool left_x = supL_x || (!supR_x && Ss.v.x >= 0.f);
    const bool left_y = supL_y || (!supR_y && Ss.v.y >= 0.f);
    const f2 SK = sel2(left_x, left_y, SL, SR);
    const f2 ir = sel2(left_x, left_y, irL, irR);
    const f2 rho = sel2(left_x, left_y, L.rho, R.rho);
    const f2 un = sel2(left_x, left_y, L.un, R.un);
    const f2 u1 = sel2(left_x, left_y, L.ut1, R.ut1);
    const f2 u2 = sel2(left_x, left_y, L.ut2, R.ut2);
    const f2 p = sel2(left_x, left_y, L.p, R.p);
    // physical flux of the selected side (euler_flux, riemann.jl:9-20)
    const f2 q2 = fma2(u2, u2, fma2(u1, u1, un * un));
    const f2 E = fma2(p, f2::splat(ig1), f2::splat(0.5f) * rho * q2);
    const f2 mun = rho * un;
    F[0] = mun;
    F[1] = fma2(mun, un, p);
    F[2] = mun * u1;
    F[3] = mun * u2;
    F[4] = (E + p) * un;
    // star correction SK (U* - U) (_hllc_star, riemann.jl:69-88), selected per
    // half (a select, so a non-finite value in an unused half never leaks)
    const f2 a = SK - un;
    const f2 ra = rho * a;
    const f2 factor = ra * rcp2(SK - Ss);
    const f2 Estar = fma2(E, ir, (Ss - un) * fma2(p, rcp2(ra), Ss));
    const bool sx = !supL_x && !supR_x, sy = !supL_y && !supR_y;
    const f2 fr = factor - rho;
    const f2 d[5] = {fr, fma2(factor, Ss, f2(-mun.v.x, -mun.v.y)), fr * u1, fr * u2,
                     fma2(factor, Estar, f2(-E.v.x, -E.v.y))};
#pragma unroll
    for (int k = 0; k < 5; ++k) F[k] = sel2(sx, sy, fma2(SK, d[k], F[k]), F[k]);
}

}  // namespace vb
