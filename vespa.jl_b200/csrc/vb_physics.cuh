// vb_physics.cuh -- ideal-gas EOS, minmod PLM and HLLC, templated on the
// reconstruction/Riemann precision T (double for VB_FP64, float for VB_MIXED).
//
// Every expression keeps the reference's evaluation order.  The VB_FP64
// translation unit is compiled with -fmad=false, so each product and sum is
// rounded separately exactly as Julia does and the results are bit-identical
// to a serial float64 evaluation of the same expressions.
#pragma once

#include "vb_common.cuh"
#include "vb_tma.cuh"

namespace vb {

// cons2prim, src/eos.jl:8-25, always evaluated in float64 (the mixed mode
// keeps the total-energy-minus-kinetic pressure recovery in float64 too).
// The pressure floor max(p, 1e-12*kinetic) is at src/eos.jl:24.
__device__ __forceinline__ void cons2prim(const double U[5], double g, double W[5])
{
    double rho = U[0];
    double inv = 1.0 / rho;
    double vx = U[1] * inv;
    double vy = U[2] * inv;
    double vz = U[3] * inv;
    double kinetic = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
    double p = (g - 1.0) * (U[4] - kinetic);
    W[0] = rho;
    W[1] = vx;
    W[2] = vy;
    W[3] = vz;
    W[4] = fmax(p, 1e-12 * kinetic);
}

// sound_speed, src/eos.jl:35
__device__ __forceinline__ double sound_speed(const double W[5], double g)
{
    return sqrt(g * W[4] / W[0]);
}

// minmod, src/reconstruct.jl:6-12
template <typename T>
__device__ __forceinline__ T minmod(T a, T b)
{
    if (a * b <= T(0)) return T(0);
    return fabs(a) < fabs(b) ? a : b;
}

// limited_slope, src/reconstruct.jl:15-16
template <typename T>
__device__ __forceinline__ T limited_slope(T l, T c, T r)
{
    return minmod<T>(c - l, r - c);
}

// ghost_state, src/driver.jl:117-122: Outflow copies, Reflecting negates the
// normal velocity (primitive index 1 + axis).  AX is the 0-based axis.
template <typename T>
__device__ __forceinline__ void ghost_state(const T W[5], int bc, int ax, T out[5])
{
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = W[k];
    if (bc == BC_REFLECTING) out[1 + ax] = -W[1 + ax];
}

// prim2cons total energy, src/eos.jl:28-32 (also euler_flux's E, riemann.jl:14)
template <typename T>
__device__ __forceinline__ T total_energy(const T W[5], T g)
{
    return W[4] / (g - T(1)) + T(0.5) * W[0] * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]);
}

// hllc_flux, src/riemann.jl:33-66 with euler_flux (9-20) and _hllc_star
// (69-88).  DIM is the 1-based face-normal axis.
template <typename T, int DIM>
__device__ __forceinline__ void hllc_flux(const T WL[5], const T WR[5], double gamma, T F[5])
{
    const T g = T(gamma);
    const T rhoL = WL[0], rhoR = WR[0];
    const T pL = WL[4], pR = WR[4];
    const T unL = WL[DIM], unR = WR[DIM];
    const T cL = sqrt(g * pL / rhoL);
    const T cR = sqrt(g * pR / rhoR);
    const T SL = fmin(unL - cL, unR - cR);
    const T SR = fmax(unL + cL, unR + cR);

    // Only the selected side's conserved state and physical flux are needed.
    // SL >= 0 -> FL;  SR <= 0 -> FR;  else the star flux of the side picked by
    // the sign of S*.  Each side's quantities are the same expressions as the
    // reference's prim2cons / euler_flux, evaluated for that side only.
    bool left, star;
    T SK, Sstar = T(0);
    if (SL >= T(0)) {
        left = true; SK = SL; star = false;
    } else if (SR <= T(0)) {
        left = false; SK = SR; star = false;
    } else {
        Sstar = (pR - pL + rhoL * unL * (SL - unL) - rhoR * unR * (SR - unR)) /
                (rhoL * (SL - unL) - rhoR * (SR - unR));
        left = Sstar >= T(0);
        SK = left ? SL : SR;
        star = true;
    }
    // value selects (not a pointer to one side) keep both states in registers
    const T rho = left ? WL[0] : WR[0], vx = left ? WL[1] : WR[1];
    const T vy = left ? WL[2] : WR[2], vz = left ? WL[3] : WR[3];
    const T p = left ? WL[4] : WR[4];
    const T W[5] = {rho, vx, vy, vz, p};
    const T un = W[DIM];
    const T E = total_energy<T>(W, g);
    // euler_flux (riemann.jl:9-20); the +0 on tangential momentum is omitted
    // (it only changes the sign of an exact zero).
    T Fk[5];
    Fk[0] = rho * un;
    Fk[1] = (rho * vx) * un;
    Fk[2] = (rho * vy) * un;
    Fk[3] = (rho * vz) * un;
    Fk[DIM] = Fk[DIM] + p;
    Fk[4] = (E + p) * un;
    if (!star) {
#pragma unroll
        for (int k = 0; k < 5; ++k) F[k] = Fk[k];
        return;
    }
    // _hllc_star (riemann.jl:69-88): F* = F + SK (U* - U)
    const T Uk[5] = {rho, rho * vx, rho * vy, rho * vz, E};
    const T factor = rho * (SK - un) / (SK - Sstar);
    T vstar[3] = {vx, vy, vz};
    vstar[DIM - 1] = Sstar;
    const T Estar = E / rho + (Sstar - un) * (Sstar + p / (rho * (SK - un)));
    const T Us[5] = {factor, factor * vstar[0], factor * vstar[1], factor * vstar[2],
                     factor * Estar};
#pragma unroll
    for (int k = 0; k < 5; ++k) F[k] = Fk[k] + SK * (Us[k] - Uk[k]);
}

// PLM face value w + h*s (src/driver.jl:227-233).  In float the product-add
// is an explicit fused multiply-add so every call site rounds identically (a
// face evaluated from both neighbouring cells must give one value); in the
// float64 unit (-fmad=false) it is a separately rounded product and sum, as
// in the reference.
__device__ __forceinline__ double face_val(double w, double h, double s) { return w + h * s; }
__device__ __forceinline__ float face_val(float w, float h, float s) { return __fmaf_rn(h, s, w); }

// The same Riemann solve behind one call for every face of the cell-centric
// kernel: in float, a non-inlined body guarantees identical instructions for
// the two evaluations of each interior face (flux conservation to the bit).
template <typename T, int DIM>
__device__ __noinline__ void hllc_flux_shared(const T *WL, const T *WR, double gamma, T *F)
{
    T l[5], r[5], f[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        l[k] = WL[k];
        r[k] = WR[k];
    }
    hllc_flux<T, DIM>(l, r, gamma, f);
#pragma unroll
    for (int k = 0; k < 5; ++k) F[k] = f[k];
}

template <typename T, int DIM>
__device__ __forceinline__ void hllc_face(const T WL[5], const T WR[5], double gamma, T F[5])
{
    if constexpr (sizeof(T) == 4)
        hllc_flux_shared<T, DIM>(WL, WR, gamma, F);
    else
        hllc_flux<T, DIM>(WL, WR, gamma, F);
}

// Float32 HLLC for VB_MIXED: the same algebra as hllc_flux (Davis speeds,
// contact speed S*, star flux F + SK (U* - U)) with approximate reciprocals
// and square roots (rcp.approx / sqrt.approx, ~1 ulp) and contracted
// multiply-adds.  ig1 = 1 / (gamma - 1).  Used where each face is evaluated
// exactly once, so conservation does not depend on rounding.
template <int DIM>
__device__ __forceinline__ void hllc_flux_fast(const float WL[5], const float WR[5], float g,
                                               float ig1, float F[5])
{
    const float rhoL = WL[0], rhoR = WR[0];
    const float pL = WL[4], pR = WR[4];
    const float unL = WL[DIM], unR = WR[DIM];
    const float irL = rcp_approx(rhoL), irR = rcp_approx(rhoR);
    const float cL = sqrt_approx(g * pL * irL);
    const float cR = sqrt_approx(g * pR * irR);
    const float SL = fminf(unL - cL, unR - cR);
    const float SR = fmaxf(unL + cL, unR + cR);
    bool left, star;
    float Sstar = 0.f;
    if (SL >= 0.f) {
        left = true; star = false;
    } else if (SR <= 0.f) {
        left = false; star = false;
    } else {
        const float aL = rhoL * (SL - unL), aR = rhoR * (SR - unR);
        Sstar = (pR - pL + unL * aL - unR * aR) * rcp_approx(aL - aR);
        left = Sstar >= 0.f;
        star = true;
    }
    const float SK = left ? SL : SR, ir = left ? irL : irR;
    const float rho = left ? WL[0] : WR[0], vx = left ? WL[1] : WR[1];
    const float vy = left ? WL[2] : WR[2], vz = left ? WL[3] : WR[3];
    const float p = left ? WL[4] : WR[4];
    const float un = DIM == 1 ? vx : (DIM == 2 ? vy : vz);
    const float E = p * ig1 + 0.5f * rho * (vx * vx + vy * vy + vz * vz);
    const float mun = rho * un;
    F[0] = mun;
    F[1] = mun * vx;
    F[2] = mun * vy;
    F[3] = mun * vz;
    F[DIM] += p;
    F[4] = (E + p) * un;
    if (!star) return;
    const float a = SK - un;
    const float ra = rho * a;                 // rho (SK - un)
    const float factor = ra * rcp_approx(SK - Sstar);
    const float Estar = E * ir + (Sstar - un) * (Sstar + p * rcp_approx(ra));
    const float vs[3] = {vx, vy, vz};
    F[0] += SK * (factor - rho);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float us = (d == DIM - 1) ? factor * Sstar : factor * vs[d];
        F[1 + d] += SK * (us - rho * vs[d]);
    }
    F[4] += SK * (factor * Estar - E);
}

// hllc_flux_fast without branches: the wave pattern becomes selects and the
// star correction is always computed, then selected (same operations, same
// results).
template <int DIM>
__device__ __forceinline__ void hllc_flux_fast_bf(const float WL[5], const float WR[5], float g,
                                                  float ig1, float F[5])
{
    const float rhoL = WL[0], rhoR = WR[0];
    const float pL = WL[4], pR = WR[4];
    const float unL = WL[DIM], unR = WR[DIM];
    const float irL = rcp_approx(rhoL), irR = rcp_approx(rhoR);
    const float cL = sqrt_approx(g * pL * irL);
    const float cR = sqrt_approx(g * pR * irR);
    const float SL = fminf(unL - cL, unR - cR);
    const float SR = fmaxf(unL + cL, unR + cR);
    const float aL = rhoL * (SL - unL), aR = rhoR * (SR - unR);
    const float Ss = (pR - pL + unL * aL - unR * aR) * rcp_approx(aL - aR);
    const bool supL = SL >= 0.f, supR = SR <= 0.f;
    const bool star = !supL && !supR;
    const bool left = supL || (star && Ss >= 0.f);
    const float Sstar = star ? Ss : 0.f;
    const float SK = left ? SL : SR, ir = left ? irL : irR;
    const float rho = left ? WL[0] : WR[0], vx = left ? WL[1] : WR[1];
    const float vy = left ? WL[2] : WR[2], vz = left ? WL[3] : WR[3];
    const float p = left ? WL[4] : WR[4];
    const float un = DIM == 1 ? vx : (DIM == 2 ? vy : vz);
    const float E = p * ig1 + 0.5f * rho * (vx * vx + vy * vy + vz * vz);
    const float mun = rho * un;
    float G[5];
    G[0] = mun;
    G[1] = mun * vx;
    G[2] = mun * vy;
    G[3] = mun * vz;
    G[DIM] += p;
    G[4] = (E + p) * un;
    const float a = SK - un;
    const float ra = rho * a;
    const float factor = ra * rcp_approx(SK - Sstar);
    const float Estar = E * ir + (Sstar - un) * (Sstar + p * rcp_approx(ra));
    const float vs[3] = {vx, vy, vz};
    F[0] = star ? G[0] + SK * (factor - rho) : G[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float us = (d == DIM - 1) ? factor * Sstar : factor * vs[d];
        F[1 + d] = star ? G[1 + d] + SK * (us - rho * vs[d]) : G[1 + d];
    }
    F[4] = star ? G[4] + SK * (factor * Estar - E) : G[4];
}

// Runtime-axis dispatch for the batched face kernel.
template <typename T>
__device__ __forceinline__ void hllc_flux_axis(const T WL[5], const T WR[5], double gamma,
                                               int dim, T F[5])
{
    if (dim == 1)
        hllc_flux<T, 1>(WL, WR, gamma, F);
    else if (dim == 2)
        hllc_flux<T, 2>(WL, WR, gamma, F);
    else
        hllc_flux<T, 3>(WL, WR, gamma, F);
}

}  // namespace vb
