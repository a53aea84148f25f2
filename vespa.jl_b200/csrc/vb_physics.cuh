// vb_physics.cuh -- ideal-gas EOS, minmod PLM and HLLC, templated on the
// reconstruction/Riemann precision T (double for VB_FP64, float for VB_MIXED).
//
// Every expression keeps the reference's evaluation order.  The VB_FP64
// translation unit is compiled with -fmad=false, so each product and sum is
// rounded separately exactly as Julia does and the results are bit-identical
// to a serial float64 evaluation of the same expressions.
#pragma once

#include "vb_common.cuh"

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
    const T *W;
    T SK, Sstar = T(0);
    bool star;
    if (SL >= T(0)) {
        W = WL; SK = SL; star = false;
    } else if (SR <= T(0)) {
        W = WR; SK = SR; star = false;
    } else {
        Sstar = (pR - pL + rhoL * unL * (SL - unL) - rhoR * unR * (SR - unR)) /
                (rhoL * (SL - unL) - rhoR * (SR - unR));
        if (Sstar >= T(0)) { W = WL; SK = SL; } else { W = WR; SK = SR; }
        star = true;
    }
    const T rho = W[0], vx = W[1], vy = W[2], vz = W[3], p = W[4];
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
