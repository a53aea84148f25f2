// vb_adjoint.cuh -- reverse-mode derivatives of the float64 hydro step, with
// every branch frozen at the choice the forward evaluation makes:
//   - cons2prim's pressure floor max(p, 1e-12*kinetic)      (src/eos.jl:24)
//   - minmod's zero / left / right choice                   (src/reconstruct.jl:6-12)
//   - HLLC's Davis speed min/max, the supersonic cases and the star side
//     picked by the sign of S*                              (src/riemann.jl:33-88)
// The forward values are recomputed with the same expressions as the forward
// kernels (this translation unit is built with -fmad=false like the float64
// stepping kernels), so every branch decision matches the forward step's bit
// for bit.  The reference has no adjoint; these are the exact derivatives of
// its piecewise-smooth map wherever no branch sits on a tie.
#pragma once

#include "vb_physics.cuh"

namespace vb {

// minmod branch code of slope(l, c, r) = minmod(c - l, r - c):
// 0 -> slope 0, 1 -> slope = c - l, 2 -> slope = r - c.
__device__ __forceinline__ unsigned minmod_code(double a, double b)
{
    if (a * b <= 0.0) return 0u;
    return fabs(a) < fabs(b) ? 1u : 2u;
}

// Reverse of cons2prim (src/eos.jl:8-25): Ub = (dW/dU)^T Wb.
__device__ __forceinline__ void cons2prim_vjp(const double U[5], double g, const double Wb[5],
                                              double Ub[5])
{
    const double rho = U[0];
    const double inv = 1.0 / rho;
    const double vx = U[1] * inv, vy = U[2] * inv, vz = U[3] * inv;
    const double v2 = vx * vx + vy * vy + vz * vz;
    const double kinetic = 0.5 * rho * v2;
    const double p = (g - 1.0) * (U[4] - kinetic);
    // fmax(p, 1e-12*kinetic) returns the floor only when p < floor
    const bool floored = !(p >= 1e-12 * kinetic);
    const double keb = floored ? 1e-12 * Wb[4] : -(g - 1.0) * Wb[4];
    const double Eb = floored ? 0.0 : (g - 1.0) * Wb[4];
    const double vbx = Wb[1] + keb * rho * vx;
    const double vby = Wb[2] + keb * rho * vy;
    const double vbz = Wb[3] + keb * rho * vz;
    double rhob = Wb[0] + keb * 0.5 * v2;
    const double invb = vbx * U[1] + vby * U[2] + vbz * U[3];
    rhob -= invb * inv * inv;
    Ub[0] = rhob;
    Ub[1] = vbx * inv;
    Ub[2] = vby * inv;
    Ub[3] = vbz * inv;
    Ub[4] = Eb;
}

// Reverse of hllc_flux<double, DIM> (vb_physics.cuh): given Fb = dJ/dF, add
// dJ/dWL and dJ/dWR into WLb / WRb (which the caller zeroes).
template <int DIM>
__device__ __forceinline__ void hllc_vjp(const double WL[5], const double WR[5], double gamma,
                                         const double Fb[5], double WLb[5], double WRb[5])
{
    const double g = gamma;
    const double rhoL = WL[0], rhoR = WR[0];
    const double pL = WL[4], pR = WR[4];
    const double unL = WL[DIM], unR = WR[DIM];
    const double cL = sqrt(g * pL / rhoL);
    const double cR = sqrt(g * pR / rhoR);
    const double aL = unL - cL, aR = unR - cR;
    const double bL = unL + cL, bR = unR + cR;
    const double SL = fmin(aL, aR);
    const double SR = fmax(bL, bR);
    const bool SL_from_L = aL <= aR;  // fmin's operand (a tie has one value)
    const bool SR_from_L = bL >= bR;

    bool left, star;
    double SK, Sstar = 0.0, Nn = 0.0, Dn = 1.0;
    if (SL >= 0.0) {
        left = true; SK = SL; star = false;
    } else if (SR <= 0.0) {
        left = false; SK = SR; star = false;
    } else {
        Nn = pR - pL + rhoL * unL * (SL - unL) - rhoR * unR * (SR - unR);
        Dn = rhoL * (SL - unL) - rhoR * (SR - unR);
        Sstar = Nn / Dn;
        left = Sstar >= 0.0;
        SK = left ? SL : SR;
        star = true;
    }
    // value selects keep both face states in registers
    const double rho = left ? WL[0] : WR[0], p = left ? WL[4] : WR[4];
    const double v[3] = {left ? WL[1] : WR[1], left ? WL[2] : WR[2], left ? WL[3] : WR[3]};
    const double un = v[DIM - 1];
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double E = p / (g - 1.0) + 0.5 * rho * v2;

    // adjoints of the selected side's primitives, E and un
    double rb = 0.0, vb[3] = {0.0, 0.0, 0.0}, pb = 0.0, Eb = 0.0, unb = 0.0;
    // side-specific adjoints feeding the wave speeds
    double rLb = 0.0, unLb = 0.0, pLb = 0.0, rRb = 0.0, unRb = 0.0, pRb = 0.0;

    // physical flux of the selected side (euler_flux, src/riemann.jl:9-20)
    rb += Fb[0] * un;
    unb += Fb[0] * rho;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        rb += Fb[1 + j] * v[j] * un;
        vb[j] += Fb[1 + j] * rho * un;
        unb += Fb[1 + j] * rho * v[j];
    }
    pb += Fb[DIM];
    Eb += Fb[4] * un;
    pb += Fb[4] * un;
    unb += Fb[4] * (E + p);

    if (star) {
        // F = Fk + SK (Us - Uk), _hllc_star (src/riemann.jl:69-88)
        const double q = rho * (SK - un);
        const double d = SK - Sstar;
        const double factor = q / d;
        const double r = p / q;
        const double A = Sstar - un, B = Sstar + r;
        const double Estar = E / rho + A * B;
        double vstar[3] = {v[0], v[1], v[2]};
        vstar[DIM - 1] = Sstar;
        const double Uk[5] = {rho, rho * v[0], rho * v[1], rho * v[2], E};
        const double Us[5] = {factor, factor * vstar[0], factor * vstar[1], factor * vstar[2],
                              factor * Estar};
        double SKb = 0.0;
#pragma unroll
        for (int k = 0; k < 5; ++k) SKb += Fb[k] * (Us[k] - Uk[k]);
        // Uk = prim2cons(W): its adjoint is -SK * Fb
        rb += -SK * Fb[0];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            rb += -SK * Fb[1 + j] * v[j];
            vb[j] += -SK * Fb[1 + j] * rho;
        }
        Eb += -SK * Fb[4];
        // Us = factor * (1, vstar, Estar): its adjoint is SK * Fb
        double factorb = SK * Fb[0] + SK * Fb[4] * Estar;
#pragma unroll
        for (int j = 0; j < 3; ++j) factorb += SK * Fb[1 + j] * vstar[j];
        double Sstarb = SK * Fb[DIM] * factor;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (j != DIM - 1) vb[j] += SK * Fb[1 + j] * factor;
        const double Estarb = SK * Fb[4] * factor;
        // Estar = E/rho + (S* - un) * (S* + p/q)
        Eb += Estarb / rho;
        rb -= Estarb * E / (rho * rho);
        const double Ab = Estarb * B, Bb = Estarb * A;
        Sstarb += Ab + Bb;
        unb -= Ab;
        pb += Bb / q;
        double qb = -Bb * r / q;
        // factor = q / d, d = SK - S*
        qb += factorb / d;
        const double db = -factorb * factor / d;
        SKb += db;
        Sstarb -= db;
        // q = rho * (SK - un)
        rb += qb * (SK - un);
        SKb += qb * rho;
        unb -= qb * rho;
        // S* = N / D
        const double Nb = Sstarb / Dn;
        const double Db = -Sstarb * Sstar / Dn;
        pRb += Nb;
        pLb -= Nb;
        rLb += Nb * unL * (SL - unL) + Db * (SL - unL);
        unLb += Nb * rhoL * (SL - 2.0 * unL) - Db * rhoL;
        double SLb = Nb * rhoL * unL + Db * rhoL;
        rRb += -Nb * unR * (SR - unR) - Db * (SR - unR);
        unRb += -Nb * rhoR * (SR - 2.0 * unR) + Db * rhoR;
        double SRb = -Nb * rhoR * unR - Db * rhoR;
        if (left) SLb += SKb; else SRb += SKb;
        // Davis speeds
        double cLb = 0.0, cRb = 0.0;
        if (SL_from_L) { unLb += SLb; cLb -= SLb; } else { unRb += SLb; cRb -= SLb; }
        if (SR_from_L) { unLb += SRb; cLb += SRb; } else { unRb += SRb; cRb += SRb; }
        // c = sqrt(g p / rho)
        if (cL > 0.0) {
            pLb += cLb * g / (2.0 * cL * rhoL);
            rLb -= cLb * cL / (2.0 * rhoL);
        }
        if (cR > 0.0) {
            pRb += cRb * g / (2.0 * cR * rhoR);
            rRb -= cRb * cR / (2.0 * rhoR);
        }
    }

    // E = p/(g-1) + 0.5 rho |v|^2 of the selected side
    pb += Eb / (g - 1.0);
    rb += Eb * 0.5 * v2;
#pragma unroll
    for (int j = 0; j < 3; ++j) vb[j] += Eb * rho * v[j];
    vb[DIM - 1] += unb;

    const double sel[5] = {rb, vb[0], vb[1], vb[2], pb};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        WLb[k] += left ? sel[k] : 0.0;
        WRb[k] += left ? 0.0 : sel[k];
    }
    WLb[0] += rLb;
    WLb[DIM] += unLb;
    WLb[4] += pLb;
    WRb[0] += rRb;
    WRb[DIM] += unRb;
    WRb[4] += pRb;
}

}  // namespace vb
