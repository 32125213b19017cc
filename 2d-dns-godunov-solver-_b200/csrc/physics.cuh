// Device physics of the explicit Godunov step: limiters, face fluxes,
// boundary ghost states and transport properties.
//
// Each function restates the reference expression by expression (file:line
// cited) so that, compiled without multiply-add contraction (-fmad=false),
// the FP64 instantiation rounds exactly like the reference's Float64 code.
// The same templates compiled for float serve the mixed-precision path.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "gd2d_internal.h"

namespace gd2d {

// Julia Base.sign: -1, +1, or x itself for +-0 and NaN.
template <class T>
__device__ __forceinline__ T jl_sign(T x) {
    return x > T(0) ? T(1) : (x < T(0) ? T(-1) : x);
}

// Julia Base.min / max for floats: NaN-propagating, -0 < +0.
template <class T>
__device__ __forceinline__ T jl_min(T x, T y) {
    bool ypick = (y < x) || (signbit(y) && !signbit(x));
    return ypick ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}
template <class T>
__device__ __forceinline__ T jl_max(T x, T y) {
    bool ypick = (y > x) || (!signbit(y) && signbit(x));
    return ypick ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}

// ------------------------------------------------------------- limiters

// Minmod_Limiter, limiters.jl:33-35.
template <class T>
__device__ __forceinline__ T lim_minmod(T x, T y, T c) {
    return (jl_sign(x) + jl_sign(y)) * fabs(x * y) / (fabs(x) + fabs(y) + c);
}
// vanLeer_LimiterA, limiters.jl:41-43.
template <class T>
__device__ __forceinline__ T lim_vanleer(T a, T b, T c) {
    return (a * b + fabs(a * b)) / (a + b + c);
}
// vanAlbada_LimiterA, limiters.jl:54-56.
template <class T>
__device__ __forceinline__ T lim_vanalbada(T a, T b, T c) {
    return (a * (b * b + c) + b * (a * a + c)) / (a * a + b * b + T(2) * c);
}
// Venkatakrishnan (JCP 1995) in the two-argument slot (extension):
// o = outer difference (Delta-), c = central difference (the bound Delta+),
// eps2 = (K*HX)^3 scaled by the caller; at a local extremum (opposite signs)
// the bound is zero, which keeps the function continuous in c.
template <class T>
__device__ __forceinline__ T lim_venkat(T o, T c, T eps2) {
    if (o * c < T(0)) c = T(0);
    const T den = c * c + T(2) * o * o + o * c + eps2;
    if (den == T(0)) return T(0);
    return ((c * c + eps2) * o + T(2) * o * o * c) / den;
}

template <class T>
__device__ __forceinline__ T limiter(int kind, T a, T b, T ksi) {
    switch (kind) {
    case LIM_MINMOD: return lim_minmod(a, b, ksi);
    case LIM_VANLEER: return lim_vanleer(a, b, ksi);
    case LIM_VANALBADA: return lim_vanalbada(a, b, ksi);
    default: return T(0);
    }
}

// ---------------------------------------------------------------- fluxes

// AUSM+ helpers, AUSMflux2dFast.jl:23-53.
template <class T> __device__ __forceinline__ T Palfa_m(T M, T A) {
    return T(0.25) * (M - T(1)) * (M - T(1)) * (T(2) + M) - A * M * (M * M - T(1)) * (M * M - T(1));
}
template <class T> __device__ __forceinline__ T Palfa_p(T M, T A) {
    return T(0.25) * (M + T(1)) * (M + T(1)) * (T(2) - M) + A * M * (M * M - T(1)) * (M * M - T(1));
}
template <class T> __device__ __forceinline__ T Mbetta_p(T M, T B) {
    return T(0.25) * (M + T(1)) * (M + T(1)) + B * (M * M - T(1)) * (M * M - T(1));
}
template <class T> __device__ __forceinline__ T Mbetta_m(T M, T B) {
    return T(-0.25) * (M - T(1)) * (M - T(1)) - B * (M * M - T(1)) * (M * M - T(1));
}
template <class T> __device__ __forceinline__ T P_m(T M, T A) {
    return (fabs(M) >= T(1)) ? T(0.5) * (T(1) - jl_sign(M)) : Palfa_m(M, A);
}
template <class T> __device__ __forceinline__ T P_p(T M, T A) {
    return (fabs(M) >= T(1)) ? T(0.5) * (T(1) + jl_sign(M)) : Palfa_p(M, A);
}
template <class T> __device__ __forceinline__ T M_p(T M, T B) {
    return (fabs(M) >= T(1)) ? T(0.5) * (M + fabs(M)) : Mbetta_p(M, B);
}
template <class T> __device__ __forceinline__ T M_m(T M, T B) {
    return (fabs(M) >= T(1)) ? T(0.5) * (M - fabs(M)) : Mbetta_m(M, B);
}

// AUSMplusFlux2dFast, AUSMflux2dFast.jl:87-175 (Liou 1996).  The reference's
// muladd at :118-119 is fma(); its product 0.5*s is exact, so the fused and
// unfused forms round identically.
template <class T>
__device__ __forceinline__ void flux_ausm_plus(T rhoL, T UL, T VL, T PL, T rhoR, T UR, T VR, T PR,
                                               T nx, T ny, T side, T gamma, T g2, T *flux) {
    T htL = fma(T(0.5), (UL * UL + VL * VL), PL / rhoL + PL / rhoL / (gamma - T(1)));
    T htR = fma(T(0.5), (UR * UR + VR * VR), PR / rhoR + PR / rhoR / (gamma - T(1)));
    // g2 = 2*(gamma-1)/(gamma+1), evaluated once per case in the same order
    T sL = sqrt(g2 * htL);
    T sR = sqrt(g2 * htR);
    T vnL = UL * nx + VL * ny;
    T vnR = UR * nx + VR * ny;
    T aL_tilda = sL * jl_min(T(1), sL / fabs(vnL));
    T aR_tilda = sR * jl_min(T(1), sR / fabs(vnR));
    T a12 = jl_min(aL_tilda, aR_tilda);
    T ML = vnL / a12;
    T MR = vnR / a12;
    T m_dot12 = M_p(ML, T(1.0 / 8.0)) + M_m(MR, T(1.0 / 8.0));
    T p12 = P_p(ML, T(3.0 / 16.0)) * PL + P_m(MR, T(3.0 / 16.0)) * PR;
    T mp = T(0.5) * (m_dot12 + fabs(m_dot12));
    T mm = T(0.5) * (m_dot12 - fabs(m_dot12));
    flux[0] = -(a12 * (mp * rhoL + mm * rhoR) + T(0)) * side;
    flux[1] = -(a12 * (mp * rhoL * UL + mm * rhoR * UR) + p12 * nx) * side;
    flux[2] = -(a12 * (mp * rhoL * VL + mm * rhoR * VR) + p12 * ny) * side;
    flux[3] = -(a12 * (mp * rhoL * htL + mm * rhoR * htR) + T(0)) * side;
}

// AUSMplusM2020Flux2dFast, AUSMflux2dFast.jl:234-284 (Chen et al. 2020).
template <class T>
__device__ __forceinline__ void flux_ausm_m2020(T rhoL, T UL, T VL, T PL, T rhoR, T UR, T VR, T PR,
                                                T nx, T ny, T side, T gamma, T g2, T *flux) {
    const T pi = T(3.141592653589793);
    T htL = fma(T(0.5), (UL * UL + VL * VL), PL / rhoL + PL / rhoL / (gamma - T(1)));
    T htR = fma(T(0.5), (UR * UR + VR * VR), PR / rhoR + PR / rhoR / (gamma - T(1)));
    T htN = T(0.5) * (htL + htR - T(0.5) * ((UL * ny - VL * nx) * (UL * ny - VL * nx) +
                                            (UR * ny - VR * nx) * (UR * ny - VR * nx)));
    T as = sqrt(g2 * htN);
    T vnL = UL * nx + VL * ny;
    T vnR = UR * nx + VR * ny;
    T a12;
    if (T(0.5) * (UL * nx + VL * ny + UR * nx + VR * ny) >= T(0))
        a12 = as * as / jl_max(fabs(vnL), as);
    else
        a12 = as * as / jl_max(fabs(vnR), as);
    T f = T(0.5) * (T(1) - cos(pi * jl_min(T(1), jl_max(fabs(vnL / a12), fabs(vnR / a12)))));
    T g = T(0.5) * (T(1) + cos(pi * jl_min(PL / PR, PR / PL)));
    T p12 = -g * gamma * (PL + PR) * T(0.5) / a12 *
            (P_p(vnL / a12, T(3.0 / 16.0)) * P_m(vnR / a12, T(3.0 / 16.0)));
    T pux = p12 * (UR - UL);
    T puy = p12 * (VR - VL);
    T ps = T(0.5) * (PL + PR) - T(0.5) * T(0.5) * (rhoL + rhoR) * a12 * (UR - UL);
    T M12 = M_p(vnL / a12, T(1.0 / 8.0)) + M_m(vnR / a12, T(1.0 / 8.0))
            - T(0.5) * (T(1) - f) * (PR - PL) * T(2) / (rhoL + rhoR) / a12 / a12 * (T(1) - g);
    T m_dot12 = (M12 >= T(0)) ? M12 * a12 * rhoL : M12 * a12 * rhoR;
    T mp = T(0.5) * (m_dot12 + fabs(m_dot12));
    T mm = T(0.5) * (m_dot12 - fabs(m_dot12));
    flux[0] = -((T(0.5) * (m_dot12 + fabs(m_dot12) * T(1)) + T(0.5) * (m_dot12 - fabs(m_dot12)) * T(1)) + T(0)) * side;
    flux[1] = -((mp * UL + mm * UR) + ps * nx + pux) * side;
    flux[2] = -((mp * VL + mm * VR) + ps * ny + puy) * side;
    flux[3] = -((mp * htL + mm * htR) + T(0)) * side;
}

// RoeFlux2dFast, RoeFlux2dFast.jl:1-197 (Roe 1981; Harten entropy fix,
// delta = 0.2, on the acoustic waves).
template <class T>
__device__ __forceinline__ void flux_roe(T rhoL, T uL, T vL, T pL, T rhoR, T uR, T vR, T pR,
                                         T nx, T ny, T side, T gammaV, T *flux) {
    T mx = -ny, my = nx;
    T unL = uL * nx + vL * ny;
    T umL = uL * mx + vL * my;
    T aL = sqrt(gammaV * pL / rhoL);
    T HL = aL * aL / (gammaV - T(1)) + T(0.5) * (uL * uL + vL * vL);
    T unR = uR * nx + vR * ny;
    T umR = uR * mx + vR * my;
    T aR = sqrt(gammaV * pR / rhoR);
    T HR = aR * aR / (gammaV - T(1)) + T(0.5) * (uR * uR + vR * vR);
    T RT = sqrt(rhoR / rhoL);
    T rho = RT * rhoL;
    T u = (uL + RT * uR) / (T(1) + RT);
    T v = (vL + RT * vR) / (T(1) + RT);
    T H = (HL + RT * HR) / (T(1) + RT);
    T a = sqrt((gammaV - T(1)) * (H - T(0.5) * (u * u + v * v)));
    T un = u * nx + v * ny;
    T um = u * mx + v * my;
    T drho = rhoR - rhoL, dp = pR - pL, dun = unR - unL, dum = umR - umL;
    T LdU1 = (dp - rho * a * dun) / (T(2) * a * a);
    T LdU2 = rho * dum;
    T LdU3 = drho - dp / (a * a);
    T LdU4 = (dp + rho * a * dun) / (T(2) * a * a);
    T ws1 = fabs(un - a), ws2 = fabs(un), ws3 = fabs(un), ws4 = fabs(un + a);
    const T dws = T(1.0 / 5.0);
    if (ws1 < dws) ws1 = T(0.5) * (ws1 * ws1 / dws + dws);
    if (ws4 < dws) ws4 = T(0.5) * (ws4 * ws4 / dws + dws);
    T Rv21 = u - a * nx, Rv31 = v - a * ny, Rv41 = H - un * a;
    T Rv22 = mx, Rv32 = my, Rv42 = um;
    T Rv23 = u, Rv33 = v, Rv43 = T(0.5) * (u * u + v * v);
    T Rv24 = u + a * nx, Rv34 = v + a * ny, Rv44 = H + un * a;
    T diss1 = T(0), diss2 = T(0), diss3 = T(0), diss4 = T(0);
    diss1 = diss1 + ws1 * LdU1 * T(1);
    diss1 = diss1 + ws2 * LdU2 * T(0);
    diss1 = diss1 + ws3 * LdU3 * T(1);
    diss1 = diss1 + ws4 * LdU4 * T(1);
    diss2 = diss2 + ws1 * LdU1 * Rv21;
    diss2 = diss2 + ws2 * LdU2 * Rv22;
    diss2 = diss2 + ws3 * LdU3 * Rv23;
    diss2 = diss2 + ws4 * LdU4 * Rv24;
    diss3 = diss3 + ws1 * LdU1 * Rv31;
    diss3 = diss3 + ws2 * LdU2 * Rv32;
    diss3 = diss3 + ws3 * LdU3 * Rv33;
    diss3 = diss3 + ws4 * LdU4 * Rv34;
    diss4 = diss4 + ws1 * LdU1 * Rv41;
    diss4 = diss4 + ws2 * LdU2 * Rv42;
    diss4 = diss4 + ws3 * LdU3 * Rv43;
    diss4 = diss4 + ws4 * LdU4 * Rv44;
    T fL1 = rhoL * unL, fL2 = rhoL * unL * uL + pL * nx, fL3 = rhoL * unL * vL + pL * ny, fL4 = rhoL * unL * HL;
    T fR1 = rhoR * unR, fR2 = rhoR * unR * uR + pR * nx, fR3 = rhoR * unR * vR + pR * ny, fR4 = rhoR * unR * HR;
    flux[0] = T(-0.5) * (fL1 + fR1 - diss1) * side;
    flux[1] = T(-0.5) * (fL2 + fR2 - diss2) * side;
    flux[2] = T(-0.5) * (fL3 + fR3 - diss3) * side;
    flux[3] = T(-0.5) * (fL4 + fR4 - diss4) * side;
}

template <int FLUX, class T>
__device__ __forceinline__ void face_flux_fn(const T *L, const T *R, T nx, T ny, T side, T gamma, T g2,
                                             T *f) {
    if (FLUX == FLUX_ROE)
        flux_roe<T>(L[0], L[1], L[2], L[3], R[0], R[1], R[2], R[3], nx, ny, side, gamma, f);
    else if (FLUX == FLUX_AUSM_M2020)
        flux_ausm_m2020<T>(L[0], L[1], L[2], L[3], R[0], R[1], R[2], R[3], nx, ny, side, gamma, g2, f);
    else
        flux_ausm_plus<T>(L[0], L[1], L[2], L[3], R[0], R[1], R[2], R[3], nx, ny, side, gamma, g2, f);
}

// ---------------------------------------------------------- thermophysics

// calcAirViscosityPowerLawFromT, thermo.jl:13-15.
__device__ __forceinline__ double visc_power_law(double T) { return 1.716e-5 * pow(T / 273.11, 2.0 / 3.0); }
// calcAirCpLow / High, thermo.jl:17-41 (Julia's literal powers: T^-2 = inv(T)^2,
// T^-1 = inv(T), T^2 = T*T, T^3 = T*T*T, T^4 = pow).
__device__ __forceinline__ double cp_low(double T) {
    double iT = 1.0 / T;
    return 2898903.0 * (iT * iT) + -56496.26 * iT + 1437.799 + -1.653609 * T + 0.003062254 * (T * T) +
           -2.279138e-6 * (T * T * T) + 6.272365e-10 * pow(T, 4.0);
}
__device__ __forceinline__ double cp_high(double T) {
    double iT = 1.0 / T;
    return 6.932494e+7 * (iT * iT) + -361053.2 * iT + 1476.665 + -0.06138349 * T + 2.027963e-5 * (T * T) +
           -3.075525e-9 * (T * T * T) + 1.888054e-13 * pow(T, 4.0);
}
// calcAirHeatCapacityFromT, thermo.jl:43-54.
__device__ __forceinline__ double cp_air(double T) {
    if (T < 200.0) return cp_low(200.0);
    else if (T > 200.0 && T < 1000.0) return cp_low(T);
    else if (T >= 1000.0 && T < 6000.0) return cp_high(T);
    else return cp_high(6000.0);
}
// calcAirConductivityFromT, thermo.jl:57-60.
__device__ __forceinline__ double air_conductivity(double T) {
    return 15.0 / 4.0 * 8.314462 / 28.9647 * visc_power_law(T) *
           (4.0 / 15.0 * cp_air(T) * 28.9647 / 8.314462 + 1.0 / 3.0);
}
// calcSutherlandViscosityOF, sutherland.jl:2-5.
template <class T>
__device__ __forceinline__ T sutherland(T t) { return T(1.4792e-6) * sqrt(t) / (T(1) + T(116) / t); }

// ------------------------------------------------------ boundary states

// computeTGV2d, initfields_TGV2d.jl:9-27.
__device__ __forceinline__ void tgv_state(const DevCase &P, double x, double y, double time, double *pv) {
    double Pp = P.tgv_P0, U = P.tgv_U0, L = P.tgv_L, mu = P.tgv_mu;
    double T = Pp / P.R;
    double F = exp(-2.0 * mu * time / L / L);
    double Fp = exp(-4.0 * mu * time / L / L);
    pv[0] = Pp / P.R / T;
    pv[1] = U * sin(x / L) * cos(y / L) * F;
    pv[2] = -U * cos(x / L) * sin(y / L) * F;
    pv[3] = Pp + 0.25 * U * U * (cos(2.0 * x / L) + cos(2.0 * y / L)) * Fp;
}

// getSymmetricalPointAboutCellEdge, calcGradients.jl:21-34.
__device__ __forceinline__ void symmetrical_point(double px, double py, double x0, double y0, double x1,
                                                  double y1, double *sp) {
    double dx = x1 - x0, dy = y1 - y0;
    double a = (dx * dx - dy * dy) / (dx * dx + dy * dy);
    double b = 2.0 * dx * dy / (dx * dx + dy * dy);
    sp[0] = a * (px - x0) + b * (py - y0) + x0;
    sp[1] = b * (px - x0) - a * (py - y0) + y0;
}

// Ghost state of a boundary face (tag slot `slot` of the case's table):
// inflow (boundaryConditions2d.jl:34-39), outflow copy (:47-52), slip wall
// by Krivodonova-Berger mirroring (bcInviscidWall.jl:21-38), analytic TGV
// at the mirror point (boundaryConditions_TGV2d.jl:16-30) and the no-slip
// isothermal wall extension (u'=-u, v'=-v, p'=p, rho'=p/(R Tw)).
template <class T>
__device__ __forceinline__ void bc_ghost(const DevCase &P, const DevMesh &m, int slot, int64_t g, int k,
                                         const T *uL, T nx, T ny, double t, T *gs) {
    switch (P.bc_kind[slot]) {
    case BC_INFLOW:
        gs[0] = T(P.bc_rho[slot]); gs[1] = T(P.bc_u[slot]); gs[2] = T(P.bc_v[slot]); gs[3] = T(P.bc_p[slot]);
        break;
    case BC_SLIP:
        gs[0] = uL[0];
        gs[1] = uL[1] * (ny * ny - nx * nx) - T(2) * nx * ny * uL[2];
        gs[2] = uL[2] * (nx * nx - ny * ny) - T(2) * nx * ny * uL[1];
        gs[3] = uL[3];
        break;
    case BC_NOSLIP_ISOTHERMAL:
        gs[0] = uL[3] / (T(P.R) * T(P.bc_Tw[slot]));
        gs[1] = -uL[1];
        gs[2] = -uL[2];
        gs[3] = uL[3];
        break;
    case BC_TGV: {
        int2 e = m.c2n[(int64_t)k * m.Nc + g];
        double2 c = m.mid[g];
        double sp[2], pv[4];
        symmetrical_point(c.x, c.y, m.xnode[e.x], m.ynode[e.x], m.xnode[e.y], m.ynode[e.y], sp);
        tgv_state(P, sp[0], sp[1], t, pv);
        gs[0] = T(pv[0]); gs[1] = T(pv[1]); gs[2] = T(pv[2]); gs[3] = T(pv[3]);
        break;
    }
    default:  // outflow
        gs[0] = uL[0]; gs[1] = uL[1]; gs[2] = uL[2]; gs[3] = uL[3];
        break;
    }
}

}  // namespace gd2d
