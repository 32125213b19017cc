/*
 * godunov2d_oracle.c -- CPU oracle for the explicit Godunov step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the FP64 CPU
 * algorithm of the reference solver (dimaZloy/2D-DNS-godunov-solver-, Julia)
 * so that the CUDA path can be checked against it.  It is test infrastructure, never
 * the product: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline arm may load it.
 *
 * Parity status: UNPINNED by reference-produced vectors.  The reference is
 * Julia (not installed here, no network) and records no golden numbers; this
 * restatement is cross-checked instead against analytic known answers
 * (flux consistency / antisymmetry / upwinding, uniform-flow preservation,
 * Green-Gauss exactness on linear fields, Taylor-Green decay) and against an
 * independent high-precision evaluation of the flux formulas
 * (tests/golden/make_golden.py).
 *
 * Evaluation order follows the Julia source expression by expression; build
 * with -ffp-contract=off so that no multiply-add is fused except where the
 * reference writes muladd (AUSMflux2dFast.jl:118-119), which is fma() here.
 *
 * Index conventions: every mesh array is the reference's column-major Julia
 * array (mesh2d_Int32, primeObjects.jl:109-135) with 1-based Int32 indices and
 * negative boundary tags, exactly as read by readMesh2dHDF5 (utilsIO.jl:107).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAX_BC 8

/* mesh2d_Int32 (primeObjects.jl:109-135); column-major (rows, cols). */
typedef struct {
    int64_t nCells, nNodes;
    int32_t nNeibCells, pad_;
    const double *xNodes, *yNodes;
    const int32_t *mesh_connectivity;  /* nCells x 7 */
    const int32_t *cell_stiffness;     /* nCells x 4 */
    const int32_t *cells2nodes;        /* nCells x 8 */
    const double *cell_edges_Nx;       /* nCells x 4 */
    const double *cell_edges_Ny;       /* nCells x 4 */
    const double *cell_edges_length;   /* nCells x 4 */
    const double *cell_areas;          /* nCells */
    const double *HX;                  /* nCells */
    const double *cell_mid_points;     /* nCells x 2 */
    const int32_t *cell_clusters;      /* nNodes x nNeibCells */
    const double *node_stencils;       /* nNodes x nNeibCells */
    const int32_t *node2cellL2up;      /* nCells x 8 */
    const int32_t *node2cellL2down;    /* nCells x 8 */
} orc_mesh;

typedef struct {
    int32_t tag, kind;
    double rho, u, v, p, Tw;
} orc_bc;

/* Enumerations shared in meaning with the product's parameter block. */
enum { ORC_FLUX_AUSM = 1, ORC_FLUX_ROE = 2, ORC_FLUX_AUSM_M2020 = 3 };
enum { ORC_LIM_NONE = 0, ORC_LIM_MINMOD = 1, ORC_LIM_VENKAT = 2,
       ORC_LIM_VANLEER = 3, ORC_LIM_VANALBADA = 4 };
enum { ORC_BC_INFLOW = 1, ORC_BC_OUTFLOW = 2, ORC_BC_SLIP = 3,
       ORC_BC_NOSLIP_ISOTHERMAL = 4, ORC_BC_TGV = 5 };
enum { ORC_VISC_NONE = 0, ORC_VISC_REFERENCE = 1, ORC_VISC_SUTHERLAND = 2,
       ORC_VISC_CONSTANT = 3 };

typedef struct {
    /* THERMOPHYSICS (thermo.jl:4-10) */
    double RGAS, Gamma, Cp, mu, kGas;
    /* CONTROLS (primeObjects.jl:233-243) subset + solver selectors */
    double CFL, dt, beta;
    double ksi;          /* Minmod constant, 1e-12 (computeslope2d.jl:116) */
    double venkat_K;     /* Venkatakrishnan K, eps^2 = (K*HX)^3 */
    double mu_ref;       /* viscosity scale for the Sutherland/constant models */
    double T_ref;        /* temperature where mu = mu_ref (Sutherland) */
    double Pr;
    double tgv_U0, tgv_P0, tgv_L, tgv_mu;  /* computeTGV2d constants */
    double minDensityConstrained, maxDensityConstrained;  /* CONTROLS, primeObjects.jl:241-242 */
    int32_t flux, limiter, viscosity, art_viscosity;
    int32_t dt_mode;     /* 0: fixed dt, 1: dt = CFL-based tau */
    int32_t init_nodes;  /* 0: node primitives zero at step 1 (reference) */
    int32_t nthreads;
    int32_t n_bc;
    int32_t densityConstrained;  /* CONTROLS flag, primeObjects.jl:240 */
    int32_t pad2_;
    orc_bc bc[ORC_MAX_BC];
} orc_params;

typedef struct {
    double dt, flowTime, tau, velmax;
    double residual[4];
    double rhoMin, rhoMax;
    double totals[4];
    double Ek;
    int64_t step;
    int32_t nonfinite, pad_;
} orc_stats;

typedef struct {
    orc_mesh m;
    orc_params p;
    /* fields2d (primeObjects.jl:85-106) */
    double *densityCells, *UxCells, *UyCells, *pressureCells, *aSoundCells, *VMAXCells;
    double *densityNodes, *UxNodes, *UyNodes, *pressureNodes;
    /* conservative work arrays of the reference top-level script (testInviscidFluxesGPUx32.jl:183-192) */
    double *UconsCellsOld, *UconsCellsNew, *UconsNodesOld, *UConsDiffCells, *Delta, *FLUXES;
    /* viscous work (calcDiffTerm.jl:37-62) and artificial viscosity */
    double *g1x[3], *g1y[3], *lap[3], *muArt, *dUdx, *dVdy;
    double *charLen; /* 2*area/perimeter per cell (local CFL length) */
    double flowTime, maxEdge, suth_ref, gamma_over_Pr;
    int64_t curIter;
    int32_t (*cellsThreads)[2];
    int32_t (*nodesThreads)[2];
} orc_state;

/* ---------------------------------------------------------------- helpers */

#define IDX(a, n, i, j) (a)[(int64_t)(i) + (int64_t)(j) * (int64_t)(n)]

/* Julia Base.sign for Float64: -1, +1, or x itself for +-0 and NaN. */
static inline double jl_sign(double x) {
    if (x > 0.0) return 1.0;
    if (x < 0.0) return -1.0;
    return x;
}

/* Julia Base.min for Float64: NaN-propagating, -0.0 < +0.0. */
static inline double jl_min(double x, double y) {
    int ypick = (y < x) || ((signbit(y) != 0) > (signbit(x) != 0));
    return ypick ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}

static inline double jl_max(double x, double y) {
    int ypick = (y > x) || ((signbit(y) != 0) < (signbit(x) != 0));
    return ypick ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}

/* -------------------------------------------------------------- limiters */

/* Minmod_Limiter, limiters.jl:33-35 (a smooth harmonic-mean form). */
double orc_minmod(double x, double y, double c) {
    return (jl_sign(x) + jl_sign(y)) * fabs(x * y) / (fabs(x) + fabs(y) + c);
}

/* vanLeer_LimiterA, limiters.jl:41-43. */
double orc_vanleer(double a, double b, double c) {
    return (a * b + fabs(a * b)) / (a + b + c);
}

/* vanAlbada_LimiterA, limiters.jl:54-56. */
double orc_vanalbada(double a, double b, double c) {
    return (a * (b * b + c) + b * (a * a + c)) / (a * a + b * b + 2.0 * c);
}

/* Venkatakrishnan (JCP 1995) smooth limiter in the two-argument slot
 * (extension; the reference has no Venkatakrishnan limiter).  o = outer
 * (upwind) difference playing Delta-, c = central difference playing the
 * bound Delta+, eps2 = (K*HX)^3 (scaled by the caller):
 *   phi = ((c^2+eps2) o + 2 o^2 c) / (c^2 + 2 o^2 + o c + eps2).
 * When c has the opposite sign the cell is a local extremum and the bound is
 * zero (c := 0), which keeps the function continuous in c. */
double orc_venkat(double o, double c, double eps2) {
    if (o * c < 0.0) c = 0.0;
    double den = c * c + 2.0 * o * o + o * c + eps2;
    if (den == 0.0) return 0.0;
    return ((c * c + eps2) * o + 2.0 * o * o * c) / den;
}

/* ---------------------------------------------------------------- fluxes */

/* AUSM+ helpers, AUSMflux2dFast.jl:23-53. */
static inline double Palfa_m(double M, double A) {
    return 0.25 * (M - 1.0) * (M - 1.0) * (2.0 + M) - A * M * (M * M - 1.0) * (M * M - 1.0);
}
static inline double Palfa_p(double M, double A) {
    return 0.25 * (M + 1.0) * (M + 1.0) * (2.0 - M) + A * M * (M * M - 1.0) * (M * M - 1.0);
}
static inline double Mbetta_p(double M, double B) {
    return 0.25 * (M + 1.0) * (M + 1.0) + B * (M * M - 1.0) * (M * M - 1.0);
}
static inline double Mbetta_m(double M, double B) {
    return -0.25 * (M - 1.0) * (M - 1.0) - B * (M * M - 1.0) * (M * M - 1.0);
}
static inline double P_m(double M, double A) {
    return (fabs(M) >= 1.0) ? 0.5 * (1.0 - jl_sign(M)) : Palfa_m(M, A);
}
static inline double P_p(double M, double A) {
    return (fabs(M) >= 1.0) ? 0.5 * (1.0 + jl_sign(M)) : Palfa_p(M, A);
}
static inline double M_p(double M, double B) {
    return (fabs(M) >= 1.0) ? 0.5 * (M + fabs(M)) : Mbetta_p(M, B);
}
static inline double M_m(double M, double B) {
    return (fabs(M) >= 1.0) ? 0.5 * (M - fabs(M)) : Mbetta_m(M, B);
}

/* AUSMplusFlux2dFast, AUSMflux2dFast.jl:87-175. */
void orc_ausm_plus(double rhoL, double UL, double VL, double PL,
                   double rhoR, double UR, double VR, double PR,
                   double nx, double ny, double side, double gamma, double *flux) {
    double htL = fma(0.5, (UL * UL + VL * VL), PL / rhoL + PL / rhoL / (gamma - 1.0));
    double htR = fma(0.5, (UR * UR + VR * VR), PR / rhoR + PR / rhoR / (gamma - 1.0));
    double sL = sqrt(2.0 * (gamma - 1.0) / (gamma + 1.0) * htL);
    double sR = sqrt(2.0 * (gamma - 1.0) / (gamma + 1.0) * htR);
    double aL_tilda = sL * jl_min(1.0, sL / fabs(UL * nx + VL * ny));
    double aR_tilda = sR * jl_min(1.0, sR / fabs(UR * nx + VR * ny));
    double a12 = jl_min(aL_tilda, aR_tilda);
    double ML = (UL * nx + VL * ny) / a12;
    double MR = (UR * nx + VR * ny) / a12;
    double m_dot12 = M_p(ML, 1.0 / 8.0) + M_m(MR, 1.0 / 8.0);
    double p12 = P_p(ML, 3.0 / 16.0) * PL + P_m(MR, 3.0 / 16.0) * PR;
    double mp = 0.5 * (m_dot12 + fabs(m_dot12));
    double mm = 0.5 * (m_dot12 - fabs(m_dot12));
    flux[0] = -(a12 * (mp * rhoL + mm * rhoR) + 0.0) * side;
    flux[1] = -(a12 * (mp * rhoL * UL + mm * rhoR * UR) + p12 * nx) * side;
    flux[2] = -(a12 * (mp * rhoL * VL + mm * rhoR * VR) + p12 * ny) * side;
    flux[3] = -(a12 * (mp * rhoL * htL + mm * rhoR * htR) + 0.0) * side;
}

/* AUSMplusM2020Flux2dFast, AUSMflux2dFast.jl:234-284 (Chen et al. 2020). */
void orc_ausm_m2020(double rhoL, double UL, double VL, double PL,
                    double rhoR, double UR, double VR, double PR,
                    double nx, double ny, double side, double gamma, double *flux) {
    const double pi = 3.141592653589793;
    double htL = fma(0.5, (UL * UL + VL * VL), PL / rhoL + PL / rhoL / (gamma - 1.0));
    double htR = fma(0.5, (UR * UR + VR * VR), PR / rhoR + PR / rhoR / (gamma - 1.0));
    double htN = 0.5 * (htL + htR - 0.5 * ((UL * ny - VL * nx) * (UL * ny - VL * nx) +
                                           (UR * ny - VR * nx) * (UR * ny - VR * nx)));
    double as = sqrt(2.0 * (gamma - 1.0) / (gamma + 1.0) * htN);
    double a12;
    if (0.5 * (UL * nx + VL * ny + UR * nx + VR * ny) >= 0)
        a12 = as * as / jl_max(fabs(UL * nx + VL * ny), as);
    else
        a12 = as * as / jl_max(fabs(UR * nx + VR * ny), as);
    double f = 0.5 * (1.0 - cos(pi * jl_min(1.0, jl_max(fabs((UL * nx + VL * ny) / a12),
                                                        fabs((UR * nx + VR * ny) / a12)))));
    double g = 0.5 * (1.0 + cos(pi * jl_min(PL / PR, PR / PL)));
    double p12 = -g * gamma * (PL + PR) * 0.5 / a12 *
                 (P_p((UL * nx + VL * ny) / a12, 3.0 / 16.0) * P_m((UR * nx + VR * ny) / a12, 3.0 / 16.0));
    double pux = p12 * (UR - UL);
    double puy = p12 * (VR - VL);
    double ps = 0.5 * (PL + PR) - 0.5 * 0.5 * (rhoL + rhoR) * a12 * (UR - UL);
    double M12 = M_p((UL * nx + VL * ny) / a12, 1.0 / 8.0) + M_m((UR * nx + VR * ny) / a12, 1.0 / 8.0)
                 - 0.5 * (1.0 - f) * (PR - PL) * 2.0 / (rhoL + rhoR) / a12 / a12 * (1.0 - g);
    double m_dot12 = (M12 >= 0.0) ? M12 * a12 * rhoL : M12 * a12 * rhoR;
    flux[0] = -((0.5 * (m_dot12 + fabs(m_dot12) * 1.0) + 0.5 * (m_dot12 - fabs(m_dot12)) * 1.0) + 0.0) * side;
    flux[1] = -((0.5 * (m_dot12 + fabs(m_dot12)) * UL + 0.5 * (m_dot12 - fabs(m_dot12)) * UR) + ps * nx + pux) * side;
    flux[2] = -((0.5 * (m_dot12 + fabs(m_dot12)) * VL + 0.5 * (m_dot12 - fabs(m_dot12)) * VR) + ps * ny + puy) * side;
    flux[3] = -((0.5 * (m_dot12 + fabs(m_dot12)) * htL + 0.5 * (m_dot12 - fabs(m_dot12)) * htR) + 0.0) * side;
}

/* RoeFlux2dFast, RoeFlux2dFast.jl:1-197 (Roe 1981, Harten fix on waves 1,4). */
void orc_roe(double rhoL, double uL, double vL, double pL,
             double rhoR, double uR, double vR, double pR,
             double nx, double ny, double side, double gammaV, double *flux) {
    double mx = -ny, my = nx;
    double unL = uL * nx + vL * ny;
    double umL = uL * mx + vL * my;
    double aL = sqrt(gammaV * pL / rhoL);
    double HL = aL * aL / (gammaV - 1.0) + 0.5 * (uL * uL + vL * vL);
    double unR = uR * nx + vR * ny;
    double umR = uR * mx + vR * my;
    double aR = sqrt(gammaV * pR / rhoR);
    double HR = aR * aR / (gammaV - 1.0) + 0.5 * (uR * uR + vR * vR);
    double RT = sqrt(rhoR / rhoL);
    double rho = RT * rhoL;
    double u = (uL + RT * uR) / (1.0 + RT);
    double v = (vL + RT * vR) / (1.0 + RT);
    double H = (HL + RT * HR) / (1.0 + RT);
    double a = sqrt((gammaV - 1.0) * (H - 0.5 * (u * u + v * v)));
    double un = u * nx + v * ny;
    double um = u * mx + v * my;
    double drho = rhoR - rhoL, dp = pR - pL, dun = unR - unL, dum = umR - umL;
    double LdU1 = (dp - rho * a * dun) / (2.0 * a * a);
    double LdU2 = rho * dum;
    double LdU3 = drho - dp / (a * a);
    double LdU4 = (dp + rho * a * dun) / (2.0 * a * a);
    double ws1 = fabs(un - a), ws2 = fabs(un), ws3 = fabs(un), ws4 = fabs(un + a);
    double dws1 = 1.0 / 5.0;
    if (ws1 < dws1) ws1 = 0.5 * (ws1 * ws1 / dws1 + dws1);
    double dws4 = 1.0 / 5.0;
    if (ws4 < dws4) ws4 = 0.5 * (ws4 * ws4 / dws4 + dws4);
    double Rv11 = 1.0, Rv21 = u - a * nx, Rv31 = v - a * ny, Rv41 = H - un * a;
    double Rv12 = 0.0, Rv22 = mx, Rv32 = my, Rv42 = um;
    double Rv13 = 1.0, Rv23 = u, Rv33 = v, Rv43 = 0.5 * (u * u + v * v);
    double Rv14 = 1.0, Rv24 = u + a * nx, Rv34 = v + a * ny, Rv44 = H + un * a;
    double diss1 = 0.0, diss2 = 0.0, diss3 = 0.0, diss4 = 0.0;
    diss1 = diss1 + ws1 * LdU1 * Rv11;
    diss1 = diss1 + ws2 * LdU2 * Rv12;
    diss1 = diss1 + ws3 * LdU3 * Rv13;
    diss1 = diss1 + ws4 * LdU4 * Rv14;
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
    double fL1 = rhoL * unL, fL2 = rhoL * unL * uL + pL * nx, fL3 = rhoL * unL * vL + pL * ny, fL4 = rhoL * unL * HL;
    double fR1 = rhoR * unR, fR2 = rhoR * unR * uR + pR * nx, fR3 = rhoR * unR * vR + pR * ny, fR4 = rhoR * unR * HR;
    flux[0] = -0.5 * (fL1 + fR1 - diss1) * side;
    flux[1] = -0.5 * (fL2 + fR2 - diss2) * side;
    flux[2] = -0.5 * (fL3 + fR3 - diss3) * side;
    flux[3] = -0.5 * (fL4 + fR4 - diss4) * side;
}

void orc_flux(int kind, const double *uL, const double *uR, double nx, double ny,
              double side, double gamma, double *flux) {
    if (kind == ORC_FLUX_ROE)
        orc_roe(uL[0], uL[1], uL[2], uL[3], uR[0], uR[1], uR[2], uR[3], nx, ny, side, gamma, flux);
    else if (kind == ORC_FLUX_AUSM_M2020)
        orc_ausm_m2020(uL[0], uL[1], uL[2], uL[3], uR[0], uR[1], uR[2], uR[3], nx, ny, side, gamma, flux);
    else
        orc_ausm_plus(uL[0], uL[1], uL[2], uL[3], uR[0], uR[1], uR[2], uR[3], nx, ny, side, gamma, flux);
}

/* --------------------------------------------------------- thermophysics */

/* calcAirViscosityPowerLawFromT, thermo.jl:13-15. */
static double visc_power_law(double T) { return 1.716e-5 * pow(T / 273.11, 2.0 / 3.0); }

/* calcAirCpLow / calcAirCpHigh, thermo.jl:17-41.  Julia lowers T^(-2) to
 * inv(T)^2, T^(-1) to inv(T), T^2 to T*T, T^3 to T*T*T; T^4 is pow(T, 4). */
static double cp_low(double T) {
    double iT = 1.0 / T;
    return 2898903.0 * (iT * iT) + -56496.26 * iT + 1437.799 + -1.653609 * T +
           0.003062254 * (T * T) + -2.279138e-6 * (T * T * T) + 6.272365e-10 * pow(T, 4.0);
}
static double cp_high(double T) {
    double iT = 1.0 / T;
    return 6.932494e+7 * (iT * iT) + -361053.2 * iT + 1476.665 + -0.06138349 * T +
           2.027963e-5 * (T * T) + -3.075525e-9 * (T * T * T) + 1.888054e-13 * pow(T, 4.0);
}
/* calcAirHeatCapacityFromT, thermo.jl:43-54 (T == 200 exactly falls to Cp(6000)). */
static double cp_air(double T) {
    if (T < 200.0) return cp_low(200.0);
    else if (T > 200.0 && T < 1000.0) return cp_low(T);
    else if (T >= 1000.0 && T < 6000.0) return cp_high(T);
    else return cp_high(6000.0);
}
/* calcAirConductivityFromT, thermo.jl:57-60. */
double orc_air_conductivity(double T) {
    return 15.0 / 4.0 * 8.314462 / 28.9647 * visc_power_law(T) *
           (4.0 / 15.0 * cp_air(T) * 28.9647 / 8.314462 + 1.0 / 3.0);
}
/* calcSutherlandViscosityOF, sutherland.jl:2-5. */
double orc_sutherland(double T) { return 1.4792e-6 * sqrt(T) / (1.0 + 116.0 / T); }

/* ---------------------------------------------------- boundary conditions */

/* getSymmetricalPointAboutCellEdge, calcGradients.jl:21-34. */
static void symmetrical_point(double px, double py, double x0, double y0, double x1, double y1,
                              double *sp) {
    double dx = x1 - x0, dy = y1 - y0;
    double a = (dx * dx - dy * dy) / (dx * dx + dy * dy);
    double b = 2.0 * dx * dy / (dx * dx + dy * dy);
    sp[0] = a * (px - x0) + b * (py - y0) + x0;
    sp[1] = b * (px - x0) - a * (py - y0) + y0;
}

/* computeTGV2d, initfields_TGV2d.jl:9-27 (U, P, L, mu are parameters). */
void orc_tgv(const orc_params *p, double x, double y, double time, double *pv) {
    double P = p->tgv_P0, U = p->tgv_U0, L = p->tgv_L, mu = p->tgv_mu;
    double T = P / p->RGAS;
    double F = exp(-2.0 * mu * time / L / L);
    double Fp = exp(-4.0 * mu * time / L / L);
    pv[0] = P / p->RGAS / T;
    pv[1] = U * sin(x / L) * cos(y / L) * F;
    pv[2] = -U * cos(x / L) * sin(y / L) * F;
    pv[3] = P + 0.25 * U * U * (cos(2.0 * x / L) + cos(2.0 * y / L)) * Fp;
}

/* Ghost state for a boundary face, dispatched on the tag in cell_stiffness.
 *  INFLOW   fixed state           (boundaryConditions2d.jl:34-39)
 *  OUTFLOW  copy of the cell      (boundaryConditions2d.jl:47-52)
 *  SLIP     Krivodonova-Berger velocity mirror (bcInviscidWall.jl:21-38)
 *  TGV      analytic state at the mirror point (boundaryConditions_TGV2d.jl:16-30)
 *  NOSLIP_ISOTHERMAL (extension): u'=-u, v'=-v, p'=p, rho'=p/(R Tw)
 * Returns 0, or -1 for a tag with no entry in the table. */
int orc_bc_ghost(const orc_state *s, int64_t i, int k, int32_t tag, const double *uL,
                 double t, double *g) {
    const orc_params *p = &s->p;
    const orc_mesh *m = &s->m;
    int64_t n = m->nCells;
    for (int b = 0; b < p->n_bc; ++b) {
        if (p->bc[b].tag != tag) continue;
        const orc_bc *bc = &p->bc[b];
        double nx = IDX(m->cell_edges_Nx, n, i, k), ny = IDX(m->cell_edges_Ny, n, i, k);
        switch (bc->kind) {
        case ORC_BC_INFLOW:
            g[0] = bc->rho; g[1] = bc->u; g[2] = bc->v; g[3] = bc->p;
            return 0;
        case ORC_BC_OUTFLOW:
            g[0] = uL[0]; g[1] = uL[1]; g[2] = uL[2]; g[3] = uL[3];
            return 0;
        case ORC_BC_SLIP:
            g[0] = uL[0];
            g[1] = uL[1] * (ny * ny - nx * nx) - 2.0 * nx * ny * uL[2];
            g[2] = uL[2] * (nx * nx - ny * ny) - 2.0 * nx * ny * uL[1];
            g[3] = uL[3];
            return 0;
        case ORC_BC_NOSLIP_ISOTHERMAL:
            g[0] = uL[3] / (p->RGAS * bc->Tw);
            g[1] = -uL[1];
            g[2] = -uL[2];
            g[3] = uL[3];
            return 0;
        case ORC_BC_TGV: {
            int index = 2 * k; /* 0-based column of node (2k-1) */
            int32_t n1 = IDX(m->cells2nodes, n, i, index) - 1;
            int32_t n2 = IDX(m->cells2nodes, n, i, index + 1) - 1;
            double sp[2];
            symmetrical_point(IDX(m->cell_mid_points, n, i, 0), IDX(m->cell_mid_points, n, i, 1),
                              m->xNodes[n1], m->yNodes[n1], m->xNodes[n2], m->yNodes[n2], sp);
            orc_tgv(p, sp[0], sp[1], t, g);
            return 0;
        }
        default:
            return -1;
        }
    }
    return -1;
}

/* ------------------------------------------------------- thread partition */

/* distibuteCellsInThreadsSA, partMesh2d.jl:2-34 (1-based inclusive ranges,
 * thread 1 absorbs the remainder).  For one thread the reference returns an
 * empty [0,0] range; here one thread covers [1, n]. */
void orc_partition(int32_t nThreads, int64_t n, int32_t (*r)[2]) {
    if (nThreads <= 1) { r[0][0] = 1; r[0][1] = (int32_t)n; return; }
    int64_t nParts = n / nThreads;
    for (int i = 1; i <= nThreads; ++i) r[i - 1][1] = (int32_t)(n - nParts * (nThreads - i));
    for (int i = 1; i <= nThreads; ++i) r[i - 1][0] = (int32_t)(r[i - 1][1] - nParts + 1);
    r[0][0] = 1;
}

typedef void (*range_fn)(orc_state *s, int64_t begin, int64_t end, void *ctx);
typedef struct { orc_state *s; int64_t b, e; range_fn fn; void *ctx; } job_t;
static void *job_run(void *a) { job_t *j = (job_t *)a; j->fn(j->s, j->b, j->e, j->ctx); return NULL; }

/* Threads.@threads over the partition ranges (0-based half-open). */
static void parallel(orc_state *s, int32_t (*ranges)[2], range_fn fn, void *ctx) {
    int nt = s->p.nthreads > 0 ? s->p.nthreads : 1;
    if (nt == 1) { fn(s, ranges[0][0] - 1, ranges[0][1], ctx); return; }
    pthread_t th[256];
    job_t jobs[256];
    for (int t = 0; t < nt; ++t) {
        jobs[t].s = s; jobs[t].b = ranges[t][0] - 1; jobs[t].e = ranges[t][1];
        jobs[t].fn = fn; jobs[t].ctx = ctx;
        pthread_create(&th[t], NULL, job_run, &jobs[t]);
    }
    for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
}

/* ----------------------------------------------------- face reconstruction */

static double limit_outer_first(const orc_state *s, double outer, double central, double eps2) {
    switch (s->p.limiter) {
    case ORC_LIM_MINMOD: return orc_minmod(outer, central, s->p.ksi);
    case ORC_LIM_VANLEER: return orc_vanleer(outer, central, s->p.ksi);
    case ORC_LIM_VANALBADA: return orc_vanalbada(outer, central, s->p.ksi);
    case ORC_LIM_VENKAT: return orc_venkat(outer, central, eps2);
    default: return 0.0;
    }
}

/* computeInterfaceSlope (7-argument boundary form), computeslope2d.jl:3-136:
 * MUSCL states on face k of cell i, limiter, then the flux with
 * (left = neighbour reconstruction, right = own reconstruction). */
static void interface_flux(const orc_state *s, int64_t i, int k, const double *uLeftp,
                           double flowTime, double *flux) {
    const orc_mesh *m = &s->m;
    int64_t n = m->nCells;
    int32_t ek = IDX(m->cell_stiffness, n, i, k);
    int32_t ek_type = IDX(m->mesh_connectivity, n, i, 1);
    double side = IDX(m->cell_edges_length, n, i, k);
    double nx = IDX(m->cell_edges_Nx, n, i, k);
    double ny = IDX(m->cell_edges_Ny, n, i, k);
    double uUpp[4] = {0, 0, 0, 0}, uDownp[4] = {0, 0, 0, 0}, uRightp[4] = {0, 0, 0, 0};
    int index = 2 * k; /* 0-based column of 2k-1 */
    double hxR = s->m.HX[i];
    if (ek >= 1 && ek <= n) {
        if (ek_type == 3) {
            int32_t pDown1 = IDX(m->node2cellL2down, n, i, index) - 1;
            int32_t pUp1 = IDX(m->node2cellL2up, n, i, index) - 1;
            uUpp[0] = s->densityNodes[pUp1]; uUpp[1] = s->UxNodes[pUp1];
            uUpp[2] = s->UyNodes[pUp1]; uUpp[3] = s->pressureNodes[pUp1];
            uDownp[0] = s->densityNodes[pDown1]; uDownp[1] = s->UxNodes[pDown1];
            uDownp[2] = s->UyNodes[pDown1]; uDownp[3] = s->pressureNodes[pDown1];
        } else if (ek_type == 2) {
            int32_t pDown1 = IDX(m->node2cellL2down, n, i, index) - 1;
            int32_t pDown2 = IDX(m->node2cellL2down, n, i, index + 1) - 1;
            int32_t pUp1 = IDX(m->node2cellL2up, n, i, index) - 1;
            int32_t pUp2 = IDX(m->node2cellL2up, n, i, index + 1) - 1;
            uUpp[0] = 0.5 * (s->densityNodes[pUp1] + s->densityNodes[pUp2]);
            uUpp[1] = 0.5 * (s->UxNodes[pUp1] + s->UxNodes[pUp2]);
            uUpp[2] = 0.5 * (s->UyNodes[pUp1] + s->UyNodes[pUp2]);
            uUpp[3] = 0.5 * (s->pressureNodes[pUp1] + s->pressureNodes[pUp2]);
            uDownp[0] = 0.5 * (s->densityNodes[pDown1] + s->densityNodes[pDown2]);
            uDownp[1] = 0.5 * (s->UxNodes[pDown1] + s->UxNodes[pDown2]);
            uDownp[2] = 0.5 * (s->UyNodes[pDown1] + s->UyNodes[pDown2]);
            uDownp[3] = 0.5 * (s->pressureNodes[pDown1] + s->pressureNodes[pDown2]);
        }
        uRightp[0] = s->densityCells[ek - 1];
        uRightp[1] = s->UxCells[ek - 1];
        uRightp[2] = s->UyCells[ek - 1];
        uRightp[3] = s->pressureCells[ek - 1];
        hxR = s->m.HX[ek - 1];
    } else {
        orc_bc_ghost(s, i, k, ek, uLeftp, flowTime, uRightp);
        for (int v = 0; v < 4; ++v) { uDownp[v] = uLeftp[v]; uUpp[v] = uRightp[v]; }
    }
    double UpLeft[4], UpRight[4];
    if (s->p.limiter == ORC_LIM_VENKAT) {
        /* Extension: each side's reconstruction evaluated in its own
         * (outer, central) roles so both cells of a face build the same
         * state; eps^2 = (K*HX)^3 scaled by the face's squared magnitude
         * of the variable, (uL^2 + uR^2)/2, so that it is dimensionless. */
        double KL = s->p.venkat_K * s->m.HX[i], KR = s->p.venkat_K * hxR;
        double e2L = KL * KL * KL, e2R = KR * KR * KR;
        for (int v = 0; v < 4; ++v) {
            double sc = 0.5 * (uLeftp[v] * uLeftp[v] + uRightp[v] * uRightp[v]);
            UpLeft[v] = uLeftp[v] + 0.5 * orc_venkat(uLeftp[v] - uDownp[v], uRightp[v] - uLeftp[v], e2L * sc);
            UpRight[v] = uRightp[v] + 0.5 * orc_venkat(uRightp[v] - uUpp[v], uLeftp[v] - uRightp[v], e2R * sc);
        }
    } else {
        for (int v = 0; v < 4; ++v) {
            UpLeft[v] = uLeftp[v] + 0.5 * limit_outer_first(s, uLeftp[v] - uDownp[v], uRightp[v] - uLeftp[v], 0.0);
            UpRight[v] = uRightp[v] - 0.5 * limit_outer_first(s, uRightp[v] - uLeftp[v], uUpp[v] - uRightp[v], 0.0);
        }
    }
    orc_flux(s->p.flux, UpRight, UpLeft, nx, ny, side, s->p.Gamma, flux);
}

/* ------------------------------------------------------ calcOneStage (a3) */

typedef struct { double beta, dt, t; } stage_ctx;

/* calcOneStageMUSCLcpuFast, calcOneStageMUSCLcpuFast.jl:3-107. */
static void stage_range(orc_state *s, int64_t b, int64_t e, void *vctx) {
    stage_ctx *c = (stage_ctx *)vctx;
    const orc_mesh *m = &s->m;
    int64_t n = m->nCells;
    for (int64_t i = b; i < e; ++i) {
        double uLeftp[4] = {s->densityCells[i], s->UxCells[i], s->UyCells[i], s->pressureCells[i]};
        double f1[4] = {0, 0, 0, 0}, f2[4] = {0, 0, 0, 0}, f3[4] = {0, 0, 0, 0}, f4[4] = {0, 0, 0, 0};
        int32_t nn = IDX(m->mesh_connectivity, n, i, 2);
        if (nn == 3) {
            interface_flux(s, i, 0, uLeftp, c->t, f1);
            interface_flux(s, i, 1, uLeftp, c->t, f2);
            interface_flux(s, i, 2, uLeftp, c->t, f3);
            for (int v = 0; v < 4; ++v) IDX(s->FLUXES, n, i, v) = f1[v] + f2[v] + f3[v];
        } else if (nn == 4) {
            interface_flux(s, i, 0, uLeftp, c->t, f1);
            interface_flux(s, i, 1, uLeftp, c->t, f2);
            interface_flux(s, i, 2, uLeftp, c->t, f3);
            interface_flux(s, i, 3, uLeftp, c->t, f4);
            for (int v = 0; v < 4; ++v) IDX(s->FLUXES, n, i, v) = f1[v] + f2[v] + f3[v] + f4[v];
        }
        double Rarea = 1.0 / m->cell_areas[i];
        for (int v = 0; v < 4; ++v)
            IDX(s->UconsCellsNew, n, i, v) = (IDX(s->UconsCellsOld, n, i, v) -
                                              IDX(s->FLUXES, n, i, v) * c->beta * c->dt * Rarea +
                                              c->beta * c->dt * IDX(s->UConsDiffCells, n, i, v));
    }
}

void orc_calc_one_stage(orc_state *s, double beta, double dt, double t) {
    stage_ctx c = {beta, dt, t};
    parallel(s, s->cellsThreads, stage_range, &c);
}

/* --------------------------------------------------- updateVariables (a9) */

/* updateVariablesSA, evaluate2d.jl:52-110 (density clamp off). */
static void update_range(orc_state *s, int64_t b, int64_t e, void *vctx) {
    (void)vctx;
    int64_t n = s->m.nCells;
    double G = s->p.Gamma;
    for (int64_t i = b; i < e; ++i) {
        if (s->p.densityConstrained == 1) {
            /* evaluate2d.jl:63-77 (the reference indexes an array that is
             * out of scope there; the clamp acts on Unew as intended). */
            if (IDX(s->UconsCellsNew, n, i, 0) >= s->p.maxDensityConstrained)
                IDX(s->UconsCellsNew, n, i, 0) = s->p.maxDensityConstrained;
            if (IDX(s->UconsCellsNew, n, i, 0) <= s->p.minDensityConstrained)
                IDX(s->UconsCellsNew, n, i, 0) = s->p.minDensityConstrained;
        }
        double U1 = IDX(s->UconsCellsNew, n, i, 0), U2 = IDX(s->UconsCellsNew, n, i, 1);
        double U3 = IDX(s->UconsCellsNew, n, i, 2), U4 = IDX(s->UconsCellsNew, n, i, 3);
        s->densityCells[i] = U1;
        s->UxCells[i] = U2 / U1;
        s->UyCells[i] = U3 / U1;
        s->pressureCells[i] = (G - 1.0) * (U4 - 0.5 * (U2 * U2 + U3 * U3) / U1);
        s->aSoundCells[i] = sqrt(G * s->pressureCells[i] / s->densityCells[i]);
        s->VMAXCells[i] = sqrt(s->UxCells[i] * s->UxCells[i] + s->UyCells[i] * s->UyCells[i]) + s->aSoundCells[i];
        for (int v = 0; v < 4; ++v) {
            IDX(s->Delta, n, i, v) = IDX(s->UconsCellsNew, n, i, v) - IDX(s->UconsCellsOld, n, i, v);
            IDX(s->UconsCellsOld, n, i, v) = IDX(s->UconsCellsNew, n, i, v);
        }
    }
}

void orc_update_variables(orc_state *s, orc_stats *st) {
    int64_t n = s->m.nCells;
    /* findmax/findmin of the density before the update (evaluate2d.jl:79-80) */
    double mx = s->densityCells[0], mn = s->densityCells[0];
    for (int64_t i = 1; i < n; ++i) {
        mx = jl_max(mx, s->densityCells[i]);
        mn = jl_min(mn, s->densityCells[i]);
    }
    if (st) { st->rhoMax = mx; st->rhoMin = mn; }
    parallel(s, s->cellsThreads, update_range, NULL);
}

/* ---------------------------------------------- cells -> nodes (a10) */

/* cells2nodesSolutionReconstructionWithStencils, utilsFVM2dp.jl:299-365.
 * (The reference loop carries @fastmath; this restatement keeps the plain
 * sum-then-divide order as written.) */
static void c2n_range(orc_state *s, int64_t b, int64_t e, void *vctx) {
    (void)vctx;
    const orc_mesh *m = &s->m;
    int64_t nn = m->nNodes, nc = m->nCells;
    for (int64_t J = b; J < e; ++J) {
        double det = 0.0;
        s->densityNodes[J] = 0.0; s->UxNodes[J] = 0.0; s->UyNodes[J] = 0.0; s->pressureNodes[J] = 0.0;
        for (int v = 0; v < 4; ++v) IDX(s->UconsNodesOld, nn, J, v) = 0.0;
        for (int j = 0; j < m->nNeibCells; ++j) {
            int32_t c = IDX(m->cell_clusters, nn, J, j);
            if (c != 0) {
                double wi = IDX(m->node_stencils, nn, J, j);
                for (int v = 0; v < 4; ++v)
                    IDX(s->UconsNodesOld, nn, J, v) += IDX(s->UconsCellsOld, nc, c - 1, v) * wi;
                s->densityNodes[J] += s->densityCells[c - 1] * wi;
                s->UxNodes[J] += s->UxCells[c - 1] * wi;
                s->UyNodes[J] += s->UyCells[c - 1] * wi;
                s->pressureNodes[J] += s->pressureCells[c - 1] * wi;
                det += wi;
            }
        }
        if (det != 0) {
            s->densityNodes[J] = s->densityNodes[J] / det;
            s->UxNodes[J] = s->UxNodes[J] / det;
            s->UyNodes[J] = s->UyNodes[J] / det;
            s->pressureNodes[J] = s->pressureNodes[J] / det;
            for (int v = 0; v < 4; ++v) IDX(s->UconsNodesOld, nn, J, v) = IDX(s->UconsNodesOld, nn, J, v) / det;
        }
    }
}

void orc_cells2nodes(orc_state *s) { parallel(s, s->nodesThreads, c2n_range, NULL); }

/* cells2nodesSolutionReconstructionWithStencilsUCons, utilsFVM2dp.jl:370-422. */
static void c2n_ucons_range(orc_state *s, int64_t b, int64_t e, void *vctx) {
    (void)vctx;
    const orc_mesh *m = &s->m;
    int64_t nn = m->nNodes, nc = m->nCells;
    for (int64_t J = b; J < e; ++J) {
        double det = 0.0;
        for (int v = 0; v < 4; ++v) IDX(s->UconsNodesOld, nn, J, v) = 0.0;
        for (int j = 0; j < m->nNeibCells; ++j) {
            int32_t c = IDX(m->cell_clusters, nn, J, j);
            if (c != 0) {
                double wi = IDX(m->node_stencils, nn, J, j);
                for (int v = 0; v < 4; ++v)
                    IDX(s->UconsNodesOld, nn, J, v) += IDX(s->UconsCellsOld, nc, c - 1, v) * wi;
                det += wi;
            }
        }
        if (det != 0)
            for (int v = 0; v < 4; ++v) IDX(s->UconsNodesOld, nn, J, v) = IDX(s->UconsNodesOld, nn, J, v) / det;
    }
}

/* ------------------------------------------------- viscous term (a13) */

/* calcPhiInCellCluster, calcGradients.jl:3-18 (unweighted cluster mean). */
static double phi_in_cluster(const orc_state *s, int32_t node1, const double *field) {
    const orc_mesh *m = &s->m;
    double phi = 0.0;
    int64_t counter = 0;
    for (int i = 0; i < m->nNeibCells; ++i) {
        int32_t cell = IDX(m->cell_clusters, m->nNodes, node1 - 1, i);
        if (cell > 0 && cell <= m->nCells) {
            phi += field[cell - 1];
            counter += 1;
        }
    }
    return counter != 0 ? phi / (double)counter : 0.0;
}

typedef struct { const double *field; double *gx, *gy; } gg_ctx;

/* calcScalarFieldGreenGaussNodesBasedGradient, calcGradients.jl:36-139.
 * gradX pairs with -ny and gradY with -nx, as in the reference (:116-126);
 * the boundary branch (:100-113) is overwritten there and omitted here.
 * Slot 4 of a triangle contributes the reference's zero-initialised value. */
static void gg_range(orc_state *s, int64_t b, int64_t e, void *vctx) {
    gg_ctx *c = (gg_ctx *)vctx;
    const orc_mesh *m = &s->m;
    int64_t n = m->nCells;
    for (int64_t C = b; C < e; ++C) {
        double side[4] = {0, 0, 0, 0}, nx[4] = {0, 0, 0, 0}, ny[4] = {0, 0, 0, 0};
        double pL[4] = {0, 0, 0, 0}, pR[4] = {0, 0, 0, 0}, fX[4], fY[4];
        int nf = IDX(m->mesh_connectivity, n, C, 2) == 4 ? 4 : 3;
        for (int k = 0; k < nf; ++k) {
            side[k] = IDX(m->cell_edges_length, n, C, k);
            nx[k] = IDX(m->cell_edges_Nx, n, C, k);
            ny[k] = IDX(m->cell_edges_Ny, n, C, k);
            pL[k] = phi_in_cluster(s, IDX(m->cells2nodes, n, C, 2 * k), c->field);
            pR[k] = phi_in_cluster(s, IDX(m->cells2nodes, n, C, 2 * k + 1), c->field);
        }
        for (int k = 0; k < 4; ++k) {
            fX[k] = 0.5 * (pL[k] + pR[k]) * -ny[k] * side[k];
            fY[k] = 0.5 * (pL[k] + pR[k]) * -nx[k] * side[k];
        }
        c->gx[C] = (fX[0] + fX[1] + fX[2] + fX[3]) / m->cell_areas[C];
        c->gy[C] = (fY[0] + fY[1] + fY[2] + fY[3]) / m->cell_areas[C];
    }
}

static void gg_gradient(orc_state *s, const double *field, double *gx, double *gy) {
    gg_ctx c = {field, gx, gy};
    parallel(s, s->cellsThreads, gg_range, &c);
}

/* The same gradient of an arbitrary cell field (nCells values), as the
 * reference's operator driver calls it (testDiffOperatorsGrads.jl:303,
 * testDiffOperatorsLaplace.jl:98-105): node values are the unweighted cluster
 * means of the field, gradX pairs with -ny and gradY with -nx. */
void orc_green_gauss_gradient(orc_state *s, const double *field, double *gx, double *gy) {
    gg_gradient(s, field, gx, gy);
}

/* nodesGradientReconstructionFastPerThread22, calcGrad.jl:3-96 (node field,
 * -nx for x); used for the velocity divergence of the artificial viscosity. */
static void node_grad_cell(const orc_state *s, int64_t C, const double *nodeField, double *gx, double *gy) {
    const orc_mesh *m = &s->m;
    int64_t n = m->nCells;
    double side[4] = {0, 0, 0, 0}, nx[4] = {0, 0, 0, 0}, ny[4] = {0, 0, 0, 0};
    double pL[4] = {0, 0, 0, 0}, pR[4] = {0, 0, 0, 0}, fX[4], fY[4];
    int nf = IDX(m->mesh_connectivity, n, C, 2) == 4 ? 4 : 3;
    for (int k = 0; k < nf; ++k) {
        side[k] = IDX(m->cell_edges_length, n, C, k);
        nx[k] = IDX(m->cell_edges_Nx, n, C, k);
        ny[k] = IDX(m->cell_edges_Ny, n, C, k);
        pL[k] = nodeField[IDX(m->cells2nodes, n, C, 2 * k) - 1];
        pR[k] = nodeField[IDX(m->cells2nodes, n, C, 2 * k + 1) - 1];
    }
    for (int k = 0; k < 4; ++k) {
        fX[k] = 0.5 * (pL[k] + pR[k]) * -nx[k] * side[k];
        fY[k] = 0.5 * (pL[k] + pR[k]) * -ny[k] * side[k];
    }
    *gx = (fX[0] + fX[1] + fX[2] + fX[3]) / m->cell_areas[C];
    *gy = (fY[0] + fY[1] + fY[2] + fY[3]) / m->cell_areas[C];
}

/* Artificial viscosity, calcArtViscosity.jl:46-75 (extension: the cell
 * value is reset to zero when the sensor is off). */
static void artvisc_range(orc_state *s, int64_t b, int64_t e, void *vctx) {
    (void)vctx;
    for (int64_t i = b; i < e; ++i) {
        double dUdx, dUdy, dVdx, dVdy;
        node_grad_cell(s, i, s->UxNodes, &dUdx, &dUdy);
        node_grad_cell(s, i, s->UyNodes, &dVdx, &dVdy);
        double divU = dUdx + dVdy;
        double HX = s->m.HX[i];
        double a = 0.05 * s->aSoundCells[i] / HX / sqrt(2.0);
        double mu = 0.0;
        if (-divU > a) {
            double tmp = divU * divU - a * a;
            if (tmp > 0.0)
                mu = 0.5 * s->densityCells[i] * HX / sqrt(2.0) * HX / sqrt(2.0) * sqrt(tmp) * 1.0e-5;
        }
        s->muArt[i] = mu;
        s->dUdx[i] = dUdx;
        s->dVdy[i] = dVdy;
    }
}

static void diff_combine_range(orc_state *s, int64_t b, int64_t e, void *vctx) {
    (void)vctx;
    int64_t n = s->m.nCells;
    const orc_params *p = &s->p;
    for (int64_t i = b; i < e; ++i) {
        double lu = s->lap[0][i], lv = s->lap[1][i], le = s->lap[2][i];
        double T = s->pressureCells[i] / s->densityCells[i] / p->RGAS;
        if (p->viscosity == ORC_VISC_REFERENCE) {
            /* calcDiffTerm.jl:105-113 (mu = 1e-2 there, passed as mu_ref) */
            double mu = p->mu_ref;
            IDX(s->UConsDiffCells, n, i, 1) = mu * lu;
            IDX(s->UConsDiffCells, n, i, 2) = mu * lv;
            IDX(s->UConsDiffCells, n, i, 3) = mu * orc_air_conductivity(T) * le;
        } else {
            /* Extension: mu(T) Sutherland scaled to mu_ref at T_ref (or a
             * constant mu_ref), plus artificial viscosity, applied to the
             * Laplacians of u, v and phi = |u|^2/2 + (gamma/Pr) e:
             * div(tau) ~ mu lap(u), div(tau.u) + div(k grad T) ~
             * mu lap(|u|^2/2) + (mu cp/Pr) lap(T). */
            double mu = (p->viscosity == ORC_VISC_SUTHERLAND)
                            ? p->mu_ref * (orc_sutherland(T) / s->suth_ref)
                            : p->mu_ref;
            double mue = mu + (p->art_viscosity ? s->muArt[i] : 0.0);
            IDX(s->UConsDiffCells, n, i, 1) = mue * lu;
            IDX(s->UConsDiffCells, n, i, 2) = mue * lv;
            IDX(s->UConsDiffCells, n, i, 3) = mue * le;
        }
    }
}

typedef struct { int var; } lap_ctx;

/* calcDiffTerm, calcDiffTerm.jl:31-121.  The node averages it builds at
 * :69-76 are passed as the unused scalarFieldNodes argument of the second
 * gradient and do not reach the result; they are not formed here. */
void orc_calc_diff_term(orc_state *s) {
    int64_t n = s->m.nCells;
    double *dummy = (double *)malloc(sizeof(double) * (size_t)n);
    double *prim3 = NULL;
    if (s->p.viscosity != ORC_VISC_REFERENCE) {
        /* Extension models diffuse primitive quantities: u, v and
         * phi = |u|^2/2 + (gamma/Pr) e, e = p / ((gamma-1) rho). */
        const double G = s->p.Gamma;
        prim3 = (double *)malloc(sizeof(double) * 3 * (size_t)n);
        for (int64_t i = 0; i < n; ++i) {
            double r = s->densityCells[i], u = s->UxCells[i], v = s->UyCells[i], pp = s->pressureCells[i];
            prim3[i] = u;
            prim3[n + i] = v;
            prim3[2 * n + i] = 0.5 * (u * u + v * v) + s->gamma_over_Pr * (pp / ((G - 1.0) * r));
        }
    }
    for (int v = 0; v < 3; ++v) {
        const double *field = prim3 ? prim3 + (int64_t)v * n : s->UconsCellsOld + (int64_t)(v + 1) * n;
        gg_gradient(s, field, s->g1x[v], s->g1y[v]);
    }
    free(prim3);
    for (int v = 0; v < 3; ++v) {
        double *d2x = s->lap[v]; /* temporarily holds d/dy(gradX) */
        double *tmp = (double *)malloc(sizeof(double) * (size_t)n);
        gg_gradient(s, s->g1x[v], d2x, dummy);
        gg_gradient(s, s->g1y[v], dummy, tmp);
        for (int64_t i = 0; i < n; ++i) s->lap[v][i] = d2x[i] + tmp[i];
        free(tmp);
    }
    free(dummy);
    if (s->p.viscosity != ORC_VISC_REFERENCE && s->p.art_viscosity)
        parallel(s, s->cellsThreads, artvisc_range, NULL);
    parallel(s, s->cellsThreads, diff_combine_range, NULL);
}

/* ------------------------------------------------------------- lifecycle */

static double *zalloc(int64_t n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

orc_state *orc_create(const orc_mesh *m, const orc_params *p) {
    orc_state *s = (orc_state *)calloc(1, sizeof(orc_state));
    s->m = *m;
    s->p = *p;
    if (s->p.nthreads < 1) s->p.nthreads = 1;
    if (s->p.nthreads > 256) s->p.nthreads = 256;
    int64_t nc = m->nCells, nn = m->nNodes;
    s->densityCells = zalloc(nc); s->UxCells = zalloc(nc); s->UyCells = zalloc(nc);
    s->pressureCells = zalloc(nc); s->aSoundCells = zalloc(nc); s->VMAXCells = zalloc(nc);
    s->densityNodes = zalloc(nn); s->UxNodes = zalloc(nn); s->UyNodes = zalloc(nn); s->pressureNodes = zalloc(nn);
    s->UconsCellsOld = zalloc(4 * nc); s->UconsCellsNew = zalloc(4 * nc); s->UconsNodesOld = zalloc(4 * nn);
    s->UConsDiffCells = zalloc(4 * nc); s->Delta = zalloc(4 * nc); s->FLUXES = zalloc(4 * nc);
    for (int v = 0; v < 3; ++v) { s->g1x[v] = zalloc(nc); s->g1y[v] = zalloc(nc); s->lap[v] = zalloc(nc); }
    s->muArt = zalloc(nc); s->dUdx = zalloc(nc); s->dVdy = zalloc(nc);
    s->cellsThreads = calloc((size_t)s->p.nthreads, sizeof(int32_t[2]));
    s->nodesThreads = calloc((size_t)s->p.nthreads, sizeof(int32_t[2]));
    orc_partition(s->p.nthreads, nc, s->cellsThreads);
    orc_partition(s->p.nthreads, nn, s->nodesThreads);
    double mx = m->HX[0];
    for (int64_t i = 1; i < nc; ++i) mx = jl_max(mx, m->HX[i]);
    s->maxEdge = mx; /* findmax(testMesh.HX), testInviscidFluxesGPUx32.jl:299 */
    s->charLen = zalloc(nc);
    for (int64_t i = 0; i < nc; ++i) {
        int nf = IDX(m->mesh_connectivity, nc, i, 2) == 4 ? 4 : 3;
        double per = 0.0;
        for (int k = 0; k < nf; ++k) per += IDX(m->cell_edges_length, nc, i, k);
        s->charLen[i] = 2.0 * m->cell_areas[i] / per;
    }
    s->suth_ref = orc_sutherland(p->T_ref);
    s->gamma_over_Pr = p->Gamma / p->Pr;
    return s;
}

void orc_destroy(orc_state *s) {
    if (!s) return;
    free(s->densityCells); free(s->UxCells); free(s->UyCells); free(s->pressureCells);
    free(s->aSoundCells); free(s->VMAXCells);
    free(s->densityNodes); free(s->UxNodes); free(s->UyNodes); free(s->pressureNodes);
    free(s->UconsCellsOld); free(s->UconsCellsNew); free(s->UconsNodesOld);
    free(s->UConsDiffCells); free(s->Delta); free(s->FLUXES);
    for (int v = 0; v < 3; ++v) { free(s->g1x[v]); free(s->g1y[v]); free(s->lap[v]); }
    free(s->muArt); free(s->dUdx); free(s->dVdy); free(s->charLen);
    free(s->cellsThreads); free(s->nodesThreads);
    free(s);
}

/* createFields2d (initfields_step2d.jl:108-119 / initfields_TGV2d.jl:47-63)
 * from given cell primitives, then phs2dcns2dcellsSA (utilsFVM2dp.jl:4-17)
 * into Uold and Unew and the conservative node average
 * (testInviscidFluxesGPUx32.jl:282-286).  Node primitives stay zero unless
 * init_nodes is set, as in the reference's first step. */
void orc_init_fields(orc_state *s, const double *rho, const double *ux, const double *uy, const double *p) {
    int64_t n = s->m.nCells;
    double G = s->p.Gamma;
    for (int64_t i = 0; i < n; ++i) {
        s->densityCells[i] = rho[i]; s->UxCells[i] = ux[i]; s->UyCells[i] = uy[i]; s->pressureCells[i] = p[i];
        s->aSoundCells[i] = sqrt(G * s->pressureCells[i] / s->densityCells[i]);
        s->VMAXCells[i] = sqrt(s->UxCells[i] * s->UxCells[i] + s->UyCells[i] * s->UyCells[i]) + s->aSoundCells[i];
    }
    for (int64_t i = 0; i < n; ++i) {
        double r = s->densityCells[i], u = s->UxCells[i], v = s->UyCells[i], pp = s->pressureCells[i];
        double U[4] = {r, r * u, r * v, pp / (G - 1.0) + 0.5 * r * (u * u + v * v)};
        for (int k = 0; k < 4; ++k) { IDX(s->UconsCellsOld, n, i, k) = U[k]; IDX(s->UconsCellsNew, n, i, k) = U[k]; }
    }
    memset(s->UConsDiffCells, 0, sizeof(double) * 4 * (size_t)n);
    parallel(s, s->nodesThreads, c2n_ucons_range, NULL);
    if (s->p.init_nodes) orc_cells2nodes(s);
    else {
        memset(s->densityNodes, 0, sizeof(double) * (size_t)s->m.nNodes);
        memset(s->UxNodes, 0, sizeof(double) * (size_t)s->m.nNodes);
        memset(s->UyNodes, 0, sizeof(double) * (size_t)s->m.nNodes);
        memset(s->pressureNodes, 0, sizeof(double) * (size_t)s->m.nNodes);
    }
    s->flowTime = 0.0;
    s->curIter = 0;
}

void orc_set_time(orc_state *s, double t) { s->flowTime = t; }

/* One explicit step in the order of testInviscidFluxesGPUx32.jl:314-401 and
 * testViscousFluxesTGV2d.jl:416-506. */
void orc_step(orc_state *s, orc_stats *st) {
    int64_t n = s->m.nCells;
    orc_stats tmp;
    if (!st) st = &tmp;
    memset(st, 0, sizeof(*st));
    double velmax = s->VMAXCells[0];
    for (int64_t i = 1; i < n; ++i) velmax = jl_max(velmax, s->VMAXCells[i]);
    double tau = s->p.CFL * s->maxEdge / jl_max(velmax, 1.0e-6);
    double dt = s->p.dt_mode == 1 ? tau : s->p.dt;
    if (s->p.dt_mode == 2) {
        /* Extension: local CFL, dt = CFL * min_i(2 A_i / P_i / VMAX_i). */
        double r = s->charLen[0] / s->VMAXCells[0];
        for (int64_t i = 1; i < n; ++i) r = jl_min(r, s->charLen[i] / s->VMAXCells[i]);
        dt = s->p.CFL * r;
    }
    if (s->p.viscosity != ORC_VISC_NONE) orc_calc_diff_term(s);
    orc_calc_one_stage(s, s->p.beta, dt, s->flowTime);
    orc_update_variables(s, st);
    orc_cells2nodes(s);
    for (int v = 0; v < 4; ++v) {
        double r = 0.0, tot = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            double d = IDX(s->Delta, n, i, v);
            r += d * d;
            tot += IDX(s->UconsCellsOld, n, i, v) * s->m.cell_areas[i];
        }
        st->residual[v] = r;
        st->totals[v] = tot;
    }
    double ek = 0.0;
    int32_t bad = 0;
    for (int64_t i = 0; i < n; ++i) {
        ek += 0.5 * s->densityCells[i] * (s->UxCells[i] * s->UxCells[i] + s->UyCells[i] * s->UyCells[i]) * s->m.cell_areas[i];
        for (int v = 0; v < 4; ++v) if (!isfinite(IDX(s->UconsCellsOld, n, i, v))) bad = 1;
        if (!(s->densityCells[i] > 0.0) || !(s->pressureCells[i] > 0.0)) bad = 1;
    }
    st->Ek = ek;
    st->nonfinite = bad;
    st->dt = dt;
    st->tau = tau;
    st->velmax = velmax;
    st->flowTime = s->flowTime;
    s->curIter += 1;
    st->step = s->curIter;
    s->flowTime += dt;
}

void orc_run(orc_state *s, int32_t nsteps, orc_stats *last) {
    for (int32_t k = 0; k < nsteps; ++k) orc_step(s, last);
}

/* Field access for the tests: 0..5 cell primitives (rho,u,v,p,a,VMAX),
 * 6..9 node primitives, 10 Uold, 11 Unew, 12 node conservatives, 13 Diff,
 * 14 Delta, 15 FLUXES, 16 artificial viscosity. */
double *orc_field(orc_state *s, int32_t which) {
    switch (which) {
    case 0: return s->densityCells; case 1: return s->UxCells; case 2: return s->UyCells;
    case 3: return s->pressureCells; case 4: return s->aSoundCells; case 5: return s->VMAXCells;
    case 6: return s->densityNodes; case 7: return s->UxNodes; case 8: return s->UyNodes;
    case 9: return s->pressureNodes; case 10: return s->UconsCellsOld; case 11: return s->UconsCellsNew;
    case 12: return s->UconsNodesOld; case 13: return s->UConsDiffCells; case 14: return s->Delta;
    case 15: return s->FLUXES; case 16: return s->muArt;
    default: return NULL;
    }
}

double orc_flow_time(const orc_state *s) { return s->flowTime; }
double orc_max_edge(const orc_state *s) { return s->maxEdge; }
int32_t orc_sizeof_params(void) { return (int32_t)sizeof(orc_params); }
int32_t orc_sizeof_mesh(void) { return (int32_t)sizeof(orc_mesh); }
int32_t orc_sizeof_stats(void) { return (int32_t)sizeof(orc_stats); }
