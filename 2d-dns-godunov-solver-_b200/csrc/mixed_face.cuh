// FP32 face arithmetic of the mixed-precision path, shared by the
// cell-centred and tile-face kernels: reconstruction + limiter + flux of one
// face (computeslope2d.jl:3-136), the diffusion source (calcDiffTerm.jl:88-113
// and the extension models) and the FP64-accumulated Euler update.
#pragma once

#include "step_kernels.cuh"

namespace gd2d {
namespace {

// computeInterfaceSlope (computeslope2d.jl:3-136) in FP32.
template <int FLUX, bool QUAD>
__device__ __forceinline__ void face_flux_f(const DevMesh &m, const DevCase &P, const float4 *__restrict__ pin,
                                            const float4 *__restrict__ nodeP, int64_t g, int k, int nbk, int dnk,
                                            int upk, int dn2k, int up2k, bool is_quad, const float *uL, float hx_own,
                                            double t, float g2, float *f) {
    const int64_t o = (int64_t)k * m.Nc + g;
    const float side = m.lenf[o], nx = m.nxf[o], ny = m.nyf[o];
    float uR[4], uUp[4], uDn[4];
    float hxR = hx_own;
    if (nbk >= 0) {
        if (QUAD && is_quad) {
            float4 a = nodeP[upk], a2 = nodeP[up2k], b = nodeP[dnk], b2 = nodeP[dn2k];
            uUp[0] = 0.5f * (a.x + a2.x); uUp[1] = 0.5f * (a.y + a2.y);
            uUp[2] = 0.5f * (a.z + a2.z); uUp[3] = 0.5f * (a.w + a2.w);
            uDn[0] = 0.5f * (b.x + b2.x); uDn[1] = 0.5f * (b.y + b2.y);
            uDn[2] = 0.5f * (b.z + b2.z); uDn[3] = 0.5f * (b.w + b2.w);
        } else {
            float4 a = nodeP[upk], b = nodeP[dnk];
            uUp[0] = a.x; uUp[1] = a.y; uUp[2] = a.z; uUp[3] = a.w;
            uDn[0] = b.x; uDn[1] = b.y; uDn[2] = b.z; uDn[3] = b.w;
        }
        float4 r = pin[nbk];
        uR[0] = r.x; uR[1] = r.y; uR[2] = r.z; uR[3] = r.w;
        if (P.limiter == LIM_VENKAT) hxR = m.hxf[nbk];
    } else {
        bc_ghost<float>(P, m, -nbk - 1, g, k, uL, nx, ny, t, uR);
        for (int v = 0; v < 4; ++v) { uDn[v] = uL[v]; uUp[v] = uR[v]; }
    }
    float UpL[4], UpR[4];
    if (P.limiter == LIM_VENKAT) {
        const float K = (float)P.venkat_K;
        const float KL = K * hx_own, KR = K * hxR;
        const float e2L = KL * KL * KL, e2R = KR * KR * KR;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float sc = 0.5f * (uL[v] * uL[v] + uR[v] * uR[v]);
            UpL[v] = uL[v] + 0.5f * lim_venkat(uL[v] - uDn[v], uR[v] - uL[v], e2L * sc);
            UpR[v] = uR[v] + 0.5f * lim_venkat(uR[v] - uUp[v], uL[v] - uR[v], e2R * sc);
        }
    } else {
        const int lk = P.limiter;
        const float ksi = (float)P.ksi;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            UpL[v] = uL[v] + 0.5f * limiter(lk, uL[v] - uDn[v], uR[v] - uL[v], ksi);
            UpR[v] = uR[v] - 0.5f * limiter(lk, uR[v] - uL[v], uUp[v] - uR[v], ksi);
        }
    }
    face_flux_fn<FLUX, float>(UpR, UpL, nx, ny, side, (float)P.gamma, g2, f);
}

// Per-case constants of the FP32 face arithmetic, read from the case record
// once per tile rather than once per face.
struct FaceConstsF {
    float gam;  // gamma
    float g2;   // 2 (gamma - 1) / (gamma + 1)
    float hk;   // gamma / (gamma - 1): p/rho + p/rho/(gamma-1) = (p/rho) hk
    float vK;   // Venkatakrishnan K
    float ksi;  // Minmod constant
    int lim;    // limiter kind
};
__device__ __forceinline__ FaceConstsF face_consts_f(const DevCase &P) {
    FaceConstsF k;
    k.gam = (float)P.gamma;
    k.g2 = (float)(2.0 * (P.gamma - 1.0) / (P.gamma + 1.0));
    k.hk = (float)(P.gamma / (P.gamma - 1.0));
    k.vK = (float)P.venkat_K;
    k.ksi = (float)P.ksi;
    k.lim = P.limiter;
    return k;
}

// The limiters of the mixed path without the reference's exact-rounding
// constraints: branch-free selects and fast division.
// Venkatakrishnan in the two-argument slot (same function as lim_venkat).
__device__ __forceinline__ float venkat_fast(float o, float c, float e2) {
    c = (o * c < 0.f) ? 0.f : c;
    const float oo = o * o;
    const float den = c * c + 2.f * oo + o * c + e2;  // >= 0
    const float num = (c * c + e2) * o + 2.f * oo * c;
    return den > 0.f ? __fdividef(num, den) : 0.f;
}
// Minmod_Limiter (limiters.jl:33-35).
__device__ __forceinline__ float minmod_fast(float x, float y, float c) {
    const float sx = x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f), sy = y > 0.f ? 1.f : (y < 0.f ? -1.f : 0.f);
    return __fdividef((sx + sy) * fabsf(x * y), fabsf(x) + fabsf(y) + c);
}

// AUSM+ (Liou 1996; the reference's variant with a12 = the smaller of the
// two numerical sound speeds, AUSMflux2dFast.jl:87-175) in FP32 for the
// mixed path: the same formulas, regrouped where that saves work --
// p/rho + p/rho/(gamma-1) = (p/rho) gamma/(gamma-1), a~ = s min(1, s/|u.n|)
// = min(s, s^2/|u.n|), the split Mach and pressure polynomials as selects,
// (m + |m|)/2 = max(m, 0) -- with fast division and square root.
// L is the neighbour's reconstruction and R the cell's own, as
// computeslope2d.jl:129 passes them.
__device__ __forceinline__ float mach_p(float M) {  // M+ with beta = 1/8
    const float q = M * M - 1.f;
    return fabsf(M) >= 1.f ? fmaxf(M, 0.f) : 0.25f * (M + 1.f) * (M + 1.f) + 0.125f * q * q;
}
__device__ __forceinline__ float mach_m(float M) {  // M- with beta = 1/8
    const float q = M * M - 1.f;
    return fabsf(M) >= 1.f ? fminf(M, 0.f) : -0.25f * (M - 1.f) * (M - 1.f) - 0.125f * q * q;
}
__device__ __forceinline__ float pres_p(float M) {  // P+ with alpha = 3/16
    const float q = M * M - 1.f;
    return fabsf(M) >= 1.f ? (M > 0.f ? 1.f : 0.f)
                           : 0.25f * (M + 1.f) * (M + 1.f) * (2.f - M) + 0.1875f * M * q * q;
}
__device__ __forceinline__ float pres_m(float M) {  // P- with alpha = 3/16
    const float q = M * M - 1.f;
    return fabsf(M) >= 1.f ? (M < 0.f ? 1.f : 0.f)
                           : 0.25f * (M - 1.f) * (M - 1.f) * (2.f + M) - 0.1875f * M * q * q;
}
__device__ __forceinline__ void ausm_plus_fast(const float *L, const float *R, float nx, float ny, float side,
                                               const FaceConstsF &k, float *flux) {
    const float rL = L[0], uL = L[1], vL = L[2], pL = L[3];
    const float rR = R[0], uR = R[1], vR = R[2], pR = R[3];
    const float htL = fmaf(0.5f, uL * uL + vL * vL, __fdividef(pL, rL) * k.hk);
    const float htR = fmaf(0.5f, uR * uR + vR * vR, __fdividef(pR, rR) * k.hk);
    const float s2L = k.g2 * htL, s2R = k.g2 * htR;
    const float vnL = uL * nx + vL * ny, vnR = uR * nx + vR * ny;
    const float aL = fminf(sqrtf(s2L), __fdividef(s2L, fabsf(vnL)));
    const float aR = fminf(sqrtf(s2R), __fdividef(s2R, fabsf(vnR)));
    const float a12 = fminf(aL, aR);
    const float ia = __fdividef(1.f, a12);
    const float ML = vnL * ia, MR = vnR * ia;
    const float mdot = mach_p(ML) + mach_m(MR);
    const float p12 = pres_p(ML) * pL + pres_m(MR) * pR;
    const float mp = a12 * fmaxf(mdot, 0.f) * rL, mm = a12 * fminf(mdot, 0.f) * rR;
    flux[0] = -(mp + mm) * side;
    flux[1] = -(mp * uL + mm * uR + p12 * nx) * side;
    flux[2] = -(mp * vL + mm * vR + p12 * ny) * side;
    flux[3] = -(mp * htL + mm * htR) * side;
}

// The face with every gathered input already in registers: r = the
// neighbour's primitives, d/u = down/up node primitives (quads: averaged),
// geometry (nx, ny, side).  Boundary faces ignore r, d, u.
template <int FLUX>
__device__ __forceinline__ void face_flux_pre(const DevMesh &m, const DevCase &P, const FaceConstsF &kc, int64_t g,
                                              int k, int nbk, const float4 &r, const float4 &dd, const float4 &uu,
                                              float nx, float ny, float side, const float *uL, float hx_own,
                                              float hxR, double t, float *f) {
    float uR[4], uUp[4], uDn[4];
    if (nbk >= 0) {
        uR[0] = r.x; uR[1] = r.y; uR[2] = r.z; uR[3] = r.w;
        uUp[0] = uu.x; uUp[1] = uu.y; uUp[2] = uu.z; uUp[3] = uu.w;
        uDn[0] = dd.x; uDn[1] = dd.y; uDn[2] = dd.z; uDn[3] = dd.w;
    } else {
        bc_ghost<float>(P, m, -nbk - 1, g, k, uL, nx, ny, t, uR);
        hxR = hx_own;
        for (int v = 0; v < 4; ++v) { uDn[v] = uL[v]; uUp[v] = uR[v]; }
    }
    float UpL[4], UpR[4];
    if (kc.lim == LIM_VENKAT) {
        const float KL = kc.vK * hx_own, KR = kc.vK * hxR;
        const float e2L = KL * KL * KL, e2R = KR * KR * KR;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float sc = 0.5f * (uL[v] * uL[v] + uR[v] * uR[v]);
            UpL[v] = uL[v] + 0.5f * venkat_fast(uL[v] - uDn[v], uR[v] - uL[v], e2L * sc);
            UpR[v] = uR[v] + 0.5f * venkat_fast(uR[v] - uUp[v], uL[v] - uR[v], e2R * sc);
        }
    } else if (kc.lim == LIM_MINMOD) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            UpL[v] = uL[v] + 0.5f * minmod_fast(uL[v] - uDn[v], uR[v] - uL[v], kc.ksi);
            UpR[v] = uR[v] - 0.5f * minmod_fast(uR[v] - uL[v], uUp[v] - uR[v], kc.ksi);
        }
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            UpL[v] = uL[v] + 0.5f * limiter(kc.lim, uL[v] - uDn[v], uR[v] - uL[v], kc.ksi);
            UpR[v] = uR[v] - 0.5f * limiter(kc.lim, uR[v] - uL[v], uUp[v] - uR[v], kc.ksi);
        }
    }
    if (FLUX == FLUX_AUSM) ausm_plus_fast(UpR, UpL, nx, ny, side, kc, f);
    else face_flux_fn<FLUX, float>(UpR, UpL, nx, ny, side, kc.gam, kc.g2, f);
}

__device__ __forceinline__ float4 avg4(const float4 &a, const float4 &b) {
    return make_float4(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z), 0.5f * (a.w + b.w));
}

// Transport model of the diffusion source (calcDiffTerm.jl:105-113; the
// Sutherland / constant extensions with artificial viscosity per
// calcArtViscosity.jl:46-75) applied to the cell's Laplacians `lap` (of
// rho u, rho v, E in the reference form; of u, v, |u|^2/2 + (gamma/Pr) e
// otherwise) and, for the artificial viscosity, its velocity divergence.
__device__ __forceinline__ void visc_source_f(const DevCase &P, const float4 &me, const float *lap, float divU,
                                              float HX, float *diff) {
    const float T = me.w / me.x / (float)P.R;
    diff[0] = 0.f;
    if (P.visc_model == VISC_REFERENCE) {
        const float mu = (float)P.mu_ref;
        diff[1] = mu * lap[0];
        diff[2] = mu * lap[1];
        diff[3] = mu * (float)air_conductivity((double)T) * lap[2];
    } else {
        const float mu = (P.visc_model == VISC_SUTHERLAND)
                             ? (float)P.mu_ref * (sutherland(T) / (float)P.suth_ref)
                             : (float)P.mu_ref;
        float mart = 0.f;
        if (P.art_visc) {
            const float aS = sqrtf((float)P.gamma * me.w / me.x);
            const float a = 0.05f * aS / HX * 0.70710678f;
            if (-divU > a) {
                const float tmp = divU * divU - a * a;
                if (tmp > 0.f) mart = 0.5f * me.x * (HX * HX * 0.5f) * sqrtf(tmp) * 1.0e-5f;
            }
        }
        const float mue = mu + mart;
        diff[1] = mue * lap[0];
        diff[2] = mue * lap[1];
        diff[3] = mue * lap[2];
    }
}

// One edge's share of the Green-Gauss sums of the diffusion source, seen
// from the cell whose inward normal (nx, ny) it has: the first-gradient node
// means A, B of the edge's two nodes give the Laplacian terms
// 0.5 (A + B).(-ny, -nx) side of each variable (calcDiffTerm.jl:88-104,
// gradX paired with -ny), and the node velocities a, b the velocity
// divergence term 0.5 (a + b).(-nx, -ny) side of the artificial viscosity.
// The other cell of the edge sees the exact negation.
__device__ __forceinline__ float4 visc_face_f(const NodeGradF &A, const NodeGradF &B, const float4 &a,
                                              const float4 &b, float nx, float ny, float side, bool art) {
    const float cx = -ny * 0.5f * side, cy = -nx * 0.5f * side;
    float4 r;
    r.x = (A.ru.x + B.ru.x) * cx + (A.ru.y + B.ru.y) * cy;
    r.y = (A.rv.x + B.rv.x) * cx + (A.rv.y + B.rv.y) * cy;
    r.z = (A.re.x + B.re.x) * cx + (A.re.y + B.re.y) * cy;
    r.w = art ? (a.y + b.y) * cy + (a.z + b.z) * cx : 0.f;
    return r;
}

// Diffusion source (calcDiffTerm.jl:88-113 and the extension models) in FP32.
template <bool QUAD>
__device__ __forceinline__ void diff_source_f(const DevMesh &m, const DevState &s, const DevCase &P, int64_t g,
                                              bool is_quad, const float4 &me, float *diff) {
    const int nf = (QUAD && is_quad) ? 4 : 3;
    float sx[3] = {0.f, 0.f, 0.f}, sy[3] = {0.f, 0.f, 0.f};
    float du = 0.f, dv = 0.f;
    const bool art = (P.visc_model != VISC_REFERENCE) && P.art_visc;
    for (int k = 0; k < nf; ++k) {
        const int64_t o = (int64_t)k * m.Nc + g;
        const float side = ld_once(m.lenf + o), nx = ld_once(m.nxf + o), ny = ld_once(m.nyf + o);
        const int2 e = ld_once(m.c2n + o);
        const NodeGradF A = s.nodeGf[e.x], B = s.nodeGf[e.y];
        sx[0] += 0.5f * (A.ru.x + B.ru.x) * -ny * side; sy[0] += 0.5f * (A.ru.y + B.ru.y) * -nx * side;
        sx[1] += 0.5f * (A.rv.x + B.rv.x) * -ny * side; sy[1] += 0.5f * (A.rv.y + B.rv.y) * -nx * side;
        sx[2] += 0.5f * (A.re.x + B.re.x) * -ny * side; sy[2] += 0.5f * (A.re.y + B.re.y) * -nx * side;
        if (art) {
            const float4 na = s.nodePf[e.x], nb = s.nodePf[e.y];
            du += 0.5f * (na.y + nb.y) * -nx * side;
            dv += 0.5f * (na.z + nb.z) * -ny * side;
        }
    }
    const float rA = ld_once(m.rareaf + g);
    const float lap[3] = {(sx[0] + sy[0]) * rA, (sx[1] + sy[1]) * rA, (sx[2] + sy[2]) * rA};
    visc_source_f(P, me, lap, (du + dv) * rA, art ? ld_once(m.hxf + g) : 0.f, diff);
}

// FP32 increment, FP64 accumulation of the Euler update
// (calcOneStageMUSCLcpuFast.jl:94-99), the densityConstrained clamp, the
// primitives recovered from the FP64 state (evaluate2d.jl:87-104) and the
// cell's contribution to the step's reductions.
// The per-cell arrays the update reads, loaded by the caller (the tile
// kernel issues these loads before its flux barrier).
struct CellInF {
    double4 U;  // FP64 conservative state before the step
    float rarea, area, charlen;
};
__device__ __forceinline__ CellInF load_cell_in_f(const DevMesh &m, const DevState &s, int64_t g) {
    CellInF r;
    r.U = ld_once(s.U + g);
    r.rarea = ld_once(m.rareaf + g);
    r.area = ld_once(m.areaf + g);
    r.charlen = ld_once(m.charlenf + g);
    return r;
}

__device__ __forceinline__ void cell_update_mixed(const DevMesh &m, const DevState &s, const DevCase &P, int64_t g,
                                                  const float4 &me, const float *F, const float *diff, double dt,
                                                  const CellInF &in, float4 *__restrict__ pout, Part &part) {
    const float bdt = (float)(P.beta * dt);
    const double4 U = in.U;
    const float rarea = in.rarea;
    const double Uo[4] = {U.x, U.y, U.z, U.w};
    double Un[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) Un[v] = Uo[v] + (double)(bdt * (diff[v] - F[v] * rarea));
    if (P.density_constrained == 1) {
        if (Un[0] >= P.rho_max) Un[0] = P.rho_max;
        if (Un[0] <= P.rho_min) Un[0] = P.rho_min;
    }
    st_once(s.U + g, make_double4(Un[0], Un[1], Un[2], Un[3]));
    const double rho = Un[0];
    const double rinv = 1.0 / rho;
    const double ux = Un[1] * rinv;
    const double uy = Un[2] * rinv;
    const double p = (P.gamma - 1.0) * (Un[3] - 0.5 * (Un[1] * ux + Un[2] * uy));
    const float a = sqrtf((float)(P.gamma * p * rinv));
    const float vmax = sqrtf((float)(ux * ux + uy * uy)) + a;
    pout[g] = make_float4((float)rho, (float)ux, (float)uy, (float)p);
    const double area = (double)in.area;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double d = Un[v] - Uo[v];
        part.res[v] = d * d;
        part.tot[v] = Un[v] * area;
    }
    part.ek = 0.5 * rho * (ux * ux + uy * uy) * area;
    part.vmax = (double)vmax;
    part.rmin = (double)(in.charlen / vmax);
    part.rhomin = (double)me.x;
    part.rhomax = (double)me.x;
    const bool ok = isfinite(Un[0]) && isfinite(Un[1]) && isfinite(Un[2]) && isfinite(Un[3]) && (rho > 0.0) &&
                    (p > 0.0);
    part.bad = ok ? 0.0 : 1.0;
}

}  // namespace
}  // namespace gd2d
