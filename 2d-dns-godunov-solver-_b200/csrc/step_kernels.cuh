// Kernels of the explicit Godunov step (FP64 state and arithmetic).
//
// One step = [viscous: grad1 cell pass, grad1 node pass] -> fused cell
// kernel -> node kernel.  The fused cell kernel does, per cell,
// calcOneStageMUSCLcpuFast (calcOneStageMUSCLcpuFast.jl:3-107) followed by
// updateVariablesSA (evaluate2d.jl:52-110) and the step's reductions; the
// last tile of each case finalizes that case's statistics and next time step
// (no device-wide barrier, no spin: a per-case ticket counter elects it).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "gd2d_internal.h"
#include "physics.cuh"

// Register budget of the node-side passes, as resident 256-thread blocks per SM.
#ifndef GD2D_NODE_MINB
#define GD2D_NODE_MINB 4
#endif

namespace gd2d {

// Programmatic dependent launch (launch_dependent): every step kernel lets
// the next one be scheduled as soon as all its blocks run, and waits for
// the previous one before it reads or writes any state.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Loads and stores of data a step touches once (per-cell and per-face mesh
// arrays, the conservative state): marked evict-first, so that the caches
// keep the gathered node and neighbour data instead.
template <class T>
__device__ __forceinline__ T ld_once(const T *p) {
    return __ldcs(p);
}
__device__ __forceinline__ double4 ld_once(const double4 *p) {
    const double2 a = __ldcs(reinterpret_cast<const double2 *>(p)), b = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st_once(double4 *p, const double4 &v) {
    __stcs(reinterpret_cast<double2 *>(p), make_double2(v.x, v.y));
    __stcs(reinterpret_cast<double2 *>(p) + 1, make_double2(v.z, v.w));
}

__device__ __forceinline__ int nbr_k(const int4 &v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

// ------------------------------------------------------- block reductions

struct Part {
    double res[4], tot[4], ek, vmax, rmin, rhomin, rhomax, bad;
    __device__ void init() {
        for (int v = 0; v < 4; ++v) { res[v] = 0.0; tot[v] = 0.0; }
        ek = 0.0; vmax = 0.0; rmin = INFINITY; rhomin = INFINITY; rhomax = -INFINITY; bad = 0.0;
    }
    __device__ void combine(const Part &o) {
        for (int v = 0; v < 4; ++v) { res[v] += o.res[v]; tot[v] += o.tot[v]; }
        ek += o.ek;
        vmax = fmax(vmax, o.vmax);
        rmin = fmin(rmin, o.rmin);
        rhomin = fmin(rhomin, o.rhomin);
        rhomax = fmax(rhomax, o.rhomax);
        bad = fmax(bad, o.bad);
    }
    __device__ void load_cg(const double *p) {
        for (int v = 0; v < 4; ++v) { res[v] = __ldcg(p + P_RES0 + v); tot[v] = __ldcg(p + P_TOT0 + v); }
        ek = __ldcg(p + P_EK); vmax = __ldcg(p + P_VMAX); rmin = __ldcg(p + P_RMIN);
        rhomin = __ldcg(p + P_RHOMIN); rhomax = __ldcg(p + P_RHOMAX); bad = __ldcg(p + P_BAD);
    }
};

// Fields of a Part in record order; 0-8 are sums, then max, min, min, max, max.
constexpr int kPartFields = 14;
__device__ __forceinline__ double part_op(int f, double a, double b) {
    if (f < 9) return a + b;
    return (f == 10 || f == 11) ? fmin(a, b) : fmax(a, b);
}

// Field f of a Part (record order).
__device__ __forceinline__ double part_get(const Part &p, int f) {
    switch (f) {
    case 0: case 1: case 2: case 3: return p.res[f];
    case 4: case 5: case 6: case 7: return p.tot[f - 4];
    case 8: return p.ek;
    case 9: return p.vmax;
    case 10: return p.rmin;
    case 11: return p.rhomin;
    case 12: return p.rhomax;
    default: return p.bad;
    }
}
__device__ __forceinline__ void part_set(Part &p, int f, double x) {
    switch (f) {
    case 0: case 1: case 2: case 3: p.res[f] = x; break;
    case 4: case 5: case 6: case 7: p.tot[f - 4] = x; break;
    case 8: p.ek = x; break;
    case 9: p.vmax = x; break;
    case 10: p.rmin = x; break;
    case 11: p.rhomin = x; break;
    case 12: p.rhomax = x; break;
    default: p.bad = x; break;
    }
}

// Records [b, e) (kPartials doubles apart) reduced by one warp in a fixed
// order: lane l folds records b + l, b + l + 32, ..., then a fixed shuffle
// tree per field.  The result is valid in lane 0.
__device__ __forceinline__ Part warp_reduce_records(const double *recs, int64_t b, int64_t e) {
    const int lane = threadIdx.x & 31;
    Part acc;
    acc.init();
    for (int64_t q = b + lane; q < e; q += 32) {
        Part o;
        o.load_cg(recs + q * kPartials);
        acc.combine(o);
    }
#pragma unroll
    for (int f = 0; f < kPartFields; ++f) {
        double x = part_get(acc, f);
        for (int off = 16; off > 0; off >>= 1) x = part_op(f, x, __shfl_down_sync(0xffffffffu, x, off));
        part_set(acc, f, x);
    }
    return acc;
}

// Per-case finalization by the warp that completed the case's last tile
// group: reduce the group records in a fixed order, publish the step
// statistics and advance time (flowTime += dt, testInviscidFluxesGPUx32.jl:401)
// and the next dt: the fixed solControls.dt the reference steps with, or
// opt-in, the tau it reports (testInviscidFluxesGPUx32.jl:299,324) or the
// local-CFL extension.
static __device__ __forceinline__ void finalize_case(const DevMesh &m, const DevState &s, int c, bool is_init) {
    const DevCase &P = m.cases[c];
    const Part acc = warp_reduce_records(s.gpart, P.group_begin, P.group_end);
    if ((threadIdx.x & 31) == 0) {
        CaseState *cs = s.cstate + c;
        double vnew = acc.vmax, rnew = acc.rmin;
        if (!is_init) {
            DevStats st;
            st.dt = cs->dt;
            st.flow_time = cs->t;
            st.velmax = cs->velmax;
            st.tau = P.CFL * P.maxEdge / jl_max(cs->velmax, 1.0e-6);
            for (int v = 0; v < 4; ++v) { st.residual[v] = acc.res[v]; st.totals[v] = acc.tot[v]; }
            st.rho_min = acc.rhomin;
            st.rho_max = acc.rhomax;
            st.kinetic_energy = acc.ek;
            st.step = cs->step + 1;
            st.nonfinite = acc.bad > 0.0 ? 1 : 0;
            st.reserved0 = 0;
            const int64_t row = (cs->step % s.ring_len) * m.ncases + c;
            s.ring[row] = st;
            s.ring_host[row] = st;  // over PCIe: the host reads it after the stream's sync
            cs->t = cs->t + cs->dt;
            cs->step = cs->step + 1;
            if (acc.bad > 0.0) cs->nonfinite = 1;
        }
        double dtn;
        if (P.dt_mode == DT_REFERENCE_TAU) dtn = P.CFL * P.maxEdge / jl_max(vnew, 1.0e-6);
        else if (P.dt_mode == DT_LOCAL_CFL) dtn = P.CFL * rnew;
        else dtn = P.dt_fixed;
        cs->dt = dtn;
        cs->velmax = vnew;
        cs->rmin = rnew;
        cs->tiles_done = 0u;
    }
}

// Field f of tile q's reduction record.  Two layouts, measured per
// precision on the 2.09M-cell viscous cylinder: FIELD_MAJOR (one row of
// ntiles doubles per field), which makes the FP64 cell kernel 10 us faster
// than records of kPartials doubles and the mixed one 6 us slower, so the
// FP64 kernels use it and the mixed kernels do not.  The layout is a
// template parameter: strides read at run time cost the mixed cell kernel
// spills and 4 us.
template <bool FIELD_MAJOR>
__device__ __forceinline__ double *part_at(const DevMesh &m, const DevState &s, int64_t q, int f) {
    return FIELD_MAJOR ? s.part + (int64_t)f * m.ntiles + q : s.part + q * kPartials + f;
}

// The tile's reduction record.  With ALIASED, the staging buffer `red`
// overlays buffers the block used for the tile, so a barrier retires them
// first; a buffer of the block's own needs none.  Each field is folded in a
// fixed order: two shuffle levels over groups of four lanes (so a quarter
// of the values go through shared memory: `red` holds kPartFields rows of
// blockDim/4), then blockDim/16 threads a field (224 of 256) fold four
// values each and a fixed shuffle tree joins them -- eight dependent levels
// in all.  The record is written by each field group's first thread.
// Nothing more happens at the tile's end: the next node pass folds the
// records (fold_field), so no tile waits for a fence or an atomic.  The
// last barrier retires `red` for the next tile of a persistent block.
template <bool FIELD_MAJOR, bool ALIASED>
__device__ __forceinline__ void tile_record(const DevMesh &m, const DevState &s, int64_t tile, const Part &p,
                                            double *red) {
    const int B = blockDim.x, t = threadIdx.x, lane = t & 31;
    const int R = B >> 2;    // values per field after the lane folds
    const int tpf = B >> 4;  // threads per field (4 values each); B is 128 or 256
    if (ALIASED) __syncthreads();
    const double v[kPartFields] = {p.res[0], p.res[1], p.res[2], p.res[3], p.tot[0], p.tot[1], p.tot[2],
                                   p.tot[3], p.ek, p.vmax, p.rmin, p.rhomin, p.rhomax, p.bad};
#pragma unroll
    for (int f = 0; f < kPartFields; ++f) {
        double x = v[f];
        x = part_op(f, x, __shfl_down_sync(0xffffffffu, x, 1));
        x = part_op(f, x, __shfl_down_sync(0xffffffffu, x, 2));
        if ((lane & 3) == 0) red[f * R + (t >> 2)] = x;
    }
    __syncthreads();
    const int f = t / tpf, i = t - f * tpf;
    if (f < kPartFields) {
        const double *row = red + f * R + i;
        double x = part_op(f, part_op(f, row[0], row[tpf]), part_op(f, row[2 * tpf], row[3 * tpf]));
        // a group's lanes are consecutive within one warp (tpf <= 16); the
        // lanes of this warp below thread kPartFields * tpf take part
        const int lim = kPartFields * tpf - (t & ~31);
        const unsigned mask = lim >= 32 ? 0xffffffffu : ((1u << lim) - 1u);
        for (int off = tpf >> 1; off > 0; off >>= 1) x = part_op(f, x, __shfl_down_sync(mask, x, off, tpf));
        if (i == 0) *part_at<FIELD_MAJOR>(m, s, tile, f) = x;
    }
    __syncthreads();
}

// Identity of field f of a Part (record order), as Part::init sets it.
__device__ __forceinline__ double part_ident(int f) {
    if (f == 10 || f == 11) return INFINITY;
    return f == 12 ? -INFINITY : 0.0;
}

// Blocks of a node pass that fold one tile group: one warp per (group,
// field) pair, so a group takes kPartFields / warps-per-block blocks.
__host__ __device__ __forceinline__ int fold_blocks_per_group(int block) {
    const int nw = block / 32;
    return (kPartFields + nw - 1) / nw;
}

// The step's two-level reduction, done by warps of the node pass that
// follows the cell kernel (the cell kernel's tile records are visible
// there: pdl_wait has returned).  One warp folds field f of tile group
// `gid` (up to kGroupTiles tiles of one case) into the group's record: lane
// l takes records l, l + 32, ..., l + kGroupTiles - 32 of the group in
// turn, then a fixed shuffle tree over the lanes.  It then counts the field
// done for the case; the warp that completes the case's last (group, field)
// pair reduces the case's group records and finalizes the case
// (finalize_case).  No thread waits on another's atomic; whichever warp
// finalizes, the order of every sum is the same, so the results are
// deterministic and do not depend on the node pass's block size.
template <bool FIELD_MAJOR>
static __device__ __forceinline__ void fold_field(const DevMesh &m, const DevState &s, int64_t gid, int f,
                                               bool is_init) {
    constexpr int kPerLane = kGroupTiles / 32;
    const int c = m.group_case[gid];
    const DevCase &P = m.cases[c];
    const int64_t t0 = P.tile_begin + (gid - P.group_begin) * kGroupTiles;
    const int n = (int)((t0 + kGroupTiles < P.tile_end) ? kGroupTiles : P.tile_end - t0);
    const int lane = threadIdx.x & 31;
    const double id = part_ident(f);
    double v[kPerLane];
#pragma unroll
    for (int j = 0; j < kPerLane; ++j) v[j] = (lane + 32 * j < n) ? __ldcg(part_at<FIELD_MAJOR>(m, s, t0 + lane + 32 * j, f)) : id;
    double x = v[0];
#pragma unroll
    for (int j = 1; j < kPerLane; ++j) x = part_op(f, x, v[j]);
    for (int off = 16; off > 0; off >>= 1) x = part_op(f, x, __shfl_down_sync(0xffffffffu, x, off));
    int last = 0;
    if (lane == 0) {
        s.gpart[gid * kPartials + f] = x;  // field f is record slot f
        __threadfence();
        const unsigned int need = (unsigned int)((P.group_end - P.group_begin) * kPartFields);
        last = (atomicAdd(&s.cstate[c].tiles_done, 1u) == need - 1u) ? 1 : 0;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {
        __threadfence();
        finalize_case(m, s, c, is_init);
    }
}

// Block b < nred of a node pass: its warps fold (group, field) pairs.
template <bool FIELD_MAJOR>
__device__ __forceinline__ void fold_block(const DevMesh &m, const DevState &s, int64_t g0, bool is_init) {
    const int bpg = fold_blocks_per_group(blockDim.x);
    const int f = (int)(blockIdx.x % bpg) * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (f < kPartFields) fold_field<FIELD_MAJOR>(m, s, g0 + blockIdx.x / bpg, f, is_init);
}

// --------------------------------------------------------- MUSCL + flux

// computeInterfaceSlope, computeslope2d.jl:3-136, for face k of cell g with
// its operands already fetched: neighbour code nbk (cell id or -(bc slot+1)),
// the neighbour's primitives r and HX (interior faces), the face geometry.
template <int FLUX, bool QUAD>
__device__ __forceinline__ void face_flux_at(const DevMesh &m, const DevCase &P, const double4 *__restrict__ nodeP,
                                             int64_t g, int k, int nbk, int dnk, int upk, int dn2k, int up2k,
                                             bool is_quad, const double *uL, const double4 &r, double hx_own,
                                             double hxR, double side, double nx, double ny, double t, double g2,
                                             double *f) {
    double uR[4], uUp[4], uDn[4];
    if (nbk >= 0) {
        if (QUAD && is_quad) {
            double4 a = nodeP[upk], a2 = nodeP[up2k], b = nodeP[dnk], b2 = nodeP[dn2k];
            uUp[0] = 0.5 * (a.x + a2.x); uUp[1] = 0.5 * (a.y + a2.y);
            uUp[2] = 0.5 * (a.z + a2.z); uUp[3] = 0.5 * (a.w + a2.w);
            uDn[0] = 0.5 * (b.x + b2.x); uDn[1] = 0.5 * (b.y + b2.y);
            uDn[2] = 0.5 * (b.z + b2.z); uDn[3] = 0.5 * (b.w + b2.w);
        } else {
            double4 a = nodeP[upk], b = nodeP[dnk];
            uUp[0] = a.x; uUp[1] = a.y; uUp[2] = a.z; uUp[3] = a.w;
            uDn[0] = b.x; uDn[1] = b.y; uDn[2] = b.z; uDn[3] = b.w;
        }
        uR[0] = r.x; uR[1] = r.y; uR[2] = r.z; uR[3] = r.w;
    } else {
        bc_ghost<double>(P, m, -nbk - 1, g, k, uL, nx, ny, t, uR);
        for (int v = 0; v < 4; ++v) { uDn[v] = uL[v]; uUp[v] = uR[v]; }
        hxR = hx_own;
    }
    double UpL[4], UpR[4];
    if (P.limiter == LIM_VENKAT) {
        // eps^2 = (K*HX)^3 times the face's (uL^2 + uR^2)/2 of each variable
        double KL = P.venkat_K * hx_own, KR = P.venkat_K * hxR;
        double e2L = KL * KL * KL, e2R = KR * KR * KR;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const double sc = 0.5 * (uL[v] * uL[v] + uR[v] * uR[v]);
            UpL[v] = uL[v] + 0.5 * lim_venkat(uL[v] - uDn[v], uR[v] - uL[v], e2L * sc);
            UpR[v] = uR[v] + 0.5 * lim_venkat(uR[v] - uUp[v], uL[v] - uR[v], e2R * sc);
        }
    } else {
        const int lk = P.limiter;
        const double ksi = P.ksi;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            UpL[v] = uL[v] + 0.5 * limiter(lk, uL[v] - uDn[v], uR[v] - uL[v], ksi);
            UpR[v] = uR[v] - 0.5 * limiter(lk, uR[v] - uL[v], uUp[v] - uR[v], ksi);
        }
    }
    face_flux_fn<FLUX, double>(UpR, UpL, nx, ny, side, P.gamma, g2, f);
}

// Face k of cell g, fetching its operands from the per-cell arrays.
template <int FLUX, bool QUAD>
__device__ __forceinline__ void face_flux(const DevMesh &m, const DevCase &P, const double4 *__restrict__ pin,
                                          const double4 *__restrict__ nodeP, int64_t g, int k, int nbk,
                                          int dnk, int upk, int dn2k, int up2k, bool is_quad, const double *uL,
                                          double hx_own, double t, double g2, double *f) {
    const int64_t o = (int64_t)k * m.Nc + g;
    const double side = m.len[o], nx = m.nx[o], ny = m.ny[o];
    double4 r = make_double4(0.0, 0.0, 0.0, 0.0);
    double hxR = hx_own;
    if (nbk >= 0) {
        r = pin[nbk];
        if (P.limiter == LIM_VENKAT) hxR = m.hx[nbk];
    }
    face_flux_at<FLUX, QUAD>(m, P, nodeP, g, k, nbk, dnk, upk, dn2k, up2k, is_quad, uL, r, hx_own, hxR, side, nx, ny,
                             t, g2, f);
}

// Second Green-Gauss pass and transport model: the diffusion source of
// calcDiffTerm (calcDiffTerm.jl:88-113; gradients per calcGradients.jl:36-139,
// artificial viscosity per calcArtViscosity.jl:46-75).
template <bool QUAD>
__device__ __forceinline__ void diff_source(const DevMesh &m, const DevState &s, const DevCase &P, int64_t g,
                                            bool is_quad, const double4 &me, double *diff) {
    const int nf = (QUAD && is_quad) ? 4 : 3;
    double sx[3] = {0.0, 0.0, 0.0}, sy[3] = {0.0, 0.0, 0.0};
    double du = 0.0, dv = 0.0;
    const bool art = (P.visc_model != VISC_REFERENCE) && P.art_visc;
    for (int k = 0; k < nf; ++k) {
        const int64_t o = (int64_t)k * m.Nc + g;
        const double side = m.len[o], nx = m.nx[o], ny = m.ny[o];
        const int2 e = ld_once(m.c2n + o);
        const NodeGrad A = s.nodeG[e.x], B = s.nodeG[e.y];
        double fx, fy;
        fx = 0.5 * (A.ru.x + B.ru.x) * -ny * side; fy = 0.5 * (A.ru.y + B.ru.y) * -nx * side;
        sx[0] = (k == 0) ? fx : sx[0] + fx; sy[0] = (k == 0) ? fy : sy[0] + fy;
        fx = 0.5 * (A.rv.x + B.rv.x) * -ny * side; fy = 0.5 * (A.rv.y + B.rv.y) * -nx * side;
        sx[1] = (k == 0) ? fx : sx[1] + fx; sy[1] = (k == 0) ? fy : sy[1] + fy;
        fx = 0.5 * (A.re.x + B.re.x) * -ny * side; fy = 0.5 * (A.re.y + B.re.y) * -nx * side;
        sx[2] = (k == 0) ? fx : sx[2] + fx; sy[2] = (k == 0) ? fy : sy[2] + fy;
        if (art) {
            const double4 na = s.nodeP[e.x], nb = s.nodeP[e.y];
            double fu = 0.5 * (na.y + nb.y) * -nx * side;
            double fv = 0.5 * (na.z + nb.z) * -ny * side;
            du = (k == 0) ? fu : du + fu;
            dv = (k == 0) ? fv : dv + fv;
        }
    }
    const double area = ld_once(m.area + g);
    double lap[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) lap[v] = sx[v] / area + sy[v] / area;
    const double T = me.w / me.x / P.R;
    diff[0] = 0.0;
    if (P.visc_model == VISC_REFERENCE) {
        const double mu = P.mu_ref;
        diff[1] = mu * lap[0];
        diff[2] = mu * lap[1];
        diff[3] = mu * air_conductivity(T) * lap[2];
    } else {
        const double mu = (P.visc_model == VISC_SUTHERLAND) ? P.mu_ref * (sutherland(T) / P.suth_ref) : P.mu_ref;
        double mart = 0.0;
        if (art) {
            const double HX = ld_once(m.hx + g);
            const double divU = du / area + dv / area;
            const double aS = sqrt(P.gamma * me.w / me.x);
            const double a = 0.05 * aS / HX / sqrt(2.0);
            if (-divU > a) {
                const double tmp = divU * divU - a * a;
                if (tmp > 0.0) mart = 0.5 * me.x * HX / sqrt(2.0) * HX / sqrt(2.0) * sqrt(tmp) * 1.0e-5;
            }
        }
        // laplacians of u, v and phi = |u|^2/2 + (gamma/Pr) e
        const double mue = mu + (P.art_visc ? mart : 0.0);
        diff[1] = mue * lap[0];
        diff[2] = mue * lap[1];
        diff[3] = mue * lap[2];
    }
}

// Euler update (calcOneStageMUSCLcpuFast.jl:94-99), the densityConstrained
// clamp (evaluate2d.jl:63-77), updateVariablesSA (evaluate2d.jl:87-104) and
// the cell's contribution to the step's reductions.
// The per-cell arrays the update reads, loaded by the caller (the tile
// kernel issues these loads before its flux barrier).
struct CellIn {
    double4 U;  // conservative state before the step
    double rarea, area, charlen;
};
__device__ __forceinline__ CellIn load_cell_in(const DevMesh &m, const DevState &s, int64_t g) {
    CellIn r;
    r.U = ld_once(s.U + g);
    r.rarea = ld_once(m.rarea + g);
    r.area = ld_once(m.area + g);
    r.charlen = ld_once(m.charlen + g);
    return r;
}

__device__ __forceinline__ void cell_update(const DevMesh &m, const DevState &s, const DevCase &P, int64_t g,
                                            const double4 &me, const double *F, const double *diff, double dt,
                                            const CellIn &in, double4 *__restrict__ pout, Part &part) {
    const double4 U = in.U;
    const double rarea = in.rarea;
    const double Uo[4] = {U.x, U.y, U.z, U.w};
    double Un[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) Un[v] = (Uo[v] - F[v] * P.beta * dt * rarea + P.beta * dt * diff[v]);
    if (P.density_constrained == 1) {
        if (Un[0] >= P.rho_max) Un[0] = P.rho_max;
        if (Un[0] <= P.rho_min) Un[0] = P.rho_min;
    }
    st_once(s.U + g, make_double4(Un[0], Un[1], Un[2], Un[3]));
    const double gam = P.gamma;
    const double rho = Un[0];
    const double ux = Un[1] / Un[0];
    const double uy = Un[2] / Un[0];
    const double p = (gam - 1.0) * (Un[3] - 0.5 * (Un[1] * Un[1] + Un[2] * Un[2]) / Un[0]);
    const double a = sqrt(gam * p / rho);
    const double vmax = sqrt(ux * ux + uy * uy) + a;
    pout[g] = make_double4(rho, ux, uy, p);
    const double area = in.area;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double d = Un[v] - Uo[v];
        part.res[v] = d * d;
        part.tot[v] = Un[v] * area;
    }
    part.ek = 0.5 * rho * (ux * ux + uy * uy) * area;
    part.vmax = vmax;
    part.rmin = in.charlen / vmax;
    part.rhomin = me.x;
    part.rhomax = me.x;
    const bool ok = isfinite(Un[0]) && isfinite(Un[1]) && isfinite(Un[2]) && isfinite(Un[3]) && (rho > 0.0) &&
                    (p > 0.0);
    part.bad = ok ? 0.0 : 1.0;
}

// ---------------------------------------------------- fused cell kernel

template <int FLUX, bool VISC, bool QUAD, int MINB>
__global__ void __launch_bounds__(256, MINB) k_cell_step(const DevMesh m, const DevState s) {
    __shared__ double s_red[kPartFields * 256];
    const int par = *s.parity;
    const double4 *__restrict__ pin = s.prim + (int64_t)par * m.Nc;
    double4 *__restrict__ pout = s.prim + (int64_t)(par ^ 1) * m.Nc;
    const double4 *__restrict__ nodeP = s.nodeP;
    for (int64_t tile = blockIdx.x; tile < m.ntiles; tile += gridDim.x) {
        const int c = m.tile_case[tile];
        const DevCase &P = m.cases[c];
        const double dt = s.cstate[c].dt, t = s.cstate[c].t;
        const int64_t g = tile * blockDim.x + threadIdx.x;
        Part part;
        part.init();
        const int4 nb = m.nbr[g];
        if (nb.x != kAbsent) {
            const bool is_quad = QUAD && (nb.w != kAbsent);
            const double4 me = pin[g];
            const double uL[4] = {me.x, me.y, me.z, me.w};
            const double gam = P.gamma;
            const double g2 = 2.0 * (gam - 1.0) / (gam + 1.0);
            const double hx_own = (P.limiter == LIM_VENKAT) ? m.hx[g] : 0.0;
            const int4 dn = m.dn[g], up = m.up[g];
            int4 dn2 = make_int4(0, 0, 0, 0), up2 = make_int4(0, 0, 0, 0);
            if (QUAD && is_quad) { dn2 = m.dn2[g]; up2 = m.up2[g]; }
            double F[4], f[4];
            face_flux<FLUX, QUAD>(m, P, pin, nodeP, g, 0, nb.x, dn.x, up.x, dn2.x, up2.x, is_quad, uL, hx_own, t, g2, F);
            face_flux<FLUX, QUAD>(m, P, pin, nodeP, g, 1, nb.y, dn.y, up.y, dn2.y, up2.y, is_quad, uL, hx_own, t, g2, f);
#pragma unroll
            for (int v = 0; v < 4; ++v) F[v] = F[v] + f[v];
            face_flux<FLUX, QUAD>(m, P, pin, nodeP, g, 2, nb.z, dn.z, up.z, dn2.z, up2.z, is_quad, uL, hx_own, t, g2, f);
#pragma unroll
            for (int v = 0; v < 4; ++v) F[v] = F[v] + f[v];
            if (QUAD && is_quad) {
                face_flux<FLUX, QUAD>(m, P, pin, nodeP, g, 3, nb.w, dn.w, up.w, dn2.w, up2.w, is_quad, uL, hx_own, t, g2, f);
#pragma unroll
                for (int v = 0; v < 4; ++v) F[v] = F[v] + f[v];
            }
            double diff[4] = {0.0, 0.0, 0.0, 0.0};
            if (VISC) diff_source<QUAD>(m, s, P, g, is_quad, me, diff);
            cell_update(m, s, P, g, me, F, diff, dt, load_cell_in(m, s, g), pout, part);
        }
        tile_record<true, false>(m, s, tile, part, s_red);
    }
}

// The fused cell kernel over tile-local face lists (GD2D_LOOP_TILE_FACES).
// Phase 1 stages the tile's primitives (and HX) in shared memory; phase 2
// runs the tile's face list, one face per thread: a face between two cells
// of the tile is computed once, from its lower-indexed cell, and its flux
// stored negated into the other cell's slot -- exact because the listed
// pairs are only those whose face state and flux are antisymmetric bit for
// bit under exchange of the two cells (checked on the host: AUSM+ with the
// Minmod or Venkatakrishnan limiter or none, negated normals, exchanged
// down/up nodes); every other face slot is computed from its own cell as in
// k_cell_step.  Phase 3 sums each cell's slots in face order
// (calcOneStageMUSCLcpuFast.jl:66-85) and finishes the cell as k_cell_step.
template <int FLUX, bool VISC, bool QUAD, int MINB>
__global__ void __launch_bounds__(256, MINB) k_cell_step_tf(const DevMesh m, const DevState s) {
    constexpr int NS = QUAD ? 4 : 3;
    // one buffer: the tile's primitives, then its flux slots; the step
    // reduction reuses it once both have been consumed
    __shared__ double4 s_mem[(1 + NS) * 256];
    __shared__ double s_hx[256];
    static_assert((1 + NS) * 256 * 4 >= kPartFields * 256, "reduction buffer");
    double4 *const s_prim = s_mem;
    double4 (*const s_flux)[256] = reinterpret_cast<double4 (*)[256]>(s_mem + 256);
    pdl_trigger();
    pdl_wait();
    const int par = *s.parity;
    const double4 *__restrict__ pin = s.prim + (int64_t)par * m.Nc;
    double4 *__restrict__ pout = s.prim + (int64_t)(par ^ 1) * m.Nc;
    const int B = blockDim.x;
    for (int64_t tile = blockIdx.x; tile < m.ntiles; tile += gridDim.x) {
        const int64_t base = tile * B;
        const int64_t g = base + threadIdx.x;
        // loads that depend on nothing go out first: the face-list bounds
        // and HX (used only with the Venkatakrishnan limiter) need not wait
        // for the case record
        const int64_t f0 = m.tf_off[tile], f1 = m.tf_off[tile + 1];
        s_prim[threadIdx.x] = pin[g];
        s_hx[threadIdx.x] = ld_once(m.hx + g);
        const int c = m.tile_case[tile];
        const DevCase &P = m.cases[c];
        const double t = s.cstate[c].t;
        const bool venkat = P.limiter == LIM_VENKAT;
        // face indices fit 32 bits (setup checks the total); the first face
        // record goes out with the staging loads and each next one before
        // the current face's gathers, so no face waits for its record
        const int fb = (int)f0 + (int)threadIdx.x, fe = (int)f1;
        int4 next = make_int4(0, 0, 0, 0);
        if (fb < fe) next = ld_once(m.tf_rec + fb);
        __syncthreads();
        const double gam = P.gamma;
        const double g2 = 2.0 * (gam - 1.0) / (gam + 1.0);
        for (int f = fb; f < fe; f += B) {
            const int4 rec = next;
            if (f + B < fe) next = ld_once(m.tf_rec + f + B);
            const TileFace tf = unpack_tile_face(rec.y);
            const double4 a4 = s_prim[tf.la];
            const double uL[4] = {a4.x, a4.y, a4.z, a4.w};
            const double hx_own = venkat ? s_hx[tf.la] : 0.0;
            double4 r = make_double4(0.0, 0.0, 0.0, 0.0);
            double hxR = hx_own;
            if (rec.x >= 0) {
                const int64_t lr = (int64_t)rec.x - base;
                if (lr >= 0 && lr < B) {
                    r = s_prim[lr];
                    if (venkat) hxR = s_hx[lr];
                } else {
                    r = pin[rec.x];
                    if (venkat) hxR = m.hx[rec.x];
                }
            }
            int2 q2 = make_int2(0, 0);
            if (QUAD && tf.quad) q2 = m.tf_q[f];
            double fv[4];
            // the face geometry of slot (la, ka) from the per-cell planes,
            // cached: the viscous source reads the same lines again
            const int64_t og = (int64_t)tf.ka * m.Nc + base + tf.la;
            face_flux_at<FLUX, QUAD>(m, P, s.nodeP, base + tf.la, tf.ka, rec.x, rec.z, rec.w, q2.x, q2.y,
                                     QUAD && tf.quad, uL, r, hx_own, hxR, m.len[og], m.nx[og], m.ny[og], t,
                                     g2, fv);
            s_flux[tf.ka][tf.la] = make_double4(fv[0], fv[1], fv[2], fv[3]);
            if (tf.lbp) s_flux[tf.kb][tf.lbp - 1] = make_double4(-fv[0], -fv[1], -fv[2], -fv[3]);
        }
        // the cell's viscous source needs no flux: evaluated before the
        // barrier, it fills the time a thread with fewer faces would wait
        // (the cell's primitives are re-read from the stage rather than
        // held in registers through the face phase)
        const double4 me = s_prim[threadIdx.x];
        const double dt = s.cstate[c].dt;
        // triangles: the viscous source is evaluated for padding cells too
        // (node 0 in their edge slots, zero area; the result is unused), and
        // a padding cell is told by its zero inverse area; quads read the
        // neighbour record, which also tells triangles from quads
        bool live = true, is_quad = false;
        if (QUAD) {
            const int4 nb = ld_once(m.nbr + g);
            live = nb.x != kAbsent;
            is_quad = nb.w != kAbsent;
        }
        double diff[4] = {0.0, 0.0, 0.0, 0.0};
        if (VISC && live) diff_source<QUAD>(m, s, P, g, is_quad, me, diff);
        // the update's own loads go out before the barrier (padded arrays:
        // in bounds for padding cells, whose values are not used)
        const CellIn cin = load_cell_in(m, s, g);
        if (!QUAD) live = cin.rarea != 0.0;
        __syncthreads();
        Part part;
        part.init();
        if (live) {
            const double4 a0 = s_flux[0][threadIdx.x], a1 = s_flux[1][threadIdx.x], a2 = s_flux[2][threadIdx.x];
            double F[4] = {a0.x + a1.x, a0.y + a1.y, a0.z + a1.z, a0.w + a1.w};
            F[0] = F[0] + a2.x; F[1] = F[1] + a2.y; F[2] = F[2] + a2.z; F[3] = F[3] + a2.w;
            if (QUAD && is_quad) {
                const double4 a3 = s_flux[NS - 1][threadIdx.x];
                F[0] = F[0] + a3.x; F[1] = F[1] + a3.y; F[2] = F[2] + a3.z; F[3] = F[3] + a3.w;
            }
            cell_update(m, s, P, g, me, F, diff, dt, cin, pout, part);
        }
        tile_record<true, true>(m, s, tile, part, reinterpret_cast<double *>(s_mem));
    }
}

// ------------------------------------------------------------ node kernel

// cells2nodesSolutionReconstructionWithStencils (utilsFVM2dp.jl:299-365):
// weighted primitive averages; with VISC also calcPhiInCellCluster's
// unweighted means of rho u, rho v, E (calcGradients.jl:3-18) for the next
// step's viscous term.  The last block flips the step parity.  The first
// `nred` blocks instead fold the cell kernel's tile groups g0, g0 + 1, ...
// (fold_block): they start first and their latency hides behind the node
// gathers; nothing here reads what they write.
// The node-side kernels are bound by the latency of their gathers; their
// register budget is capped for 4 resident blocks per SM (more warps in
// flight; measured faster than the unconstrained 76-register build).
template <bool VISC, bool UNIT>
__global__ void __launch_bounds__(256, GD2D_NODE_MINB) k_node_avg(const DevMesh m, const DevState s, int flip, int zero_prims,
                                                  int64_t n0, int64_t n1, int64_t g0, int nred, int is_init) {
    pdl_trigger();
    pdl_wait();
    if ((int)blockIdx.x < nred) {
        fold_block<true>(m, s, g0, is_init != 0);
        return;
    }
    const int64_t bid = (int64_t)blockIdx.x - nred, nblk = (int64_t)gridDim.x - nred;
    const int par = *s.parity;
    const double4 *__restrict__ src = s.prim + (int64_t)(flip ? (par ^ 1) : par) * m.Nc;
    const int W = m.cluster_w;
    for (int64_t J = n0 + bid * blockDim.x + threadIdx.x; J < n1; J += nblk * blockDim.x) {
        bool prim_form = false;
        double gop = 0.0, gam = 0.0;
        if (VISC) {
            const DevCase &P = m.cases[ld_once(m.node_case + J)];
            prim_form = P.visc_model != VISC_REFERENCE;
            gop = P.gamma_over_Pr;
            gam = P.gamma;
        }
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, det = 0.0;
        double c0 = 0.0, c1 = 0.0, c2 = 0.0;
        int cnt = 0;
        auto add = [&](int c, const double4 &p, double w) {
            a0 = a0 + p.x * w; a1 = a1 + p.y * w; a2 = a2 + p.z * w; a3 = a3 + p.w * w;
            det = det + w;
            if (VISC) {
                if (prim_form) {
                    // u, v, phi = |u|^2/2 + (gamma/Pr) p / ((gamma-1) rho)
                    const double ph = 0.5 * (p.y * p.y + p.z * p.z) + gop * (p.w / ((gam - 1.0) * p.x));
                    c0 = c0 + p.y; c1 = c1 + p.z; c2 = c2 + ph;
                } else {
                    const double4 u = s.U[c];
                    c0 = c0 + u.y; c1 = c1 + u.z; c2 = c2 + u.w;
                }
                ++cnt;
            }
        };
        // all cluster indices first, then the gathers in an unrolled
        // sequence the compiler can overlap (sums keep the reference order)
        int ci[kMaxCluster];
#pragma unroll
        for (int j = 0; j < kMaxCluster; ++j) ci[j] = (j < W) ? ld_once(m.cl + (int64_t)j * m.Nn + J) : -1;
#pragma unroll
        for (int j = 0; j < kMaxCluster; ++j)
            if (ci[j] >= 0) add(ci[j], src[ci[j]], UNIT ? 1.0 : ld_once(m.wt + (int64_t)j * m.Nn + J));
        for (int j = kMaxCluster; j < W; ++j) {
            const int c = ld_once(m.cl + (int64_t)j * m.Nn + J);
            if (c >= 0) add(c, src[c], UNIT ? 1.0 : ld_once(m.wt + (int64_t)j * m.Nn + J));
        }
        if (det != 0.0) { a0 = a0 / det; a1 = a1 / det; a2 = a2 / det; a3 = a3 / det; }
        s.nodeP[J] = zero_prims ? make_double4(0.0, 0.0, 0.0, 0.0) : make_double4(a0, a1, a2, a3);
        if (VISC) {
            if (cnt != 0) {
                const double dc = (double)cnt;
                s.nodeC[J] = make_double4(c0 / dc, c1 / dc, c2 / dc, 0.0);
            } else {
                s.nodeC[J] = make_double4(0.0, 0.0, 0.0, 0.0);
            }
        }
    }
    if (flip) {
        // Every warp of the block has read the parity once the barrier is
        // passed; the block that completes the count flips it.  Nothing in
        // this kernel reads what the others wrote, so no fence: stream order
        // makes the flip and the node values visible to the next kernel.
        __syncthreads();
        if (threadIdx.x == 0 && atomicAdd(s.node_done, 1u) == (unsigned int)nblk - 1u) {
            *s.node_done = 0u;
            *s.parity = par ^ 1;
        }
    }
}

// ------------------------------------------------------ viscous passes

// First Green-Gauss gradient of rho u, rho v, E from the unweighted node
// means (calcScalarFieldGreenGaussNodesBasedGradient, calcGradients.jl:36-139:
// gradX pairs with -ny, gradY with -nx).
template <bool QUAD>
__global__ void __launch_bounds__(256, GD2D_NODE_MINB) k_grad1_cells(const DevMesh m, const DevState s) {
    constexpr int NF = QUAD ? 4 : 3;
    pdl_trigger();
    pdl_wait();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < m.Nc; g += (int64_t)gridDim.x * blockDim.x) {
        // Every per-cell load is issued before any of them is tested, so a
        // cell costs two trips to memory (its own arrays, then the node
        // gathers).  Padding cells (zero area, node 0 in their edge slots)
        // are dropped at the store; a triangle's fourth edge has zero length.
        const double area = ld_once(m.area + g);
        double side[NF], nx[NF], ny[NF];
        int2 e[NF];
#pragma unroll
        for (int k = 0; k < NF; ++k) {
            const int64_t o = (int64_t)k * m.Nc + g;
            side[k] = ld_once(m.len + o);
            nx[k] = ld_once(m.nx + o);
            ny[k] = ld_once(m.ny + o);
            e[k] = ld_once(m.c2n + o);
        }
        const int nf = (QUAD && side[NF - 1] != 0.0) ? 4 : 3;
        double sx[3] = {0.0, 0.0, 0.0}, sy[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < NF; ++k) {
            if (k >= nf) break;
            const double4 A = s.nodeC[e[k].x], B = s.nodeC[e[k].y];
            double fx, fy;
            fx = 0.5 * (A.x + B.x) * -ny[k] * side[k]; fy = 0.5 * (A.x + B.x) * -nx[k] * side[k];
            sx[0] = (k == 0) ? fx : sx[0] + fx; sy[0] = (k == 0) ? fy : sy[0] + fy;
            fx = 0.5 * (A.y + B.y) * -ny[k] * side[k]; fy = 0.5 * (A.y + B.y) * -nx[k] * side[k];
            sx[1] = (k == 0) ? fx : sx[1] + fx; sy[1] = (k == 0) ? fy : sy[1] + fy;
            fx = 0.5 * (A.z + B.z) * -ny[k] * side[k]; fy = 0.5 * (A.z + B.z) * -nx[k] * side[k];
            sx[2] = (k == 0) ? fx : sx[2] + fx; sy[2] = (k == 0) ? fy : sy[2] + fy;
        }
        if (area == 0.0) continue;
        NodeGrad r;
        r.ru = make_double2(sx[0] / area, sy[0] / area);
        r.rv = make_double2(sx[1] / area, sy[1] / area);
        r.re = make_double2(sx[2] / area, sy[2] / area);
        s.g1[g] = r;
    }
}

// Unweighted node means of the first gradients (calcPhiInCellCluster on the
// gradient fields, calcGradients.jl:3-18).
static __global__ void __launch_bounds__(256, GD2D_NODE_MINB) k_grad1_nodes(const DevMesh m, const DevState s) {
    const int W = m.cluster_w;
    pdl_trigger();
    pdl_wait();
    for (int64_t J = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; J < m.Nn; J += (int64_t)gridDim.x * blockDim.x) {
        double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int cnt = 0;
        auto add = [&](const NodeGrad &q) {
            v[0] = v[0] + q.ru.x; v[1] = v[1] + q.ru.y; v[2] = v[2] + q.rv.x;
            v[3] = v[3] + q.rv.y; v[4] = v[4] + q.re.x; v[5] = v[5] + q.re.y;
            ++cnt;
        };
        int ci[kMaxCluster];
#pragma unroll
        for (int j = 0; j < kMaxCluster; ++j) ci[j] = (j < W) ? ld_once(m.cl + (int64_t)j * m.Nn + J) : -1;
#pragma unroll
        for (int j = 0; j < kMaxCluster; ++j)
            if (ci[j] >= 0) add(s.g1[ci[j]]);
        for (int j = kMaxCluster; j < W; ++j) {
            const int c = ld_once(m.cl + (int64_t)j * m.Nn + J);
            if (c >= 0) add(s.g1[c]);
        }
        NodeGrad r;
        if (cnt != 0) {
            const double dc = (double)cnt;
            r.ru = make_double2(v[0] / dc, v[1] / dc);
            r.rv = make_double2(v[2] / dc, v[3] / dc);
            r.re = make_double2(v[4] / dc, v[5] / dc);
        } else {
            r.ru = r.rv = r.re = make_double2(0.0, 0.0);
        }
        s.nodeG[J] = r;
    }
}

// ------------------------------------------------------------ state init

// phs2dcns2dcellsSA (utilsFVM2dp.jl:4-17) on the current primitives and the
// reductions that give the first step's dt (createFields2d's VMAX).
static __global__ void __launch_bounds__(256) k_init_state(const DevMesh m, const DevState s, int64_t t0, int64_t t1) {
    __shared__ double s_red[kPartFields * 256];
    const int par = *s.parity;
    const double4 *__restrict__ pin = s.prim + (int64_t)par * m.Nc;
    for (int64_t tile = t0 + blockIdx.x; tile < t1; tile += gridDim.x) {
        const int c = m.tile_case[tile];
        const DevCase &P = m.cases[c];
        const int64_t g = tile * blockDim.x + threadIdx.x;
        Part part;
        part.init();
        const int4 nb = m.nbr[g];
        if (nb.x != kAbsent) {
            const double4 q = pin[g];
            const double G = P.gamma;
            const double r = q.x, u = q.y, v = q.z, pp = q.w;
            s.U[g] = make_double4(r, r * u, r * v, pp / (G - 1.0) + 0.5 * r * (u * u + v * v));
            const double a = sqrt(G * pp / r);
            const double vmax = sqrt(u * u + v * v) + a;
            part.vmax = vmax;
            part.rmin = m.charlen[g] / vmax;
        }
        tile_record<true, false>(m, s, tile, part, s_red);
    }
}

// ------------------------------------------------------- face-loop variants

// One thread per face: the flux seen from cell a (face slot ka), added to a
// and subtracted from the neighbour b (FACE_COLOURED: into Facc, faces of
// one launch never share a cell) or stored in the slots (a, ka) and (b, kb)
// (FACE_SLOTS).  face = (a, neighbour code of slot ka, ka | kb << 8, -).
template <int FLUX, bool QUAD, bool SLOTS>
__global__ void __launch_bounds__(256) k_face_flux(const DevMesh m, const DevState s, const int4 *__restrict__ faces,
                                                   int64_t f0, int64_t f1, int tile_cells,
                                                   double4 *__restrict__ Facc, double4 *__restrict__ Fslot) {
    const int64_t f = f0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= f1) return;
    const int par = *s.parity;
    const double4 *__restrict__ pin = s.prim + (int64_t)par * m.Nc;
    const int4 fc = faces[f];
    const int64_t a = fc.x;
    const int nbk = fc.y, ka = fc.z & 255, kb = fc.z >> 8;
    const int c = m.tile_case[a / tile_cells];
    const DevCase &P = m.cases[c];
    const double t = s.cstate[c].t;
    const int4 nb = m.nbr[a];
    const bool is_quad = QUAD && (nb.w != kAbsent);
    const double4 me = pin[a];
    const double uL[4] = {me.x, me.y, me.z, me.w};
    const double gam = P.gamma;
    const double g2 = 2.0 * (gam - 1.0) / (gam + 1.0);
    const double hx_own = (P.limiter == LIM_VENKAT) ? m.hx[a] : 0.0;
    const int4 dn = m.dn[a], up = m.up[a];
    int4 dn2 = make_int4(0, 0, 0, 0), up2 = make_int4(0, 0, 0, 0);
    if (QUAD && is_quad) { dn2 = m.dn2[a]; up2 = m.up2[a]; }
    double fv[4];
    face_flux<FLUX, QUAD>(m, P, pin, s.nodeP, a, ka, nbk, nbr_k(dn, ka), nbr_k(up, ka), nbr_k(dn2, ka),
                          nbr_k(up2, ka), is_quad, uL, hx_own, t, g2, fv);
    if (SLOTS) {
        Fslot[(int64_t)ka * m.Nc + a] = make_double4(fv[0], fv[1], fv[2], fv[3]);
        if (nbk >= 0) Fslot[(int64_t)kb * m.Nc + nbk] = make_double4(-fv[0], -fv[1], -fv[2], -fv[3]);
    } else {
        double4 x = Facc[a];
        Facc[a] = make_double4(x.x + fv[0], x.y + fv[1], x.z + fv[2], x.w + fv[3]);
        if (nbk >= 0) {
            double4 y = Facc[nbk];
            Facc[nbk] = make_double4(y.x - fv[0], y.y - fv[1], y.z - fv[2], y.w - fv[3]);
        }
    }
}

// Euler update and updateVariablesSA after a face loop: the cell kernel's
// second half, with the face-flux sum read back (FACE_SLOTS: summed in face
// order k = 1..nf as calcOneStageMUSCLcpuFast.jl:66-85; FACE_COLOURED: the
// accumulator, reset to zero for the next step).
template <bool VISC, bool QUAD, bool SLOTS, int MINB>
__global__ void __launch_bounds__(256, MINB) k_face_update(const DevMesh m, const DevState s,
                                                          double4 *__restrict__ Facc,
                                                          const double4 *__restrict__ Fslot) {
    __shared__ double s_red[kPartFields * 256];
    const int par = *s.parity;
    const double4 *__restrict__ pin = s.prim + (int64_t)par * m.Nc;
    double4 *__restrict__ pout = s.prim + (int64_t)(par ^ 1) * m.Nc;
    for (int64_t tile = blockIdx.x; tile < m.ntiles; tile += gridDim.x) {
        const int c = m.tile_case[tile];
        const DevCase &P = m.cases[c];
        const double dt = s.cstate[c].dt;
        const int64_t g = tile * blockDim.x + threadIdx.x;
        Part part;
        part.init();
        const int4 nb = m.nbr[g];
        if (nb.x != kAbsent) {
            const bool is_quad = QUAD && (nb.w != kAbsent);
            const double4 me = pin[g];
            double F[4];
            if (SLOTS) {
                double4 a0 = Fslot[g], a1 = Fslot[m.Nc + g], a2 = Fslot[2 * m.Nc + g];
                F[0] = a0.x + a1.x + a2.x; F[1] = a0.y + a1.y + a2.y;
                F[2] = a0.z + a1.z + a2.z; F[3] = a0.w + a1.w + a2.w;
                if (QUAD && is_quad) {
                    double4 a3 = Fslot[3 * m.Nc + g];
                    F[0] = F[0] + a3.x; F[1] = F[1] + a3.y; F[2] = F[2] + a3.z; F[3] = F[3] + a3.w;
                }
            } else {
                double4 a0 = Facc[g];
                F[0] = a0.x; F[1] = a0.y; F[2] = a0.z; F[3] = a0.w;
                Facc[g] = make_double4(0.0, 0.0, 0.0, 0.0);
            }
            double diff[4] = {0.0, 0.0, 0.0, 0.0};
            if (VISC) diff_source<QUAD>(m, s, P, g, is_quad, me, diff);
            cell_update(m, s, P, g, me, F, diff, dt, load_cell_in(m, s, g), pout, part);
        }
        tile_record<true, false>(m, s, tile, part, s_red);
    }
}

// ------------------------------------ the reference's functions one at a time

// calcOneStageMUSCLcpuFast alone (calcOneStageMUSCLcpuFast.jl:3-107): FLUXES
// and Unew from the current primitives, node primitives, Uold and Diff
// (diff may be NULL: zero), with the caller's beta, dt and flowTime.  One
// tile of blockDim cells per block, as the fused kernel.
template <int FLUX, bool QUAD>
__global__ void __launch_bounds__(256) k_stage_only(const DevMesh m, const DevState s, double beta, double dt,
                                                    double t, const double4 *__restrict__ diffs,
                                                    double4 *__restrict__ unew, double4 *__restrict__ fluxes) {
    const int par = *s.parity;
    const double4 *__restrict__ pin = s.prim + (int64_t)par * m.Nc;
    const int64_t tile = blockIdx.x;
    const int c = m.tile_case[tile];
    const DevCase &P = m.cases[c];
    const int64_t g = tile * blockDim.x + threadIdx.x;
    const int4 nb = m.nbr[g];
    if (nb.x == kAbsent) return;
    const bool is_quad = QUAD && (nb.w != kAbsent);
    const double4 me = pin[g];
    const double uL[4] = {me.x, me.y, me.z, me.w};
    const double gam = P.gamma;
    const double g2 = 2.0 * (gam - 1.0) / (gam + 1.0);
    const double hx_own = (P.limiter == LIM_VENKAT) ? m.hx[g] : 0.0;
    const int4 dn = m.dn[g], up = m.up[g];
    int4 dn2 = make_int4(0, 0, 0, 0), up2 = make_int4(0, 0, 0, 0);
    if (QUAD && is_quad) { dn2 = m.dn2[g]; up2 = m.up2[g]; }
    double F[4], f[4];
    face_flux<FLUX, QUAD>(m, P, pin, s.nodeP, g, 0, nb.x, dn.x, up.x, dn2.x, up2.x, is_quad, uL, hx_own, t, g2, F);
    face_flux<FLUX, QUAD>(m, P, pin, s.nodeP, g, 1, nb.y, dn.y, up.y, dn2.y, up2.y, is_quad, uL, hx_own, t, g2, f);
    for (int v = 0; v < 4; ++v) F[v] = F[v] + f[v];
    face_flux<FLUX, QUAD>(m, P, pin, s.nodeP, g, 2, nb.z, dn.z, up.z, dn2.z, up2.z, is_quad, uL, hx_own, t, g2, f);
    for (int v = 0; v < 4; ++v) F[v] = F[v] + f[v];
    if (QUAD && is_quad) {
        face_flux<FLUX, QUAD>(m, P, pin, s.nodeP, g, 3, nb.w, dn.w, up.w, dn2.w, up2.w, is_quad, uL, hx_own, t, g2, f);
        for (int v = 0; v < 4; ++v) F[v] = F[v] + f[v];
    }
    double diff[4] = {0.0, 0.0, 0.0, 0.0};
    if (diffs) {
        const double4 d = diffs[g];
        diff[0] = d.x; diff[1] = d.y; diff[2] = d.z; diff[3] = d.w;
    }
    const double rarea = m.rarea[g];
    const double4 U = s.U[g];
    const double Uo[4] = {U.x, U.y, U.z, U.w};
    double Un[4];
    for (int v = 0; v < 4; ++v) Un[v] = (Uo[v] - F[v] * beta * dt * rarea + beta * dt * diff[v]);
    unew[g] = make_double4(Un[0], Un[1], Un[2], Un[3]);
    fluxes[g] = make_double4(F[0], F[1], F[2], F[3]);
}

// updateVariablesSA alone (evaluate2d.jl:52-110): primitives of Unew in
// place, Delta = Unew - Uold, Uold <- Unew (density clamp as configured).
static __global__ void __launch_bounds__(256) k_update_only(const DevMesh m, const DevState s, double4 *__restrict__ unew,
                                                     double4 *__restrict__ delta) {
    const int par = *s.parity;
    double4 *__restrict__ prim = s.prim + (int64_t)par * m.Nc;
    const int64_t tile = blockIdx.x;
    const DevCase &P = m.cases[m.tile_case[tile]];
    const int64_t g = tile * blockDim.x + threadIdx.x;
    if (m.nbr[g].x == kAbsent) return;
    double4 un = unew[g];
    if (P.density_constrained == 1) {
        if (un.x >= P.rho_max) un.x = P.rho_max;
        if (un.x <= P.rho_min) un.x = P.rho_min;
        unew[g] = un;
    }
    const double G = P.gamma;
    const double rho = un.x, ux = un.y / un.x, uy = un.z / un.x;
    const double p = (G - 1.0) * (un.w - 0.5 * (un.y * un.y + un.z * un.z) / un.x);
    prim[g] = make_double4(rho, ux, uy, p);
    const double4 uo = s.U[g];
    delta[g] = make_double4(un.x - uo.x, un.y - uo.y, un.z - uo.z, un.w - uo.w);
    s.U[g] = un;
}

// calcDiffTerm alone (calcDiffTerm.jl:31-121): the diffusion source from
// the first-gradient node means (the grad1 passes must have run).
template <bool QUAD>
__global__ void __launch_bounds__(256) k_diff_only(const DevMesh m, const DevState s, double4 *__restrict__ diffs) {
    const int par = *s.parity;
    const double4 *__restrict__ pin = s.prim + (int64_t)par * m.Nc;
    const int64_t tile = blockIdx.x;
    const DevCase &P = m.cases[m.tile_case[tile]];
    const int64_t g = tile * blockDim.x + threadIdx.x;
    const int4 nb = m.nbr[g];
    if (nb.x == kAbsent) return;
    double diff[4];
    diff_source<QUAD>(m, s, P, g, QUAD && nb.w != kAbsent, pin[g], diff);
    diffs[g] = make_double4(diff[0], diff[1], diff[2], diff[3]);
}

}  // namespace gd2d
