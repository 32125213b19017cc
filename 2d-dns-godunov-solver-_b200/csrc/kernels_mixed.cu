// Mixed-precision step kernels: FP32 gathers, reconstruction, face fluxes
// and viscous terms (FP32 geometry and primitives), FP64 conservative state,
// Euler-update accumulation, primitive recovery and all reductions.
//
// Same dataflow as the FP64 kernels (step_kernels.cuh), with the primitives
// packed as float4 so each neighbour or node gather is one 128-bit load.
// Built with fast FP32 division and square root; the error of this path is
// reported against the FP64 oracle rather than asserted bit-exact.
#include "mixed_face.cuh"

// Register budget of the mixed node-side passes, as resident 256-thread
// blocks per SM.
#ifndef GD2D_NODE_MINB_MIXED
#define GD2D_NODE_MINB_MIXED 6
#endif

namespace gd2d {

namespace {

template <int FLUX, bool VISC, bool QUAD, int MINB>
__global__ void __launch_bounds__(256, MINB) k_cell_step_mixed(const DevMesh m, const DevState s) {
    __shared__ double s_red[kPartFields * 256];
    const int par = *s.parity;
    const float4 *__restrict__ pin = s.primf + (int64_t)par * m.Nc;
    float4 *__restrict__ pout = s.primf + (int64_t)(par ^ 1) * m.Nc;
    const float4 *__restrict__ nodeP = s.nodePf;
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
            const float4 me = pin[g];
            const float uL[4] = {me.x, me.y, me.z, me.w};
            const float gam = (float)P.gamma;
            const float g2 = 2.f * (gam - 1.f) / (gam + 1.f);
            const float hx_own = (P.limiter == LIM_VENKAT) ? m.hxf[g] : 0.f;
            const int4 dn = m.dn[g], up = m.up[g];
            int4 dn2 = make_int4(0, 0, 0, 0), up2 = make_int4(0, 0, 0, 0);
            if (QUAD && is_quad) { dn2 = m.dn2[g]; up2 = m.up2[g]; }
            // every gather of faces 0-2 issued before any arithmetic (boundary
            // faces load the cell itself and node 0, which they then ignore)
            const int64_t Nc = m.Nc;
            const float4 R0 = pin[nb.x >= 0 ? nb.x : g], R1 = pin[nb.y >= 0 ? nb.y : g], R2 = pin[nb.z >= 0 ? nb.z : g];
            float4 D0 = nodeP[dn.x], D1 = nodeP[dn.y], D2 = nodeP[dn.z];
            float4 W0 = nodeP[up.x], W1 = nodeP[up.y], W2 = nodeP[up.z];
            const float nx0 = m.nxf[g], nx1 = m.nxf[Nc + g], nx2 = m.nxf[2 * Nc + g];
            const float ny0 = m.nyf[g], ny1 = m.nyf[Nc + g], ny2 = m.nyf[2 * Nc + g];
            const float l0 = m.lenf[g], l1 = m.lenf[Nc + g], l2 = m.lenf[2 * Nc + g];
            float h0 = hx_own, h1 = hx_own, h2 = hx_own;
            if (P.limiter == LIM_VENKAT) {
                if (nb.x >= 0) h0 = m.hxf[nb.x];
                if (nb.y >= 0) h1 = m.hxf[nb.y];
                if (nb.z >= 0) h2 = m.hxf[nb.z];
            }
            if (QUAD && is_quad) {
                D0 = avg4(D0, nodeP[dn2.x]); D1 = avg4(D1, nodeP[dn2.y]); D2 = avg4(D2, nodeP[dn2.z]);
                W0 = avg4(W0, nodeP[up2.x]); W1 = avg4(W1, nodeP[up2.y]); W2 = avg4(W2, nodeP[up2.z]);
            }
            float F[4], f[4];
            const FaceConstsF kc = face_consts_f(P);
            face_flux_pre<FLUX>(m, P, kc, g, 0, nb.x, R0, D0, W0, nx0, ny0, l0, uL, hx_own, h0, t, F);
            face_flux_pre<FLUX>(m, P, kc, g, 1, nb.y, R1, D1, W1, nx1, ny1, l1, uL, hx_own, h1, t, f);
#pragma unroll
            for (int v = 0; v < 4; ++v) F[v] += f[v];
            face_flux_pre<FLUX>(m, P, kc, g, 2, nb.z, R2, D2, W2, nx2, ny2, l2, uL, hx_own, h2, t, f);
#pragma unroll
            for (int v = 0; v < 4; ++v) F[v] += f[v];
            if (QUAD && is_quad) {
                face_flux_f<FLUX, QUAD>(m, P, pin, nodeP, g, 3, nb.w, dn.w, up.w, dn2.w, up2.w, is_quad, uL, hx_own, t, g2, f);
#pragma unroll
                for (int v = 0; v < 4; ++v) F[v] += f[v];
            }
            float diff[4] = {0.f, 0.f, 0.f, 0.f};
            if (VISC) diff_source_f<QUAD>(m, s, P, g, is_quad, me, diff);
            cell_update_mixed(m, s, P, g, me, F, diff, dt, load_cell_in_f(m, s, g), pout, part);
        }
        tile_record<false, false>(m, s, tile, part, s_red);
    }
}

// Node-side kernels: gather-latency bound, registers capped for 6
// resident blocks per SM.
template <bool VISC, bool UNIT>
__global__ void __launch_bounds__(256, GD2D_NODE_MINB_MIXED) k_node_avg_mixed(const DevMesh m, const DevState s, int flip, int zero_prims,
                                                        int64_t n0, int64_t n1, int64_t g0, int nred, int is_init) {
    pdl_trigger();
    pdl_wait();
    if ((int)blockIdx.x < nred) {
        fold_block<false>(m, s, g0, is_init != 0);
        return;
    }
    const int64_t bid = (int64_t)blockIdx.x - nred, nblk = (int64_t)gridDim.x - nred;
    const int par = *s.parity;
    const float4 *__restrict__ src = s.primf + (int64_t)(flip ? (par ^ 1) : par) * m.Nc;
    const int W = m.cluster_w;
    for (int64_t J = n0 + bid * blockDim.x + threadIdx.x; J < n1; J += nblk * blockDim.x) {
        bool prim_form = false;
        float gop = 0.f, gam = 0.f;
        if (VISC) {
            const DevCase &P = m.cases[ld_once(m.node_case + J)];
            prim_form = P.visc_model != VISC_REFERENCE;
            gop = (float)P.gamma_over_Pr;
            gam = (float)P.gamma;
        }
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, det = 0.f;
        float c0 = 0.f, c1 = 0.f, c2 = 0.f;
        int cnt = 0;
        auto add = [&](int c, const float4 &p, float w) {
            a0 += p.x * w; a1 += p.y * w; a2 += p.z * w; a3 += p.w * w;
            det += w;
            if (VISC) {
                if (prim_form) {
                    c0 += p.y; c1 += p.z; c2 += 0.5f * (p.y * p.y + p.z * p.z) + gop * (p.w / ((gam - 1.f) * p.x));
                } else {
                    const double4 u = s.U[c];
                    c0 += (float)u.y; c1 += (float)u.z; c2 += (float)u.w;
                }
                ++cnt;
            }
        };
        int ci[kMaxCluster];
#pragma unroll
        for (int j = 0; j < kMaxCluster; ++j) ci[j] = (j < W) ? ld_once(m.cl + (int64_t)j * m.Nn + J) : -1;
#pragma unroll
        for (int j = 0; j < kMaxCluster; ++j)
            if (ci[j] >= 0) add(ci[j], src[ci[j]], UNIT ? 1.f : (float)ld_once(m.wt + (int64_t)j * m.Nn + J));
        for (int j = kMaxCluster; j < W; ++j) {
            const int c = ld_once(m.cl + (int64_t)j * m.Nn + J);
            if (c >= 0) add(c, src[c], UNIT ? 1.f : (float)ld_once(m.wt + (int64_t)j * m.Nn + J));
        }
        if (det != 0.f) { const float r = 1.f / det; a0 *= r; a1 *= r; a2 *= r; a3 *= r; }
        s.nodePf[J] = zero_prims ? make_float4(0.f, 0.f, 0.f, 0.f) : make_float4(a0, a1, a2, a3);
        if (VISC) {
            const float r = cnt ? 1.f / (float)cnt : 0.f;
            s.nodeCf[J] = make_float4(c0 * r, c1 * r, c2 * r, 0.f);
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

template <bool QUAD>
__global__ void __launch_bounds__(256, GD2D_NODE_MINB_MIXED) k_grad1_cells_mixed(const DevMesh m, const DevState s) {
    constexpr int NF = QUAD ? 4 : 3;
    pdl_trigger();
    pdl_wait();
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < m.Nc; g += (int64_t)gridDim.x * blockDim.x) {
        // all per-cell loads first (two trips to memory per cell); padding
        // cells have zero inverse area and are dropped at the store,
        // triangles have a zero-length fourth edge; each edge's weights
        // are n * len, rounded once
        const float rA = ld_once(m.rareaf + g);
        float nlx[NF], nly[NF];
        int2 e[NF];
#pragma unroll
        for (int k = 0; k < NF; ++k) {
            const int64_t o = (int64_t)k * m.Nc + g;
            nlx[k] = ld_once(m.nlxf + o);
            nly[k] = ld_once(m.nlyf + o);
            e[k] = ld_once(m.c2n + o);
        }
        const int nf = (QUAD && ld_once(m.lenf + (int64_t)(NF - 1) * m.Nc + g) != 0.f) ? 4 : 3;
        float sx[3] = {0.f, 0.f, 0.f}, sy[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < NF; ++k) {
            if (k >= nf) break;
            const float4 A = s.nodeCf[e[k].x], B = s.nodeCf[e[k].y];
            sx[0] += 0.5f * (A.x + B.x) * -nly[k]; sy[0] += 0.5f * (A.x + B.x) * -nlx[k];
            sx[1] += 0.5f * (A.y + B.y) * -nly[k]; sy[1] += 0.5f * (A.y + B.y) * -nlx[k];
            sx[2] += 0.5f * (A.z + B.z) * -nly[k]; sy[2] += 0.5f * (A.z + B.z) * -nlx[k];
        }
        if (rA == 0.f) continue;
        NodeGradF r;
        r.ru = make_float2(sx[0] * rA, sy[0] * rA);
        r.rv = make_float2(sx[1] * rA, sy[1] * rA);
        r.re = make_float2(sx[2] * rA, sy[2] * rA);
        s.g1f[g] = r;
    }
}

__global__ void __launch_bounds__(256, GD2D_NODE_MINB_MIXED) k_grad1_nodes_mixed(const DevMesh m, const DevState s) {
    const int W = m.cluster_w;
    pdl_trigger();
    pdl_wait();
    for (int64_t J = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; J < m.Nn; J += (int64_t)gridDim.x * blockDim.x) {
        float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int cnt = 0;
        auto add = [&](const NodeGradF &q) {
            v[0] += q.ru.x; v[1] += q.ru.y; v[2] += q.rv.x; v[3] += q.rv.y; v[4] += q.re.x; v[5] += q.re.y;
            ++cnt;
        };
        int ci[kMaxCluster];
#pragma unroll
        for (int j = 0; j < kMaxCluster; ++j) ci[j] = (j < W) ? ld_once(m.cl + (int64_t)j * m.Nn + J) : -1;
#pragma unroll
        for (int j = 0; j < kMaxCluster; ++j)
            if (ci[j] >= 0) add(s.g1f[ci[j]]);
        for (int j = kMaxCluster; j < W; ++j) {
            const int c = ld_once(m.cl + (int64_t)j * m.Nn + J);
            if (c >= 0) add(s.g1f[c]);
        }
        const float r = cnt ? 1.f / (float)cnt : 0.f;
        NodeGradF o;
        o.ru = make_float2(v[0] * r, v[1] * r);
        o.rv = make_float2(v[2] * r, v[3] * r);
        o.re = make_float2(v[4] * r, v[5] * r);
        s.nodeGf[J] = o;
    }
}

// U holds FP64 primitives on entry: conservatives (utilsFVM2dp.jl:4-17) and
// the FP32 primitives are written, with the first dt's reductions.
__global__ void __launch_bounds__(256) k_init_state_mixed(const DevMesh m, const DevState s, int64_t t0, int64_t t1) {
    __shared__ double s_red[kPartFields * 256];
    const int par = *s.parity;
    float4 *__restrict__ pout = s.primf + (int64_t)par * m.Nc;
    for (int64_t tile = t0 + blockIdx.x; tile < t1; tile += gridDim.x) {
        const int c = m.tile_case[tile];
        const DevCase &P = m.cases[c];
        const int64_t g = tile * blockDim.x + threadIdx.x;
        Part part;
        part.init();
        const int4 nb = m.nbr[g];
        if (nb.x != kAbsent) {
            const double4 q = s.U[g];
            const double G = P.gamma;
            const double r = q.x, u = q.y, v = q.z, pp = q.w;
            s.U[g] = make_double4(r, r * u, r * v, pp / (G - 1.0) + 0.5 * r * (u * u + v * v));
            pout[g] = make_float4((float)r, (float)u, (float)v, (float)pp);
            const double a = sqrt(G * pp / r);
            const double vmax = sqrt(u * u + v * v) + a;
            part.vmax = vmax;
            part.rmin = (double)m.charlenf[g] / vmax;
        }
        tile_record<false, false>(m, s, tile, part, s_red);
    }
}

int grid_for_m(int64_t work, int block) {
    int64_t g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148LL * 64) g = 148 * 64;
    return (int)g;
}

template <int FLUX, bool VISC, bool QUAD>
cudaError_t cell_step_m(const DevMesh &m, const DevState &s, const LaunchCfg &lc, cudaStream_t st) {
    int grid = lc.persistent ? lc.grid : (int)m.ntiles;
    if (lc.min_blocks >= 4) k_cell_step_mixed<FLUX, VISC, QUAD, 4><<<grid, lc.block, 0, st>>>(m, s);
    else if (lc.min_blocks == 3) k_cell_step_mixed<FLUX, VISC, QUAD, 3><<<grid, lc.block, 0, st>>>(m, s);
    else k_cell_step_mixed<FLUX, VISC, QUAD, 2><<<grid, lc.block, 0, st>>>(m, s);
    return cudaGetLastError();
}

template <int FLUX>
cudaError_t cell_step_flux_m(const DevMesh &m, const DevState &s, bool visc, bool quads, const LaunchCfg &lc,
                             cudaStream_t st) {
    if (visc) return quads ? cell_step_m<FLUX, true, true>(m, s, lc, st) : cell_step_m<FLUX, true, false>(m, s, lc, st);
    return quads ? cell_step_m<FLUX, false, true>(m, s, lc, st) : cell_step_m<FLUX, false, false>(m, s, lc, st);
}

}  // namespace

cudaError_t launch_cell_step_mixed(const DevMesh &m, const DevState &s, int flux, bool visc, bool quads,
                                   const LaunchCfg &lc, cudaStream_t st) {
    switch (flux) {
    case FLUX_ROE: return cell_step_flux_m<FLUX_ROE>(m, s, visc, quads, lc, st);
    case FLUX_AUSM_M2020: return cell_step_flux_m<FLUX_AUSM_M2020>(m, s, visc, quads, lc, st);
    default: return cell_step_flux_m<FLUX_AUSM>(m, s, visc, quads, lc, st);
    }
}

cudaError_t launch_node_avg_mixed(const DevMesh &m, const DevState &s, bool visc, bool flip_parity, bool zero_prims,
                                  int64_t n0, int64_t n1, int64_t g0, int64_t g1, bool red_init, const LaunchCfg &lc,
                                  cudaStream_t st) {
    const int b = lc.node_block;
    const int nred = (int)(g1 > g0 ? g1 - g0 : 0) * fold_blocks_per_group(b);
    const int grid = grid_for_m(n1 - n0, b) + nred;
    const bool unit = m.unit_weights != 0;
    const int fl = (int)flip_parity, zp = (int)zero_prims, ri = (int)red_init;
    if (visc) {
        if (unit) return launch_dependent(k_node_avg_mixed<true, true>, grid, b, st, m, s, fl, zp, n0, n1, g0, nred, ri);
        return launch_dependent(k_node_avg_mixed<true, false>, grid, b, st, m, s, fl, zp, n0, n1, g0, nred, ri);
    }
    if (unit) return launch_dependent(k_node_avg_mixed<false, true>, grid, b, st, m, s, fl, zp, n0, n1, g0, nred, ri);
    return launch_dependent(k_node_avg_mixed<false, false>, grid, b, st, m, s, fl, zp, n0, n1, g0, nred, ri);
}

cudaError_t launch_visc_grad_mixed(const DevMesh &m, const DevState &s, const LaunchCfg &lc, cudaStream_t st) {
    const int b = lc.node_block;
    cudaError_t e = (m.nfmax == 4) ? launch_dependent(k_grad1_cells_mixed<true>, grid_for_m(m.Nc, b), b, st, m, s)
                                   : launch_dependent(k_grad1_cells_mixed<false>, grid_for_m(m.Nc, b), b, st, m, s);
    if (e != cudaSuccess) return e;
    return launch_dependent(k_grad1_nodes_mixed, grid_for_m(m.Nn, b), b, st, m, s);
}

cudaError_t launch_init_state_mixed(const DevMesh &m, const DevState &s, int64_t t0, int64_t t1, const LaunchCfg &lc,
                                    cudaStream_t st) {
    k_init_state_mixed<<<(int)(t1 - t0), lc.block, 0, st>>>(m, s, t0, t1);
    return cudaGetLastError();
}

}  // namespace gd2d
