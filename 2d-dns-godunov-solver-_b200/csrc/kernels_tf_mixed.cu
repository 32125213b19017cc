// Mixed-precision instantiations of the tile-face cell kernel.  Built with
// -use_fast_math like kernels_mixed.cu.
#include "mixed_face.cuh"

namespace gd2d {

namespace {

// Mixed-precision cell kernel over tile-local face lists: the FP64
// k_cell_step_tf's schedule (tile primitives staged in shared memory, a face
// shared by two cells of the tile evaluated once with its flux stored negated
// for the other cell, slots summed in face order) with this file's FP32 face
// arithmetic and FP64 update.  With VISC a first pass over the face list
// evaluates each listed edge's share of the diffusion source's Green-Gauss
// sums (the Laplacian terms of the three variables and the velocity
// divergence of the artificial viscosity, visc_face_f) into a second set of
// slots, negated for the other cell of a shared edge like the flux; the cell
// phase sums them and applies the transport model.  So an edge shared by two
// cells of the tile is gathered and evaluated once, and the per-cell face
// geometry and edge-node arrays are not read at all.  The viscous pass is
// separate from the flux pass (which re-reads the face records from L1):
// one fused pass held both passes' gathers in registers at once and spilled
// (2.09M-cell cylinder: 0.214 ms fused, 0.209 ms in two passes).
template <int FLUX, bool VISC, bool QUAD, int MINB>
__global__ void __launch_bounds__(256, MINB) k_cell_step_tf_mixed(const DevMesh m, const DevState s) {
    constexpr int NS = QUAD ? 4 : 3;
    // one buffer: the tile's primitives, flux slots and (VISC) viscous
    // slots, which the step reduction reuses once they have been consumed;
    // declared as double4 for its 32-byte alignment (float4 views need 16)
    constexpr int kTileBytes = (1 + NS * (VISC ? 2 : 1)) * 256 * 16;
    constexpr int kRedBytes = kPartFields * 256 * 8;
    constexpr int kBufBytes = kTileBytes > kRedBytes ? kTileBytes : kRedBytes;
    __shared__ double4 s_buf[kBufBytes / 32];
    __shared__ float s_hx[256];
    float4 *const s_prim = reinterpret_cast<float4 *>(s_buf);
    float4 (*const s_flux)[256] = reinterpret_cast<float4 (*)[256]>(s_prim + 256);
    float4 (*const s_visc)[256] = reinterpret_cast<float4 (*)[256]>(s_prim + 256 * (1 + NS));
    pdl_trigger();
    pdl_wait();
    const int par = *s.parity;
    const float4 *__restrict__ pin = s.primf + (int64_t)par * m.Nc;
    float4 *__restrict__ pout = s.primf + (int64_t)(par ^ 1) * m.Nc;
    const float4 *__restrict__ nodeP = s.nodePf;
    const int B = blockDim.x;
    for (int64_t tile = blockIdx.x; tile < m.ntiles; tile += gridDim.x) {
        const int64_t base = tile * B;
        const int64_t g = base + threadIdx.x;
        // loads that depend on nothing go out first: the face-list bounds
        // and HX (Venkatakrishnan limiter, artificial viscosity) need not
        // wait for the case record
        const int64_t f0 = m.tf_off[tile], f1 = m.tf_off[tile + 1];
        s_prim[threadIdx.x] = pin[g];
        s_hx[threadIdx.x] = ld_once(m.hxf + g);
        const int c = m.tile_case[tile];
        const DevCase &P = m.cases[c];
        const double t = s.cstate[c].t;
        const FaceConstsF kc = face_consts_f(P);
        const bool venkat = kc.lim == LIM_VENKAT;
        const bool art = VISC && P.visc_model != VISC_REFERENCE && P.art_visc;
        // face indices fit 32 bits (setup checks the total)
        const int fb = (int)f0 + (int)threadIdx.x, fe = (int)f1;
        // the viscous pass's first face record goes out with the staging
        // loads and each next one before the current face's gathers, so a
        // thread with two faces does not wait for its second record (the
        // cached loads leave the records in L1 for the flux pass)
        int pk = 0; int2 pe = make_int2(0, 0); float pnx = 0.f, pny = 0.f, pln = 0.f;
        if (VISC && fb < fe) {
            pk = m.tf_rec[fb].y; pe = ld_once(m.tf_e + fb);
            pnx = m.tf_nxf[fb]; pny = m.tf_nyf[fb]; pln = m.tf_lenf[fb];
        }
        __syncthreads();
        if (VISC) {
            for (int f = fb; f < fe; f += B) {
                const TileFace tf = unpack_tile_face(pk);
                const float nxf = pnx, nyf = pny, lenf = pln;
                const int2 e = pe;
                if (f + B < fe) {
                    pk = m.tf_rec[f + B].y; pe = ld_once(m.tf_e + f + B);
                    pnx = m.tf_nxf[f + B]; pny = m.tf_nyf[f + B]; pln = m.tf_lenf[f + B];
                }
                const NodeGradF GA = s.nodeGf[e.x], GB = s.nodeGf[e.y];
                float4 na = make_float4(0.f, 0.f, 0.f, 0.f), nb = na;
                if (art) { na = nodeP[e.x]; nb = nodeP[e.y]; }
                const float4 vv = visc_face_f(GA, GB, na, nb, nxf, nyf, lenf, art);
                s_visc[tf.ka][tf.la] = vv;
                if (tf.lbp) s_visc[tf.kb][tf.lbp - 1] = make_float4(-vv.x, -vv.y, -vv.z, -vv.w);
            }
        }
        for (int f = fb; f < fe; f += B) {
            const int4 rec = ld_once(m.tf_rec + f);
            const TileFace tf = unpack_tile_face(rec.y);
            const float4 a4 = s_prim[tf.la];
            const float uL[4] = {a4.x, a4.y, a4.z, a4.w};
            const float hx_own = venkat ? s_hx[tf.la] : 0.f;
            const float nxf = ld_once(m.tf_nxf + f), nyf = ld_once(m.tf_nyf + f), lenf = ld_once(m.tf_lenf + f);
            float4 r = a4, dd = a4, uu = a4;
            float hxR = hx_own;
            if (rec.x >= 0) {
                const int lr = rec.x - (int)base;
                if (lr >= 0 && lr < B) {
                    r = s_prim[lr];
                    if (venkat) hxR = s_hx[lr];
                } else {
                    r = pin[rec.x];
                    if (venkat) hxR = m.hxf[rec.x];
                }
                dd = nodeP[rec.z];
                uu = nodeP[rec.w];
                if (QUAD && tf.quad) {
                    const int2 q2 = m.tf_q[f];
                    dd = avg4(dd, nodeP[q2.x]);
                    uu = avg4(uu, nodeP[q2.y]);
                }
            }
            float fv[4];
            face_flux_pre<FLUX>(m, P, kc, base + tf.la, tf.ka, rec.x, r, dd, uu, nxf, nyf, lenf, uL, hx_own, hxR, t,
                                fv);
            s_flux[tf.ka][tf.la] = make_float4(fv[0], fv[1], fv[2], fv[3]);
            if (tf.lbp) s_flux[tf.kb][tf.lbp - 1] = make_float4(-fv[0], -fv[1], -fv[2], -fv[3]);
        }
        const double dt = s.cstate[c].dt;
        // the update's own loads go out before the barrier (padded arrays:
        // in bounds for padding cells, whose values are not used)
        const CellInF cin = load_cell_in_f(m, s, g);
        // a padding cell has zero inverse area (quads: the neighbour record
        // also tells triangles from quads)
        bool live = cin.rarea != 0.f, is_quad = false;
        if (QUAD) {
            const int4 nbq = ld_once(m.nbr + g);
            live = nbq.x != kAbsent;
            is_quad = nbq.w != kAbsent;
        }
        __syncthreads();
        Part part;
        part.init();
        if (live) {
            const float4 me = s_prim[threadIdx.x];
            const float4 a0 = s_flux[0][threadIdx.x], a1 = s_flux[1][threadIdx.x], a2 = s_flux[2][threadIdx.x];
            float F[4] = {a0.x + a1.x + a2.x, a0.y + a1.y + a2.y, a0.z + a1.z + a2.z, a0.w + a1.w + a2.w};
            if (QUAD && is_quad) {
                const float4 a3 = s_flux[NS - 1][threadIdx.x];
                F[0] += a3.x; F[1] += a3.y; F[2] += a3.z; F[3] += a3.w;
            }
            float diff[4] = {0.f, 0.f, 0.f, 0.f};
            if (VISC) {
                const float4 v0 = s_visc[0][threadIdx.x], v1 = s_visc[1][threadIdx.x], v2 = s_visc[2][threadIdx.x];
                float V[4] = {v0.x + v1.x + v2.x, v0.y + v1.y + v2.y, v0.z + v1.z + v2.z, v0.w + v1.w + v2.w};
                if (QUAD && is_quad) {
                    const float4 v3 = s_visc[NS - 1][threadIdx.x];
                    V[0] += v3.x; V[1] += v3.y; V[2] += v3.z; V[3] += v3.w;
                }
                const float rA = cin.rarea;
                const float lap[3] = {V[0] * rA, V[1] * rA, V[2] * rA};
                visc_source_f(P, me, lap, V[3] * rA, s_hx[threadIdx.x], diff);
            }
            cell_update_mixed(m, s, P, g, me, F, diff, dt, cin, pout, part);
        }
        tile_record<false, true>(m, s, tile, part, reinterpret_cast<double *>(s_buf));
    }
}

template <int FLUX, bool VISC, bool QUAD>
cudaError_t cell_step_tf_m(const DevMesh &m, const DevState &s, const LaunchCfg &lc, cudaStream_t st) {
    const int grid = lc.persistent ? lc.grid : (int)m.ntiles;
    if (lc.min_blocks >= 4) return launch_dependent(k_cell_step_tf_mixed<FLUX, VISC, QUAD, 4>, grid, lc.block, st, m, s);
    if (lc.min_blocks == 3) return launch_dependent(k_cell_step_tf_mixed<FLUX, VISC, QUAD, 3>, grid, lc.block, st, m, s);
    return launch_dependent(k_cell_step_tf_mixed<FLUX, VISC, QUAD, 2>, grid, lc.block, st, m, s);
}

template <int FLUX>
cudaError_t cell_step_tf_flux_m(const DevMesh &m, const DevState &s, bool visc, bool quads, const LaunchCfg &lc,
                                cudaStream_t st) {
    if (visc) return quads ? cell_step_tf_m<FLUX, true, true>(m, s, lc, st) : cell_step_tf_m<FLUX, true, false>(m, s, lc, st);
    return quads ? cell_step_tf_m<FLUX, false, true>(m, s, lc, st) : cell_step_tf_m<FLUX, false, false>(m, s, lc, st);
}

}  // namespace

cudaError_t launch_cell_step_tf_mixed(const DevMesh &m, const DevState &s, int flux, bool visc, bool quads,
                                      const LaunchCfg &lc, cudaStream_t st) {
    switch (flux) {
    case FLUX_ROE: return cell_step_tf_flux_m<FLUX_ROE>(m, s, visc, quads, lc, st);
    case FLUX_AUSM_M2020: return cell_step_tf_flux_m<FLUX_AUSM_M2020>(m, s, visc, quads, lc, st);
    default: return cell_step_tf_flux_m<FLUX_AUSM>(m, s, visc, quads, lc, st);
    }
}

}  // namespace gd2d
