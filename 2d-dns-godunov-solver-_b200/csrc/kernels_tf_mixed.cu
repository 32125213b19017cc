// Mixed-precision instantiations of the tile-face cell kernel.  Built with
// -use_fast_math like kernels_mixed.cu.
#include "mixed_face.cuh"

namespace gd2d {

namespace {

// Mixed-precision cell kernel over tile-local face lists: the FP64
// k_cell_step_tf's schedule (tile primitives staged in shared memory, a face
// shared by two cells of the tile evaluated once with its flux stored negated
// for the other cell, slots summed in face order) with this file's FP32 face
// arithmetic and FP64 update.
template <int FLUX, bool VISC, bool QUAD, int MINB>
__global__ void __launch_bounds__(256, MINB) k_cell_step_tf_mixed(const DevMesh m, const DevState s) {
    constexpr int NS = QUAD ? 4 : 3;
    // one buffer for the step reduction; the tile's primitives and flux
    // slots live in it until the reduction retires them
    // declared as double4 for its 32-byte alignment (float4 views need 16)
    __shared__ double4 s_buf[kPartFields * 256 / 4];
    __shared__ float s_hx[256];
    static_assert((1 + NS) * 256 * 16 <= kPartFields * 256 * 8, "tile buffers");
    double *const s_red = reinterpret_cast<double *>(s_buf);
    float4 *const s_prim = reinterpret_cast<float4 *>(s_buf);
    float4 (*const s_flux)[256] = reinterpret_cast<float4 (*)[256]>(s_prim + 256);
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
        // and HX (used only with the Venkatakrishnan limiter) need not wait
        // for the case record
        const int64_t f0 = m.tf_off[tile], f1 = m.tf_off[tile + 1];
        s_prim[threadIdx.x] = pin[g];
        s_hx[threadIdx.x] = ld_once(m.hxf + g);
        const int c = m.tile_case[tile];
        const DevCase &P = m.cases[c];
        const double t = s.cstate[c].t;
        const bool venkat = P.limiter == LIM_VENKAT;
        __syncthreads();
        const float gam = (float)P.gamma;
        const float g2 = 2.f * (gam - 1.f) / (gam + 1.f);
        for (int64_t f = f0 + threadIdx.x; f < f1; f += B) {
            const int4 rec = ld_once(m.tf_rec + f);
            const TileFace tf = unpack_tile_face(rec.y);
            const float4 a4 = s_prim[tf.la];
            const float uL[4] = {a4.x, a4.y, a4.z, a4.w};
            const float hx_own = venkat ? s_hx[tf.la] : 0.f;
            float4 r = a4, dd = a4, uu = a4;
            float hxR = hx_own;
            if (rec.x >= 0) {
                const int64_t lr = (int64_t)rec.x - base;
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
            face_flux_pre<FLUX>(m, P, base + tf.la, tf.ka, rec.x, r, dd, uu, ld_once(m.tf_nxf + f), ld_once(m.tf_nyf + f),
                                ld_once(m.tf_lenf + f),
                                uL, hx_own, hxR, t, g2, fv);
            s_flux[tf.ka][tf.la] = make_float4(fv[0], fv[1], fv[2], fv[3]);
            if (tf.lbp) s_flux[tf.kb][tf.lbp - 1] = make_float4(-fv[0], -fv[1], -fv[2], -fv[3]);
        }
        // the viscous source needs no flux: evaluated before the barrier
        // (the cell's primitives re-read from the stage, not held through
        // the face phase)
        const float4 me = s_prim[threadIdx.x];
        const double dt = s.cstate[c].dt;
        const int4 nb = ld_once(m.nbr + g);
        const bool is_quad = QUAD && (nb.w != kAbsent);
        float diff[4] = {0.f, 0.f, 0.f, 0.f};
        // triangles: evaluated for padding cells too (node 0 in their edge
        // slots; the result is unused), so its loads need not wait for nb
        if (VISC && (!QUAD || nb.x != kAbsent)) diff_source_f<QUAD>(m, s, P, g, is_quad, me, diff);
        // the update's own loads go out before the barrier (padded arrays:
        // in bounds for padding cells, whose values are not used)
        const CellInF cin = load_cell_in_f(m, s, g);
        __syncthreads();
        Part part;
        part.init();
        if (nb.x != kAbsent) {
            const float4 a0 = s_flux[0][threadIdx.x], a1 = s_flux[1][threadIdx.x], a2 = s_flux[2][threadIdx.x];
            float F[4] = {a0.x + a1.x + a2.x, a0.y + a1.y + a2.y, a0.z + a1.z + a2.z, a0.w + a1.w + a2.w};
            if (QUAD && is_quad) {
                const float4 a3 = s_flux[NS - 1][threadIdx.x];
                F[0] += a3.x; F[1] += a3.y; F[2] += a3.z; F[3] += a3.w;
            }
            cell_update_mixed(m, s, P, g, me, F, diff, dt, cin, pout, part);
        }
        tile_epilogue(m, s, tile, c, part, s_red, false);
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
