// FP64 instantiations of the step kernels.  This translation unit is built
// with -fmad=false: like the reference's Julia Float64 code, no multiply-add
// is contracted except the explicit fma() standing for the reference's
// muladd, so results round exactly like the CPU restatement.
#include "step_kernels.cuh"

namespace gd2d {

namespace {

int grid_for(int64_t work, int block) {
    int64_t g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148LL * 64) g = 148 * 64;
    return (int)g;
}

template <int FLUX, bool VISC, bool QUAD>
cudaError_t cell_step(const DevMesh &m, const DevState &s, const LaunchCfg &lc, cudaStream_t st) {
    int grid = lc.persistent ? lc.grid : (int)m.ntiles;
    // register budget chosen by the launch configuration (blocks per SM)
    if (lc.min_blocks >= 4) k_cell_step<FLUX, VISC, QUAD, 4><<<grid, lc.block, 0, st>>>(m, s);
    else if (lc.min_blocks == 3) k_cell_step<FLUX, VISC, QUAD, 3><<<grid, lc.block, 0, st>>>(m, s);
    else k_cell_step<FLUX, VISC, QUAD, 2><<<grid, lc.block, 0, st>>>(m, s);
    return cudaGetLastError();
}

template <int FLUX>
cudaError_t cell_step_flux(const DevMesh &m, const DevState &s, bool visc, bool quads, const LaunchCfg &lc,
                           cudaStream_t st) {
    if (visc) return quads ? cell_step<FLUX, true, true>(m, s, lc, st) : cell_step<FLUX, true, false>(m, s, lc, st);
    return quads ? cell_step<FLUX, false, true>(m, s, lc, st) : cell_step<FLUX, false, false>(m, s, lc, st);
}

}  // namespace

cudaError_t launch_cell_step_f64(const DevMesh &m, const DevState &s, int flux, bool visc, bool quads,
                                 const LaunchCfg &lc, cudaStream_t st) {
    switch (flux) {
    case FLUX_ROE: return cell_step_flux<FLUX_ROE>(m, s, visc, quads, lc, st);
    case FLUX_AUSM_M2020: return cell_step_flux<FLUX_AUSM_M2020>(m, s, visc, quads, lc, st);
    default: return cell_step_flux<FLUX_AUSM>(m, s, visc, quads, lc, st);
    }
}

cudaError_t launch_node_avg_f64(const DevMesh &m, const DevState &s, bool visc, bool flip_parity, bool zero_prims,
                                int64_t n0, int64_t n1, int64_t g0, int64_t g1, bool red_init, const LaunchCfg &lc,
                                cudaStream_t st) {
    const int b = lc.node_block;
    const int nred = (int)(g1 > g0 ? g1 - g0 : 0) * fold_blocks_per_group(b);
    const int grid = grid_for(n1 - n0, b) + nred;
    const bool unit = m.unit_weights != 0;
    const int fl = (int)flip_parity, zp = (int)zero_prims, ri = (int)red_init;
    if (visc) {
        if (unit) return launch_dependent(k_node_avg<true, true>, grid, b, st, m, s, fl, zp, n0, n1, g0, nred, ri);
        return launch_dependent(k_node_avg<true, false>, grid, b, st, m, s, fl, zp, n0, n1, g0, nred, ri);
    }
    if (unit) return launch_dependent(k_node_avg<false, true>, grid, b, st, m, s, fl, zp, n0, n1, g0, nred, ri);
    return launch_dependent(k_node_avg<false, false>, grid, b, st, m, s, fl, zp, n0, n1, g0, nred, ri);
}

cudaError_t launch_visc_grad_f64(const DevMesh &m, const DevState &s, const LaunchCfg &lc, cudaStream_t st) {
    const int b = lc.node_block;
    cudaError_t e = (m.nfmax == 4) ? launch_dependent(k_grad1_cells<true>, grid_for(m.Nc, b), b, st, m, s)
                                   : launch_dependent(k_grad1_cells<false>, grid_for(m.Nc, b), b, st, m, s);
    if (e != cudaSuccess) return e;
    return launch_dependent(k_grad1_nodes, grid_for(m.Nn, b), b, st, m, s);
}

cudaError_t launch_init_state_f64(const DevMesh &m, const DevState &s, int64_t t0, int64_t t1, const LaunchCfg &lc,
                                  cudaStream_t st) {
    k_init_state<<<(int)(t1 - t0), lc.block, 0, st>>>(m, s, t0, t1);
    return cudaGetLastError();
}

cudaError_t launch_face_flux_f64(const DevMesh &m, const DevState &s, int flux, bool quads, bool slots,
                                 const int4 *faces, int64_t f0, int64_t f1, double4 *Facc, double4 *Fslot,
                                 const LaunchCfg &lc, cudaStream_t st) {
    if (f1 <= f0) return cudaSuccess;
    const int b = 256;
    const int grid = (int)((f1 - f0 + b - 1) / b);
    const int tc = lc.block;
#define GD2D_FACE(F)                                                                                          \
    do {                                                                                                      \
        if (quads) {                                                                                          \
            if (slots) k_face_flux<F, true, true><<<grid, b, 0, st>>>(m, s, faces, f0, f1, tc, Facc, Fslot);   \
            else k_face_flux<F, true, false><<<grid, b, 0, st>>>(m, s, faces, f0, f1, tc, Facc, Fslot);        \
        } else {                                                                                              \
            if (slots) k_face_flux<F, false, true><<<grid, b, 0, st>>>(m, s, faces, f0, f1, tc, Facc, Fslot);  \
            else k_face_flux<F, false, false><<<grid, b, 0, st>>>(m, s, faces, f0, f1, tc, Facc, Fslot);       \
        }                                                                                                     \
    } while (0)
    if (flux == FLUX_ROE) GD2D_FACE(FLUX_ROE);
    else if (flux == FLUX_AUSM_M2020) GD2D_FACE(FLUX_AUSM_M2020);
    else GD2D_FACE(FLUX_AUSM);
#undef GD2D_FACE
    return cudaGetLastError();
}

cudaError_t launch_face_update_f64(const DevMesh &m, const DevState &s, bool visc, bool quads, bool slots,
                                   double4 *Facc, const double4 *Fslot, const LaunchCfg &lc, cudaStream_t st) {
    const int grid = lc.persistent ? lc.grid : (int)m.ntiles;
#define GD2D_UPD(V, Q, S) k_face_update<V, Q, S, 3><<<grid, lc.block, 0, st>>>(m, s, Facc, Fslot)
    if (visc) {
        if (quads) { if (slots) GD2D_UPD(true, true, true); else GD2D_UPD(true, true, false); }
        else { if (slots) GD2D_UPD(true, false, true); else GD2D_UPD(true, false, false); }
    } else {
        if (quads) { if (slots) GD2D_UPD(false, true, true); else GD2D_UPD(false, true, false); }
        else { if (slots) GD2D_UPD(false, false, true); else GD2D_UPD(false, false, false); }
    }
#undef GD2D_UPD
    return cudaGetLastError();
}

cudaError_t launch_stage_only_f64(const DevMesh &m, const DevState &s, int flux, bool quads, double beta, double dt,
                                  double t, const double4 *diffs, double4 *unew, double4 *fluxes, const LaunchCfg &lc,
                                  cudaStream_t st) {
    const int grid = (int)m.ntiles, b = lc.block;
#define GD2D_STAGE(F)                                                                                    \
    (quads ? (k_stage_only<F, true><<<grid, b, 0, st>>>(m, s, beta, dt, t, diffs, unew, fluxes), 0)      \
           : (k_stage_only<F, false><<<grid, b, 0, st>>>(m, s, beta, dt, t, diffs, unew, fluxes), 0))
    if (flux == FLUX_ROE) GD2D_STAGE(FLUX_ROE);
    else if (flux == FLUX_AUSM_M2020) GD2D_STAGE(FLUX_AUSM_M2020);
    else GD2D_STAGE(FLUX_AUSM);
#undef GD2D_STAGE
    return cudaGetLastError();
}

cudaError_t launch_update_only_f64(const DevMesh &m, const DevState &s, double4 *unew, double4 *delta,
                                   const LaunchCfg &lc, cudaStream_t st) {
    k_update_only<<<(int)m.ntiles, lc.block, 0, st>>>(m, s, unew, delta);
    return cudaGetLastError();
}

cudaError_t launch_diff_only_f64(const DevMesh &m, const DevState &s, double4 *diffs, const LaunchCfg &lc,
                                 cudaStream_t st) {
    if (m.nfmax == 4) k_diff_only<true><<<(int)m.ntiles, lc.block, 0, st>>>(m, s, diffs);
    else k_diff_only<false><<<(int)m.ntiles, lc.block, 0, st>>>(m, s, diffs);
    return cudaGetLastError();
}

}  // namespace gd2d

// ------------------------------------------ reference order <-> device order
//
// Fields cross the ABI in the reference's layout: column-major [n x 4]
// matrices (or four columns) indexed by the reference's cell / node ids.
// These kernels do the reordering on the device, so the host only copies
// contiguous blocks (a permutation on the host is a cache miss per value).

namespace gd2d {

namespace {

int reorder_grid(int64_t n) {
    int64_t g = (n + 255) / 256;
    if (g < 1) g = 1;
    if (g > 148LL * 32) g = 148 * 32;
    return (int)g;
}

// dst[j] = (a[i], b[i], c[i], d[i]) with i = perm[j]: reference rows to
// device-order records.
__global__ void __launch_bounds__(256) k_cols_to_dev(const double *__restrict__ a, const double *__restrict__ b,
                                                     const double *__restrict__ c, const double *__restrict__ d,
                                                     const int32_t *__restrict__ perm, int64_t n,
                                                     double4 *__restrict__ dst) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = perm[j];
        dst[j] = make_double4(a[i], b[i], c[i], d[i]);
    }
}

// Conservative reference rows to device-order primitives, the formula of
// the primitives recovery (evaluate2d.jl:87-104) in the same order; this
// translation unit has no multiply-add contraction, like the host code it
// replaces.
__global__ void __launch_bounds__(256) k_cons_to_prims(const double *__restrict__ u, int64_t n,
                                                       const int32_t *__restrict__ perm, double G,
                                                       double4 *__restrict__ dst) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = perm[j];
        const double U1 = u[i], U2 = u[i + n], U3 = u[i + 2 * n], U4 = u[i + 3 * n];
        dst[j] = make_double4(U1, U2 / U1, U3 / U1, (G - 1.0) * (U4 - 0.5 * (U2 * U2 + U3 * U3) / U1));
    }
}

// dst[i + v n] = component v of src[inv[i]]: device-order records to
// reference-order columns (FP32 records widened exactly).
template <class T4>
__global__ void __launch_bounds__(256) k_dev_to_cols(const T4 *__restrict__ src, const int32_t *__restrict__ inv,
                                                     int64_t n, double *__restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T4 r = src[inv[i]];
        dst[i] = (double)r.x;
        dst[i + n] = (double)r.y;
        dst[i + 2 * n] = (double)r.z;
        dst[i + 3 * n] = (double)r.w;
    }
}

}  // namespace

cudaError_t launch_cols_to_dev(const double *cols, const int32_t *perm, int64_t n, double4 *dst, cudaStream_t st) {
    k_cols_to_dev<<<reorder_grid(n), 256, 0, st>>>(cols, cols + n, cols + 2 * n, cols + 3 * n, perm, n, dst);
    return cudaGetLastError();
}

cudaError_t launch_cons_to_prims(const double *cols, const int32_t *perm, int64_t n, double gamma, double4 *dst,
                                 cudaStream_t st) {
    k_cons_to_prims<<<reorder_grid(n), 256, 0, st>>>(cols, n, perm, gamma, dst);
    return cudaGetLastError();
}

cudaError_t launch_dev_to_cols(const double4 *src, const int32_t *inv, int64_t n, double *cols, cudaStream_t st) {
    k_dev_to_cols<double4><<<reorder_grid(n), 256, 0, st>>>(src, inv, n, cols);
    return cudaGetLastError();
}

cudaError_t launch_dev_to_cols_f(const float4 *src, const int32_t *inv, int64_t n, double *cols, cudaStream_t st) {
    k_dev_to_cols<float4><<<reorder_grid(n), 256, 0, st>>>(src, inv, n, cols);
    return cudaGetLastError();
}

}  // namespace gd2d
