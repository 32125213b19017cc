// FP64 instantiations of the tile-face cell kernel (k_cell_step_tf).  Built
// with -fmad=false like kernels_f64.cu: results are bit-identical to the
// cell-centred kernel and the CPU restatement.
#include "step_kernels.cuh"

namespace gd2d {

namespace {

template <int FLUX, bool VISC, bool QUAD>
cudaError_t cell_step_tf(const DevMesh &m, const DevState &s, const LaunchCfg &lc, cudaStream_t st) {
    const int grid = lc.persistent ? lc.grid : (int)m.ntiles;
    if (lc.min_blocks >= 4) return launch_dependent(k_cell_step_tf<FLUX, VISC, QUAD, 4>, grid, lc.block, st, m, s);
    if (lc.min_blocks == 3) return launch_dependent(k_cell_step_tf<FLUX, VISC, QUAD, 3>, grid, lc.block, st, m, s);
    return launch_dependent(k_cell_step_tf<FLUX, VISC, QUAD, 2>, grid, lc.block, st, m, s);
}

template <int FLUX>
cudaError_t cell_step_tf_flux(const DevMesh &m, const DevState &s, bool visc, bool quads, const LaunchCfg &lc,
                              cudaStream_t st) {
    if (visc) return quads ? cell_step_tf<FLUX, true, true>(m, s, lc, st) : cell_step_tf<FLUX, true, false>(m, s, lc, st);
    return quads ? cell_step_tf<FLUX, false, true>(m, s, lc, st) : cell_step_tf<FLUX, false, false>(m, s, lc, st);
}

}  // namespace

cudaError_t launch_cell_step_tf_f64(const DevMesh &m, const DevState &s, int flux, bool visc, bool quads,
                                    const LaunchCfg &lc, cudaStream_t st) {
    switch (flux) {
    case FLUX_ROE: return cell_step_tf_flux<FLUX_ROE>(m, s, visc, quads, lc, st);
    case FLUX_AUSM_M2020: return cell_step_tf_flux<FLUX_AUSM_M2020>(m, s, visc, quads, lc, st);
    default: return cell_step_tf_flux<FLUX_AUSM>(m, s, visc, quads, lc, st);
    }
}

}  // namespace gd2d
