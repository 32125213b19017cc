// Internal device-side data structures of the godunov2d library.
//
// Layout in HBM (all cases of a handle concatenated; every case's cell range
// padded to a multiple of kCellPad so that a tile of the cell kernel never
// straddles two cases):
//   per cell  : int4 nbr (neighbour cell or -(bc_slot+1), kAbsent for no face),
//               int4 dn/up (down/up node per face; quads: dn2/up2 second node),
//               int2 c2n[k] (edge node pair, viscous and TGV only),
//               geometry planes nx[k], ny[k], len[k] (k < faces), rarea, area,
//               hx, charlen, mid (x,y);
//   state     : double4 U (rho, rho u, rho v, E) updated in place,
//               prim[2] double4 (rho, u, v, p) double-buffered by step parity;
//   per node  : double4 nodeP (weighted primitive average),
//               double4 nodeC (unweighted mean of rho u, rho v, E) and
//               NodeGrad nodeG (unweighted mean of the first gradients),
//               ELL cluster lists cl[w][node] / wt[w][node].
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gd2d {

constexpr int kCellPad = 1024;      // case cell ranges are multiples of this
constexpr int kMaxBC = 8;
constexpr int32_t kAbsent = INT32_MIN;
constexpr int kPartials = 16;       // doubles per tile partial record
constexpr int kGroupTiles = 256;    // tiles per group of the two-level step reduction
constexpr int kMaxCluster = 8;

enum FluxKind { FLUX_AUSM = 1, FLUX_ROE = 2, FLUX_AUSM_M2020 = 3 };
enum LimKind { LIM_NONE = 0, LIM_MINMOD = 1, LIM_VENKAT = 2, LIM_VANLEER = 3, LIM_VANALBADA = 4 };
enum BcKind { BC_INFLOW = 1, BC_OUTFLOW = 2, BC_SLIP = 3, BC_NOSLIP_ISOTHERMAL = 4, BC_TGV = 5 };
enum ViscKind { VISC_NONE = 0, VISC_REFERENCE = 1, VISC_SUTHERLAND = 2, VISC_CONSTANT = 3 };
enum DtMode { DT_FIXED = 0, DT_REFERENCE_TAU = 1, DT_LOCAL_CFL = 2 };

// Partial record slots.
enum PartSlot {
    P_RES0 = 0, P_TOT0 = 4, P_EK = 8, P_VMAX = 9, P_RMIN = 10, P_RHOMIN = 11, P_RHOMAX = 12,
    P_BAD = 13
};

// Per-case constants (read-only on the device).
struct DevCase {
    double gamma, R, CFL, dt_fixed, beta, ksi, venkat_K;
    double mu_ref, suth_ref, gamma_over_Pr, maxEdge;
    double tgv_U0, tgv_P0, tgv_L, tgv_mu;
    double rho_min, rho_max;          // densityConstrained clamp
    double bc_rho[kMaxBC], bc_u[kMaxBC], bc_v[kMaxBC], bc_p[kMaxBC], bc_Tw[kMaxBC];
    int32_t bc_kind[kMaxBC];
    int32_t dt_mode, visc_model, art_visc, limiter;
    int32_t density_constrained, pad_;
    int64_t cell_begin, cell_end;   // padded global cell range [begin, end)
    int64_t tile_begin, tile_end;   // tiles of the cell kernel
    int64_t group_begin, group_end; // tile groups (kGroupTiles tiles each, the last one shorter)
};

// Per-case mutable step state (device).
struct CaseState {
    double t, dt, velmax, rmin;
    int64_t step;
    unsigned int tiles_done;  // (tile group, record field) pairs of the case folded this step
    int32_t nonfinite;
};

// Mirrors gd2d_stats (include/godunov2d.h).
struct DevStats {
    double dt, flow_time, tau, velmax;
    double residual[4];
    double rho_min, rho_max;
    double totals[4];
    double kinetic_energy;
    int64_t step;
    int32_t nonfinite;
    int32_t reserved0;
};

struct NodeGrad {  // unweighted node means of the first gradients
    double2 ru, rv, re;  // (gradX, gradY) of rho u, rho v, E
};

struct DevMesh {
    int64_t Nc, Nn;          // padded totals
    int32_t ncases, nfmax;   // nfmax: 3 or 4
    int32_t cluster_w;       // ELL width of the cluster lists
    int32_t unit_weights;    // all node_stencils on live slots are 1.0
    int64_t ntiles;
    const int4 *nbr;
    const int4 *dn, *up, *dn2, *up2;     // dn2/up2 only with quads
    const int2 *c2n;                     // [nfmax][Nc] edge node pairs
    const double *nx, *ny, *len;         // [nfmax][Nc]
    const double *rarea, *area, *hx, *charlen;
    const double2 *mid;                  // TGV only
    const double *xnode, *ynode;         // TGV only
    const int32_t *cl;                   // [cluster_w][Nn], -1 = empty
    const double *wt;                    // [cluster_w][Nn] (NULL if unit weights)
    const int32_t *tile_case;            // [ntiles]
    const int32_t *group_case;           // [ngroups] case of each tile group of the step reduction
    int64_t ngroups;
    const int32_t *node_case;            // [Nn] (viscous only)
    const DevCase *cases;
    // mixed precision: FP32 copies of the geometry (the FP64 planes are not allocated)
    const float *nxf, *nyf, *lenf;       // [nfmax][Nc]
    const float *nlxf, *nlyf;            // [nfmax][Nc] (viscous) nx * len, ny * len, rounded once to FP32
    const float *rareaf, *areaf, *hxf, *charlenf;
    // tile-local face lists (GD2D_LOOP_TILE_FACES): faces of tile t are
    // [tf_off[t], tf_off[t+1]); tf_rec = (neighbour code, packed slots, dn, up)
    // with packed = la | ka << 10 | (lb + 1) << 12 | kb << 22 | quad << 24
    // (lb + 1 = 0: the face is not shared with another cell of the tile);
    // tf_q = (dn2, up2) for quads; mixed precision: the face geometry of
    // slot (la, ka) (the FP64 kernel reads it from the per-cell planes)
    const int64_t *tf_off;               // [ntiles + 1]
    const int4 *tf_rec;
    const int2 *tf_q;
    const int2 *tf_e;                    // (viscous) edge node pair of slot (la, ka)
    const float *tf_nxf, *tf_nyf, *tf_lenf;
};

// Fields of a packed tile-face slot record.
struct TileFace {
    int la, ka, lbp, kb;
    bool quad;
};
__host__ __device__ __forceinline__ TileFace unpack_tile_face(int32_t w) {
    TileFace f;
    f.la = w & 1023;
    f.ka = (w >> 10) & 3;
    f.lbp = (w >> 12) & 1023;
    f.kb = (w >> 22) & 3;
    f.quad = ((w >> 24) & 1) != 0;
    return f;
}
__host__ __device__ __forceinline__ int32_t pack_tile_face(int la, int ka, int lbp, int kb, bool quad) {
    return (int32_t)(la | (ka << 10) | (lbp << 12) | (kb << 22) | ((quad ? 1 : 0) << 24));
}

struct NodeGradF {  // FP32 node means of the first gradients
    float2 ru, rv, re;
};

struct DevState {
    double4 *U;        // [Nc]
    double4 *prim;     // [2][Nc]
    double4 *nodeP;    // [Nn]
    double4 *nodeC;    // [Nn] (viscous)
    NodeGrad *g1;      // [Nc] (viscous) first gradients per cell
    NodeGrad *nodeG;   // [Nn] (viscous)
    double *part;      // tile records (FP64: field f of tile q at [f * ntiles + q]; mixed: [q * kPartials + f])
    double *gpart;     // [ngroups][kPartials] group records
    CaseState *cstate; // [ncases]
    DevStats *ring;    // [ring_len][ncases]
    DevStats *ring_host;  // the host's page-locked, mapped copy of ring, written alongside it
    int32_t *parity;   // step parity (which prim buffer is current)
    unsigned int *node_done;
    int32_t ring_len;
    int32_t pad_;
    // mixed precision: FP32 primitives for the gathers (U stays FP64)
    float4 *primf;     // [2][Nc]
    float4 *nodePf;    // [Nn]
    float4 *nodeCf;    // [Nn] (viscous)
    NodeGradF *g1f;    // [Nc] (viscous)
    NodeGradF *nodeGf; // [Nn] (viscous)
};

struct LaunchCfg {
    int block;       // cell kernel threads per block (tile size)
    int node_block;
    int persistent;
    int grid;        // persistent grid size
    int min_blocks;  // register budget of the cell kernel: blocks per SM (2, 3, 4)
};

// Message reported by gd2d_last_error(NULL) for calls without a handle.
void set_handleless_error(const char *msg);

// Launch of a step kernel as a programmatic dependent of the kernel before
// it on the stream: it may be scheduled once every block of that kernel has
// started (each calls pdl_trigger first), and its threads wait in pdl_wait
// until that kernel has finished and its writes are visible.  This hides
// the launch gap and fills the last wave of one step kernel with the next.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*kernel)(KArgs...), int grid, int block, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Launchers implemented in kernels_f64.cu.
cudaError_t launch_cell_step_f64(const DevMesh &m, const DevState &s, int flux, bool visc, bool quads,
                                 const LaunchCfg &lc, cudaStream_t st);
cudaError_t launch_cell_step_tf_f64(const DevMesh &m, const DevState &s, int flux, bool visc, bool quads,
                                    const LaunchCfg &lc, cudaStream_t st);
// Reordering between the reference's column-major rows and device order
// (cols: [n x 4] column-major; perm[j] = reference row of device record j;
// inv[i] = device record of reference row i).
cudaError_t launch_cols_to_dev(const double *cols, const int32_t *perm, int64_t n, double4 *dst, cudaStream_t st);
cudaError_t launch_cons_to_prims(const double *cols, const int32_t *perm, int64_t n, double gamma, double4 *dst,
                                 cudaStream_t st);
cudaError_t launch_dev_to_cols(const double4 *src, const int32_t *inv, int64_t n, double *cols, cudaStream_t st);
cudaError_t launch_dev_to_cols_f(const float4 *src, const int32_t *inv, int64_t n, double *cols, cudaStream_t st);
// Node pass over nodes [n0, n1).  Its first blocks also complete the step
// reduction of the tile records of groups [g0, g1) that the cell kernel (or
// the state initialisation, red_init) wrote: the last group of each case
// finalizes the case (statistics, flowTime, the next dt).  g0 == g1: none.
cudaError_t launch_node_avg_f64(const DevMesh &m, const DevState &s, bool visc, bool flip_parity,
                                bool zero_prims, int64_t n0, int64_t n1, int64_t g0, int64_t g1, bool red_init,
                                const LaunchCfg &lc, cudaStream_t st);
cudaError_t launch_visc_grad_f64(const DevMesh &m, const DevState &s, const LaunchCfg &lc, cudaStream_t st);
cudaError_t launch_init_state_f64(const DevMesh &m, const DevState &s, int64_t t0, int64_t t1, const LaunchCfg &lc,
                                  cudaStream_t st);

// Face-loop variants (FP64, kernels_f64.cu): fluxes of faces [f0, f1), then
// the per-cell update.
cudaError_t launch_face_flux_f64(const DevMesh &m, const DevState &s, int flux, bool quads, bool slots,
                                 const int4 *faces, int64_t f0, int64_t f1, double4 *Facc, double4 *Fslot,
                                 const LaunchCfg &lc, cudaStream_t st);
cudaError_t launch_face_update_f64(const DevMesh &m, const DevState &s, bool visc, bool quads, bool slots,
                                   double4 *Facc, const double4 *Fslot, const LaunchCfg &lc, cudaStream_t st);

// The reference's functions one at a time (FP64, kernels_f64.cu).
cudaError_t launch_stage_only_f64(const DevMesh &m, const DevState &s, int flux, bool quads, double beta, double dt,
                                  double t, const double4 *diffs, double4 *unew, double4 *fluxes, const LaunchCfg &lc,
                                  cudaStream_t st);
cudaError_t launch_update_only_f64(const DevMesh &m, const DevState &s, double4 *unew, double4 *delta,
                                   const LaunchCfg &lc, cudaStream_t st);
cudaError_t launch_diff_only_f64(const DevMesh &m, const DevState &s, double4 *diffs, const LaunchCfg &lc,
                                 cudaStream_t st);

// Launchers implemented in kernels_mixed.cu (FP32 reconstruction, fluxes and
// viscous terms; FP64 state update and reductions).
cudaError_t launch_cell_step_mixed(const DevMesh &m, const DevState &s, int flux, bool visc, bool quads,
                                   const LaunchCfg &lc, cudaStream_t st);
cudaError_t launch_cell_step_tf_mixed(const DevMesh &m, const DevState &s, int flux, bool visc, bool quads,
                                      const LaunchCfg &lc, cudaStream_t st);
cudaError_t launch_node_avg_mixed(const DevMesh &m, const DevState &s, bool visc, bool flip_parity,
                                  bool zero_prims, int64_t n0, int64_t n1, int64_t g0, int64_t g1, bool red_init,
                                  const LaunchCfg &lc, cudaStream_t st);
cudaError_t launch_visc_grad_mixed(const DevMesh &m, const DevState &s, const LaunchCfg &lc, cudaStream_t st);
// U holds the case's FP64 primitives on entry and its conservatives on exit.
cudaError_t launch_init_state_mixed(const DevMesh &m, const DevState &s, int64_t t0, int64_t t1,
                                    const LaunchCfg &lc, cudaStream_t st);

}  // namespace gd2d
