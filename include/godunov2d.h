/*
 * godunov2d.h -- C ABI of the B200 explicit Godunov step.
 *
 * Drop-in boundary for the hot path of dimaZloy/2D-DNS-godunov-solver-
 * (Julia).  The reference has no FFI: its "interface" is the Julia call
 * shape of the step loop.  Each entry point below names the reference code
 * it replaces (file:line in the reference project).  Julia binds these with
 * ccall; ctypes and C++ bind them the same way (no torch types, plain
 * pointers and sizes).
 *
 * Arrays crossing this boundary are the reference's own Julia arrays:
 * column-major (rows, cols) Float64/Int32 matrices with 1-based indices and
 * negative boundary tags, e.g. an (nCells,4) conservative matrix is four
 * contiguous planes rho, rho*u, rho*v, E.  Nothing is copied on the host
 * side beyond a one-time reordering at setup.
 *
 * Ownership: the library owns all device memory of a handle.  Threading: a
 * handle is driven by one host thread at a time and runs on one CUDA
 * stream; distinct handles may be used concurrently.  Every call returns 0
 * or a negative GD2D_ERR_* code; gd2d_last_error() gives the message.
 */
#ifndef GODUNOV2D_H
#define GODUNOV2D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GD2D_ABI_VERSION 1
#define GD2D_MAX_BC 8

enum gd2d_status {
    GD2D_OK = 0,
    GD2D_ERR_ARG = -1,       /* invalid argument or handle */
    GD2D_ERR_MESH = -2,      /* mesh fails a structural invariant */
    GD2D_ERR_CUDA = -3,      /* CUDA runtime error */
    GD2D_ERR_NONFINITE = -4, /* NaN/Inf or non-positive density/pressure in the state */
    GD2D_ERR_TIMEOUT = -5,   /* a bounded device wait gave up */
    GD2D_ERR_OOM = -6,       /* device allocation failed */
    GD2D_ERR_STATE = -7      /* call out of order (e.g. propagate before set_state) */
};

/* Face flux (computeslope2d.jl:129-132 selects it by editing source). */
enum gd2d_flux { GD2D_FLUX_AUSM_PLUS = 1, GD2D_FLUX_ROE = 2, GD2D_FLUX_AUSM_PLUS_M2020 = 3 };
/* Slope limiter (limiters.jl); VENKAT is an extension. */
enum gd2d_limiter { GD2D_LIM_NONE = 0, GD2D_LIM_MINMOD = 1, GD2D_LIM_VENKAT = 2,
                    GD2D_LIM_VANLEER = 3, GD2D_LIM_VANALBADA = 4 };
/* Boundary kinds addressed by the negative tags of cell_stiffness. */
enum gd2d_bc_kind { GD2D_BC_INFLOW = 1, GD2D_BC_OUTFLOW = 2, GD2D_BC_SLIP_WALL = 3,
                    GD2D_BC_NOSLIP_ISOTHERMAL = 4, GD2D_BC_TGV_ANALYTIC = 5 };
/* Viscous source: REFERENCE = calcDiffTerm.jl as written (constant mu,
 * air conductivity); SUTHERLAND / CONSTANT are extensions. */
enum gd2d_viscosity { GD2D_VISC_NONE = 0, GD2D_VISC_REFERENCE = 1, GD2D_VISC_SUTHERLAND = 2,
                      GD2D_VISC_CONSTANT = 3 };
/* Time step: FIXED = solControls.dt, what the reference steps with
 * (testInviscidFluxesGPUx32.jl:301, flowTime += dt at :401).
 * REFERENCE_TAU = step with tau = CFL*max(HX)/max(VMAX), which the reference
 * computes and reports every step (testInviscidFluxesGPUx32.jl:299,324) but
 * does not step with.  LOCAL_CFL = CFL*min(2A/P/VMAX) (extension).  tau is
 * reported in gd2d_stats under every mode. */
enum gd2d_dt_mode { GD2D_DT_FIXED = 0, GD2D_DT_REFERENCE_TAU = 1, GD2D_DT_LOCAL_CFL = 2 };
enum gd2d_precision { GD2D_PREC_F64 = 0, GD2D_PREC_MIXED = 1 };
enum gd2d_order { GD2D_ORDER_NATURAL = 0, GD2D_ORDER_HILBERT = 1, GD2D_ORDER_RCM = 2 };
/* CELL: one thread per cell evaluates its own faces (each interior face
 * twice, no atomics).  FACE_COLOURED: one thread per face, faces grouped in
 * colours no two of which touch the same cell, accumulating into the cells.
 * FACE_SLOTS: one thread per face, each side's flux stored in its own
 * (cell, face) slot and summed in face order by the update (FP64 only).
 * TILE_FACES: one fused kernel over per-tile face lists; a face between two
 * cells of one tile is evaluated once when its flux is exactly antisymmetric
 * (AUSM+ with Minmod/Venkatakrishnan/no limiter), results bit-identical to
 * CELL (FP64 only). */
enum gd2d_loop { GD2D_LOOP_CELL = 0, GD2D_LOOP_FACE_COLOURED = 1, GD2D_LOOP_FACE_SLOTS = 2,
                 GD2D_LOOP_TILE_FACES = 3 };

/* mesh2d_Int32 (primeObjects.jl:109-135) as read by readMesh2dHDF5
 * (utilsIO.jl:107-252).  All matrices column-major. */
typedef struct gd2d_mesh_view {
    int64_t n_cells;
    int64_t n_nodes;
    int32_t n_neib_cells;                /* columns of cell_clusters / node_stencils (8) */
    int32_t reserved0;
    const double *x_nodes, *y_nodes;     /* [n_nodes] */
    const int32_t *mesh_connectivity;    /* [n_cells x 7]: id, type (3 tri / 2 quad), n, nodes */
    const int32_t *cell_stiffness;       /* [n_cells x 4]: neighbour id or negative tag */
    const int32_t *cells2nodes;          /* [n_cells x 8]: node pair of each edge */
    const double *cell_edges_Nx;         /* [n_cells x 4]: unit inward normals */
    const double *cell_edges_Ny;         /* [n_cells x 4] */
    const double *cell_edges_length;     /* [n_cells x 4] */
    const double *cell_areas;            /* [n_cells] */
    const double *HX;                    /* [n_cells]: longest edge */
    const double *cell_mid_points;       /* [n_cells x 2] */
    const int32_t *cell_clusters;        /* [n_nodes x n_neib_cells], 0-padded */
    const double *node_stencils;         /* [n_nodes x n_neib_cells] */
    const int32_t *node2cellL2up;        /* [n_cells x 8] */
    const int32_t *node2cellL2down;      /* [n_cells x 8] */
} gd2d_mesh_view;

typedef struct gd2d_bc {
    int32_t tag;   /* negative tag as stored in cell_stiffness */
    int32_t kind;  /* gd2d_bc_kind */
    double rho, u, v, p;  /* INFLOW state */
    double Tw;            /* NOSLIP_ISOTHERMAL wall temperature */
} gd2d_bc;

/* THERMOPHYSICS (thermo.jl:4-10), CONTROLS (primeObjects.jl:233-243) and
 * the solver selectors, per case. */
typedef struct gd2d_params {
    double RGAS, Gamma, Cp, mu, kGas;
    double CFL, dt, beta;   /* beta = bettaKJ of calcOneStageMUSCLcpuFast (1.0) */
    double ksi;             /* Minmod constant (computeslope2d.jl:116: 1e-12) */
    double venkat_K;        /* eps^2 = (K*HX)^3 */
    double mu_ref;          /* REFERENCE: mu (1e-2); SUTHERLAND: mu(T_ref); CONSTANT: mu */
    double T_ref;
    double Pr;
    double tgv_U0, tgv_P0, tgv_L, tgv_mu;  /* computeTGV2d (initfields_TGV2d.jl:9-27) */
    double start_time;
    double min_density, max_density;  /* minDensityConstrained / maxDensityConstrained */
    int32_t flux, limiter, viscosity, art_viscosity;
    int32_t dt_mode;
    int32_t init_nodes;     /* 0: node primitives zero in step 1, as the reference */
    int32_t n_bc;
    int32_t density_constrained;  /* densityConstrained: clamp the new density (evaluate2d.jl:63-77) */
    gd2d_bc bc[GD2D_MAX_BC];
} gd2d_params;

/* Launch / layout choices of a handle (NULL = defaults or autotuned). */
typedef struct gd2d_launch {
    int32_t precision;      /* gd2d_precision */
    int32_t order;          /* gd2d_order */
    int32_t loop;           /* gd2d_loop */
    int32_t block;          /* threads per block of the cell kernel (0 = default) */
    int32_t node_block;     /* threads per block of the node kernel (0 = default) */
    int32_t persistent;     /* 1: grid-stride persistent cell kernel */
    int32_t graph_steps;    /* steps per captured CUDA graph (0 = default, 1 = eager) */
    int32_t min_blocks;     /* cell kernel blocks per SM the register budget targets: 2, 3, 4 (0 = default) */
    int32_t device;         /* CUDA device ordinal of the handle (the library links its own CUDA
                               runtime, so the caller's current device does not carry over) */
    int32_t reserved0;
    void *stream;           /* cudaStream_t to run on (on `device`); NULL: the handle's own */
} gd2d_launch;

/* Per-case diagnostics of one step (the reference's dynControls fields,
 * evaluate2d.jl:6-48 residuals, and conserved totals). */
typedef struct gd2d_stats {
    double dt, flow_time, tau, velmax;
    double residual[4];     /* sum over cells of (Unew - Uold)^2 per variable */
    double rho_min, rho_max;/* of the density entering the step (evaluate2d.jl:79-80) */
    double totals[4];       /* sum of U * area after the step */
    double kinetic_energy;  /* sum of 0.5 rho |u|^2 area after the step */
    int64_t step;
    int32_t nonfinite;      /* 1 if any cell left the admissible set */
    int32_t reserved0;
} gd2d_stats;

typedef struct gd2d_handle gd2d_handle;

int gd2d_abi_version(void);

/* Message of the last failed call on h (h may be NULL for setup failures). */
const char *gd2d_last_error(const gd2d_handle *h);

/* setupSolver: readMesh2dHDF5 result + setupSolver_*.jl globals + device
 * buffers (testInviscidFluxesGPUx32.jl:137-277, cuda_data_x32.jl:2-50).
 * n_cases independent meshes advance together in one launch per kernel. */
int gd2d_setup(gd2d_handle **out, int32_t n_cases, const gd2d_mesh_view *meshes,
               const gd2d_params *params, const gd2d_launch *launch);

/* createFields2d + phs2dcns2dcellsSA + the conservative node average
 * (initfields_*.jl createFields2d, utilsFVM2dp.jl:4-17, 370-422).
 * Host arrays that are page-locked (cudaHostAlloc / cudaHostRegister, or
 * pinned by the caller's CUDA binding) are copied to the device directly;
 * pageable ones go through the library's own page-locked stage.  The same
 * holds for every host array of gd2d_set_conservative and gd2d_get_state. */
int gd2d_set_state(gd2d_handle *h, int32_t icase, const double *density, const double *ux,
                   const double *uy, const double *pressure);

/* Restart from a conservative state (nCells x 4) and time
 * (loadPrevResults.jl:3-38): U is kept exactly, the primitives, the next dt
 * and (rebuild_nodes != 0) the node values are recomputed from it as a step
 * would, so an FP64 run restarted from gd2d_get_state's Ucons and its
 * flowTime continues bit for bit. */
int gd2d_set_conservative(gd2d_handle *h, int32_t icase, const double *ucons, double flow_time,
                          int32_t rebuild_nodes);

/* The step loop body, nsteps times (testInviscidFluxesGPUx32.jl:314-401,
 * testViscousFluxesTGV2d.jl:416-506): dt from the CFL reduction,
 * calcDiffTerm, calcOneStageMUSCLcpuFast, updateVariablesSA,
 * cells2nodesSolutionReconstructionWithStencils, residuals, flowTime += dt.
 * stats_out: [n_cases] stats of the last step (may be NULL). */
int gd2d_propagate(gd2d_handle *h, int32_t nsteps, gd2d_stats *stats_out);

/* Per-step stats of the last min(nsteps, capacity) steps of case icase,
 * oldest first; returns the count written. */
int gd2d_get_history(gd2d_handle *h, int32_t icase, gd2d_stats *out, int32_t capacity);

/* Fields in reference ordering (the permutation applied at setup is undone
 * exactly).  Any pointer may be NULL.  ucons/prims: [nCells x 4]
 * (prims = rho, u, v, p); node_prims: [nNodes x 4]. */
int gd2d_get_state(gd2d_handle *h, int32_t icase, double *ucons, double *prims, double *node_prims);

/* Reference functions one at a time, on the handle's state (for callers that
 * keep the reference's loop and for parity checks). */
/* calcOneStageMUSCLcpuFast(cellsThreads, beta, dt, t, ..., Uold, FLUXES, Diff, Unew)
 * (calcOneStageMUSCLcpuFast.jl:3-107): writes Unew (and FLUXES if fluxes != NULL,
 * [nCells x 4] host) without touching Uold or the primitives. */
int gd2d_calc_one_stage(gd2d_handle *h, int32_t icase, double beta, double dt, double flow_time,
                        double *fluxes, double *unew);
/* updateVariablesSA (evaluate2d.jl:52-110): primitives, VMAX, Delta, Uold <- Unew. */
int gd2d_update_variables(gd2d_handle *h, int32_t icase, double *delta);
/* cells2nodesSolutionReconstructionWithStencils (utilsFVM2dp.jl:299-365). */
int gd2d_cells_to_nodes(gd2d_handle *h);
/* calcDiffTerm (calcDiffTerm.jl:31-121): Diff [nCells x 4] from Uold. */
int gd2d_calc_diff_term(gd2d_handle *h, int32_t icase, double *diff);

/* Autotuner (no counterpart in the reference, whose CPU loop has no launch
 * shape): times candidate launch shapes on this handle's own data and keeps
 * the fastest -- cell-kernel register budget (min_blocks 2/3/4) x
 * persistence, node-pass block (64/128/256), steps per graph (8/32/128,
 * unless the launch record given to gd2d_setup set graph_steps, which is
 * kept) -- by coordinate search, `steps_per_trial` steps each (<= 0: 64).  Every
 * device array a step touches is saved first and restored after the trials,
 * so propagation continues bit-identically.  Needs gd2d_set_state on every
 * case; allocates a temporary copy of the state.  `chosen` (may be NULL)
 * receives the new launch shape; gd2d_last_timing's total is its ms/step. */
int gd2d_autotune(gd2d_handle *h, int32_t steps_per_trial, gd2d_launch *chosen);

/* Device time of the kernels of the last propagate call (CUDA events on the
 * handle's stream): total ms and ms of the fused cell kernel. */
int gd2d_last_timing(gd2d_handle *h, double *total_ms, double *cell_kernel_ms, int64_t *launches);

int gd2d_destroy(gd2d_handle *h);

/* updateVariablesSA + residuals on caller-owned DEVICE arrays, allocating
 * nothing.  No counterpart in the reference: it exists for callers that
 * cannot let a library allocate -- memory owned by their own pool (Julia's
 * CUDA.jl, a caching allocator) or an allocation-free step loop (cudaMalloc
 * synchronises the device and is not allowed during stream capture).
 * d_unew, d_uold, d_prims: [n_cells x 4] column-major device arrays (d_uold is
 * overwritten with d_unew, d_prims receives rho, u, v, p); d_stats: 6 device
 * doubles = sum of (Unew-Uold)^2 per variable, max VMAX, non-finite flag.
 * The only scratch is a fixed 4 MiB array inside the library (one per GPU,
 * held until exit), so n_cells is limited to 16,777,216 (larger: GD2D_ERR_ARG).
 * The first call on a device looks that array up (again after the device's
 * context is recreated, e.g. by cudaDeviceReset) and should come before any
 * stream capture; calls that overlap on the GPU share the array and race.
 * Runs on `stream` (NULL: the legacy default stream). */
int gd2d_update_variables_noalloc(const double *d_unew, double *d_uold, double *d_prims, int64_t n_cells,
                                  double gamma, double *d_stats, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GODUNOV2D_H */
