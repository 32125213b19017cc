/* A plain C caller of libgodunov2d: the reference's setup -> createFields2d
 * -> step loop -> read-back sequence through the C ABI alone, without the
 * Python package.  The mesh, the case parameters and the initial state come
 * from "case_data.h", generated by tests/test_c_abi.py from the same case
 * the Python binding runs, so the two results can be compared bit for bit.
 * Prints the conservative state after NSTEPS steps, one value per line. */
#include <stdio.h>
#include <string.h>

#include "godunov2d.h"
#include "case_data.h"

int main(void) {
    gd2d_mesh_view mv;
    memset(&mv, 0, sizeof mv);
    mv.n_cells = N_CELLS;
    mv.n_nodes = N_NODES;
    mv.n_neib_cells = N_NEIB;
    mv.x_nodes = x_nodes;
    mv.y_nodes = y_nodes;
    mv.mesh_connectivity = mesh_connectivity;
    mv.cell_stiffness = cell_stiffness;
    mv.cells2nodes = cells2nodes;
    mv.cell_edges_Nx = cell_edges_Nx;
    mv.cell_edges_Ny = cell_edges_Ny;
    mv.cell_edges_length = cell_edges_length;
    mv.cell_areas = cell_areas;
    mv.HX = HX;
    mv.cell_mid_points = cell_mid_points;
    mv.cell_clusters = cell_clusters;
    mv.node_stencils = node_stencils;
    mv.node2cellL2up = node2cellL2up;
    mv.node2cellL2down = node2cellL2down;

    gd2d_params p;
    memset(&p, 0, sizeof p);
    p.RGAS = CASE_RGAS;
    p.Gamma = CASE_GAMMA;
    p.Cp = 1000.0;
    p.CFL = CASE_CFL;
    p.beta = 1.0;
    p.ksi = 1.0e-12;
    p.venkat_K = 5.0;
    p.T_ref = 300.0;
    p.Pr = 0.72;
    p.min_density = 0.01;
    p.max_density = 10.0;
    p.flux = GD2D_FLUX_AUSM_PLUS;
    p.limiter = GD2D_LIM_MINMOD;
    p.viscosity = GD2D_VISC_NONE;
    p.dt_mode = GD2D_DT_LOCAL_CFL;
    p.n_bc = 3;
    p.bc[0].tag = -1; p.bc[0].kind = GD2D_BC_INFLOW;
    p.bc[0].rho = IN_RHO; p.bc[0].u = IN_U; p.bc[0].v = 0.0; p.bc[0].p = IN_P;
    p.bc[1].tag = -2; p.bc[1].kind = GD2D_BC_OUTFLOW;
    p.bc[2].tag = -3; p.bc[2].kind = GD2D_BC_SLIP_WALL;

    gd2d_launch launch;
    memset(&launch, 0, sizeof launch);  /* FP64, cell loop, device 0 */
    launch.order = GD2D_ORDER_HILBERT;

    gd2d_handle *h = NULL;
    if (gd2d_setup(&h, 1, &mv, &p, &launch) != GD2D_OK) {
        fprintf(stderr, "setup: %s\n", gd2d_last_error(NULL));
        return 1;
    }
    if (gd2d_set_state(h, 0, rho0, ux0, uy0, p0) != GD2D_OK) {
        fprintf(stderr, "set_state: %s\n", gd2d_last_error(h));
        return 1;
    }
    gd2d_stats st;
    if (gd2d_propagate(h, NSTEPS, &st) != GD2D_OK) {
        fprintf(stderr, "propagate: %s\n", gd2d_last_error(h));
        return 1;
    }
    static double ucons[4 * N_CELLS];
    if (gd2d_get_state(h, 0, ucons, NULL, NULL) != GD2D_OK) {
        fprintf(stderr, "get_state: %s\n", gd2d_last_error(h));
        return 1;
    }
    for (int i = 0; i < 4 * N_CELLS; ++i) printf("%.17g\n", ucons[i]);
    printf("step %lld dt %.17g\n", (long long)st.step, st.dt);
    gd2d_destroy(h);
    return 0;
}
