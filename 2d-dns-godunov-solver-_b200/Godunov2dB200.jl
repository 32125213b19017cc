# Godunov2dB200 -- Julia binding of libgodunov2d.so (include/godunov2d.h).
#
# Drop-in for the step loop of the reference's drivers
# (testInviscidFluxesGPUx32.jl:314-447, testViscousFluxesTGV2d.jl:416-552):
# the reference's own mesh2d_Int32 and field arrays are passed with
# pointer(...), column-major, 1-based, no copies.  Every call runs the
# library's sm_100a kernels; there is no CPU fallback.  The struct layouts
# below mirror the C header field for field (tests/test_julia_binding.py
# checks names, order and sizes against the header and the ctypes binding).
#
#   include("Godunov2dB200.jl"); using .Godunov2dB200
#   h = Godunov2dB200.setup([testMesh], [params])
#   Godunov2dB200.set_state(h, 0, testfields2d)
#   st = Godunov2dB200.propagate(h, 100)
module Godunov2dB200

const lib = get(ENV, "GD2D_LIB", joinpath(@__DIR__, "libgodunov2d.so"))

const GD2D_MAX_BC = 8

# enum values of the header
const FLUX_AUSM_PLUS, FLUX_ROE, FLUX_AUSM_PLUS_M2020 = Int32(1), Int32(2), Int32(3)
const LIM_NONE, LIM_MINMOD, LIM_VENKAT, LIM_VANLEER, LIM_VANALBADA = Int32.(0:4)
const BC_INFLOW, BC_OUTFLOW, BC_SLIP_WALL, BC_NOSLIP_ISOTHERMAL, BC_TGV_ANALYTIC = Int32.(1:5)
const VISC_NONE, VISC_REFERENCE, VISC_SUTHERLAND, VISC_CONSTANT = Int32.(0:3)
const DT_FIXED, DT_REFERENCE_TAU, DT_LOCAL_CFL = Int32.(0:2)
const PREC_F64, PREC_MIXED = Int32(0), Int32(1)
const ORDER_NATURAL, ORDER_HILBERT, ORDER_RCM = Int32.(0:2)
const LOOP_CELL, LOOP_FACE_COLOURED, LOOP_FACE_SLOTS, LOOP_TILE_FACES = Int32.(0:3)

# gd2d_mesh_view: mesh2d_Int32 (primeObjects.jl:109-135)
struct MeshView
    n_cells::Int64
    n_nodes::Int64
    n_neib_cells::Int32
    reserved0::Int32
    x_nodes::Ptr{Float64}
    y_nodes::Ptr{Float64}
    mesh_connectivity::Ptr{Int32}
    cell_stiffness::Ptr{Int32}
    cells2nodes::Ptr{Int32}
    cell_edges_Nx::Ptr{Float64}
    cell_edges_Ny::Ptr{Float64}
    cell_edges_length::Ptr{Float64}
    cell_areas::Ptr{Float64}
    HX::Ptr{Float64}
    cell_mid_points::Ptr{Float64}
    cell_clusters::Ptr{Int32}
    node_stencils::Ptr{Float64}
    node2cellL2up::Ptr{Int32}
    node2cellL2down::Ptr{Int32}
end

# gd2d_bc
struct BC
    tag::Int32
    kind::Int32
    rho::Float64
    u::Float64
    v::Float64
    p::Float64
    Tw::Float64
end

# gd2d_params: THERMOPHYSICS (thermo.jl:4-10), CONTROLS (primeObjects.jl:233-243)
struct Params
    RGAS::Float64
    Gamma::Float64
    Cp::Float64
    mu::Float64
    kGas::Float64
    CFL::Float64
    dt::Float64
    beta::Float64
    ksi::Float64
    venkat_K::Float64
    mu_ref::Float64
    T_ref::Float64
    Pr::Float64
    tgv_U0::Float64
    tgv_P0::Float64
    tgv_L::Float64
    tgv_mu::Float64
    start_time::Float64
    min_density::Float64
    max_density::Float64
    flux::Int32
    limiter::Int32
    viscosity::Int32
    art_viscosity::Int32
    dt_mode::Int32
    init_nodes::Int32
    n_bc::Int32
    density_constrained::Int32
    bc::NTuple{8,BC}
end

# gd2d_launch
struct Launch
    precision::Int32
    order::Int32
    loop::Int32
    block::Int32
    node_block::Int32
    persistent::Int32
    graph_steps::Int32
    min_blocks::Int32
    device::Int32
    reserved0::Int32
    stream::Ptr{Cvoid}
end

# gd2d_stats: dynControls fields, residuals (evaluate2d.jl:6-48), totals
struct Stats
    dt::Float64
    flow_time::Float64
    tau::Float64
    velmax::Float64
    residual::NTuple{4,Float64}
    rho_min::Float64
    rho_max::Float64
    totals::NTuple{4,Float64}
    kinetic_energy::Float64
    step::Int64
    nonfinite::Int32
    reserved0::Int32
end

MeshView(m) = MeshView(m.nCells, m.nNodes, m.nNeibCells, Int32(0),
    pointer(m.xNodes), pointer(m.yNodes), pointer(m.mesh_connectivity),
    pointer(m.cell_stiffness), pointer(m.cells2nodes), pointer(m.cell_edges_Nx),
    pointer(m.cell_edges_Ny), pointer(m.cell_edges_length), pointer(m.cell_areas),
    pointer(m.HX), pointer(m.cell_mid_points), pointer(m.cell_clusters),
    pointer(m.node_stencils), pointer(m.node2cellL2up), pointer(m.node2cellL2down))

# The defaults of the C library: FP64, Hilbert order, cell loop, library-chosen shapes, device 0.
default_launch(; precision=PREC_F64, order=ORDER_HILBERT, loop=LOOP_CELL, device=0) =
    Launch(precision, order, loop, 0, 0, 0, 0, 0, Int32(device), 0, C_NULL)

abi_version() = ccall((:gd2d_abi_version, lib), Cint, ())
last_error(h=C_NULL) = unsafe_string(ccall((:gd2d_last_error, lib), Cstring, (Ptr{Cvoid},), h))
check(rc, h=C_NULL) = rc < 0 ? error("godunov2d: $(last_error(h)) ($rc)") : rc

# setupSolver: readMesh2dHDF5 result + setupSolver_*.jl globals + device buffers
# (testInviscidFluxesGPUx32.jl:137-277).  The library copies what it needs.
function setup(meshes::Vector, params::Vector{Params}; launch::Launch=default_launch())
    views = [MeshView(m) for m in meshes]
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve meshes views params begin
        check(ccall((:gd2d_setup, lib), Cint,
              (Ptr{Ptr{Cvoid}}, Int32, Ptr{MeshView}, Ptr{Params}, Ref{Launch}),
              h, length(meshes), views, params, launch))
    end
    return h[]
end

# createFields2d + phs2dcns2dcellsSA (initfields_*.jl, utilsFVM2dp.jl:4-17);
# icase is 0-based like the C ABI
set_state(h, icase, f) = check(ccall((:gd2d_set_state, lib), Cint,
    (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
    h, icase, f.densityCells, f.UxCells, f.UyCells, f.pressureCells), h)

# restart from (nCells x 4) conservatives and flowTime (loadPrevResults.jl:3-38)
set_conservative(h, icase, Ucons::Matrix{Float64}, flow_time, rebuild_nodes=true) =
    check(ccall((:gd2d_set_conservative, lib), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Float64, Int32),
          h, icase, Ucons, flow_time, rebuild_nodes ? 1 : 0), h)

# the step loop body nsteps times; returns the last step's stats per case
function propagate(h, nsteps, ncases=1)
    st = Vector{Stats}(undef, ncases)
    check(ccall((:gd2d_propagate, lib), Cint, (Ptr{Cvoid}, Int32, Ptr{Stats}), h, nsteps, st), h)
    return st
end

# per-step stats of the last steps of a case, oldest first
function get_history(h, icase, capacity=1024)
    st = Vector{Stats}(undef, capacity)
    n = check(ccall((:gd2d_get_history, lib), Cint, (Ptr{Cvoid}, Int32, Ptr{Stats}, Int32),
                    h, icase, st, capacity), h)
    return st[1:n]
end

# fields back in reference order (any array may be C_NULL)
get_state!(h, icase, Ucons, prims, nodeprims) = check(ccall((:gd2d_get_state, lib), Cint,
    (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), h, icase, Ucons, prims, nodeprims), h)

# calcOneStageMUSCLcpuFast(cellsThreads, beta, dt, t, ..., Uold, FLUXES, Diff, Unew)
calc_one_stage!(h, icase, beta, dt, t, FLUXES, Unew) = check(ccall((:gd2d_calc_one_stage, lib), Cint,
    (Ptr{Cvoid}, Int32, Float64, Float64, Float64, Ptr{Float64}, Ptr{Float64}),
    h, icase, beta, dt, t, FLUXES, Unew), h)
# updateVariablesSA (evaluate2d.jl:52-110)
update_variables!(h, icase, Delta) = check(ccall((:gd2d_update_variables, lib), Cint,
    (Ptr{Cvoid}, Int32, Ptr{Float64}), h, icase, Delta), h)
# cells2nodesSolutionReconstructionWithStencils (utilsFVM2dp.jl:299-365)
cells_to_nodes!(h) = check(ccall((:gd2d_cells_to_nodes, lib), Cint, (Ptr{Cvoid},), h), h)
# calcDiffTerm (calcDiffTerm.jl:31-121)
calc_diff_term!(h, icase, Diff) = check(ccall((:gd2d_calc_diff_term, lib), Cint,
    (Ptr{Cvoid}, Int32, Ptr{Float64}), h, icase, Diff), h)

# time launch shapes on the handle's own state (saved and restored around
# the trials) and keep the fastest; returns the chosen Launch
function autotune!(h, steps_per_trial=64)
    l = Ref{Launch}()
    check(ccall((:gd2d_autotune, lib), Cint, (Ptr{Cvoid}, Int32, Ref{Launch}), h, steps_per_trial, l), h)
    return l[]
end

# device time of the last propagate call: (total ms, cell-kernel ms, kernel launches)
function last_timing(h)
    t, c, n = Ref{Float64}(0), Ref{Float64}(0), Ref{Int64}(0)
    check(ccall((:gd2d_last_timing, lib), Cint, (Ptr{Cvoid}, Ref{Float64}, Ref{Float64}, Ref{Int64}),
                h, t, c, n), h)
    return t[], c[], n[]
end

destroy(h) = ccall((:gd2d_destroy, lib), Cint, (Ptr{Cvoid},), h)

# updateVariablesSA on device arrays the caller owns (e.g. CuArrays from
# CUDA.jl's pool: pass pointer(cuarray)), allocating nothing; limits and
# concurrency rules as in the header.  d_stats: 6 device doubles.
update_variables_noalloc!(d_unew, d_uold, d_prims, n_cells, gamma, d_stats, stream=C_NULL) =
    check(ccall((:gd2d_update_variables_noalloc, lib), Cint,
          (Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Float64, Ptr{Float64}, Ptr{Cvoid}),
          d_unew, d_uold, d_prims, n_cells, gamma, d_stats, stream))

end # module
