# FEMToolsB200Ext — FEMTools.jl package extension that runs the dynamic-relaxation
# Stokes and thermal solves on libfemtools_b200 (sm_100a) instead of the
# KernelAbstractions CUDABackend kernels.
#
# Hook: FEMTools loads CUDA support through a package extension
# (ext/FEMToolsCUDAExt.jl:6 of FEMTools.jl); this file is a second extension on the
# same weak dependency. Project.toml of FEMTools.jl gains
#
#     [weakdeps]
#     CUDA = "052768ef-5323-5732-b1bb-66c8b64840ba"
#     [extensions]
#     FEMToolsB200Ext = "CUDA"
#
# The methods below are more specific than FEMTools' own `solve!`
# (src/stokes/solvers/DR.jl:302), `solve_coupled!` (:89) and the thermal `solve!`
# (src/heat_diffusion/solvers/DR.jl:50): they take states whose arrays are
# `CuArray`s, so a script written for the CUDABackend runs on the B200 library
# unchanged. `FEMToolsB200Ext.ENABLED[] = false` sends every call back to the
# KernelAbstractions path. The library is found through ENV["FEMTOOLS_B200_LIB"]
# (a path to libfemtools_b200.so) or the dynamic loader's search path.
#
# Every struct below mirrors include/femtools_b200.h field for field (isbits, C
# layout); tests/test_julia_extension.py checks the field lists against the header.
module FEMToolsB200Ext

using CUDA
using FEMTools
using FEMTools: StokesDR, MixedMesh, Mesh, DirichletBoundaryCondition, DruckerPrager, ThermalDiffusionDR

const LIB = get(ENV, "FEMTOOLS_B200_LIB", "libfemtools_b200")
const ENABLED = Ref(true)
const MAX_PHASES = 16

# status codes and enumerations of include/femtools_b200.h
const OK = Cint(0)
const F64, F32 = Int32(0), Int32(1)
const PHASE_NODAL, PHASE_CELL, PHASE_ELEMENT_NODE = Int32(0), Int32(1), Int32(2)
const FIELD_NONE, FIELD_IP, FIELD_NODAL = Int32(0), Int32(1), Int32(2)
const PRECISION_FP64, PRECISION_MIXED = Int32(0), Int32(1)

# ---- struct mirrors ----------------------------------------------------------

struct StokesMaterialC                      # femb200_stokes_material
    nphases::Int32
    eta::NTuple{16, Float64}
    eta_b::NTuple{16, Float64}
    G::NTuple{16, Float64}
    alpha::NTuple{16, Float64}
    rho0::NTuple{16, Float64}
    K::NTuple{16, Float64}
    g::NTuple{3, Float64}
    Tref::Float64
    plastic::Int32
    cos_phi::NTuple{16, Float64}
    sin_phi::NTuple{16, Float64}
    sin_psi::NTuple{16, Float64}
    C::NTuple{16, Float64}
    eta_reg::NTuple{16, Float64}
    Kb::NTuple{16, Float64}
    use_scaling_eta::Int32
    scaling_eta::NTuple{16, Float64}
end

struct StokesProblemC                       # femb200_stokes_problem
    dim::Int32
    nv::Int32
    np::Int32
    nq::Int32
    dtype::Int32
    geo_dtype::Int32
    nels::Int64
    nnodes::Int64
    nnodesP::Int64
    el2n::Ptr{Cvoid}
    dofsP::Ptr{Cvoid}
    el2nP::Ptr{Cvoid}
    geo_v::Ptr{Cvoid}
    geo_P::Ptr{Cvoid}
    v::NTuple{3, Ptr{Cvoid}}
    rate::NTuple{3, Ptr{Cvoid}}
    Rv::NTuple{3, Ptr{Cvoid}}
    Rv0::NTuple{3, Ptr{Cvoid}}
    dRdv::NTuple{3, Ptr{Cvoid}}
    PC::NTuple{3, Ptr{Cvoid}}
    P::Ptr{Cvoid}
    P0::Ptr{Cvoid}
    gammaP::Ptr{Cvoid}
    T::Ptr{Cvoid}
    T0::Ptr{Cvoid}
    Q::Ptr{Cvoid}
    Pf::Ptr{Cvoid}
    RP::Ptr{Cvoid}
    M_P::Ptr{Cvoid}
    Pnum::Ptr{Cvoid}
    phases_v::Ptr{Cvoid}
    phases_v_layout::Int32
    phases_P::Ptr{Cvoid}
    phases_P_layout::Int32
    tau_old::NTuple{6, Ptr{Cvoid}}
    tau_old_layout::Int32
    tau::NTuple{6, Ptr{Cvoid}}
    P_old::Ptr{Cvoid}
    P_old_layout::Int32
    viscosity_ip::Ptr{Cvoid}
    body_force::NTuple{3, Ptr{Cvoid}}
    bc_dofs::NTuple{3, Ptr{Cvoid}}
    bc_vals::NTuple{3, Ptr{Cvoid}}
    bc_n::NTuple{3, Int64}
    mat::StokesMaterialC
end

struct StokesControlsC                      # femb200_stokes_controls
    dt::Float64
    pressure_factor::Float64
    tolerance::Float64
    max_iterations::Int64
    check_interval::Int64
    iter_max::Int64
    max_ph_iterations::Int64
    rel_drop0::Float64
    freeze_jacobian::Int32
    finite_K::Int32
    assemble_scaling::Int32
    throw_on_failure::Int32
    precision::Int32
    cfl_v::Float64
    c_fact::Float64
    history::Ptr{Float64}
    history_capacity::Int64
end

struct StokesStatsC                         # femb200_stokes_stats
    itPH::Int64
    iter::Int64
    err::Float64
    err_abs::Float64
    err_rel::Float64
    err_v::Float64
    err_P::Float64
    converged::Int32
    reached_total_iter::Int32
    lambda_max::Float64
    lambda_max_gershgorin::Float64
    jacobian_assemblies::Int64
    history_len::Int64
    err_T::Float64
    thermal_iterations::Int64
    defect_corrections::Int64
end

struct ThermalProblemC                      # femb200_thermal_problem
    dim::Int32
    nv::Int32
    nq::Int32
    dtype::Int32
    geo_dtype::Int32
    nels::Int64
    nnodes::Int64
    el2n::Ptr{Cvoid}
    geo::Ptr{Cvoid}
    T::Ptr{Cvoid}
    T0::Ptr{Cvoid}
    rate::Ptr{Cvoid}
    R::Ptr{Cvoid}
    R0::Ptr{Cvoid}
    dRdT::Ptr{Cvoid}
    PC::Ptr{Cvoid}
    P::Ptr{Cvoid}
    source::Ptr{Cvoid}
    source_ip::Ptr{Cvoid}
    phases::Ptr{Cvoid}
    phases_layout::Int32
    bc_dofs::Ptr{Cvoid}
    bc_vals::Ptr{Cvoid}
    bc_n::Int64
    nphases::Int32
    k::NTuple{16, Float64}
    Cp::NTuple{16, Float64}
    rho0::NTuple{16, Float64}
    alpha::NTuple{16, Float64}
    K::NTuple{16, Float64}
    cfl::Float64
    c_fact::Float64
    eps::Float64
end

struct ThermalControlsC                     # femb200_thermal_controls
    dt::Float64
    Tref::Float64
    tolerance::Float64
    max_iterations::Int64
    check_interval::Int64
    throw_on_failure::Int32
end

struct ThermalStatsC                        # femb200_thermal_stats
    converged::Int32
    iterations::Int64
    residual::Float64
end

# ---- handles ------------------------------------------------------------------

mutable struct Handle
    ptr::Ptr{Cvoid}
end

# one library handle per (task-local) CUDA device; the handle owns only scratch
const HANDLES = Dict{Int, Handle}()
const HANDLE_LOCK = ReentrantLock()

function handle()
    dev = CUDA.deviceid(CUDA.device())
    lock(HANDLE_LOCK) do
        get!(HANDLES, dev) do
            r = Ref{Ptr{Cvoid}}(C_NULL)
            rc = ccall((:femb200_create, LIB), Cint, (Ref{Ptr{Cvoid}},), r)
            rc == OK || error("femb200_create failed (status $rc): no usable sm_100a device?")
            h = Handle(r[])
            finalizer(x -> ccall((:femb200_destroy, LIB), Cint, (Ptr{Cvoid},), x.ptr), h)
            h
        end
    end
end

function bind_stream(h::Handle)
    rc = ccall((:femb200_set_stream, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), h.ptr,
               reinterpret(Ptr{Cvoid}, CUDA.stream().handle))
    rc == OK || throw_status(h, rc)
    return h
end

last_error(h::Handle) = unsafe_string(ccall((:femb200_last_error, LIB), Cstring, (Ptr{Cvoid},), h.ptr))

# The library's messages are the reference's (DR.jl:332-335, :574-575, :711-712,
# utils.jl:155), so the error a caller sees is the one FEMTools would raise.
throw_status(h::Handle, rc) = error(last_error(h))

# ---- conversions ----------------------------------------------------------------

dptr(::Nothing) = C_NULL
dptr(x::CuArray) = reinterpret(Ptr{Cvoid}, pointer(x))
dtype_code(::Type{Float64}) = F64
dtype_code(::Type{Float32}) = F32
dtype_code(T) = throw(ArgumentError("libfemtools_b200 runs Float64 or Float32 states, got $T"))

pad16(t::Tuple, fill) = ntuple(i -> i <= length(t) ? Float64(t[i]) : Float64(fill), Val(MAX_PHASES))

function phase_layout(ph, nnodes, nels)
    ph isa CuArray{Int32} || throw(ArgumentError("phases must be a CuArray{Int32}"))
    ndims(ph) == 1 && length(ph) == nnodes && return PHASE_NODAL
    ndims(ph) == 2 && size(ph, 2) == nels && return size(ph, 1) == 1 ? PHASE_CELL : PHASE_ELEMENT_NODE
    throw(DimensionMismatch("phases of size $(size(ph)) fit neither nodes nor elements"))
end

# SymmetricTensor3D stores (xx, yy, zz, yz, xz, xy); the library reads the
# assembler order (xx, yy, zz, xy, xz, yz) (src/stokes/types/stokes_types.jl:316-318).
tensor_ptrs(::Nothing, D) = ntuple(_ -> C_NULL, Val(6))
tensor_ptrs(t, D) = D == 3 ?
    (dptr(t.xx), dptr(t.yy), dptr(t.zz), dptr(t.xy), dptr(t.xz), dptr(t.yz)) :
    (dptr(t.xx), dptr(t.yy), dptr(t.xy), C_NULL, C_NULL, C_NULL)

function field_layout(t, nq, nels, nnodes)
    t === nothing && return FIELD_NONE
    n = length(t.xx)
    n == nq * nels && return FIELD_IP
    n == nnodes && return FIELD_NODAL
    throw(DimensionMismatch("stress history of length $n is neither nq × nels nor nodal"))
end

vec3(f, D) = D == 3 ? (dptr(f.x), dptr(f.y), dptr(f.z)) : (dptr(f.x), dptr(f.y), C_NULL)

function material_c(dr::StokesDR, plastic, viscosity, scaling_viscosity)
    n = length(dr.η)
    eta = viscosity isa Tuple ? viscosity : dr.η
    pl = plastic isa DruckerPrager
    plastic === nothing || pl ||
        throw(ArgumentError("libfemtools_b200 solves DruckerPrager plasticity or none, got $(typeof(plastic))"))
    z = ntuple(_ -> 0.0, Val(MAX_PHASES))
    use_s = scaling_viscosity isa Tuple && scaling_viscosity !== eta
    g = ntuple(i -> i <= length(dr.g) ? Float64(dr.g[i]) : 0.0, Val(3))
    return StokesMaterialC(
        Int32(n), pad16(eta, 1), pad16(dr.ηb, 1), pad16(dr.G, Inf), pad16(dr.α, 0), pad16(dr.ρ0, 1),
        pad16(dr.K, Inf), g, Float64(dr.Tref), Int32(pl),
        pl ? pad16(plastic.cosϕ, 1) : z, pl ? pad16(plastic.sinϕ, 0) : z, pl ? pad16(plastic.sinΨ, 0) : z,
        pl ? pad16(plastic.C, 0) : z, pl ? pad16(plastic.η_reg, 0) : z, pl ? pad16(plastic.Kb, Inf) : z,
        Int32(use_s), use_s ? pad16(scaling_viscosity, 1) : z,
    )
end

function stokes_problem(dr::StokesDR{<:Any, D}, mesh::MixedMesh{D}, bc_v; plastic = nothing,
                        viscosity = dr.η, scaling_viscosity = viscosity, phases_v = dr.phases_v,
                        P_old = nothing, body_force = nothing) where {D}
    geo = mesh.geometry
    geo === nothing && throw(ArgumentError("mesh has no geometry cache; build it with MixedMesh(backend, …)"))
    nv, np = size(mesh.el2n, 1), size(mesh.DoFsP, 1)
    nq = size(geo.geo_P, 1)
    FP = eltype(dr.v.x)
    nels, nn, nP = mesh.nels, mesh.nnodes, mesh.nnodesP
    eta_ip = viscosity isa CuArray ? dptr(viscosity) : C_NULL
    bf = body_force === nothing ? ntuple(_ -> C_NULL, Val(3)) : vec3(body_force, D)
    bcd = ntuple(i -> i <= D ? dptr(bc_v[i].DoFs) : C_NULL, Val(3))
    bcv = ntuple(i -> i <= D ? dptr(bc_v[i].vals) : C_NULL, Val(3))
    bcn = ntuple(i -> i <= D ? Int64(length(bc_v[i].DoFs)) : Int64(0), Val(3))
    return StokesProblemC(
        Int32(D), Int32(nv), Int32(np), Int32(nq), dtype_code(FP), dtype_code(eltype(geo.geo_P)),
        Int64(nels), Int64(nn), Int64(nP),
        dptr(mesh.el2n), dptr(mesh.DoFsP), dptr(mesh.el2nP), dptr(geo.geo_v), dptr(geo.geo_P),
        vec3(dr.v, D), vec3(dr.∂v∂τ, D), vec3(dr.Rv, D), vec3(dr.Rv0, D), vec3(dr.∂Rv∂v, D), vec3(dr.PC_v, D),
        dptr(dr.P), dptr(dr.P0), dptr(dr.γP), dptr(dr.T), dptr(dr.T0), dptr(dr.Q), dptr(dr.Pf), dptr(dr.RP),
        dptr(dr.M_P), dptr(dr.Pnum),
        dptr(phases_v), phase_layout(phases_v, nn, nels),
        dptr(dr.phases_P), phase_layout(dr.phases_P, nP, nels),
        tensor_ptrs(dr.τ_old, D), field_layout(dr.τ_old, nq, nels, nn),
        tensor_ptrs(dr.τ, D),
        dptr(P_old), P_old === nothing ? FIELD_NONE : (length(P_old) == nq * nels ? FIELD_IP : FIELD_NODAL),
        eta_ip, bf, bcd, bcv, bcn,
        material_c(dr, plastic, viscosity, scaling_viscosity),
    )
end

function stokes_controls(dr; dt, pressure_factor = 50, tolerance = 1.0e-6, max_iterations = 50_000,
                         check_interval = 50, iterMax = 50_000, max_ph_iterations = 1000, rel_drop0 = 1.0e-2,
                         freeze_jacobian = nothing, finite_K = false, assemble_scaling = true,
                         throw_on_failure = true, precision = :fp64)
    precision in (:fp64, :mixed) || throw(ArgumentError("precision must be :fp64 or :mixed"))
    return StokesControlsC(
        Float64(dt), Float64(pressure_factor), Float64(tolerance), Int64(max_iterations), Int64(check_interval),
        Int64(iterMax), Int64(max_ph_iterations), Float64(rel_drop0),
        Int32(freeze_jacobian === nothing ? -1 : freeze_jacobian), Int32(finite_K), Int32(assemble_scaling),
        Int32(throw_on_failure), precision === :mixed ? PRECISION_MIXED : PRECISION_FP64,
        Float64(dr.CFL_v), Float64(dr.c_fact), Ptr{Float64}(C_NULL), Int64(0),
    )
end

stats_tuple(s::StokesStatsC) = (;
    converged = s.converged != 0, iter = Int(s.iter), iterations = Int(s.iter), itPH = Int(s.itPH),
    err = s.err, residual = s.err_abs, err_abs = s.err_abs, err_rel = s.err_rel, err_v = s.err_v, err_P = s.err_P,
    λmax = s.lambda_max, jacobian_assemblies = Int(s.jacobian_assemblies), reached_total_iter = s.reached_total_iter != 0,
    err_T = s.err_T, thermal_iterations = Int(s.thermal_iterations),
)

function thermal_problem(th::ThermalDiffusionDR, mesh, bc::DirichletBoundaryCondition; source_ip = nothing)
    geo = mesh.geometry
    nv = size(mesh.el2n, 1)
    nq = size(geo, 1)
    D = nv == 27 ? 3 : 2
    n = length(th.k)
    return ThermalProblemC(
        Int32(D), Int32(nv), Int32(nq), dtype_code(eltype(th.T)), dtype_code(eltype(th.T)),
        Int64(mesh.nels), Int64(mesh.nnodes),
        dptr(mesh.el2n), dptr(geo), dptr(th.T), dptr(th.T0), dptr(th.∂T∂τ), dptr(th.R), dptr(th.R0), dptr(th.∂R∂T),
        dptr(th.PC), dptr(th.P), dptr(th.source), dptr(source_ip),
        dptr(th.phases), phase_layout(th.phases, mesh.nnodes, mesh.nels),
        dptr(bc.DoFs), dptr(bc.vals), Int64(length(bc.DoFs)),
        Int32(n), pad16(th.k, 1), pad16(th.Cp, 1), pad16(th.ρ0, 1), pad16(th.α, 0), pad16(th.K, Inf),
        Float64(th.CFL), Float64(th.c_fact), Float64(th.ϵ),
    )
end

# ---- the solves -------------------------------------------------------------------

const CuStokesDR{D} = StokesDR{<:Any, D, <:Any, <:Any, <:CuArray}

function FEMTools.solve!(dr::CuStokesDR{D}, mesh::MixedMesh{D}, bc_v::NTuple{D, DirichletBoundaryCondition};
                         dt, pressure_factor = 50, viscosity = dr.η, scaling_viscosity = viscosity,
                         phases_v = dr.phases_v, plastic = nothing, finite_K = false, tolerance = 1.0e-6,
                         max_iterations = 50_000, check_interval = 50, throw_on_failure = true, workgroup = 256,
                         precision = :fp64, body_force = nothing, P_old = nothing, ordered_scatter = false,
                         kwargs...) where {D}
    if !ENABLED[]
        return invoke(FEMTools.solve!, Tuple{StokesDR{<:Any, D}, MixedMesh{D}, NTuple{D, DirichletBoundaryCondition}},
                      dr, mesh, bc_v; dt, pressure_factor, viscosity, scaling_viscosity, phases_v, plastic, finite_K,
                      tolerance, max_iterations, check_interval, throw_on_failure, workgroup, kwargs...)
    end
    h = bind_stream(handle())
    p = Ref(stokes_problem(dr, mesh, bc_v; plastic, viscosity, scaling_viscosity, phases_v, P_old, body_force))
    c = Ref(stokes_controls(dr; dt, pressure_factor, tolerance, max_iterations, check_interval, finite_K,
                            throw_on_failure, precision, kwargs...))
    st = Ref{StokesStatsC}()
    # ordered_scatter = true: a reproducible mixed-precision solve (colour-ordered scatter)
    ccall((:femb200_set_ordered_scatter, LIB), Cint, (Ptr{Cvoid}, Int32), h.ptr, Int32(ordered_scatter))
    rc = GC.@preserve dr mesh bc_v viscosity phases_v body_force P_old begin
        ccall((:femb200_solve_stokes, LIB), Cint,
              (Ptr{Cvoid}, Ref{StokesProblemC}, Ref{StokesControlsC}, Ref{StokesStatsC}), h.ptr, p, c, st)
    end
    ccall((:femb200_set_ordered_scatter, LIB), Cint, (Ptr{Cvoid}, Int32), h.ptr, Int32(0))
    rc == OK || throw_status(h, rc)
    return stats_tuple(st[])
end

function FEMTools.solve!(th::ThermalDiffusionDR{<:Any, <:CuArray}, mesh::Mesh, bc::DirichletBoundaryCondition;
                         dt, Tref = eltype(th.T)(273), tolerance = th.ϵ, max_iterations = 10_000,
                         check_interval = 100, throw_on_failure = true, kwargs...)
    if !ENABLED[]
        return invoke(FEMTools.solve!, Tuple{ThermalDiffusionDR, Mesh, DirichletBoundaryCondition}, th, mesh, bc;
                      dt, Tref, kwargs...)
    end
    h = bind_stream(handle())
    t = Ref(thermal_problem(th, mesh, bc))
    c = Ref(ThermalControlsC(Float64(dt), Float64(Tref), Float64(tolerance), Int64(max_iterations),
                             Int64(check_interval), Int32(throw_on_failure)))
    st = Ref{ThermalStatsC}()
    rc = GC.@preserve th mesh bc begin
        ccall((:femb200_solve_thermal, LIB), Cint,
              (Ptr{Cvoid}, Ref{ThermalProblemC}, Ref{ThermalControlsC}, Ref{ThermalStatsC}), h.ptr, t, c, st)
    end
    rc == OK || throw_status(h, rc)
    s = st[]
    return (; converged = s.converged != 0, iterations = Int(s.iterations), residual = s.residual)
end

function FEMTools.solve_coupled!(thermal::ThermalDiffusionDR{<:Any, <:CuArray}, stokes::CuStokesDR{D},
                                 thermal_mesh::Mesh, stokes_mesh::MixedMesh{D}, bc_T::DirichletBoundaryCondition,
                                 bc_v::NTuple{D, DirichletBoundaryCondition}; dt, Tref = eltype(thermal.T)(273),
                                 workgroup = 256, shear_heating = false, plastic = nothing, pressure_factor = 50,
                                 tolerance = 1.0e-6, max_iterations = 50_000, check_interval = 50,
                                 throw_on_failure = true, kwargs...) where {D}
    if !ENABLED[]
        return invoke(FEMTools.solve_coupled!,
                      Tuple{ThermalDiffusionDR, StokesDR{<:Any, D}, Mesh, MixedMesh{D}, DirichletBoundaryCondition,
                            NTuple{D, DirichletBoundaryCondition}},
                      thermal, stokes, thermal_mesh, stokes_mesh, bc_T, bc_v; dt, Tref, workgroup, shear_heating,
                      plastic, pressure_factor, tolerance, max_iterations, check_interval, throw_on_failure, kwargs...)
    end
    thermal_mesh.nnodes == stokes_mesh.nnodes ||
        throw(DimensionMismatch("thermal mesh nodes must match the Stokes velocity-node layout"))
    h = bind_stream(handle())
    t = Ref(thermal_problem(thermal, thermal_mesh, bc_T))
    p = Ref(stokes_problem(stokes, stokes_mesh, bc_v; plastic))
    c = Ref(stokes_controls(stokes; dt, pressure_factor, tolerance, max_iterations, check_interval,
                            throw_on_failure, kwargs...))
    nq = size(stokes_mesh.geometry.geo_P, 1)
    phi = shear_heating ? CUDA.zeros(eltype(stokes.v.x), nq * stokes_mesh.nels) : nothing
    st = Ref{StokesStatsC}()
    rc = GC.@preserve thermal stokes thermal_mesh stokes_mesh bc_T bc_v phi begin
        ccall((:femb200_solve_coupled, LIB), Cint,
              (Ptr{Cvoid}, Ref{ThermalProblemC}, Ref{StokesProblemC}, Ref{StokesControlsC}, Float64, Int32, Ptr{Cvoid},
               Ref{StokesStatsC}),
              h.ptr, t, p, c, Float64(Tref), Int32(shear_heating), dptr(phi), st)
    end
    rc == OK || throw_status(h, rc)
    return stats_tuple(st[])
end

end # module
