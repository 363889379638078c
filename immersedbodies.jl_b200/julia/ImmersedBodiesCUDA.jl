"""
    ImmersedBodiesCUDA

A drop-in `AbstractSolver` for ImmersedBodies.jl whose `advance!` runs on a B200
through `libibpm_b200.so` (C ABI: `include/ibpm_b200.h`).

    using ImmersedBodies, ImmersedBodiesCUDA
    solve(prob; t=1.0, solver_kw=(; gpu=true))   # the reference's solve, GPU solver
    solver = GpuCnabSolver(State(prob))          # or build it by hand
    solve!(solver; t=1.0)                        # ImmersedBodies' own driver loop

Host callbacks (`freestream_vel(t)`, each `MovingRigidBody`'s `motion(t)`, a
`MovingGrid`'s `motion(t)`) are evaluated here each step and passed to the
library as scalars; the library never calls back into Julia.  `state.index`,
`state.t` and `state.fb` are refreshed after every step; the full fields are
copied back by `getstate(solver)` / `sync!(solver)`.
"""
module ImmersedBodiesCUDA

using ImmersedBodies
using ImmersedBodies: State, Problem, CNAB, AbstractSolver, StaticBody, MovingRigidBody, StaticGrid,
    MovingGrid, n_panels, timestep, gridstep, inc_time_index!, set_time_index!, update_vars!
import ImmersedBodies: advance!, getstate, create_solver

export GpuCnabSolver, sync!, level_vorticity, level_x_velocity, level_y_velocity, set_warm_start!,
    set_rebuild_transform!

const libibpm = get(ENV, "IBPM_B200_LIB", joinpath(@__DIR__, "..", "lib", "libibpm_b200.so"))

const IBPM_OK = Cint(0)

struct IbpmProblem
    nx::Int32; ny::Int32; nlevel::Int32
    h::Float64; x0::Float64; y0::Float64
    Re::Float64; dt::Float64
    npanel::Int32; nbody::Int32
    body_kind::Ptr{Int32}; body_start::Ptr{Int32}
    body_xb::Ptr{Float64}; body_ds::Ptr{Float64}
    grid_moving::Int32
end

struct IbpmOptions
    precision::Int32; device::Int32; cg_maxiter::Int32
    cg_reltol::Float64; cg_abstol::Float64
end

struct IbpmStepParams
    freestream::NTuple{2,Float64}
    grid_motion::NTuple{6,Float64}
    body_motion::Ptr{Float64}
end

mutable struct IbpmStateView
    index::Int64; t0::Float64
    q::Ptr{Float64}; q0::Ptr{Float64}; gamma::Ptr{Float64}; psi::Ptr{Float64}
    nonlin1::Ptr{Float64}; nonlin2::Ptr{Float64}
    xb::Ptr{Float64}; ds::Ptr{Float64}; ub::Ptr{Float64}; fbt::Ptr{Float64}
    freestream::NTuple{2,Float64}
end

_err(h) = unsafe_string(ccall((:ibpm_last_error, libibpm), Cstring, (Ptr{Cvoid},), h))

function _check(h, rc)
    rc < 0 && error(_err(h))   # e.g. "Panel index=... outside allowed region" (coupling.jl:40)
    rc
end

mutable struct GpuCnabSolver <: AbstractSolver
    state::State{CNAB}
    handle::Ptr{Cvoid}
    motion::Matrix{Float64}   # nbody x 6, row-major when passed (transposed copy)
    moving::Vector{Bool}
    stale::Bool
end

function GpuCnabSolver(state::State{CNAB}; cg=(), device=0, fftw=())  # fftw: the CPU solver's option, unused
    prob = state.prob
    bodies = prob.bodies
    parts = bodies.preset
    kinds = Int32[p.body isa MovingRigidBody ? 1 : 0 for p in parts]
    starts = Int32[[first(p.panel_range) - 1 for p in parts]; n_panels(bodies)]
    xb = reduce(vcat, [ImmersedBodies.bodypanels(p.body).xb for p in parts])
    ds = reduce(vcat, [ImmersedBodies.bodypanels(p.body).ds for p in parts])
    grid = prob.fluid.grid
    base = grid.base
    opt = IbpmOptions(0, device, get(cg, :maxiter, 5000), get(cg, :reltol, 1e-12), get(cg, :abstol, 0.0))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve kinds starts xb ds begin
        p = IbpmProblem(base.n[1], base.n[2], grid.nlevel, base.h, base.x0[1], base.x0[2],
            prob.fluid.Re, timestep(prob), n_panels(bodies), length(parts),
            pointer(kinds), pointer(starts), pointer(xb), pointer(ds),
            prob.fluid.grid_motion isa MovingGrid ? 1 : 0)
        rc = ccall((:ibpm_create, libibpm), Cint, (Ref{IbpmProblem}, Ref{IbpmOptions}, Ref{Ptr{Cvoid}}),
            p, opt, h)
        rc == IBPM_OK || error(_err(C_NULL))
    end
    # _init_body_motion!: static bodies take their reference panels
    for part in parts
        if part.body isa StaticBody
            state.panels.xb[part.panel_range, :] .= part.body.panels.xb
            state.panels.ds[part.panel_range] .= part.body.panels.ds
            state.panels.ub[part.panel_range, :] .= 0
        end
    end
    solver = GpuCnabSolver(state, h[], zeros(6, length(parts)), [k == 1 for k in kinds], false)
    finalizer(s -> ccall((:ibpm_destroy, libibpm), Cvoid, (Ptr{Cvoid},), s.handle), solver)
    _upload!(solver)
    solver
end

create_solver(state::State{CNAB}, ::Val{:gpu}; kw...) = GpuCnabSolver(state; kw...)

# solve(prob; solver_kw) builds its solver with create_solver(State(prob); solver_kw...)
# (src/solver.jl:71-74, 152), and Julia does not dispatch on keywords.  At load time
# the reference's create_solver(::State{CNAB}; kw...) is therefore replaced by one
# that takes a `gpu` keyword: gpu=true builds a GpuCnabSolver (keywords cg, device),
# gpu=false (the default) builds the reference's CnabSolver exactly as before.  The
# replacement runs in __init__, not at precompile time, where overwriting another
# module's method is not allowed.
function __init__()
    Core.eval(ImmersedBodies, quote
        create_solver(state::State{CNAB}; gpu::Bool=false, kw...) =
            gpu ? $(GpuCnabSolver)(state; kw...) : CnabSolver(state; kw...)
    end)
    nothing
end

function _view(s::State)
    IbpmStateView(s.index, s.t0, pointer(s.q), pointer(s.q0), pointer(s.Γ), pointer(s.ψ),
        pointer(s.nonlin[1]), pointer(s.nonlin[2]), pointer(s.panels.xb), pointer(s.panels.ds),
        pointer(s.panels.ub), pointer(s.F̃b), Tuple(s.freestream_vel))
end

function _upload!(solver::GpuCnabSolver)
    s = solver.state
    GC.@preserve s begin
        v = _view(s)
        _check(solver.handle, ccall((:ibpm_set_state, libibpm), Cint, (Ptr{Cvoid}, Ref{IbpmStateView}),
            solver.handle, v))
    end
end

"""
    sync!(solver::GpuCnabSolver)

Copy the full device state (q, q0, Γ, ψ, nonlin, panels, F̃b) into `solver.state`.
"""
function sync!(solver::GpuCnabSolver)
    s = solver.state
    GC.@preserve s begin
        v = _view(s)
        _check(solver.handle, ccall((:ibpm_get_state, libibpm), Cint, (Ptr{Cvoid}, Ref{IbpmStateView}),
            solver.handle, v))
    end
    update_vars!(s)
    solver.stale = false
    s
end

getstate(solver::GpuCnabSolver) = solver.stale ? sync!(solver) : solver.state

function advance!(solver::GpuCnabSolver)
    state = solver.state
    prob = state.prob
    inc_time_index!(state)
    t = state.t
    state.freestream_vel = prob.fluid.freestream_vel(t)
    gm = prob.fluid.grid_motion
    g = if gm isa MovingGrid
        m = gm(t)
        (m.center[1], m.center[2], m.vel[1], m.vel[2], m.angle, m.angular_vel)
    else
        (0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    end
    for (b, part) in enumerate(prob.bodies.preset)
        if solver.moving[b]
            m = part.body.motion(t)
            solver.motion[:, b] .= (m.pos[1], m.pos[2], m.vel[1], m.vel[2], m.angle, m.angular_vel)
        end
    end
    motion = solver.motion
    GC.@preserve motion begin
        prm = IbpmStepParams(Tuple(state.freestream_vel), g, any(solver.moving) ? pointer(motion) : C_NULL)
        rc = ccall((:ibpm_advance, libibpm), Cint, (Ptr{Cvoid}, Int64, Ref{IbpmStepParams}),
            solver.handle, 1, prm)
        rc < 0 && set_time_index!(state, state.index - 1)
        _check(solver.handle, rc)
    end
    fb = state.fb
    GC.@preserve fb _check(solver.handle, ccall((:ibpm_get_forces, libibpm), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}), solver.handle, pointer(fb), C_NULL))
    solver.stale = true
    nothing
end

# One level of the reference's output fields (vorticity!, x_velocity!, y_velocity!,
# src/problem.jl:715-866), computed on the device; only that level is copied back.
function _level_field(solver::GpuCnabSolver, field::Integer, level::Integer, dims)
    out = Matrix{Float64}(undef, dims...)
    GC.@preserve out _check(solver.handle, ccall((:ibpm_get_field, libibpm), Cint,
        (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}), solver.handle, field, level, pointer(out)))
    out
end
_base_n(solver) = solver.state.prob.fluid.grid.base.n
level_vorticity(solver::GpuCnabSolver, level::Integer=1) =
    _level_field(solver, 0, level, (_base_n(solver)[1] - 1, _base_n(solver)[2] - 1))
level_x_velocity(solver::GpuCnabSolver, level::Integer=1) =
    _level_field(solver, 1, level, (_base_n(solver)[1] + 1, _base_n(solver)[2]))
level_y_velocity(solver::GpuCnabSolver, level::Integer=1) =
    _level_field(solver, 2, level, (_base_n(solver)[1], _base_n(solver)[2] + 1))

# CG initial guess for moving bodies: :previous (the reference's start), :extrapolated,
# :projected over the last `depth` solutions (1..16), or :direct (B^-1 b with B
# assembled and inverted on the GPU every `depth` steps, FP64 only); plain CG then
# runs to the configured tolerance.  :preconditioned is :direct with CG
# preconditioned by that inverse (not the reference's iteration; same stopping
# rule); :preconditioned_extrapolated also starts CG from the stale error
# extrapolated over the last steps.  (The learned mode needs a network made with
# ibpm_net_*.)
function set_warm_start!(solver::GpuCnabSolver, mode::Symbol=:projected; depth::Integer=16)
    m = Dict(:previous => 0, :extrapolated => 2, :projected => 3, :direct => 4, :preconditioned => 5,
        :preconditioned_extrapolated => 6)[mode]
    _check(solver.handle, ccall((:ibpm_set_warm_start, libibpm), Cint, (Ptr{Cvoid}, Int32, Ptr{Cvoid}, Int32),
        solver.handle, m, C_NULL, depth))
    solver
end

# How the preconditioned modes assemble the B they invert: 0 with the step's FP64
# transforms, 3 (or 1) with dense DST-I passes on the tensor cores of split-BF16
# (or BF16) operands; nx = ny in {256, 512}.
function set_rebuild_transform!(solver::GpuCnabSolver, products::Integer=3)
    _check(solver.handle, ccall((:ibpm_set_rebuild_transform, libibpm), Cint, (Ptr{Cvoid}, Int32),
        solver.handle, products))
    solver
end

end # module
