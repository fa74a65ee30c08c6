"""
    SymCodeB200

Julia binding of `libsymcode.so` (C ABI in `include/symcode.h`): the B200 path
behind SymmetryCode.jl's solver and closure calls.  Each method takes the same
arguments as the reference function it replaces and operates on `CuArray`s of
the reference layout (`Complex{T}` of size `(n÷2+1, n, n)`, column-major).

This file is not executed in this repository's test suite (no Julia toolchain
in the build environment); the same entry points are exercised from Python.
"""
module SymCodeB200

using CUDA
using ChainRulesCore  # a dependency of Zygote, which the reference already uses (Project.toml)
using JLD2            # the reference's own field-file format (src/solver.jl:76-86, src/data.jl:200-216)

const LIB = get(ENV, "SYMCODE_LIB", joinpath(@__DIR__, "..", "libsymcode.so"))

struct SCForcing
    enabled::Cint
    eps::Cdouble
end

function check(status::Cint)
    status == 0 && return nothing
    msg = unsafe_string(ccall((:sc_last_error_string, LIB), Cstring, ()))
    error("libsymcode error $(status): $(msg)")
end

"Device plan standing in for `Grid{D}(; l, n)` + `getcache(grid)` (src/solver.jl:147, :956)."
mutable struct Plan
    ptr::Ptr{Cvoid}
    D::Int
    n::Int
    l::Float64
    T::DataType
end

function Plan(D::Int, n::Int, l::Real, ::Type{T}) where {T <: Union{Float32, Float64}}
    ref = Ref{Ptr{Cvoid}}(C_NULL)
    ws = Ref{Csize_t}(0)
    check(ccall((:sc_plan_create, LIB), Cint, (Ptr{Ptr{Cvoid}}, Cint, Cint, Cdouble, Cint, Ptr{Csize_t}),
        ref, D, n, l, T === Float32 ? 0 : 1, ws))
    p = Plan(ref[], D, n, Float64(l), T)
    finalizer(p -> ccall((:sc_plan_destroy, LIB), Cint, (Ptr{Cvoid},), p.ptr), p)
    return p
end

stream() = CUDA.stream().handle
ptrs(u) = [Base.unsafe_convert(CuPtr{Cvoid}, pointer(c)) for c in u]

"`convectiondiffusion!(du, u, grid, cache; visc)` (src/solver.jl:949)."
function convectiondiffusion!(du, u, p::Plan; visc)
    check(ccall((:sc_rhs, LIB), Cint, (Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Ptr{CuPtr{Cvoid}}, Cdouble, Ptr{Cvoid}),
        p.ptr, ptrs(u), ptrs(du), visc, stream()))
    return nothing
end

"`wray3!(convectiondiffusion!, u, Δt, grid, cache; visc)` (src/solver.jl:968)."
function wray3!(u, Δt, p::Plan; visc)
    check(ccall((:sc_wray3_step, LIB), Cint, (Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Cdouble, Cdouble, Ptr{Cvoid}),
        p.ptr, ptrs(u), Δt, visc, stream()))
    return u
end

"RK4 steps with optional linear band forcing at injection rate `eps` (new)."
function rk4!(u, Δt, p::Plan; visc, nsteps = 1, eps = nothing)
    f = Ref(SCForcing(isnothing(eps) ? 0 : 1, isnothing(eps) ? 0.0 : eps))
    check(ccall((:sc_rk4_steps, LIB), Cint,
        (Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Cdouble, Cdouble, Cint, Ptr{SCForcing}, Ptr{Cvoid}),
        p.ptr, ptrs(u), Δt, visc, nsteps, f, stream()))
    return u
end

"`sfs!(; τ, ubar, u, g_dns, g_les, Δ)` (src/data.jl:625) for several widths at once."
function sfs!(ubars, τs, u, dns::Plan, les::Plan, Δs)
    d = Cdouble[isnothing(x) ? -1.0 : x for x in Δs]
    check(ccall((:sc_filter_sfs, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Ptr{Cdouble}, Cint, Ptr{CuPtr{Cvoid}}, Ptr{CuPtr{Cvoid}}, Ptr{Cvoid}),
        dns.ptr, les.ptr, ptrs(u), d, length(d), reduce(vcat, ptrs.(ubars)), reduce(vcat, ptrs.(τs)), stream()))
    return nothing
end

"`filter_reynolds(ubar, g_les, visc, Δ)` (src/solver.jl:768-774)."
function filter_reynolds(ubar, les::Plan, visc, Δ)
    re = Ref{Cdouble}(0)
    check(ccall((:sc_filter_reynolds, LIB), Cint, (Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Cdouble, Cdouble, Ptr{Cdouble},
        Ptr{Cvoid}), les.ptr, ptrs(ubar), visc, Δ, re, stream()))
    return re[]
end

"""
    FieldSeries(nfilters)

Host-side accumulator of the filtered-field series that `create_data`
(src/data.jl:170-197) writes per filter width: `inputs[k]` (ū per snapshot),
`outputs[k]` (τ per snapshot), `redelta[k]` (Re_Δ per snapshot), with ū and τ
as NamedTuples of host `Array{Complex{T},3}` in the reference's spectral layout
and component names, so `fieldsfile` data written from this path loads with
the reference's own readers (src/experiment.jl:203-207, src/data.jl:656-803).
"""
struct FieldSeries
    inputs::Vector{Vector{Any}}
    outputs::Vector{Vector{Any}}
    redelta::Vector{Vector{Float64}}
end
FieldSeries(nfilters::Integer) = FieldSeries([Any[] for _ in 1:nfilters], [Any[] for _ in 1:nfilters],
                                             [Float64[] for _ in 1:nfilters])

"""
    push_snapshot!(series, u, dns, les, Δs, visc)

One snapshot of `create_data`'s filter loop (src/data.jl:185-192): `sfs!` of the
DNS field `u` at every Δ in one call (the DNS products are shared), then the
device->host copies `map(Array, ubar)` / `map(Array, τ)` and `filter_reynolds`.
"""
function push_snapshot!(series::FieldSeries, u, dns::Plan, les::Plan, Δs, visc)
    T = les.T
    sz = (les.n ÷ 2 + 1, ntuple(_ -> les.n, les.D - 1)...)
    nt = les.D == 3 ? 6 : 3
    ubars = [[CUDA.zeros(Complex{T}, sz) for _ in 1:les.D] for _ in Δs]
    τs = [[CUDA.zeros(Complex{T}, sz) for _ in 1:nt] for _ in Δs]
    sfs!(ubars, τs, u, dns, les, Δs)
    vnames = les.D == 3 ? (:x, :y, :z) : (:x, :y)
    tnames = les.D == 3 ? (:xx, :yy, :zz, :xy, :yz, :zx) : (:xx, :yy, :xy)
    for (k, Δ) in enumerate(Δs)
        push!(series.inputs[k], NamedTuple{vnames}(Tuple(map(Array, ubars[k]))))
        push!(series.outputs[k], NamedTuple{tnames}(Tuple(map(Array, τs[k]))))
        push!(series.redelta[k], filter_reynolds(ubars[k], les, visc, Δ))
    end
    return series
end

"""
    save_fieldsfile(file, series, k; Δ, Δ_factor, visc)

Write filter `k` of `series` as the reference's `fieldsfile` (src/data.jl:207-211):
`jldsave` to a temporary file and `mv` over `file` (the atomic write of
`jldsave_atomic`, src/solver.jl:76-86), with the keys `inputs`, `outputs`,
`redelta`, `Δ`, `Δ_factor`, `visc`.
"""
function save_fieldsfile(file, series::FieldSeries, k::Integer; Δ, Δ_factor, visc)
    tmp = tempname(dirname(file); cleanup = false)
    try
        jldsave(tmp; inputs = [x for x in series.inputs[k]], outputs = [x for x in series.outputs[k]],
                redelta = series.redelta[k], Δ, Δ_factor, visc)
        mv(tmp, file; force = true)
    catch
        isfile(tmp) && rm(tmp; force = true)
        rethrow()
    end
    return file
end

"""
    load_fieldsfile(file) -> (; inputs, outputs, redelta, Δ, Δ_factor, visc)

Read a `fieldsfile` (written by the reference or by `save_fieldsfile`) back;
`CuArray.(values(inputs[i]))` gives the device fields for this library's calls.
"""
load_fieldsfile(file) = (; (Symbol(k) => v for (k, v) in JLD2.load(file))...)

"A closure `model(u, G)` bound to a plan (`create_clark`, `create_dynamic_smagorinsky`, ...)."
mutable struct Closure
    ptr::Ptr{Cvoid}
    plan::Plan
end

function Closure(p::Plan, kind::Integer, Δ::Real, params::Vector{Float64} = Float64[])
    ref = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:sc_closure_create, LIB), Cint, (Ptr{Ptr{Cvoid}}, Ptr{Cvoid}, Cint, Cdouble, Ptr{Cdouble}, Cint),
        ref, p.ptr, kind, Δ, params, length(params)))
    c = Closure(ref[], p)
    finalizer(c -> ccall((:sc_closure_destroy, LIB), Cint, (Ptr{Cvoid},), c.ptr), c)
    return c
end
create_clark(Δ, p) = Closure(p, 1, Δ)
create_smagorinsky(CS, Δ, p) = Closure(p, 2, Δ, [Float64(CS)])
create_verstappen(C, Δ, p) = Closure(p, 3, Δ, [Float64(C)])
create_dynamic_smagorinsky(Δ, p) = Closure(p, 4, Δ)
create_bardina(s, Δ, p) = Closure(p, 5, Δ, [Float64(s)])

"`les!(du, u, grid, cache; model, visc)` (src/les.jl:4)."
function les!(du, u, p::Plan; model::Union{Nothing, Closure}, visc)
    m = isnothing(model) ? C_NULL : model.ptr
    check(ccall((:sc_les_rhs, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Ptr{CuPtr{Cvoid}}, Cdouble, Ptr{Cvoid}),
        p.ptr, m, ptrs(u), ptrs(du), visc, stream()))
    return nothing
end

"`energy(u)` (src/solver.jl:643), FP64 on the device."
function energy(u, p::Plan)
    e = Ref{Cdouble}(0)
    check(ccall((:sc_energy, LIB), Cint, (Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Ptr{Cdouble}, Ptr{Cvoid}),
        p.ptr, ptrs(u), e, stream()))
    return e[]
end

"`propose_timestep(u, grid, visc, cache)` (src/solver.jl:931-947), without the `cfl` factor."
function propose_timestep(u, p::Plan, visc)
    dt = Ref{Cdouble}(0)
    check(ccall((:sc_propose_timestep, LIB), Cint, (Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Cdouble, Ptr{Cdouble}, Ptr{Cvoid}),
        p.ptr, ptrs(u), visc, dt, stream()))
    return dt[]
end

"`spectrum(u, grid)` (src/solver.jl:693-699) on shells 1..nshell."
function spectrum(u, p::Plan, nshell::Integer)
    s = zeros(Cdouble, nshell)
    check(ccall((:sc_spectrum, LIB), Cint, (Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Cint, Ptr{Cdouble}, Ptr{Cvoid}),
        p.ptr, ptrs(u), nshell, s, stream()))
    return s
end

"""
CNN closure (new): `ws[l]`, `bs[l]` in PyTorch conv3d order (Cout, Cin, 3, 3, 3),
flattened column-major as Julia stores `permutedims(w, (5, 4, 3, 2, 1))`.
`tensorcores = true` selects the tcgen05 BF16 network (FP32 plans, n = 64 or 128);
`split = true` (tensor cores only) evaluates every convolution as three passes
over hi/lo operand parts (`SC_CLOPT_CNN_SPLIT`), about FP32 accuracy.
"""
function create_cnn(Δ, visc, p::Plan, ws::Vector{Vector{Float32}}, bs::Vector{Vector{Float32}};
                    mu = 0.0, sigma = 1.0, tensorcores = true, split = false)
    ref = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve ws bs begin
        wp = [pointer(w) for w in ws]
        bp = [pointer(b) for b in bs]
        f = tensorcores ? :sc_cnn_closure_create : :sc_cnn_fp_closure_create
        check(ccall((f, LIB), Cint,
            (Ptr{Ptr{Cvoid}}, Ptr{Cvoid}, Cdouble, Cdouble, Ptr{Ptr{Float32}}, Ptr{Ptr{Float32}}, Cdouble, Cdouble),
            ref, p.ptr, Δ, visc, wp, bp, mu, sigma))
    end
    c = Closure(ref[], p)
    finalizer(c -> ccall((:sc_closure_destroy, LIB), Cint, (Ptr{Cvoid},), c.ptr), c)
    split && set_option(c, SC_CLOPT_CNN_SPLIT, 1)
    return c
end

const SC_CLOPT_CNN_SPLIT = Cint(1)

"Closure options (`sc_closure_set_option`): `SC_CLOPT_CNN_SPLIT` => 0 | 1."
set_option(c::Closure, option::Integer, value::Integer) =
    check(ccall((:sc_closure_set_option, LIB), Cint, (Ptr{Cvoid}, Cint, Clonglong), c.ptr, option, value))

"""
Pointwise learned closures: `fullchain(setup, mlp(...))` (`kind = :mlp`) and `tbnn`
(`kind = :tbnn`).  `ws[l]` is the layer's `(c_in, c_out)` PointwiseConv weight
(Julia memory order), `bs[l]` its bias (absent for the last layer).
"""
function create_pointwise(kind::Symbol, Δ, visc, p::Plan, ws::Vector{Matrix{Float64}}, bs::Vector{Vector{Float64}};
                          use_redelta = false, mu = 0.0, sigma = 1.0)
    widths = Cint[size(ws[1], 1); [size(w, 2) for w in ws]]
    θ = Float64[]
    for (l, w) in enumerate(ws)
        append!(θ, vec(w))
        l < length(ws) && append!(θ, bs[l])
    end
    f = kind === :tbnn ? :sc_tbnn_closure_create : :sc_mlp_closure_create
    ref = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((f, LIB), Cint,
        (Ptr{Ptr{Cvoid}}, Ptr{Cvoid}, Cdouble, Cdouble, Cint, Ptr{Cint}, Ptr{Cdouble}, Cint, Cdouble, Cdouble),
        ref, p.ptr, Δ, visc, length(ws), widths, θ, use_redelta, mu, sigma))
    c = Closure(ref[], p)
    finalizer(c -> ccall((:sc_closure_destroy, LIB), Cint, (Ptr{Cvoid},), c.ptr), c)
    return c
end

"The a-posteriori reductions of `solve_les!` (src/les.jl:94-148) for one LES state."
function les_diagnostics(u, p::Plan; model::Union{Nothing, Closure} = nothing, uref = nothing, visc, nshell)
    out = zeros(Cdouble, 4)
    spec = zeros(Cdouble, nshell)
    tr = zeros(Cdouble, nshell)
    m = isnothing(model) ? C_NULL : model.ptr
    r = isnothing(uref) ? Ptr{CuPtr{Cvoid}}(C_NULL) : ptrs(uref)
    check(ccall((:sc_les_diagnostics, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Ptr{CuPtr{Cvoid}}, Cdouble, Cint, Ptr{Cdouble}, Ptr{Cdouble},
         Ptr{Cdouble}, Ptr{Cvoid}),
        p.ptr, m, ptrs(u), r, visc, nshell, out, spec, tr, stream()))
    return (; e_post = out[1], ke = out[2], eps_visc = out[3], eps_sfs = out[4], spectrum = spec, transfer = tr)
end

"The CNN's flat parameter vector θ (weights then biases per layer)."
function set_params!(c::Closure, θ::Vector{Float64})
    check(ccall((:sc_closure_set_params, LIB), Cint, (Ptr{Cvoid}, Ptr{Cdouble}), c.ptr, θ))
    return c
end
function num_params(c::Closure)
    n = Ref{Clonglong}(0)
    check(ccall((:sc_closure_num_params, LIB), Cint, (Ptr{Cvoid}, Ptr{Clonglong}), c.ptr, n))
    return Int(n[])
end

"Trajectory of `nsteps` RK4 steps with closure `c` (device bytes, compact states)."
function rollout_record(c::Closure, u0, p::Plan; Δt, visc, nsteps)
    nb = ccall((:sc_rollout_traj_bytes, LIB), Csize_t, (Ptr{Cvoid}, Cint), p.ptr, nsteps)
    traj = CuArray{UInt8}(undef, nb)
    check(ccall((:sc_rollout_record, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, Cdouble, Cdouble, Cint, CuPtr{Cvoid}, Ptr{Cvoid}),
        p.ptr, c.ptr, ptrs(u0), Δt, visc, nsteps, pointer(traj), stream()))
    return traj
end

"(loss, dloss/dθ) of the trajectory MSE against `traj` by the hand-written adjoint."
function rollout_adjoint(c::Closure, u0, traj, p::Plan; Δt, visc, nsteps, ckpt_every = 5)
    loss = Ref{Cdouble}(0)
    grad = zeros(Cdouble, num_params(c))
    check(ccall((:sc_rollout_adjoint, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, CuPtr{Cvoid}, Cdouble, Cdouble, Cint, Cint, Ptr{Cdouble},
         Ptr{Cdouble}, Ptr{Cvoid}),
        p.ptr, c.ptr, ptrs(u0), pointer(traj), Δt, visc, nsteps, ckpt_every, loss, grad, stream()))
    return loss[], grad
end

"""
    rollout_loss(θ, c, u0, traj, p; Δt, visc, nsteps, ckpt_every = 5)

Trajectory-MSE loss L = 1/nsteps Σ_s ⟨u_s - u*_s, u_s - u*_s⟩ of an RK4 LES
rollout from `u0` with closure `c` at parameters `θ` against the target
trajectory `traj` (`rollout_record`).  Zygote differentiates it through the
`rrule` below, whose pullback is the hand-written adjoint
(`sc_rollout_adjoint`: RK4 stages recomputed from checkpoints every
`ckpt_every` steps) instead of tracing the solver (the reference's in-place
KernelAbstractions kernels, src/solver.jl:434-521, are not differentiable by
Zygote).
"""
function rollout_loss(θ::AbstractVector{<:Real}, c::Closure, u0, traj, p::Plan; Δt, visc, nsteps,
                      ckpt_every = 5)
    set_params!(c, Vector{Float64}(θ))
    loss = Ref{Cdouble}(0)
    check(ccall((:sc_rollout_loss, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{CuPtr{Cvoid}}, CuPtr{Cvoid}, Cdouble, Cdouble, Cint, Ptr{Cdouble}, Ptr{Cvoid}),
        p.ptr, c.ptr, ptrs(u0), pointer(traj), Δt, visc, nsteps, loss, stream()))
    return loss[]
end

# Only θ is differentiated: the initial state, the target trajectory, the
# closure object and the plan get NoTangent (the C ABI returns dL/dθ only).
function ChainRulesCore.rrule(::typeof(rollout_loss), θ::AbstractVector{<:Real}, c::Closure, u0, traj, p::Plan;
                              Δt, visc, nsteps, ckpt_every = 5)
    set_params!(c, Vector{Float64}(θ))
    loss, grad = rollout_adjoint(c, u0, traj, p; Δt, visc, nsteps, ckpt_every)
    function rollout_loss_pullback(ȳ)
        dθ = ProjectTo(θ)(unthunk(ȳ) .* grad)
        return (NoTangent(), dθ, NoTangent(), NoTangent(), NoTangent(), NoTangent())
    end
    return loss, rollout_loss_pullback
end

end # module
