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
`tensorcores = true` selects the tcgen05 BF16 network (FP32 plans, n = 64 or 128).
"""
function create_cnn(Δ, visc, p::Plan, ws::Vector{Vector{Float32}}, bs::Vector{Vector{Float32}};
                    mu = 0.0, sigma = 1.0, tensorcores = true)
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
    return c
end

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

end # module
