# FlexibleFMMB200: the drop-in of FlexibleFMM.jl's FMM entry points onto libfmmb (sm_100a),
# through `ccall` into the C ABI of include/fmmb.h.
#
#   using FlexibleFMM, FlexibleFMMB200
#   m = SphericalHarmonics(Laplace3D(); p=10)
#   f = FlexibleFMMB200.FMM(m, points; ppl=64, bbox=(SVector(0.0, 0.0, 0.0), 1.0))
#   st = FlexibleFMMB200.build_expansions(f, points, τ)                 # src/fmm.jl:306-314
#   u = FlexibleFMMB200.evaluate_at_sources(f, st)                      # src/evaluate.jl:111-132
#   g = FlexibleFMMB200.evaluate(f, st, targets; output=Gradient())     # src/evaluate.jl:81-102
#
# The argument meanings and the exceptions are the reference's: status 1 → ArgumentError,
# 2 → DimensionMismatch. Points are `Vector{SVector{3,Float64}}` (their memory is the 3 × N
# interleaved array the ABI takes); outputs come back in the original order.
module FlexibleFMMB200

using FlexibleFMM: FlexibleFMM, SphericalHarmonics, StokesHarmonics, CubeKernelIndependent, KernelIndependent,
    Laplace3D, Laplace2D, Yukawa3D, Stokeslet3D, Potential, Gradient, Pressure, Dipole
using StaticArrays: SVector, SMatrix

const libfmmb = get(ENV, "FMMB_LIB", joinpath(@__DIR__, "..", "libfmmb.so"))

const FMMB_PRECISION_FP64 = Cint(0)
const FMMB_PRECISION_MIXED = Cint(1)
const FMMB_OUTPUT_POTENTIAL = Cint(1)
const FMMB_OUTPUT_GRADIENT = Cint(2)

struct MethodDesc
    method::Int32
    kernel::Int32
    p::Int32
    reserved::Int32
    tol::Float64
    kappa::Float64
    pc::Int32
    reserved2::Int32
    d::Float64
    pinv_rtol::Float64
end

struct TreeOpts
    ppl::Int32
    max_levels::Int32
    has_bbox::Int32
    reserved::Int32
    origin::NTuple{3,Float64}
    width::Float64
end

function check(rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:fmmb_last_error, libfmmb), Cstring, ()))
    rc == 1 && throw(ArgumentError(msg))
    rc == 2 && throw(DimensionMismatch(msg))
    error("fmmb error $rc: $msg")
end

mutable struct Context
    h::Ptr{Cvoid}
    function Context(device::Integer=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:fmmb_ctx_create, libfmmb), Cint, (Cint, Ref{Ptr{Cvoid}}), device, r))
        c = new(r[])
        finalizer(x -> ccall((:fmmb_ctx_destroy, libfmmb), Cint, (Ptr{Cvoid},), x.h), c)
    end
end
const DEFAULT_CONTEXT = Ref{Union{Nothing,Context}}(nothing)
default_context() = something(DEFAULT_CONTEXT[], (DEFAULT_CONTEXT[] = Context(0)))

"""
    OperatorCache(method)  (src/operators/cache.jl:19-22)
"""
const DeviceMethod = Union{SphericalHarmonics,StokesHarmonics,CubeKernelIndependent{3},KernelIndependent}
_kernel_id(m::SphericalHarmonics) = m.kernel isa Laplace3D ? Int32(1) : m.kernel isa Yukawa3D ? Int32(2) :
    throw(ArgumentError("the device method is written for Laplace3D and Yukawa3D"))
_kappa(m::SphericalHarmonics) = m.kernel isa Yukawa3D ? Float64(m.kernel.k) : 0.0
_kappa(m::StokesHarmonics) = 0.0
_kernel_id(m::StokesHarmonics) = m.kernel isa Stokeslet3D ? Int32(3) :
    throw(ArgumentError("the device Stokes method is written for Stokeslet3D"))

_method_desc(m::Union{SphericalHarmonics,StokesHarmonics}) =
    MethodDesc(1, _kernel_id(m), Int32(m.p), 0, m isa SphericalHarmonics ? m.tol : 0.0, _kappa(m), 0, 0, 0.0, 0.0)
# CubeKernelIndependent{3}(Laplace3D(); p, pc, d, pinv_rtol): the spectral-M2L method on cube surfaces
_method_desc(m::CubeKernelIndependent{3}) = m.kernel isa Laplace3D ?
    MethodDesc(2, 1, Int32(m.p), 0, 0.0, 0.0, Int32(m.pc), 0, Float64(m.d), Float64(m.pinv_rtol)) :
    throw(ArgumentError("the device cube KI method is written for Laplace3D"))

# KernelIndependent(Laplace2D(); nequiv, pinv_rtol): the 2D circle method; the ABI takes its points as
# 3 × N with z = 0 (`embed2`) and a bbox whose z origin is −width/2
_method_desc(m::KernelIndependent) = m.kernel isa Laplace2D ?
    MethodDesc(3, 4, Int32(m.nequiv), 0, 0.0, 0.0, 0, 0, 0.0, Float64(m.pinv_rtol)) :
    throw(ArgumentError("the device circle KI method is written for Laplace2D"))
embed2(pts::AbstractVector{SVector{2,Float64}}) = [SVector(p[1], p[2], 0.0) for p in pts]

mutable struct OperatorCache
    method::DeviceMethod
    ctx::Context
    h::Ptr{Cvoid}
    function OperatorCache(m::DeviceMethod; ctx::Context=default_context())
        d = Ref(_method_desc(m))
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:fmmb_cache_create, libfmmb), Cint, (Ptr{Cvoid}, Ref{MethodDesc}, Ref{Ptr{Cvoid}}), ctx.h, d, r))
        c = new(m, ctx, r[])
        finalizer(x -> ccall((:fmmb_cache_destroy, libfmmb), Cint, (Ptr{Cvoid},), x.h), c)
    end
end

"""
    FMM(method, sources; ppl=50, bbox=nothing, cache=OperatorCache(method), max_levels=30)  (src/fmm.jl:31-49)
"""
mutable struct FMM
    method::DeviceMethod
    cache::OperatorCache
    h::Ptr{Cvoid}
    n::Int
end
function FMM(m::DeviceMethod, sources::AbstractVector{SVector{3,Float64}}; ppl::Integer=50, bbox=nothing,
             cache::OperatorCache=OperatorCache(m), max_levels::Integer=30)
    cache.method === m || throw(ArgumentError("the cache was built for a different method"))
    pts = collect(sources)
    o = bbox === nothing ? TreeOpts(ppl, max_levels, 0, 0, (0.0, 0.0, 0.0), 0.0) :
        TreeOpts(ppl, max_levels, 1, 0, Tuple(Float64.(bbox[1])), Float64(bbox[2]))
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:fmmb_plan_create, libfmmb), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64, Ref{TreeOpts}, Ref{Ptr{Cvoid}}),
                cache.h, pts, length(pts), Ref(o), r))
    f = FMM(m, cache, r[], length(pts))
    finalizer(x -> ccall((:fmmb_plan_destroy, libfmmb), Cint, (Ptr{Cvoid},), x.h), f)
end
"""
    BatchFMM(method, sets; ppl=50, cache=OperatorCache(method), max_levels=30)

Several independent FMMs in one plan (no reference counterpart; fmmb_batch_plan_create): each
point set of `sets` its own tree in its own box (each set's `square_bbox`, fitted by `fit_box!`
in order), one tree build and one launch per pass for all of them; an `FMM` whose sources,
densities and outputs are the sets' concatenated in order, each set's results bitwise those of
its own `FMM` built with the same cache.
"""
function BatchFMM(m::DeviceMethod, sets::AbstractVector{<:AbstractVector{SVector{3,Float64}}}; ppl::Integer=50,
                  cache::OperatorCache=OperatorCache(m), max_levels::Integer=30)
    cache.method === m || throw(ArgumentError("the cache was built for a different method"))
    pts = reduce(vcat, collect.(sets))
    counts = Int64[length(x) for x in sets]
    o = TreeOpts(ppl, max_levels, 0, 0, (0.0, 0.0, 0.0), 0.0)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:fmmb_batch_plan_create, libfmmb), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Int64}, Int64, Ref{TreeOpts}, Ptr{Float64}, Ref{Ptr{Cvoid}}),
                cache.h, pts, counts, length(counts), Ref(o), C_NULL, r))
    f = FMM(m, cache, r[], length(pts))
    finalizer(x -> ccall((:fmmb_plan_destroy, libfmmb), Cint, (Ptr{Cvoid},), x.h), f)
end
# the circle method's 2D points and square: the plane z = 0 of the cube (the gradients it returns
# are 3-vectors with a zero z component)
function FMM(m::KernelIndependent, sources::AbstractVector{SVector{2,Float64}}; ppl::Integer=50, bbox=nothing,
             cache::OperatorCache=OperatorCache(m), max_levels::Integer=30)
    pts = collect(sources)
    bbox === nothing && (bbox = FlexibleFMM.square_bbox(pts))
    b3 = ((Float64(bbox[1][1]), Float64(bbox[1][2]), -Float64(bbox[2]) / 2), Float64(bbox[2]))
    return FMM(m, embed2(pts); ppl, bbox=b3, cache, max_levels)
end

"""
    FMMState  (src/fmm.jl:64-94): the expansions of one right-hand side on the device.
"""
mutable struct FMMState
    fmm::FMM
    h::Ptr{Cvoid}
    function FMMState(f::FMM; precision::Symbol=:fp64)
        prec = precision === :mixed ? FMMB_PRECISION_MIXED : FMMB_PRECISION_FP64
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:fmmb_state_create, libfmmb), Cint, (Ptr{Cvoid}, Cint, Ref{Ptr{Cvoid}}), f.h, prec, r))
        s = new(f, r[])
        finalizer(x -> ccall((:fmmb_state_destroy, libfmmb), Cint, (Ptr{Cvoid},), x.h), s)
    end
end

function build_expansions!(st::FMMState, f::FMM, sources::AbstractVector{SVector{3,Float64}}, τ::AbstractVector{<:Real})
    length(sources) == f.n || throw(DimensionMismatch("expected $(f.n) sources in group 1"))
    length(τ) == f.n || throw(DimensionMismatch("expected $(f.n) densities in group 1"))
    pts = collect(sources)
    tau = Vector{Float64}(τ)
    check(ccall((:fmmb_build_expansions, libfmmb), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64),
                st.h, pts, tau, f.n))
    return st
end
# The launch shapes of this state timed on its own inputs and the fastest kept (fmmb_autotune);
# no result depends on them. Returns (block targets, FP64 chunk variant, near-field warps,
# M2L ms, near-field ms).
function autotune!(st::FMMState, f::FMM, sources::AbstractVector{SVector{3,Float64}}, τ::AbstractVector{<:Real};
                   tune_blocks::Bool=true)
    length(sources) == f.n || throw(DimensionMismatch("expected $(f.n) sources"))
    length(τ) == f.n || throw(DimensionMismatch("expected $(f.n) densities"))
    pts = collect(sources)
    tau = Vector{Float64}(τ)
    out = zeros(Float64, 5)
    check(ccall((:fmmb_autotune, libfmmb), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Cint, Ptr{Float64}),
                st.h, pts, tau, f.n, tune_blocks ? 1 : 0, out))
    return (Int(out[1]), Int(out[2]), Int(out[3]), out[4], out[5])
end

# Dipole densities, alone or as (charge, Dipole) tuples per source (src/sources.jl:16-31)
function build_expansions!(st::FMMState, f::FMM, sources::AbstractVector{SVector{3,Float64}},
                           τ::AbstractVector{<:Union{Dipole{3,Float64},Tuple{Float64,Dipole{3,Float64}}}})
    length(sources) == f.n || throw(DimensionMismatch("expected $(f.n) sources in group 1"))
    length(τ) == f.n || throw(DimensionMismatch("expected $(f.n) densities in group 1"))
    pts = collect(sources)
    dip = [t isa Dipole ? t.d : t[2].d for t in τ]
    q = eltype(τ) <: Dipole ? nothing : Float64[t[1] for t in τ]
    check(ccall((:fmmb_build_expansions_dipoles, libfmmb), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{SVector{3,Float64}}, Int64),
                st.h, pts, q === nothing ? C_NULL : pointer(q), dip, f.n))
    return st
end
build_expansions!(st::FMMState, f::FMM, sources, τ) =
    throw(ArgumentError("densities of type $(eltype(τ)) are not supported by SphericalHarmonics"))
build_expansions(f::FMM, sources, τ; precision::Symbol=:fp64) = build_expansions!(FMMState(f; precision), f, sources, τ)

_flag(::Potential) = FMMB_OUTPUT_POTENTIAL
_flag(::Gradient) = FMMB_OUTPUT_GRADIENT
_flag(out) = throw(ArgumentError("output $(typeof(out)) is not available with SphericalHarmonics"))

function evaluate_at_sources(f::FMM, st::FMMState, g::Int=1; output=Potential())
    g == 1 || throw(ArgumentError("group $g of 1"))
    flag = _flag(output)
    if output isa Potential
        out = Vector{Float64}(undef, f.n)
        check(ccall((:fmmb_evaluate_at_sources, libfmmb), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}),
                    st.h, flag, out, C_NULL))
    else
        out = Vector{SVector{3,Float64}}(undef, f.n)
        check(ccall((:fmmb_evaluate_at_sources, libfmmb), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{SVector{3,Float64}}),
                    st.h, flag, C_NULL, out))
    end
    return out
end

function evaluate(f::FMM, st::FMMState, targets::AbstractVector{SVector{3,Float64}}; output=Potential())
    flag = _flag(output)
    tg = collect(targets)
    nt = length(tg)
    if output isa Potential
        out = Vector{Float64}(undef, nt)
        check(ccall((:fmmb_evaluate, libfmmb), Cint, (Ptr{Cvoid}, Ptr{SVector{3,Float64}}, Int64, Cint, Ptr{Float64}, Ptr{Float64}),
                    st.h, tg, nt, flag, out, C_NULL))
    else
        out = Vector{SVector{3,Float64}}(undef, nt)
        check(ccall((:fmmb_evaluate, libfmmb), Cint,
                    (Ptr{Cvoid}, Ptr{SVector{3,Float64}}, Int64, Cint, Ptr{Float64}, Ptr{SVector{3,Float64}}),
                    st.h, tg, nt, flag, C_NULL, out))
    end
    return out
end

# ---------------------------------------------------------------- the request server (no reference counterpart)
struct ServerOpts; slots::Int32; ppl::Int32; hbm_budget::Int64; group_max::Int32; reserved::Int32
                   group_points::Int64; end
struct Request
    xyz::Ptr{Float64}; tau::Ptr{Float64}; n::Int64; tol::Float64; kernel::Int32; p::Int32
    outputs::Int32; precision::Int32; ppl::Int32; pot::Ptr{Float64}; grad::Ptr{SVector{3,Float64}}
    kappa::Float64
end
struct RequestInfo
    status::Int32; p::Int32; precision::Int32; slot::Int32
    queued_s::Float64; run_s::Float64; latency_s::Float64; bytes_estimate::Int64
    plan_s::Float64; matvec_s::Float64; device_s::Float64; group::Int32; reserved::Int32
end

"""A continuous-batching FMM request server on one GPU: `submit` queues a Laplace3D FMM at the
sources (potential and gradient, self excluded) whose order and precision path follow `tol`;
`wait` returns the results. Requests overlap on `slots` streams as device memory allows."""
mutable struct Server
    h::Ptr{Cvoid}
    live::Dict{Int64,Any}
    function Server(device::Integer=0; slots::Integer=2, ppl::Integer=0, hbm_budget::Integer=0,
                    group_max::Integer=0, group_points::Integer=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:fmmb_server_create, libfmmb), Cint, (Cint, Ref{ServerOpts}, Ref{Ptr{Cvoid}}),
                    device, ServerOpts(slots, ppl, hbm_budget, group_max, 0, group_points), r))
        s = new(r[], Dict{Int64,Any}())
        finalizer(x -> ccall((:fmmb_server_destroy, libfmmb), Cint, (Ptr{Cvoid},), x.h), s)
        return s
    end
end

"""`submit(server, sources, τ; tol, kappa=nothing)`: a Laplace3D FMM, or Yukawa3D(kappa) on the FP64
path, at the sources (potential and gradient, self excluded)."""
function submit(s::Server, sources::AbstractVector{SVector{3,Float64}}, τ::AbstractVector{Float64}; tol::Real=1e-6,
                kappa::Union{Nothing,Real}=nothing)
    length(τ) == length(sources) || throw(DimensionMismatch("one charge per source"))
    x, t = collect(sources), collect(τ)
    pot = Vector{Float64}(undef, length(x))
    grad = Vector{SVector{3,Float64}}(undef, length(x))
    req = Request(Base.unsafe_convert(Ptr{Float64}, pointer(reinterpret(Float64, x))), pointer(t), length(x), tol,
                  kappa === nothing ? 1 : 2, 0, 3, -1, 0, pointer(pot), pointer(grad),
                  kappa === nothing ? 0.0 : Float64(kappa))
    return _submit(s, req, (x, t, pot, grad))
end

"""`submit_stokes(server, sources, stokeslets; tol, p=0, ppl=0)`: a StokesHarmonics(Stokeslet3D())
FMM (velocities at the sources, self excluded, FP64); `wait` returns (velocities, nothing, info)."""
function submit_stokes(s::Server, sources::AbstractVector{SVector{3,Float64}}, f::AbstractVector{SVector{3,Float64}};
                       tol::Real=1e-6, p::Integer=0, ppl::Integer=0)
    length(f) == length(sources) || throw(DimensionMismatch("one Stokeslet per source"))
    x, fs = collect(sources), collect(f)
    vel = Vector{SVector{3,Float64}}(undef, length(x))
    req = Request(Base.unsafe_convert(Ptr{Float64}, pointer(reinterpret(Float64, x))),
                  Base.unsafe_convert(Ptr{Float64}, pointer(reinterpret(Float64, fs))), length(x), tol, 3, p, 0, -1, ppl,
                  Base.unsafe_convert(Ptr{Float64}, pointer(reinterpret(Float64, vel))), C_NULL, 0.0)
    return _submit(s, req, (x, fs, vel, nothing))
end

function _submit(s::Server, req::Request, bufs)
    ticket = Ref{Int64}(0)
    check(ccall((:fmmb_server_submit, libfmmb), Cint, (Ptr{Cvoid}, Ref{Request}, Ref{Int64}), s.h, req, ticket))
    s.live[ticket[]] = bufs      # rooted until the request is waited for
    return ticket[]
end

function Base.wait(s::Server, ticket::Int64)
    info = Ref{RequestInfo}()
    rc = ccall((:fmmb_server_wait, libfmmb), Cint, (Ptr{Cvoid}, Int64, Float64, Ref{RequestInfo}), s.h, ticket, -1.0, info)
    x, t, pot, grad = pop!(s.live, ticket)
    check(rc)
    return pot, grad, info[]
end

# ---------------------------------------------------------------- the Stokes plan API (src/stokes_api.jl)
"""
    StokesFMMPlan(sources; targets=nothing, method=:harmonics, p=16, ppl=200, bbox=nothing)  (src/stokes_api.jl:20-62)

A plan of StokesHarmonics(Stokeslet3D(); p) on the device: the tree and operators for a fixed
geometry, reused by every `stokes_fmm_eval!`. With targets, the box covers the sources and the
targets (`square_bbox` of both, as the reference plan fits it) and the evaluation is there.
"""
struct StokesFMMPlan
    fmm::FMM
    state::FMMState
    sources::Vector{SVector{3,Float64}}
    targets::Union{Nothing,Vector{SVector{3,Float64}}}
end
function StokesFMMPlan(sources::AbstractVector{SVector{3,Float64}}; method::Symbol=:harmonics, p::Integer=16,
                       ppl::Integer=200, bbox=nothing, targets=nothing)
    method === :harmonics || throw(ArgumentError("the device path provides method=:harmonics"))
    pts = collect(sources)
    tgs = targets === nothing ? nothing : collect(SVector{3,Float64}, targets)
    bbox === nothing && (bbox = FlexibleFMM.square_bbox(tgs === nothing ? pts : vcat(pts, tgs)))
    f = FMM(StokesHarmonics(Stokeslet3D(); p=p), pts; ppl, bbox)
    return StokesFMMPlan(f, FMMState(f), pts, tgs)
end

# fmmb_stokes_densities
struct StokesDensitiesC
    stokeslets::Ptr{Cvoid}
    stresslets::Ptr{Cvoid}
    stressvecs::Ptr{Cvoid}
    doublets::Ptr{Cvoid}
    weights::Ptr{Cvoid}
end
_dptr(::Nothing) = C_NULL
_dptr(a::Vector) = Ptr{Cvoid}(pointer(a))
# a density array as the library reads it: Float64 (weights) or SVector{3,Float64} per source
_dcollect(::Nothing, n, name, ::Type) = nothing
function _dcollect(a::AbstractVector, n, name, ::Type{T}) where {T}
    length(a) == n || throw(DimensionMismatch("$name has length $(length(a)), expected $n"))
    return collect(T, a)
end

function _stokes_call!(out_src, out_trg, plan::StokesFMMPlan, tg, stokeslets, stresslets, stressvecs, doublets,
                       weights, output)
    n = length(plan.sources)
    (stresslets === nothing) == (stressvecs === nothing) ||
        throw(ArgumentError("stresslets and stressvecs must be given together"))
    (stokeslets !== nothing || stresslets !== nothing || doublets !== nothing) ||
        throw(ArgumentError("provide at least one of stokeslets, stresslets, doublets"))
    code = output isa Pressure ? Cint(1) : output isa Gradient ? Cint(2) : output isa Potential ? Cint(0) :
        throw(ArgumentError("Stokes outputs are Velocity(), Pressure() and Gradient()"))
    out_src === nothing || length(out_src) == n || throw(DimensionMismatch("expected $n outputs at the sources"))
    nt = tg === nothing ? 0 : length(tg)
    out_trg === nothing || length(out_trg) == nt || throw(DimensionMismatch("expected $nt outputs at the targets"))
    V = SVector{3,Float64}
    arrs = (_dcollect(stokeslets, n, "stokeslets", V), _dcollect(stresslets, n, "stresslets", V),
            _dcollect(stressvecs, n, "stressvecs", V), _dcollect(doublets, n, "doublets", V),
            _dcollect(weights, n, "weights", Float64))
    # the library writes ∂u_i/∂t_j at 9k + 3i + j: read as an SMatrix that is the transpose
    T = code == 1 ? Float64 : code == 2 ? SMatrix{3,3,Float64,9} : SVector{3,Float64}
    rs = out_src === nothing ? nothing : Vector{T}(undef, n)
    rt = out_trg === nothing ? nothing : Vector{T}(undef, nt)
    tgv = tg === nothing ? nothing : collect(SVector{3,Float64}, tg)
    GC.@preserve arrs rs rt tgv begin
        d = Ref(StokesDensitiesC(map(_dptr, arrs)...))
        check(ccall((:fmmb_stokes_eval_src_trg, libfmmb), Cint,
                    (Ptr{Cvoid}, Ptr{SVector{3,Float64}}, Ref{StokesDensitiesC}, Int64, Ptr{Cvoid}, Int64, Cint,
                     Ptr{Cvoid}, Ptr{Cvoid}),
                    plan.state.h, plan.sources, d, n, _dptr(tgv), nt, code, _dptr(rs), _dptr(rt)))
    end
    fix(r) = code == 2 ? map(transpose, r) : r
    out_src === nothing || copyto!(out_src, fix(rs))
    out_trg === nothing || copyto!(out_trg, fix(rt))
    return nothing
end

"""
    stokes_fmm_eval!(out, plan; stokeslets=nothing, stresslets=nothing, stressvecs=nothing,
                     doublets=nothing, weights=nothing, targets=nothing, output=Velocity())  (src/stokes_api.jl:72-123)

Velocities (`Vector{SVector{3,Float64}}`), with `output=Pressure()` pressures (`Vector{Float64}`), or
with `output=Gradient()` velocity gradients (`Vector{SMatrix{3,3,Float64,9}}`, [i, j] = ∂u_i/∂t_j)
at the plan's targets (or `targets`), or at the sources of a self plan with the i = j term skipped.
Stokeslets, stresslet strengths with their stressvecs, and doublets are `SVector{3,Float64}` per
source; weights multiply the stokeslets, the stresslet strengths and the doublets.
"""
function stokes_fmm_eval!(out::AbstractVector, plan::StokesFMMPlan; stokeslets=nothing, stresslets=nothing,
                          stressvecs=nothing, doublets=nothing, weights=nothing, targets=nothing, output=Potential())
    tg = targets === nothing ? plan.targets : targets
    if tg === nothing
        _stokes_call!(out, nothing, plan, nothing, stokeslets, stresslets, stressvecs, doublets, weights, output)
    else
        _stokes_call!(nothing, out, plan, tg, stokeslets, stresslets, stressvecs, doublets, weights, output)
    end
    return out
end

"""
    stokes_fmm_eval_src_trg!(out_src, out_trg, plan; ...)  (src/stokes_api.jl:125-146)

One expansion build, two evaluations: at the sources (i = j skipped) and at the plan's targets.
"""
function stokes_fmm_eval_src_trg!(out_src::AbstractVector, out_trg::AbstractVector, plan::StokesFMMPlan;
                                  stokeslets=nothing, stresslets=nothing, stressvecs=nothing, doublets=nothing,
                                  weights=nothing, targets=nothing, output=Potential())
    tg = targets === nothing ? plan.targets : targets
    tg === nothing && throw(ArgumentError("the plan has no targets"))
    _stokes_call!(out_src, out_trg, plan, tg, stokeslets, stresslets, stressvecs, doublets, weights, output)
    return out_src, out_trg
end

end # module