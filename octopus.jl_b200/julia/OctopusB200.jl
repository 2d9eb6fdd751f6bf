"""
    OctopusB200

Julia side of the drop-in: routes Octopus.jl's strong-strong PIC collision to libocto_b200.so
(hand-written sm_100a kernels behind a C ABI, include/octo_b200.h) with `ccall`.

`B200PICPoissonSolver` composes an ordinary `PICPoissonSolver` (the pattern of
`GaussianPICPoissonSolver`, src/tasks/strongstrong/gaussian_pic.jl:87-92), so the
`PICPoissonSolver` keywords stay the API and no method of `collide!(::PICPoissonSolver, ...)`
is overwritten.  Beams stay `Beam{CUDABackend}` with `CuArray` SoA coordinates; the library
kicks them in place on the task's stream.

This file is loaded after Octopus (`include("OctopusB200.jl")` or as a package extension).
"""
module OctopusB200

using CUDA
import Octopus
using Octopus: Beam, CUDABackend, TrackingContext, PICPoissonSolver, GaussianPICPoissonSolver, LongitudinalSlicing,
               AbstractPoissonSolver, StrongStrongTask

const LIB = get(ENV, "OCTO_B200_LIB", joinpath(@__DIR__, "..", "build", "libocto_b200.so"))

# include/octo_b200.h: octo_beam
struct OctoBeam
    n::Int64
    dtype::Int32
    reserved::Int32
    x::CuPtr{Float64}; px::CuPtr{Float64}; y::CuPtr{Float64}
    py::CuPtr{Float64}; z::CuPtr{Float64}; pz::CuPtr{Float64}
end

# include/octo_b200.h: octo_beam_params (BeamParams, src/beam/Beam.jl:29-35)
struct OctoBeamParams
    charge::Float64; mc2::Float64; E0::Float64; r0::Float64; npart::Float64
end

# include/octo_b200.h: octo_pic_options (PICPoissonSolver fields, interface.jl:1350-1382)
struct OctoPicOptions
    nx::Int32; ny::Int32; deposit_method::Int32; lum_deposit_method::Int32
    lum_nx::Int32; lum_ny::Int32; green_type::Int32; green_cache::Int32
    field_derivative::Int32; slice_interpolation::Int32; interaction_grid::Int32; grid_extent::Int32
    grid_extent_sigma::Float64; min_extent_x::Float64; min_extent_y::Float64; grid_quantize::Float64
    green_min_ratio::Float64; green_growth::Float64
    longitudinal_kick::Int32; slicing_method1::Int32; slicing_method2::Int32
    nslices1::Int32; nslices2::Int32; center_position1::Int32; center_position2::Int32
    positions1::Ptr{Float64}; positions2::Ptr{Float64}
    has_kbb1::Int32; has_kbb2::Int32; has_lum_scale::Int32
    kbb1::Float64; kbb2::Float64; lum_scale::Float64
    precision::Int32; gaussian::Int32; margin_sigma::Float64; neutralize::Int32
    solver::Int32; gaussian_when_luminosity::Int32; ignore_centroid1::Int32; ignore_centroid2::Int32
    virtual_drift::Int32; include_sigma_xy::Int32; min_sigma::Float64
    resolution1::Int32; resolution2::Int32
    coupling_tol::Float64
end

# include/octo_b200.h: octo_collide_report
mutable struct OctoCollideReport
    status::Int32; role::Int32; pair_i::Int32; pair_j::Int32; direction::Int32; n_batches::Int32
    turn::Int64; first_index::Int64; dropped::Int64
    green_hits::Int64; green_misses::Int64; green_rebuilds::Int64; kernel_launches::Int64
    replayed::Int32; pad::Int32
    OctoCollideReport() = new(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
end

"""
    B200PICPoissonSolver(; kwargs...)

`PICPoissonSolver(; kwargs...)` run on libocto_b200.  Every keyword is the reference's.
"""
struct B200PICPoissonSolver{T<:Real} <: AbstractPoissonSolver
    pic::PICPoissonSolver{T}
end
B200PICPoissonSolver(; kwargs...) = B200PICPoissonSolver(PICPoissonSolver(; kwargs...))

"""
    B200GaussianPICPoissonSolver(; margin_sigma=5.0, neutralize=true, coupling_tol=Inf, kwargs...)

`GaussianPICPoissonSolver(; ...)` (gaussian_pic.jl:87-112) run on libocto_b200: the uncoupled subtraction, or
the coupled (rotated) one above a finite `coupling_tol`.
"""
struct B200GaussianPICPoissonSolver{T<:Real} <: AbstractPoissonSolver
    gpic::GaussianPICPoissonSolver{T}
    pic::PICPoissonSolver{T}
end
function B200GaussianPICPoissonSolver(; kwargs...)
    g = GaussianPICPoissonSolver(; kwargs...)
    return B200GaussianPICPoissonSolver(g, g.pic)
end
"""
    B200GaussianPoissonSolver(; kwargs...)

`GaussianPoissonSolver(; kwargs...)`, the soft-Gaussian strong-strong solver (interface.jl:949-1020,
gaussian.jl), run on libocto_b200: the uncoupled or coupled (`include_sigma_xy`) covariance with the
:hirata, :chromatic or :exact virtual drift, on Float64 or Float32 beams.  `pic` only carries the slicings, kbb and luminosity-scale overrides and
`longitudinal_kick` into the shared options struct.
"""
struct B200GaussianPoissonSolver{T<:Real} <: AbstractPoissonSolver
    soft::Octopus.GaussianPoissonSolver
    pic::PICPoissonSolver{T}
end
function B200GaussianPoissonSolver(; kwargs...)
    g = Octopus.GaussianPoissonSolver(; kwargs...)
    g.virtual_drift isa Union{Octopus.HirataParaxialDrift,Octopus.ChromaticDrift,Octopus.ExactHamiltonianDrift} ||
        throw(ArgumentError("the B200 backend's soft-Gaussian solver implements the :hirata, :chromatic and :exact drifts"))
    pic = PICPoissonSolver(; grid=(8, 8), kbb1=g.kbb1, kbb2=g.kbb2, luminosity_scale=g.luminosity_scale,
                           slicing1=g.slicing1, slicing2=g.slicing2, longitudinal_kick=g.longitudinal_kick,
                           luminosity_schedule=g.luminosity_schedule)
    return B200GaussianPoissonSolver(g, pic)
end
const B200Solver = Union{B200PICPoissonSolver,B200GaussianPICPoissonSolver,B200GaussianPoissonSolver}
_gaussian_of(::Union{B200PICPoissonSolver,B200GaussianPoissonSolver}) = nothing
_gaussian_of(s::B200GaussianPICPoissonSolver) = s.gpic
_soft_of(::Union{B200PICPoissonSolver,B200GaussianPICPoissonSolver}) = nothing
_soft_of(s::B200GaussianPoissonSolver) = s.soft

_sym(v, table) = Int32(table[Symbol(v)])

# OCTO_SLICING_* codes; the aliases of interface.jl:793-797 map to their methods
const _SLICING_CODE = Dict(:normal_quantile => 0, :gaussian => 0, :Gaussian => 0, :specified => 1,
                           :equal_area => 2, :equal_count => 3, :equal_width => 4, :equal_spaced => 4)

function _slicing_fields(s::LongitudinalSlicing)
    haskey(_SLICING_CODE, s.method) || throw(ArgumentError(
        "unsupported longitudinal slicing method $(repr(s.method))"))
    return (Int32(_SLICING_CODE[s.method]), Int32(s.nslices), s.center_position === :centroid ? Int32(0) : Int32(1),
            Int32(s.resolution))
end

function _options(p::PICPoissonSolver, keep::Vector{Any}, precision::Integer=0, gaussian=nothing; soft=nothing)
    m1, n1, c1, r1 = _slicing_fields(p.slicing1)
    m2, n2, c2, r2 = _slicing_fields(p.slicing2)
    pos1 = Float64.(p.slicing1.positions); pos2 = Float64.(p.slicing2.positions)
    push!(keep, pos1, pos2)
    lg = p.luminosity_grid === nothing ? (0, 0) : p.luminosity_grid
    ldm = p.luminosity_deposit_method === nothing ? Int32(-1) : _sym(p.luminosity_deposit_method, Dict(:CIC => 0, :TSC => 1))
    ig = Symbol(p.interaction_grid)
    return OctoPicOptions(
        Int32(p.grid[1]), Int32(p.grid[2]), _sym(p.deposit_method, Dict(:CIC => 0, :TSC => 1)), ldm,
        Int32(lg[1]), Int32(lg[2]), _sym(p.green_type, Dict(:integrated => 0, :standard => 1, :lattice => 2)),
        _sym(p.green_cache, Dict(:none => 0, :slice_pair => 1)),
        p.field_derivative === :fourth ? Int32(4) : Int32(2), p.slice_interpolation === :quadratic ? Int32(1) : Int32(0),
        _sym(ig, Dict(:slice_pair => 0, :source_slice => 1, :node => 2)), p.grid_extent === :extrema ? Int32(0) : Int32(1),
        Float64(p.grid_extent_sigma), Float64(p.min_transverse_extent[1]), Float64(p.min_transverse_extent[2]),
        Float64(p.grid_quantize), Float64(p.slice_pair_green_min_ratio), Float64(p.slice_pair_green_growth),
        Int32(p.longitudinal_kick), m1, m2, n1, n2, c1, c2,
        isempty(pos1) ? Ptr{Float64}(C_NULL) : pointer(pos1), isempty(pos2) ? Ptr{Float64}(C_NULL) : pointer(pos2),
        Int32(p.kbb1 !== nothing), Int32(p.kbb2 !== nothing), Int32(p.luminosity_scale !== nothing),
        p.kbb1 === nothing ? 0.0 : Float64(p.kbb1), p.kbb2 === nothing ? 0.0 : Float64(p.kbb2),
        p.luminosity_scale === nothing ? 0.0 : Float64(p.luminosity_scale), Int32(precision),
        Int32(gaussian !== nothing), gaussian === nothing ? 5.0 : Float64(gaussian.margin_sigma),
        Int32(gaussian === nothing ? 1 : gaussian.neutralize),
        # soft-Gaussian solver fields (solver, gaussian_when_luminosity, ignore_centroid1/2, virtual_drift,
        # include_sigma_xy, min_sigma)
        Int32(soft === nothing ? 0 : 1), Int32(soft === nothing ? 2 : soft.gaussian_when_luminosity),
        Int32(soft === nothing ? 0 : soft.ignore_centroid1), Int32(soft === nothing ? 0 : soft.ignore_centroid2),
        Int32(soft === nothing ? 0 : soft.virtual_drift isa Octopus.ChromaticDrift ? 1 :
              soft.virtual_drift isa Octopus.ExactHamiltonianDrift ? 2 : 0),
        Int32(soft === nothing ? 0 : soft.include_sigma_xy), soft === nothing ? 0.0 : Float64(soft.min_sigma),
        r1, r2, gaussian === nothing ? Inf : Float64(gaussian.coupling_tol))
end

"""Context: device workspaces and the slice-pair Green cache (the twin of task.runtime_cache)."""
mutable struct Context
    ptr::Ptr{Cvoid}
    # T = Float64: the plain form; T = Float32: the precision form (FP32 particles, planes and FFTs)
    function Context(p::PICPoissonSolver, ::Type{T}=Float64, gaussian=nothing; soft=nothing) where {T<:Union{Float32,Float64}}
        keep = Any[]
        opts = Ref(_options(p, keep, T === Float32 ? 1 : 0, gaussian; soft=soft))
        ptr = GC.@preserve keep ccall((:octo_create, LIB), Ptr{Cvoid}, (Int32, Ref{OctoPicOptions}),
                                      Int32(CUDA.device().handle), opts)
        ptr == C_NULL && error("octo_create failed")
        c = new(ptr)
        finalizer(c) do c
            c.ptr == C_NULL || ccall((:octo_destroy, LIB), Cvoid, (Ptr{Cvoid},), c.ptr)
            c.ptr = C_NULL
        end
        return c
    end
end

function _last_error(ctx::Context)
    buf = Vector{UInt8}(undef, 1024)
    ccall((:octo_last_error, LIB), Int32, (Ptr{Cvoid}, Ptr{UInt8}, Int64), ctx.ptr, buf, length(buf))
    return unsafe_string(pointer(buf))
end

_octo_beam(b::Beam) = OctoBeam(Int64(length(b.rep.x)), Int32(eltype(b.rep.x) === Float32 ? 1 : 0), Int32(0),
    pointer(b.rep.x), pointer(b.rep.px), pointer(b.rep.y), pointer(b.rep.py), pointer(b.rep.z), pointer(b.rep.pz))
_octo_params(b::Beam) = OctoBeamParams(Float64(b.params.charge), Float64(b.params.mc2), Float64(b.params.E0),
                                       Float64(b.params.r0), Float64(b.params.npart))

function _collide!(ctx::Context, solver::B200Solver, beam1::Beam, beam2::Beam, turn::Integer)
    eltype(beam1.rep.x) === eltype(beam2.rep.x) && eltype(beam1.rep.x) in (Float32, Float64) || throw(ArgumentError(
        "the B200 backend takes two Float64 (plain form) or two Float32 (precision form) beams"))
    b1 = Ref(_octo_beam(beam1)); b2 = Ref(_octo_beam(beam2))
    p1 = Ref(_octo_params(beam1)); p2 = Ref(_octo_params(beam2))
    lum = Ref(NaN)
    rep = OctoCollideReport()
    compute = Octopus._pic_compute_luminosity(solver.pic, turn < 0 ? nothing : TrackingContext(turn=Int64(turn)))
    rc = ccall((:octo_pic_collide, LIB), Int32,
               (Ptr{Cvoid}, Ref{OctoBeam}, Ref{OctoBeam}, Ref{OctoBeamParams}, Ref{OctoBeamParams}, Int64, Int32,
                Ref{Float64}, Ref{OctoCollideReport}, Ptr{Cvoid}),
               ctx.ptr, b1, b2, p1, p2, Int64(turn), Int32(compute), lum, rep, CUDA.stream().handle)
    rc == 0 || throw(ArgumentError(_last_error(ctx)))
    Octopus._pic_report_dropped_count(rep.dropped)   # warns exactly as pic_cpu.jl:445-457 does
    return Float64(lum[])
end

"""autotune!(ctx, beam1, beam2; rounds=2) -> shape index: times collides of copies of the beams in each
launch shape (octo_pic_autotune) and keeps the fastest for this context; results do not depend on it."""
function autotune!(ctx::Context, beam1::Beam, beam2::Beam; rounds::Integer=2)
    c1 = deepcopy(beam1); c2 = deepcopy(beam2)
    b1 = Ref(_octo_beam(c1)); b2 = Ref(_octo_beam(c2))
    p1 = Ref(_octo_params(c1)); p2 = Ref(_octo_params(c2))
    choice = Ref(Int32(-1))
    rc = GC.@preserve c1 c2 ccall((:octo_pic_autotune, LIB), Int32,
               (Ptr{Cvoid}, Ref{OctoBeam}, Ref{OctoBeam}, Ref{OctoBeamParams}, Ref{OctoBeamParams}, Int32,
                Ref{Int32}, Ptr{Cvoid}),
               ctx.ptr, b1, b2, p1, p2, Int32(rounds), choice, CUDA.stream().handle)
    rc == 0 || throw(ArgumentError(_last_error(ctx)))
    return Int(choice[])
end

"""collide!(solver, beam1, beam2, CUDABackend[, ctx]) on libocto_b200: a fresh (cold) context per call,
as the reference's public collide! builds a fresh Green cache (pic_cuda.jl:94-126)."""
function Octopus.collide!(solver::B200Solver, beam1::Beam, beam2::Beam, ::Type{CUDABackend},
                          ctx::Union{Nothing,TrackingContext}=nothing)
    c = Context(solver.pic, eltype(beam1.rep.x), _gaussian_of(solver); soft=_soft_of(solver))
    try
        return _collide!(c, solver, beam1, beam2, ctx === nothing ? -1 : ctx.turn)
    finally
        finalize(c)
    end
end

# Task path: one persistent context per (label, solver) in task.runtime_cache (pic_cuda.jl:127-137).
function Octopus._strong_strong_collide_backend!(task::StrongStrongTask, label::Symbol,
                                                 solver::B200Solver, beam1::Beam, beam2::Beam,
                                                 ::Type{CUDABackend}, ctx::TrackingContext)
    T = eltype(beam1.rep.x)
    key = (:octo_b200_context, label, T, solver.pic.grid, objectid(solver))
    c = get!(() -> Context(solver.pic, T, _gaussian_of(solver); soft=_soft_of(solver)), task.runtime_cache, key)::Context
    return _collide!(c, solver, beam1, beam2, ctx.turn)
end

Octopus._pic_compute_luminosity(solver::B200Solver, ctx) = Octopus._pic_compute_luminosity(solver.pic, ctx)

# ---------------------------------------------------------------- line tracking between collisions
# include/octo_b200.h: octo_element
struct OctoElement
    kind::Int32; nharm::Int32; mode::Int32; is_damping::Int32; is_excitation::Int32; reserved::Int32
    rng_id::UInt64
    p::NTuple{40,Float64}
end

function _elem(kind, p::Vector{Float64}; nharm=0, mode=0, is_damping=0, is_excitation=0, rng_id=0)
    q = zeros(40); q[1:length(p)] .= p
    return OctoElement(Int32(kind), Int32(nharm), Int32(mode), Int32(is_damping), Int32(is_excitation), Int32(0),
                       UInt64(rng_id), Tuple(q))
end
_f(v) = Float64[Float64(x) for x in v]
_par(spec, k) = Octopus.param(spec, k)

# One element spec -> octo_element (the OCTO_ELEM_* layouts of include/octo_b200.h).
_octo_element(s::Octopus.ElementSpec{:linear6d}) = _elem(1, _f(Octopus.compile_runtime(s).matrix))
function _octo_element(s::Octopus.ElementSpec{:thin_crab_cavity})
    N = _par(s, :N); p = zeros(25); p[1] = Float64(_par(s, :frequency))
    for h in 1:N
        p[1 + h] = _par(s, :strengthX)[h]; p[9 + h] = _par(s, :strengthY)[h]; p[17 + h] = _par(s, :phase)[h]
    end
    return _elem(2, p; nharm=N)
end
_octo_element(s::Octopus.ElementSpec{:lorentz_boost}) = _elem(3, [Float64(_par(s, :angle))])
_octo_element(s::Octopus.ElementSpec{:rev_lorentz_boost}) = _elem(4, [Float64(_par(s, :angle))])
_octo_element(s::Octopus.ElementSpec{:chromaticity_kick}) =
    _elem(5, vcat(_f(_par(s, :xi)), _f(_par(s, :beta))[1:2], _f(_par(s, :alpha))[1:2],
                  _f(_par(s, :zeta)), _f(_par(s, :eta)), _f(_par(s, :R))))
function _octo_element(s::Octopus.ElementSpec{:lumped_radiation})
    m = Octopus.tracking_method(s)
    mode = m isa Octopus.Damping6DMap ? 1 : m isa Octopus.Diffusion6DMap ? 2 : 0
    p = vcat(_f(_par(s, :damping_turns)), _f(_par(s, :beta)), _f(_par(s, :alpha)), _f(_par(s, :sigma)),
             _f(_par(s, :zeta)), _f(_par(s, :eta)), _f(_par(s, :R)))
    return _elem(6, p; mode=mode, is_damping=Int(Octopus.getparam(s, :is_damping, true)),
                 is_excitation=Int(Octopus.getparam(s, :is_excitation, true)), rng_id=_par(s, :rng_id))
end
_octo_element(s::Octopus.ElementSpec{:crab_dispersion}) = _elem(7, [Float64(_par(s, k)) for k in (:zeta1, :zeta2, :zeta3, :zeta4)])
_octo_element(s::Octopus.ElementSpec{:momentum_dispersion}) = _elem(8, [Float64(_par(s, k)) for k in (:eta1, :eta2, :eta3, :eta4)])
_octo_element(s::Octopus.ElementSpec{:xy_coupling}) =
    _elem(9, [Float64(_par(s, k)) for k in (:r1, :r2, :r3, :r4)]; mode=Int(Octopus.getparam(s, :mode, Octopus.XY_MODEA)))

_flatten(e) = (e,)
_flatten(t::Tuple) = Tuple(Iterators.flatten(map(_flatten, t)))

const _SCRATCH = Ref{Union{Nothing,Context}}(nothing)
function _scratch_context()
    if _SCRATCH[] === nothing
        _SCRATCH[] = Context(PICPoissonSolver(grid=(8, 8), slicing=LongitudinalSlicing(nslices=1, method=:normal_quantile)))
    end
    return _SCRATCH[]::Context
end

_octo_rep(r) = OctoBeam(Int64(length(r.x)), Int32(eltype(r.x) === Float32 ? 1 : 0), Int32(0),
    pointer(r.x), pointer(r.px), pointer(r.y), pointer(r.py), pointer(r.z), pointer(r.pz))

"""
    track_line!(rep, specs, turns=1; context=TrackingContext())

track!(rep, elems, turns; context) (src/track/phase6d_track.jl:10-35) on libocto_b200 for a line of the
zero-length elements around the collision (Linear6D, thin crab cavity, Lorentz boost pair, chromaticity kick,
lumped radiation, crab/momentum dispersion, xy coupling), given as their `ElementSpec`s, nested tuples
expanded as fusedTrack does: one fused device pass on the task's stream.  The radiation draws use
`context.seed`, `context.rng_method` and turn `context.turn + t - 1` for particle index i, as the
reference's fused CUDA kernel does, so results match it to the ulps of the device's libm.
"""
function track_line!(rep, specs::Tuple, turns::Integer=1; context::TrackingContext=TrackingContext())
    elems = OctoElement[_octo_element(s) for s in _flatten(specs)]
    c = _scratch_context()
    b = Ref(_octo_rep(rep))
    rc = GC.@preserve rep elems ccall((:octo_track_line, LIB), Int32,
               (Ptr{Cvoid}, Ref{OctoBeam}, Ptr{OctoElement}, Int32, Int64, Int32, UInt64, Int32, Ptr{Cvoid}),
               c.ptr, b, elems, Int32(length(elems)), Int64(context.turn), Int32(turns), UInt64(context.seed),
               Int32(context.rng_method), CUDA.stream().handle)
    rc == 0 || throw(ArgumentError(_last_error(c)))
    return rep
end

# ---------------------------------------------------------------- moment rows on the device
"""
    moment_row!(row, rep, moments; turn, mask_lost=Octopus.allow_lost_particles())

One MomentObserver row (src/tasks/BeamObservers.jl:1013-1040, 1254-1271) of `rep` computed on the device into
`row::CuVector{Float64}` of length `1 + length(moments)` (typically a row view of the observer's device record
matrix): `row[1] = turn`, then each `Moment`'s mean (order 1) or central moment.  No host synchronisation; the
caller copies the record matrix to the host when it flushes.
"""
function moment_row!(row::CuArray{Float64}, rep, moments; turn::Integer,
                     mask_lost::Bool=Octopus.allow_lost_particles())
    powers = Int32[p for m in moments for p in m.powers]
    c = _scratch_context()
    b = Ref(_octo_rep(rep))
    rc = GC.@preserve rep row powers ccall((:octo_beam_moments, LIB), Int32,
               (Ptr{Cvoid}, Ref{OctoBeam}, Ptr{Int32}, Int32, Int32, Int64, CuPtr{Float64}, Ptr{Cvoid}),
               c.ptr, b, powers, Int32(length(moments)), Int32(mask_lost), Int64(turn), pointer(row),
               CUDA.stream().handle)
    rc == 0 || throw(ArgumentError(_last_error(c)))
    return row
end

end # module
