# PhotonPropB200 — Julia binding of libphotonprop_b200.so (include/photonprop_b200.h).
#
# Drop-in for PhotonProp.jl's propagation (src/photon_prop_cuda.jl):
# `propagate_distance(distance, medium, n_ph_gen)` returns the same columns as
# the reference's DataFrame, and `propagate_pairs` runs any number of
# source-target pairs through the batched B200 kernel.  The structs below are
# isbits mirrors of the C structs (field order, types and sizes must match).
#
# Julia is not installed in the build container, so this file is not executed
# by the test suite; tests/test_host_library.py checks the same struct sizes
# and the Python binding calls the same entry points with the same arguments.
module PhotonPropB200

export PPMediumDesc, PPSpectrumDesc, PPPmtDesc, PPPair, PPRunOpts, PPHit
export Context, propagate_pairs, propagate_distance, default_opts, make_photon_fits, get_dir_reweight
export propagate_device!, propagate_device_noalloc!

const libpp = get(ENV, "PHOTONPROP_B200_LIB",
                  joinpath(@__DIR__, "..", "libphotonprop_b200.so"))

const PP_OK = Cint(0)
const PP_ERR_OVERFLOW = Cint(3)
const PP_MODE_COMPAT = Cint(0)
const PP_MODE_PHYSICAL = Cint(1)
const PP_EMITTER_ISOTROPIC = Cint(0)
const PP_EMITTER_CHERENKOV_CONE = Cint(1)
const PP_EMITTER_CASCADE = Cint(2)          # CherenkovAngularEmission, physical mode
const PP_OPT_PMT_WEIGHT = UInt32(1)
const PP_OPT_NORMALIZE = UInt32(2)
const PP_OPT_NO_HITS = UInt32(4)
const PP_OPT_COMPACT_HITS = UInt32(8)
const PP_OPT_CASCADE = UInt32(16)
const PP_STATS = 8

struct PPMediumDesc            # WaterProperties (src/medium.jl:23-50) + absorption table
    salinity::Cdouble          # permille
    pressure::Cdouble          # atm
    temperature::Cdouble       # degC
    vol_conc_small_part::Cdouble
    vol_conc_large_part::Cdouble
    radiation_length::Cdouble
    n_abs::Int32               # 0: the reference's 6-knot table
    pad::Int32
    abs_wl::NTuple{32,Cdouble}
    abs_len::NTuple{32,Cdouble}
end

PPMediumDesc(salinity, pressure_atm, temperature, small, large; radiation_length=36.08) =
    PPMediumDesc(salinity, pressure_atm, temperature, small, large, radiation_length,
                 Int32(0), Int32(0), ntuple(_ -> 0.0, 32), ntuple(_ -> 0.0, 32))

struct PPSpectrumDesc          # CherenkovSpectrum / Monochromatic (src/spectrum.jl)
    kind::Int32                # 0 Cherenkov, 1 monochromatic
    n_knots::Int32
    wl_min::Cdouble
    wl_max::Cdouble
end

struct PPPmtDesc               # PMT acceptance table (src/detection.jl:18-33)
    n::Int32
    pad::Int32
    wavelength::NTuple{256,Cdouble}
    acceptance::NTuple{256,Cdouble}
end

function PPPmtDesc(wl::AbstractVector, acc::AbstractVector)
    n = length(wl)
    @assert n == length(acc) && n <= 256
    PPPmtDesc(Int32(n), Int32(0), ntuple(i -> i <= n ? Float64(wl[i]) : 0.0, 256),
              ntuple(i -> i <= n ? Float64(acc[i]) : 0.0, 256))
end

struct PPPair                  # PhotonSource + DetectionSphere, 80 bytes
    pos::NTuple{3,Cfloat}
    t0::Cfloat
    dir::NTuple{3,Cfloat}
    track_len::Cfloat
    target::NTuple{3,Cfloat}
    radius::Cfloat
    n_photons::Int64
    seed::UInt64
    emitter::Int32
    reserved::NTuple{3,Int32}
end

struct PPRunOpts
    mode::Int32
    max_steps::Int32
    g::Cfloat
    t_max::Cfloat
    hist_t0::Cfloat
    hist_bin_width::Cfloat
    hist_bins::Int32
    flags::UInt32
    block_size::Int32
    blocks_per_sm::Int32
    chunk_photons::Int32
    reserved::Int32
end

struct PPHit                   # 64 bytes
    pos::NTuple{3,Cfloat}
    time::Cfloat
    dir0::NTuple{3,Cfloat}
    weight::Cfloat
    dir::NTuple{3,Cfloat}
    wavelength::Cfloat
    dist::Cfloat
    pair::UInt32
    photon::UInt64
end

@assert sizeof(PPPair) == 80 && sizeof(PPHit) == 64 && sizeof(PPRunOpts) == 48

check(st, ctx=C_NULL) = st == PP_OK ? nothing :
    error("photonprop_b200 status $(st): " * unsafe_string(ccall((:pp_last_error, libpp), Cstring, (Ptr{Cvoid},), ctx)))

function default_opts(mode::Integer)
    r = Ref{PPRunOpts}()
    check(ccall((:pp_default_opts, libpp), Cint, (Int32, Ref{PPRunOpts}), Int32(mode), r))
    r[]
end

mutable struct Context
    ptr::Ptr{Cvoid}
    function Context(medium::PPMediumDesc, spectrum::PPSpectrumDesc, pmt::Union{PPPmtDesc,Nothing}=nothing;
                     device::Integer=0)
        out = Ref{Ptr{Cvoid}}(C_NULL)
        st = pmt === nothing ?
            ccall((:pp_create, libpp), Cint, (Ref{Ptr{Cvoid}}, Cint, Ref{PPMediumDesc}, Ref{PPSpectrumDesc}, Ptr{Cvoid}),
                  out, device, medium, spectrum, C_NULL) :
            ccall((:pp_create, libpp), Cint, (Ref{Ptr{Cvoid}}, Cint, Ref{PPMediumDesc}, Ref{PPSpectrumDesc}, Ref{PPPmtDesc}),
                  out, device, medium, spectrum, pmt)
        check(st)
        ctx = new(out[])
        finalizer(c -> c.ptr == C_NULL || ccall((:pp_destroy, libpp), Cvoid, (Ptr{Cvoid},), c.ptr), ctx)
        ctx
    end
end

"""
    propagate_pairs(ctx, pairs, opts; hit_capacity) -> (hits, n_hits, stats, hist)

Batched persistent kernel over all pairs (`pp_propagate`).  `stats` is
PP_STATS x n_pairs (hits, Σw, Σw², Σw·t, Σw·t², Σw·ln t, photons, 0) and
`hist` hist_bins x n_pairs (column-major views of the C row-major arrays).
"""
function propagate_pairs(ctx::Context, pairs::Vector{PPPair}, opts::PPRunOpts; hit_capacity::Integer=1 << 20)
    n = length(pairs)
    hits = Vector{PPHit}(undef, hit_capacity)
    stats = zeros(Float64, PP_STATS, n)
    hist = zeros(Float64, max(opts.hist_bins, 1), n)
    nh = Ref{Int64}(0)
    st = ccall((:pp_propagate, libpp), Cint,
               (Ptr{Cvoid}, Ptr{PPPair}, Int64, Ref{PPRunOpts}, Ptr{PPHit}, Int64, Ref{Int64}, Ptr{Cdouble}, Ptr{Cdouble}),
               ctx.ptr, pairs, n, opts, hits, hit_capacity, nh, stats, opts.hist_bins > 0 ? hist : C_NULL)
    st == PP_ERR_OVERFLOW || check(st, ctx.ptr)
    (hits[1:min(nh[], hit_capacity)], nh[], stats, hist)
end

"""
    propagate_device!(ctx, d_pairs, n_pairs, opts, d_hits, hit_capacity, d_counters, d_stats, d_hist, stream)

`pp_propagate_device` on device buffers (raw device addresses, e.g.
`UInt(pointer(A))` of CuArrays: `d_pairs` n_pairs `PPPair`s, `d_hits`
hit_capacity `PPHit`s, `d_counters` 4 `UInt64`, `d_stats` PP_STATS x n_pairs
and `d_hist` hist_bins x n_pairs `Float64`), asynchronous on the `CUstream`
`stream` (CUDA.jl: `CUDA.stream().handle`; `C_NULL` for the default stream).
"""
function propagate_device!(ctx::Context, d_pairs, n_pairs::Integer, opts::PPRunOpts, d_hits, hit_capacity::Integer,
                           d_counters, d_stats, d_hist, stream=C_NULL)
    check(ccall((:pp_propagate_device, libpp), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ref{PPRunOpts}, Ptr{Cvoid}, Int64, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid},
                 Ptr{Cvoid}),
                ctx.ptr, Ptr{Cvoid}(UInt(d_pairs)), n_pairs, opts, Ptr{Cvoid}(UInt(d_hits)), hit_capacity,
                Ptr{Cvoid}(UInt(d_counters)), Ptr{Cvoid}(UInt(d_stats)), Ptr{Cvoid}(UInt(d_hist)),
                Ptr{Cvoid}(UInt(stream))), ctx.ptr)
    nothing
end

"""
    propagate_device_noalloc!(ctx, d_pairs, n_pairs, opts, d_hits, hit_capacity, d_counters, d_stats, d_hist, stream)

The same call for code that keeps all device memory in CUDA.jl's pool
(`pp_propagate_device_noalloc`): the library allocates nothing, its work-queue
scratch being a fixed ~512 KiB device array.  At most 65536 pairs per call;
make the first call on a device before any stream capture; calls that
overlap on the GPU race on the shared scratch, so issue them on one stream.
"""
function propagate_device_noalloc!(ctx::Context, d_pairs, n_pairs::Integer, opts::PPRunOpts, d_hits,
                                   hit_capacity::Integer, d_counters, d_stats, d_hist, stream=C_NULL)
    check(ccall((:pp_propagate_device_noalloc, libpp), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ref{PPRunOpts}, Ptr{Cvoid}, Int64, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid},
                 Ptr{Cvoid}),
                ctx.ptr, Ptr{Cvoid}(UInt(d_pairs)), n_pairs, opts, Ptr{Cvoid}(UInt(d_hits)), hit_capacity,
                Ptr{Cvoid}(UInt(d_counters)), Ptr{Cvoid}(UInt(d_stats)), Ptr{Cvoid}(UInt(d_hist)),
                Ptr{Cvoid}(UInt(stream))), ctx.ptr)
    nothing
end

const C_VAC = 0.299792458  # m/ns

"""
    propagate_distance(ctx, medium, distance, n_ph_gen; seed=0)

`propagate_distance` of src/photon_prop_cuda.jl:588-644 in reference-compatible
mode: isotropic source at the origin, 0.21 m sphere at (0, 0, distance).
Returns a NamedTuple of the reference's columns (tres, initial_theta, ref_ix,
abs_weight, dist_travelled, wavelength).
"""
function propagate_distance(ctx::Context, medium::PPMediumDesc, distance::Real, n_ph_gen::Integer; seed::Integer=0)
    r = 0.21f0
    pair = PPPair((0f0, 0f0, 0f0), 0f0, (0f0, 0f0, 1f0), 0f0, (0f0, 0f0, Float32(distance)), r,
                  Int64(n_ph_gen), UInt64(seed), PP_EMITTER_ISOTROPIC, (Int32(0), Int32(0), Int32(0)))
    opts = default_opts(PP_MODE_COMPAT)
    hits, nh, _, _ = propagate_pairs(ctx, [pair], opts; hit_capacity=max(1024, n_ph_gen ÷ 20 + 1024))
    sort!(hits, by=h -> h.photon)
    wl = [Float64(h.wavelength) for h in hits]
    d = [Float64(h.dist) for h in hits]
    m = Ref(medium)
    ref_ix = [ccall((:pp_refractive_index, libpp), Cdouble, (Ref{PPMediumDesc}, Cdouble), m, x) for x in wl]
    labs = [ccall((:pp_absorption_length, libpp), Cdouble, (Ref{PPMediumDesc}, Cdouble), m, x) for x in wl]
    n800 = ccall((:pp_refractive_index, libpp), Cdouble, (Ref{PPMediumDesc}, Cdouble), m, 800.0)
    tgeo = (distance - r) / (C_VAC / n800)
    (tres=d ./ (C_VAC ./ ref_ix) .- tgeo, initial_theta=[acos(clamp(Float64(h.dir0[3]), -1, 1)) for h in hits],
     ref_ix=ref_ix, abs_weight=exp.(-d ./ labs), dist_travelled=d, wavelength=wl)
end

"""
    sobol_1d(lb, ub, n)

The first n points of Sobol.jl's one-dimensional `SobolSeq([lb], [ub])`
(the bit-reversed Gray code of k = 1, 2, ...).
"""
sobol_1d(lb, ub, n) = [lb + (ub - lb) * bitreverse(UInt32(k ⊻ (k >> 1))) / 2.0^32 for k in 1:n]

"""
    make_photon_fits(ctx, n_photons_per_dist, n_distances, n_angles, max_dist=300f0; seed=0)

`make_photon_fits` of src/modelling.jl:86-111 as one library call
(`pp_propagate_fit`): every distance propagates in one batched launch and
every (distance, angle) is reweighted and fitted on the device.  Returns a
NamedTuple of the reference's DataFrame columns.
"""
function make_photon_fits(ctx::Context, n_photons_per_dist::Integer, n_distances::Integer, n_angles::Integer,
                          max_dist::Real=300f0; seed::Integer=0, hit_capacity::Integer=1 << 27)
    distances = Float32.(10 .^ sobol_1d(0.0, Float64(Float32(log10(Float32(max_dist)))), n_distances))
    obs_angles = sobol_1d(0.0, Float64(pi), n_angles)
    pairs = [PPPair((0f0, 0f0, 0f0), 0f0, (0f0, 0f0, 1f0), 0f0, (0f0, 0f0, d), 0.21f0, Int64(n_photons_per_dist),
                    ccall((:pp_pair_seed, libpp), UInt64, (UInt64, UInt64), UInt64(seed), UInt64(i - 1)),
                    PP_EMITTER_ISOTROPIC, (Int32(0), Int32(0), Int32(0))) for (i, d) in enumerate(distances)]
    o = default_opts(PP_MODE_COMPAT)
    opts = PPRunOpts(o.mode, o.max_steps, o.g, o.t_max, o.hist_t0, o.hist_bin_width, Int32(0),
                     o.flags | PP_OPT_PMT_WEIGHT, o.block_size, o.blocks_per_sm, o.chunk_photons, o.reserved)
    fits = Array{Cdouble}(undef, 3, n_angles, n_distances)
    nh = Ref{Int64}(0)
    check(ccall((:pp_propagate_fit, libpp), Cint,
                (Ptr{Cvoid}, Ptr{PPPair}, Int64, Ref{PPRunOpts}, Ptr{Cdouble}, Int32, Int64, Ref{Int64},
                 Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
                ctx.ptr, pairs, n_distances, opts, obs_angles, n_angles, hit_capacity, nh, fits, C_NULL, C_NULL,
                C_NULL), ctx.ptr)
    (obs_angle=repeat(obs_angles, n_distances), fit_alpha=vec(fits[1, :, :]), fit_theta=vec(fits[2, :, :]),
     det_fraction=vec(fits[3, :, :]), distance=repeat(Float64.(distances), inner=n_angles))
end

"""
    get_dir_reweight(thetas, obs_angle, ref_ixs)

src/modelling.jl:46-49 through the library's FP64 host function.
"""
function get_dir_reweight(thetas::AbstractVector{Float64}, obs_angle::Real, ref_ixs::AbstractVector{Float64})
    out = similar(thetas)
    check(ccall((:pp_dir_reweight, libpp), Cint, (Ptr{Cdouble}, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Int64),
                thetas, obs_angle, ref_ixs, out, length(thetas)))
    out
end

end # module
