# B200FrequencyDriftRateTransformsExt -- FrequencyDriftRateTransforms.jl on libfdrb200.so.
#
# A package extension of FrequencyDriftRateTransforms (loaded with CUDA, like the
# reference's ext/CUDAFrequencyDriftRateTransformsExt.jl) whose methods ccall the C ABI of
# libfdrb200.so (include/fdr_b200.h) for Float32 CuArrays.  It replaces, for
# CuMatrix{Float32} spectrograms, the reference's CuArray path: the cuFFT plans and C2R
# output of ext/CUDAFrequencyDriftRateTransformsExt.jl:50-103 and the CUDA.jl broadcasts of
# src/zdtfdr.jl, src/intfdr.jl, src/fftfdr.jl and src/fdrutils.jl.
#
# Installation (a maintainer's change to the reference package):
#   Project.toml  [extensions] B200FrequencyDriftRateTransformsExt = "CUDA"
#   ext/B200FrequencyDriftRateTransformsExt.jl = this file
#   ENV["FDR_B200_LIB"] = path of libfdrb200.so (default: ../libfdrb200.so from here)
#
# Conventions: every library call is ordered on the task-local CUDA.jl stream; a nonzero
# fdr_status becomes error(fdr_last_error_string()) (the reference's errors are Julia
# exceptions too); the library's indices are zero-based and are returned 1-based here.
#
# ZDTWorkspace(spectrogram::CuMatrix{Float32}, ...) returns a B200ZDTWorkspace (the
# reference's ZDTWorkspace struct holds Julia FFT plans, which this path does not use); it
# has the reference workspace's fields (Nf, Nt, r0, δr, Nr, Nl, factors and, on first use,
# F, Y, Yf, Ys, V as CuArrays on the library's buffers), so the reference's generic
# functions that read them keep working.
module B200FrequencyDriftRateTransformsExt

import FrequencyDriftRateTransforms
const FDRT = FrequencyDriftRateTransforms
import FrequencyDriftRateTransforms: ZDTWorkspace, input!, preprocess!, convolve!,
                                     postprocess!, output!, zdtfdr!, zdtfdr,
                                     intshift!, intfdr!, fftfdr_workspace,
                                     fftfdr_workspace!, fdshiftsum!, fdshiftsum, fdshift!,
                                     fdshift, fftfdr!, fftfdr, fdrstats, fdrnormalize!,
                                     findprotohits, fdrsynchronize

using CUDA: CUDA, CuArray, CuMatrix, CuVector, CuPtr

const libfdrb200 = get(ENV, "FDR_B200_LIB", joinpath(@__DIR__, "..", "libfdrb200.so"))

# fdr_status codes, flags and window codes (include/fdr_b200.h)
const FDR_OK = Cint(0)
const FDR_ERR_CAPACITY = Cint(6)
const FDR_WINDOW_RECT = Cint(0)
const FDR_WINDOW_HAMMING = Cint(1)
const FDR_WINDOW_CUSTOM = Cint(2)
const FDR_ZDT_OUTPUT_ALIGNED = UInt32(0x1)
const FDR_SNR_F64 = Cint(1)
const FDR_SNR_F32 = Cint(2)
const FDR_RATES_F64 = Cint(0)
const FDR_RATES_F32 = Cint(1)

# the task-local stream as the library's fdr_stream_t
curstream() = Ptr{Cvoid}(CUDA.stream().handle)

function check(st::Cint)
    st == FDR_OK && return nothing
    msg = unsafe_string(ccall((:fdr_last_error_string, libfdrb200), Cstring, ()))
    error(msg)
end

# fdr_zdt_info (include/fdr_b200.h)
struct ZDTInfo
    Nf::Int64
    Nt::Int64
    Nr::Int64
    Nl::Int64
    K::Int64
    r0::Float32
    dr::Float32
    flags::UInt32
    fused::Int32
    bytes::Int64
    nfactors::Int32
    factors::NTuple{8,Int64}
end

# ---------------------------------------------------------------------------------------
# ZDTWorkspace (src/zdtfdr.jl:10-103; plan_ffts! ext/CUDAFrequencyDriftRateTransformsExt.jl:50-82)
# ---------------------------------------------------------------------------------------
mutable struct B200ZDTWorkspace
    handle::Ptr{Cvoid}
    Nf::Int
    Nt::Int
    r0::Float32
    δr::Float32
    Nr::Int
    Nl::Int
    factors::Union{Tuple,AbstractVector}
    buffers::Union{Nothing,NTuple{3,CuMatrix{ComplexF32}}}
end

# ZDTWorkspace(spectrogram, r0, δr, Nr, factors; output_aligned) (zdtfdr.jl:37-75): the
# library allocates the workspace, runs input! and computes V; the range form
# (zdtfdr.jl:78-87) reaches this method through the reference's own constructor.
function ZDTWorkspace(spectrogram::CuMatrix{Float32}, r0::Real, δr::Real, Nr::Integer,
                      factors::Union{Tuple,AbstractVector}=(2, 3, 5); output_aligned=false)
    Nf, Nt = size(spectrogram)
    f = Int64[Int64(x) for x in factors]
    h = Ref{Ptr{Cvoid}}(C_NULL)
    flags = output_aligned ? FDR_ZDT_OUTPUT_ALIGNED : UInt32(0)
    check(ccall((:fdr_zdt_create, libfdrb200), Cint,
                (Ref{Ptr{Cvoid}}, CuPtr{Float32}, Int64, Int64, Float32, Float32, Int64,
                 Ptr{Int64}, Cint, UInt32, Ptr{Cvoid}),
                h, spectrogram, Nf, Nt, Float32(r0), Float32(δr), Nr, f, length(f), flags,
                curstream()))
    info = Ref{ZDTInfo}()
    check(ccall((:fdr_zdt_get_info, libfdrb200), Cint, (Ptr{Cvoid}, Ref{ZDTInfo}), h[], info))
    ws = B200ZDTWorkspace(h[], Nf, Nt, info[].r0, info[].dr, Int(Nr), Int(info[].Nl),
                          factors, nothing)
    finalizer(ws) do w
        if w.handle != C_NULL
            ccall((:fdr_zdt_destroy, libfdrb200), Cint, (Ptr{Cvoid},), w.handle)
            w.handle = C_NULL
        end
    end
    return ws
end

# F (K x Nt), Y (K x Nl) with Yf / Ys its first Nt / Nr columns, V (K x Nl): the library's
# staged buffers (allocated on first access for a workspace that runs the fused kernels).
function workspace_buffers(ws::B200ZDTWorkspace)
    if ws.buffers === nothing
        pF, pY, pV = Ref{Ptr{Cvoid}}(C_NULL), Ref{Ptr{Cvoid}}(C_NULL), Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:fdr_zdt_buffers, libfdrb200), Cint,
                    (Ptr{Cvoid}, Ref{Ptr{Cvoid}}, Ref{Ptr{Cvoid}}, Ref{Ptr{Cvoid}}),
                    ws.handle, pF, pY, pV))
        K = ws.Nf ÷ 2 + 1
        wrap(p, n) = unsafe_wrap(CuArray, CuPtr{ComplexF32}(UInt(p)), (K, n); own=false)
        ws.buffers = (wrap(pF[], ws.Nt), wrap(pY[], ws.Nl), wrap(pV[], ws.Nl))
    end
    return ws.buffers
end

function Base.getproperty(ws::B200ZDTWorkspace, name::Symbol)
    name === :F && return workspace_buffers(ws)[1]
    name === :Y && return workspace_buffers(ws)[2]
    name === :V && return workspace_buffers(ws)[3]
    name === :Yf && return view(workspace_buffers(ws)[2], :, 1:getfield(ws, :Nt))
    name === :Ys && return view(workspace_buffers(ws)[2], :, 1:getfield(ws, :Nr))
    return getfield(ws, name)
end

Base.propertynames(::B200ZDTWorkspace) =
    (:Nf, :Nt, :r0, :δr, :Nr, :Nl, :factors, :F, :Yf, :Y, :Ys, :V)

# Base.show (zdtfdr.jl:89-99)
function Base.show(io::IO, ws::B200ZDTWorkspace)
    print(io, typeof(ws))
    print(io, "(Nf=", ws.Nf)
    print(io, ",Nt=", ws.Nt)
    print(io, ",r0=", ws.r0)
    print(io, ",δr=", ws.δr)
    print(io, ",Nr=", ws.Nr)
    print(io, ",Nl=", ws.Nl)
    print(io, ",", ws.factors)
    print(io, ")")
end

# Base.sizeof (zdtfdr.jl:101-103): the device bytes the workspace owns.
function Base.sizeof(ws::B200ZDTWorkspace)
    info = Ref{ZDTInfo}()
    check(ccall((:fdr_zdt_get_info, libfdrb200), Cint, (Ptr{Cvoid}, Ref{ZDTInfo}), ws.handle, info))
    return Int(info[].bytes)
end

# ---------------------------------------------------------------------------------------
# Windows (zdtfdr.jl:297-321): :rect, :hamming, Val forms, or w(k, Nf)
# ---------------------------------------------------------------------------------------
window_args(::Val{:rect}, ws) = (FDR_WINDOW_RECT, CuPtr{Float64}(0))
window_args(::Val{:hamming}, ws) = (FDR_WINDOW_HAMMING, CuPtr{Float64}(0))
window_args(::Val{S}, ws) where {S} = error("unsupported window type ($S)")
window_args(w::Symbol, ws) = window_args(Val(w), ws)
window_args(w::Function, ws) =
    (FDR_WINDOW_CUSTOM, CuArray(Float64[Float64(w(k, ws.Nf)) for k in 0:ws.Nf÷2]))

# ---------------------------------------------------------------------------------------
# Staged functions (zdtfdr.jl:209-331; output! ext:94-103)
# ---------------------------------------------------------------------------------------
function input!(ws::B200ZDTWorkspace, spectrogram::CuMatrix{Float32})
    check(ccall((:fdr_zdt_input, libfdrb200), Cint, (Ptr{Cvoid}, CuPtr{Float32}, Ptr{Cvoid}),
                ws.handle, spectrogram, curstream()))
    return ws.F
end

function preprocess!(ws::B200ZDTWorkspace, r0::Float32=ws.r0)
    check(ccall((:fdr_zdt_preprocess, libfdrb200), Cint, (Ptr{Cvoid}, Float32, Ptr{Cvoid}),
                ws.handle, r0, curstream()))
    return nothing
end

preprocess!(ws::B200ZDTWorkspace, r0::Real) = preprocess!(ws, Float32(r0))

function convolve!(ws::B200ZDTWorkspace)
    check(ccall((:fdr_zdt_convolve, libfdrb200), Cint, (Ptr{Cvoid}, Ptr{Cvoid}),
                ws.handle, curstream()))
    return nothing
end

function postprocess_code!(ws::B200ZDTWorkspace, code::Cint, vals)
    check(ccall((:fdr_zdt_postprocess, libfdrb200), Cint,
                (Ptr{Cvoid}, Cint, CuPtr{Float64}, Ptr{Cvoid}),
                ws.handle, code, vals, curstream()))
    return nothing
end

postprocess!(w::Function, ws::B200ZDTWorkspace) = postprocess_code!(ws, window_args(w, ws)...)
postprocess!(w::Val{:hamming}, ws::B200ZDTWorkspace) = postprocess_code!(ws, window_args(w, ws)...)
postprocess!(w::Val{:rect}, ws::B200ZDTWorkspace) = postprocess_code!(ws, window_args(w, ws)...)
postprocess!(::Val{S}, ws::B200ZDTWorkspace) where {S} = error("unsupported window type ($S)")
postprocess!(w::Symbol, ws::B200ZDTWorkspace) = postprocess!(Val(w), ws)
postprocess!(ws::B200ZDTWorkspace) = postprocess!(Val(:rect), ws)

# output! may clobber Ys, like the reference's CuArray method (ext:84-93).
function output!(dest::CuMatrix{Float32}, ws::B200ZDTWorkspace)
    check(ccall((:fdr_zdt_output, libfdrb200), Cint, (Ptr{Cvoid}, CuPtr{Float32}, Ptr{Cvoid}),
                ws.handle, dest, curstream()))
    return dest
end

# ---------------------------------------------------------------------------------------
# zdtfdr! / zdtfdr (zdtfdr.jl:349-421): one fdr_zdt_execute call runs input! (when a
# spectrogram is given) and every (dest, r0) pair, with the fused kernels when eligible.
# ---------------------------------------------------------------------------------------
function execute!(w, dests, ws::B200ZDTWorkspace, spectrogram, r0)
    ds = collect(dests)
    n = length(ds)
    r0s = Float32[Float32(r) for (_, r) in zip(ds, Iterators.cycle(r0))]
    ptrs = CuPtr{Float32}[pointer(d) for d in ds]
    code, vals = window_args(w, ws)
    sp = spectrogram === nothing ? CuPtr{Float32}(0) : pointer(spectrogram)
    for d in ds
        size(d) == (ws.Nf, ws.Nr) || error("dest has size $(size(d)), expected ($(ws.Nf), $(ws.Nr))")
    end
    check(ccall((:fdr_zdt_execute, libfdrb200), Cint,
                (Ptr{Cvoid}, CuPtr{Float32}, Ptr{Float32}, Int64, Ptr{CuPtr{Float32}}, Cint,
                 CuPtr{Float64}, Ptr{Cvoid}),
                ws.handle, sp, r0s, n, ptrs, code, vals, curstream()))
    return dests
end

function zdtfdr!(w::Union{Function,Symbol,Val}, dests, ws::B200ZDTWorkspace,
                 spectrogram=nothing; r0=ws.r0)
    return execute!(w, dests, ws, spectrogram, r0)
end

# dest as one matrix (zdtfdr.jl:370-378); also resolves the reference's
# zdtfdr!(w, dest::AbstractMatrix{<:Real}, workspace, ...) against the method above.
function zdtfdr!(w::Union{Function,Symbol,Val}, dest::AbstractMatrix{<:Real},
                 ws::B200ZDTWorkspace, spectrogram=nothing; r0::Real=ws.r0)
    dest isa CuMatrix{Float32} || error("dest must be a CuMatrix{Float32}")
    execute!(w, (dest,), ws, spectrogram, r0)
    return dest
end

# No dest (zdtfdr.jl:382-396): the result stays in ws.Ys (before the output FFT).
function zdtfdr!(w::Union{Function,Symbol,Val}, ws::B200ZDTWorkspace, spectrogram=nothing;
                 r0::Real=ws.r0)
    if spectrogram !== nothing
        input!(ws, spectrogram)
    end
    preprocess!(ws, r0)
    convolve!(ws)
    postprocess!(w, ws)
    return nothing
end

zdtfdr!(ws::B200ZDTWorkspace, spectrogram=nothing; r0::Real=ws.r0) =
    zdtfdr!(Val(:rect), ws, spectrogram; r0=r0)

# Allocating forms (zdtfdr.jl:412-421): the dest is a CuMatrix{Float32}, never ws.Ys's
# staged buffer.
function zdtfdr(w::Union{Function,Symbol,Val}, ws::B200ZDTWorkspace, spectrogram=nothing;
                r0::Real=ws.r0)
    dest = CuMatrix{Float32}(undef, ws.Nf, ws.Nr)
    return zdtfdr!(w, dest, ws, spectrogram; r0=r0)
end

zdtfdr(ws::B200ZDTWorkspace, spectrogram=nothing; r0::Real=ws.r0) =
    zdtfdr(Val(:rect), ws, spectrogram; r0=r0)

# zdtfdr! followed by findprotohits(dests, threshold; snr) in one library call (the fused
# threshold scan); returns the proto-hits like findprotohits.
function zdtfdr_protohits!(dests, ws::B200ZDTWorkspace, spectrogram, threshold;
                           snr::Bool=true, r0=ws.r0, w=Val(:rect))
    ds = collect(dests)
    r0s = Float32[Float32(r) for (_, r) in zip(ds, Iterators.cycle(r0))]
    ptrs = CuPtr{Float32}[pointer(d) for d in ds]
    code, vals = window_args(w, ws)
    sp = spectrogram === nothing ? CuPtr{Float32}(0) : pointer(spectrogram)
    cap = 1 << 20
    hits = CuArray{Int64}(undef, 2, cap)
    n = Ref{Int64}(0)
    thr = Ref{Float64}(0)
    st = ccall((:fdr_zdtfdr_protohits, libfdrb200), Cint,
               (Ptr{Cvoid}, CuPtr{Float32}, Ptr{Float32}, Int64, Ptr{CuPtr{Float32}}, Cint,
                CuPtr{Float64}, Float64, Cint, CuPtr{Int64}, Int64, Ref{Int64}, Ref{Float64},
                Ptr{Cvoid}),
               ws.handle, sp, r0s, length(ds), ptrs, code, vals, Float64(threshold),
               snr_mode(threshold, snr), hits, cap, n, thr, curstream())
    if st == FDR_ERR_CAPACITY  # the FDR and the threshold are computed: collect the hits
        return findprotohits(ds, thr[])
    end
    check(st)
    return hits_to_indices(hits, n[])
end

# ---------------------------------------------------------------------------------------
# intfdr.jl: shifts round(rate*(t-1)) are formed here, in the rate's own arithmetic, as
# intshift! (intfdr.jl:10) forms them; the sums are bit-exact with the CPU reference.
# ---------------------------------------------------------------------------------------
function intshift!(dout::CuMatrix{Float32}, din::CuMatrix{Float32}, rate::Union{Float32,Float64})
    @assert size(din) == size(dout)
    Nf, Nt = size(din)
    rt = rate isa Float32 ? FDR_RATES_F32 : FDR_RATES_F64
    check(ccall((:fdr_intshift, libfdrb200), Cint,
                (CuPtr{Float32}, Int64, Int64, Float64, Cint, CuPtr{Float32}, Ptr{Cvoid}),
                din, Nf, Nt, Float64(rate), rt, dout, curstream()))
    return dout
end

function intfdr!(fdr::CuMatrix{Float32}, spectrogram::CuMatrix{Float32}, rates)
    Nf, Nt = size(spectrogram)
    Nr = length(rates)
    @assert size(fdr) == (Nf, Nr)
    shifts = Int64[Int64(round(r * (t - 1))) for t in 1:Nt, r in rates]  # shifts[t, j]
    check(ccall((:fdr_intfdr_shifts, libfdrb200), Cint,
                (CuPtr{Float32}, Int64, Int64, Ptr{Int64}, Int64, CuPtr{Float32}, Ptr{Cvoid}),
                spectrogram, Nf, Nt, shifts, Nr, fdr, curstream()))
    return fdr
end

# The Taylor-tree integer FDR (the reference's README.md:88-92; no counterpart in the reference code):
# columns d = dmin..dmax of fdr, drift d channels over Nt-1 steps.
function taylorfdr!(fdr::CuMatrix{Float32}, spectrogram::CuMatrix{Float32}, drange::UnitRange{<:Integer})
    Nf, Nt = size(spectrogram)
    @assert size(fdr) == (Nf, length(drange))
    check(ccall((:fdr_taylor_tree, libfdrb200), Cint,
                (CuPtr{Float32}, Int64, Int64, Cint, Cint, CuPtr{Float32}, Ptr{Cvoid}),
                spectrogram, Nf, Nt, first(drange), last(drange), fdr, curstream()))
    return fdr
end

# ---------------------------------------------------------------------------------------
# fftfdr.jl (:39-148)
# ---------------------------------------------------------------------------------------
mutable struct B200FFTWorkspace
    handle::Ptr{Cvoid}
    Nf::Int
    Nt::Int
    dest_rfft::CuMatrix{ComplexF32}
end

function fftfdr_workspace(spectrogram::CuMatrix{Float32}; bunaligned=true)
    Nf, Nt = size(spectrogram)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:fdr_fftfdr_workspace, libfdrb200), Cint,
                (Ref{Ptr{Cvoid}}, CuPtr{Float32}, Int64, Int64, Ptr{Cvoid}),
                h, spectrogram, Nf, Nt, curstream()))
    pF = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:fdr_fftfdr_rfft_buffer, libfdrb200), Cint, (Ptr{Cvoid}, Ref{Ptr{Cvoid}}), h[], pF))
    F = unsafe_wrap(CuArray, CuPtr{ComplexF32}(UInt(pF[])), (Nf ÷ 2 + 1, Nt); own=false)
    ws = B200FFTWorkspace(h[], Nf, Nt, F)
    finalizer(ws) do w
        if w.handle != C_NULL
            ccall((:fdr_fftfdr_destroy, libfdrb200), Cint, (Ptr{Cvoid},), w.handle)
            w.handle = C_NULL
        end
    end
    return ws
end

function fftfdr_workspace!(ws::B200FFTWorkspace, spectrogram::CuMatrix{Float32}; bunaligned=true)
    Nf, Nt = size(spectrogram)
    (Nf, Nt) == (ws.Nf, ws.Nt) || error("input spectrogram has unexpected size")
    check(ccall((:fdr_fftfdr_workspace_update, libfdrb200), Cint,
                (Ptr{Cvoid}, CuPtr{Float32}, Int64, Int64, Ptr{Cvoid}),
                ws.handle, spectrogram, Nf, Nt, curstream()))
    return ws
end

function fdshiftsum!(dest::CuVector{Float32}, ws::B200FFTWorkspace, rate)
    check(ccall((:fdr_fdshiftsum, libfdrb200), Cint, (Ptr{Cvoid}, Float32, CuPtr{Float32}, Ptr{Cvoid}),
                ws.handle, Float32(rate), dest, curstream()))
    return dest
end

fdshiftsum(ws::B200FFTWorkspace, rate) = fdshiftsum!(CuVector{Float32}(undef, ws.Nf), ws, rate)

function fdshift!(dest::CuMatrix{Float32}, ws::B200FFTWorkspace, rate)
    check(ccall((:fdr_fdshift, libfdrb200), Cint, (Ptr{Cvoid}, Float32, CuPtr{Float32}, Ptr{Cvoid}),
                ws.handle, Float32(rate), dest, curstream()))
    return dest
end

fdshift(ws::B200FFTWorkspace, rate) = fdshift!(CuMatrix{Float32}(undef, ws.Nf, ws.Nt), ws, rate)

function fftfdr!(fdr::CuMatrix{Float32}, ws::B200FFTWorkspace, rates)
    Nr = length(rates)
    @assert size(fdr) == (ws.Nf, Nr)
    rs = Float32[Float32(r) for r in rates]
    check(ccall((:fdr_fftfdr, libfdrb200), Cint,
                (Ptr{Cvoid}, Ptr{Float32}, Int64, CuPtr{Float32}, Ptr{Cvoid}),
                ws.handle, rs, Nr, fdr, curstream()))
    return fdr
end

fftfdr(ws::B200FFTWorkspace, rates) = fftfdr!(CuMatrix{Float32}(undef, ws.Nf, length(rates)), ws, rates)

# ---------------------------------------------------------------------------------------
# fdrutils.jl (:39-169)
# ---------------------------------------------------------------------------------------
const FDRBatches = Union{AbstractVector{<:CuMatrix{Float32}},Tuple{Vararg{CuMatrix{Float32}}}}

function stats(mats)
    ptrs = CuPtr{Float32}[pointer(m) for m in mats]
    Nf, Nrb = size(first(mats))
    m = Ref{Float64}(0)
    s = Ref{Float64}(0)
    check(ccall((:fdr_stats, libfdrb200), Cint,
                (Ptr{CuPtr{Float32}}, Int64, Int64, Int64, Ref{Float64}, Ref{Float64}, Ptr{Cvoid}),
                ptrs, length(ptrs), Nf, Nrb, m, s, curstream()))
    return (Float32(m[]), Float32(s[]))  # the library's values are Float32
end

fdrstats(fdr::CuMatrix{Float32}) = stats((fdr,))
fdrstats(fdrs::FDRBatches) = stats(fdrs)

function normalize!(mats, m::Float32, s::Float32)
    ptrs = CuPtr{Float32}[pointer(x) for x in mats]
    Nf, Nrb = size(first(mats))
    check(ccall((:fdr_normalize, libfdrb200), Cint,
                (Ptr{CuPtr{Float32}}, Int64, Int64, Int64, Float32, Float32, Ptr{Cvoid}),
                ptrs, length(ptrs), Nf, Nrb, m, s, curstream()))
    return nothing
end

# (x - m) / s in Float32, as the reference's broadcast computes it for Float32 m and s.
fdrnormalize!(fdr::CuMatrix{Float32}, m::Float32, s::Float32) = (normalize!((fdr,), m, s); fdr)
fdrnormalize!(fdrs::FDRBatches, m::Float32, s::Float32) = (normalize!(fdrs, m, s); fdrs)

# The type Julia promotes fdrdenormalize(snr, m, s) = snr*s + m to, for Float32 m and s.
snr_mode(threshold, snr::Bool) =
    !snr ? Cint(0) : (threshold isa Union{Integer,Float32} ? FDR_SNR_F32 : FDR_SNR_F64)

function hits_to_indices(hits::CuArray{Int64}, n::Integer)
    h = Array(view(hits, :, 1:n))
    return CartesianIndex{2}[CartesianIndex(Int(h[1, i]) + 1, Int(h[2, i]) + 1) for i in 1:n]
end

function protohits(mats, threshold, snr::Bool)
    Nf, Nrb = size(first(mats))
    ptrs = CuPtr{Float32}[pointer(m) for m in mats]
    cap = 1 << 20
    while true
        hits = CuArray{Int64}(undef, 2, max(cap, 1))
        n = Ref{Int64}(0)
        thr = Ref{Float64}(0)
        st = ccall((:fdr_findprotohits, libfdrb200), Cint,
                   (Ptr{CuPtr{Float32}}, Int64, Int64, Int64, Float64, Cint, CuPtr{Int64}, Int64,
                    Ref{Int64}, Ref{Float64}, Ptr{Cvoid}),
                   ptrs, length(ptrs), Nf, Nrb, Float64(threshold), snr_mode(threshold, snr),
                   hits, cap, n, thr, curstream())
        if st == FDR_ERR_CAPACITY
            cap = Int(n[])  # retry with the true count
            continue
        end
        check(st)
        return hits_to_indices(hits, n[])
    end
end

findprotohits(fdr::CuMatrix{Float32}, threshold; snr::Bool=false) = protohits((fdr,), threshold, snr)
findprotohits(fdrs::FDRBatches, threshold; snr::Bool=false) = protohits(fdrs, threshold, snr)

# fdrsynchronize (fdrutils.jl:129-130): synchronises the task's stream and reports a bounded
# wait of the library's TMA-fed kernels that ran out.  (Narrower than the reference's
# CuArray method, ext:26-28, which it leaves in place for other element types.)
function fdrsynchronize(::Type{<:CuArray{Float32}})
    check(ccall((:fdr_synchronize, libfdrb200), Cint, (Ptr{Cvoid},), curstream()))
    return nothing
end

end # module B200FrequencyDriftRateTransformsExt
