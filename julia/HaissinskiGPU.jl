# HaissinskiGPU.jl -- drop-in GPU method of StochasticHaissinski.longitudinal_evolve!
#
# Adds a method of the reference's evolution entry point
#     longitudinal_evolve!(particles, params, buffers, comm, use_mpi)
# (src/evolution.jl:206-212) that dispatches on a `GPUBackend` passed in the
# `comm` position and runs the whole turn loop in libhaissinski_gpu.so through
# ccall.  The particle arrays are the caller's StructArray fields (updated in
# place); the return value is the reference's (σ_E, σ_z, E0) tuple.
#
# The bin grid is built here with Julia's own `range`, exactly as
# src/evolution.jl:270-274 does, and handed to the library so that bins agree
# bit for bit with the reference.
module HaissinskiGPU

using StructArrays
using StochasticHaissinski
using StochasticHaissinski: Particle, SimulationParameters, SimulationBuffers

export GPUBackend, scan_voltages

const libhj = get(ENV, "HAISSINSKI_GPU_LIB",
                  joinpath(@__DIR__, "..", "haissinskijulia_b200", "libhaissinski_gpu.so"))

# Mirrors of the POD structs in include/haissinski_gpu.h (same field order).
struct HjParams
    E0::Float64
    mass::Float64
    voltage::Float64
    harmonic::Int64
    radius::Float64
    pipe_radius::Float64
    α_c::Float64
    ϕs::Float64
    freq_rf::Float64
    n_turns::Int64
    use_wakefield::UInt8
    update_η::UInt8
    update_E0::UInt8
    SR_damping::UInt8
    use_excitation::UInt8
    pad1::UInt8
    pad2::UInt8
    pad3::UInt8
end

struct HjWake
    wake_factor::Float64
    wake_sqrt::Float64
    ctau::Float64
    sin_coef::Float64
    population::Float64
    half_width_sigmas::Float64
    delta_std::Float64
end

struct HjGrid
    nbins::Int64
    edge_first::Float64
    edge_last::Float64
    edge_step::Float64
    centers::Ptr{Float64}
end

struct HjResult
    sigma_E::Float64
    sigma_z::Float64
    E0::Float64
    sigma_E0_initial::Float64
    sigma_z0_initial::Float64
    mean_z::Float64
    mean_dE::Float64
    turns::Int64
end

"""A library context on one CUDA device; pass it where the reference takes `comm`."""
mutable struct GPUBackend
    ctx::Ptr{Cvoid}
    device::Int32
    seed::UInt64
    function GPUBackend(device::Integer = 0; seed::Integer = 0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:hj_create, libhj), Int32, (Int32, Ref{Ptr{Cvoid}}), device, r)
        st == 0 || error("hj_create failed: ", unsafe_string(ccall((:hj_status_string, libhj), Cstring, (Int32,), st)))
        b = new(r[], Int32(device), UInt64(seed))
        finalizer(b) do x
            ccall((:hj_destroy, libhj), Cvoid, (Ptr{Cvoid},), x.ctx)
        end
        return b
    end
end

# The C mirror of a SimulationParameters, optionally with another RF voltage
# (one point of a voltage sweep).
HjParams(p::SimulationParameters; voltage::Real = p.voltage) =
    HjParams(p.E0, p.mass, Float64(voltage), p.harmonic, p.radius, p.pipe_radius, p.α_c,
             p.ϕs, p.freq_rf, p.n_turns, p.use_wakefield, p.update_η, p.update_E0,
             p.SR_damping, p.use_excitation, 0, 0, 0)
to_c(p::SimulationParameters) = HjParams(p)

function reference_wake(p::HjParams)
    w = Ref{HjWake}()
    ccall((:hj_wake_reference, libhj), Int32, (Ref{HjParams}, Ref{HjWake}), p, w)
    return w[]
end

function check(b::GPUBackend, st::Int32)
    st == 0 && return nothing
    name = unsafe_string(ccall((:hj_status_string, libhj), Cstring, (Int32,), st))
    msg = unsafe_string(ccall((:hj_last_error, libhj), Cstring, (Ptr{Cvoid},), b.ctx))
    error("$name: $msg")
end

# Single-pass sample std of src/utils.jl:569-606 (what the MPI branch uses for σ_z0).
function global_std(x::AbstractVector{Float64})
    s = 0.0; s2 = 0.0
    @inbounds for v in x
        s += v; s2 += v * v
    end
    n = length(x)
    n <= 1 && return 0.0
    m = s / n
    return sqrt(max(0.0, ((s2 / n) - m * m) * n / (n - 1)))
end

function StochasticHaissinski.longitudinal_evolve!(
        particles::StructArray{Particle{Float64}}, params::SimulationParameters,
        buffers::SimulationBuffers{Float64}, backend::GPUBackend, use_mpi::Bool = false;
        wake::Union{HjWake,Nothing} = nothing,
        qe_draws::Union{Matrix{Float64},Nothing} = nothing)
    z = particles.coordinates.z
    dE = particles.coordinates.ΔE
    n = length(z)
    pc = to_c(params)
    w = wake === nothing ? reference_wake(pc) : wake
    nbins = length(buffers.λ)
    res = Ref{HjResult}()
    # bins exactly as src/evolution.jl:270-274
    z_width = w.half_width_sigmas * global_std(z)
    z_width < 1e-9 && (z_width = 1e-6)
    edges = range(-z_width, z_width, length = nbins + 1)
    centers = collect((edges[1:end-1] + edges[2:end]) ./ 2)
    GC.@preserve z dE centers qe_draws begin
        grid = Ref(HjGrid(nbins, first(edges), last(edges), step(edges), pointer(centers)))
        draws = qe_draws === nothing ? Ptr{Float64}(C_NULL) : pointer(qe_draws)
        st = ccall((:hj_evolve, libhj), Int32,
                   (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Ref{HjParams}, Ref{HjWake},
                    Int64, Ref{HjGrid}, Ptr{Float64}, UInt64, Ref{HjResult}),
                   backend.ctx, pointer(z), pointer(dE), n, pc, w, nbins, grid, draws,
                   backend.seed, res)
        check(backend, st)
    end
    r = res[]
    return r.sigma_E, r.sigma_z, r.E0
end

"""
    scan_voltages(backend, params, voltages, n, σ_z, σ_E, nbins; wake, block_turns = 64)

The voltage scan of scan_parameter (src/parameter_sensitivity/scan.jl:182-184)
with every point a bunch of one batch on the GPU: n independent Gaussian
particles per point generated on the device (seed = the point's index),
params.n_turns turns each, all points advancing together.  Returns, per
voltage, (σ_E, σ_z, E0, cor(z, ΔE)) of the final particles -- the inputs of
compute_fom (src/parameter_sensitivity/figures_of_merit.jl:16-48).
"""
function scan_voltages(backend::GPUBackend, params::SimulationParameters,
                       voltages::AbstractVector{<:Real}, n::Integer, σ_z::Real, σ_E::Real,
                       nbins::Integer; wake::Union{HjWake,Nothing} = nothing,
                       block_turns::Integer = 64)
    k = length(voltages)
    bt = Ref{Ptr{Cvoid}}(C_NULL)
    check(backend, ccall((:hj_batch_create, libhj), Int32,
                         (Ptr{Cvoid}, Int64, Int32, Int32, Int64, Int32, Ref{Ptr{Cvoid}}),
                         backend.ctx, Int64(k) * (n + 4), k, nbins, 65536, -1, bt))
    ids = zeros(Int64, k)
    out = Vector{NTuple{4,Float64}}(undef, k)
    try
        for (i, V) in enumerate(voltages)
            p = HjParams(params; voltage = V)
            w = wake === nothing ? reference_wake(p) : wake
            id = Ref{Int64}(0)
            check(backend, ccall((:hj_batch_add_gaussian, libhj), Int32,
                                 (Ptr{Cvoid}, Int64, Float64, Float64, UInt64, Ref{HjParams},
                                  Ref{HjWake}, Int64, UInt64, Int64, Ref{Int64}),
                                 bt[], n, σ_z, σ_E, UInt64(i), p, w, nbins, UInt64(i),
                                 params.n_turns, id))
            ids[i] = id[]
        end
        done = Int64[]
        finished = zeros(Int64, k)
        while length(done) < k
            check(backend, ccall((:hj_batch_advance, libhj), Int32, (Ptr{Cvoid}, Int64),
                                 bt[], block_turns))
            nd = Ref{Int32}(0)
            check(backend, ccall((:hj_batch_poll, libhj), Int32,
                                 (Ptr{Cvoid}, Ptr{Int64}, Int32, Ref{Int32}),
                                 bt[], finished, k, nd))
            append!(done, finished[1:nd[]])
            nd[] == 0 && continue
            # retire the finished points at once; they leave the batch here
            res = Vector{HjResult}(undef, nd[])
            corr = zeros(Float64, nd[])
            check(backend, ccall((:hj_batch_take_many, libhj), Int32,
                                 (Ptr{Cvoid}, Int32, Ptr{Int64}, Ptr{Ptr{Float64}},
                                  Ptr{Ptr{Float64}}, Ptr{HjResult}, Ptr{Float64}),
                                 bt[], nd[], finished, C_NULL, C_NULL, res, corr))
            for (j, id) in enumerate(finished[1:nd[]])
                i = findfirst(==(id), ids)
                ids[i] = -1                           # taken
                out[i] = (res[j].sigma_E, res[j].sigma_z, res[j].E0, corr[j])
            end
        end
    finally
        ccall((:hj_batch_destroy, libhj), Cvoid, (Ptr{Cvoid},), bt[])
    end
    return out
end

end # module
