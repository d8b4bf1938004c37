# PFWB200.jl — Julia binding of libpfw_b200.so for PotentialFrameWork.jl.
#
# A maintainer adds this module next to the package (or as a package
# extension) to make the B200 library a drop-in behind the reference's own
# API: `evaluate!(::CUDAWorkspace, sys, p; request)`, `neighbour_list(sys,
# cutoff; backend=CUDAWorkspace())` and the AtomsCalculators methods through
# `neighbourlist=cuda_ws`.  Units are stripped at the same boundary as
# `NeighbourList/storage.jl:74-78`; species are mapped to channels by strict
# identity as `storage.jl:157-170`.  Not executable in the build container
# (no Julia); the ctypes binding pfw_b200/lib.py exercises the same ABI.
module PFWB200

using AtomsBase, Unitful, StaticArrays
import AtomsCalculators as AC
using PotentialFrameWork
const PP = PotentialFrameWork.PairPotentials
const NL = PotentialFrameWork.NeighbourList

const libpfw = get(ENV, "PFW_B200_LIB", joinpath(@__DIR__, "..", "lib", "libpfw_b200.so"))

const PFW_OK, PFW_EINVAL, PFW_EDOMAIN, PFW_ESHAPE = 0, 1, 2, 3
const REQ_E, REQ_F, REQ_V = UInt32(1), UInt32(2), UInt32(4)

struct Options
    precision::Int32
    bruteforce_threshold::Int32
    device::Int32
    reserved::Int32
end

mutable struct CUDAWorkspace
    handle::Ptr{Cvoid}
    function CUDAWorkspace(; precision=Float64, bruteforce_threshold=32, device=0)
        opt = Ref(Options(precision === Float64 ? 0 : 1, bruteforce_threshold, device, 0))
        h = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:pfw_ws_create, libpfw), Cint, (Ref{Options}, Ref{Ptr{Cvoid}}), opt, h)
        rc == PFW_OK || error("pfw_ws_create failed ($rc): no CUDA device or invalid options")
        w = new(h[])
        finalizer(w -> ccall((:pfw_ws_destroy, libpfw), Cvoid, (Ptr{Cvoid},), w.handle), w)
    end
end

function check(w::CUDAWorkspace, rc)
    rc == PFW_OK && return nothing
    msg = unsafe_string(ccall((:pfw_last_error, libpfw), Cstring, (Ptr{Cvoid},), w.handle))
    rc == PFW_EINVAL && throw(ArgumentError(msg))
    rc == PFW_EDOMAIN && throw(DomainError(0, msg))
    rc == PFW_ESHAPE && throw(DimensionMismatch(msg))
    error("libpfw_b200: $msg ($rc)")
end

# Numeric Å geometry in original order; cell columns are cell vectors.
function upload!(w::CUDAWorkspace, sys, channels::Vector{Int32})
    n = length(sys)
    X = Matrix{Float64}(undef, 3, n)
    for i = 1:n, a = 1:3
        X[a, i] = ustrip(u"Å", AtomsBase.position(sys, i)[a])
    end
    cv = AtomsBase.cell_vectors(sys)
    H = Float64[ustrip(u"Å", cv[j][a]) for a = 1:3, j = 1:3]
    pbc = UInt8.(collect(AtomsBase.periodicity(sys)))
    check(w, ccall((:pfw_set_geometry, libpfw), Cint,
                   (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{UInt8}, Ptr{Int32}),
                   w.handle, n, X, H, pbc, channels))
end

function channels_for(sys, labels)
    map(1:length(sys)) do i
        s = ChemicalSpecies(AtomsBase.species(sys, i))
        k = findfirst(l -> isequal(l, s), labels)
        isnothing(k) && throw(ArgumentError("potential has no parameters for species $s"))
        Int32(k - 1)
    end
end

bind_model!(w, p::PP.SmoothPair) =
    check(w, ccall((:pfw_pair_model_smooth, libpfw), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Float64),
                   w.handle, length(p.labels), Matrix{Float64}(transpose(p.amplitudes)), p.radius))
bind_model!(w, p::PP.RadialPotential{<:PP.LennardJonesRadial}) =
    check(w, ccall((:pfw_pair_model_lj, libpfw), Cint, (Ptr{Cvoid}, Float64, Float64, Float64),
                   w.handle, p.radial.epsilon, p.radial.sigma, p.radius))

request_bits(::PP.EnergyForcesVirial) = REQ_E | REQ_F | REQ_V
request_bits(::PP.EnergyOnly) = REQ_E
request_bits(props::Tuple) = reduce(|, (p isa AC.Energy ? REQ_E : p isa AC.Forces ? REQ_F : REQ_V for p in props); init=UInt32(0))

"""evaluate!(w::CUDAWorkspace, sys, p; request) — same contract as
PairPotentials.evaluate! (evaluation.jl:31-52): owning, original-order,
unitful outputs; topology rebuilt on every call."""
function PP.evaluate!(w::CUDAWorkspace, sys, p; request=PP.EnergyForcesVirial(), parallel=false, parameters=nothing)
    isnothing(parameters) || (p = PP.with_parameters(p, parameters))
    labels = p isa PP.SmoothPair ? p.labels : [ChemicalSpecies(AtomsBase.species(sys, 1))]
    ch = p isa PP.SmoothPair ? channels_for(sys, labels) : zeros(Int32, length(sys))
    upload!(w, sys, ch)
    bind_model!(w, p)
    n = length(sys)
    E = Ref(0.0); F = zeros(3, n); W = zeros(3, 3)
    check(w, ccall((:pfw_evaluate, libpfw), Cint, (Ptr{Cvoid}, Int32, UInt32, Ref{Float64}, Ptr{Float64}, Ptr{Float64}),
                   w.handle, 0, request_bits(request), E, F, W))
    request isa PP.EnergyOnly && return (; energy=E[] * u"eV")
    (; energy=E[] * u"eV", forces=F * u"eV/Å", virial=W * u"eV")
end

"""neighbour_list(sys, cutoff; backend=CUDAWorkspace()) — materialised directed
snapshot (interface.jl:67-96) returned as NL.NeighbourSnapshot."""
function NL.neighbour_list(sys::AtomsBase.AbstractSystem{3}, cutoff, w::CUDAWorkspace; int_type=Int32)
    upload!(w, sys, zeros(Int32, length(sys)))
    c = Float64(ustrip(u"Å", cutoff isa Unitful.Length ? cutoff : cutoff * u"Å"))
    M = Ref{Int64}(0)
    check(w, ccall((:pfw_neighbour_count, libpfw), Cint, (Ptr{Cvoid}, Float64, Ref{Int64}), w.handle, c, M))
    n = length(sys)
    offs = zeros(Int64, n + 1); js = zeros(Int32, M[]); S = zeros(Int32, 3, M[]); R = zeros(3, M[])
    check(w, ccall((:pfw_neighbour_fill, libpfw), Cint,
                   (Ptr{Cvoid}, Ptr{Int64}, Ptr{Int32}, Ptr{Int32}, Ptr{Float64}), w.handle, offs, js, S, R))
    idx = [int_type.(js[offs[i]+1:offs[i+1]] .+ 1) for i = 1:n]
    disp = [[SVector{3}(R[:, k]) for k = offs[i]+1:offs[i+1]] for i = 1:n]
    shf = [[SVector{3,int_type}(S[:, k]) for k = offs[i]+1:offs[i+1]] for i = 1:n]
    NL.NeighbourSnapshot(idx, disp, shf)
end

"""set_skin!(w, skin) — Verlet skin reuse of the pair list (pfw_pair_set_skin,
the reference's gpu_skin!, NeighbourList/gpu.jl:404-549); 0 rebuilds on every
call as evaluate! does."""
set_skin!(w::CUDAWorkspace, skin) =
    check(w, ccall((:pfw_pair_set_skin, libpfw), Cint, (Ptr{Cvoid}, Float64), w.handle,
                   Float64(ustrip(u"Å", skin isa Unitful.Length ? skin : skin * u"Å"))))

"""evaluate_batch!(w, systems, p; request) — energies, forces and virials of
many independent structures in one launch (pfw_set_batch + pfw_evaluate_batch),
as a loop of evaluate! calls would return them."""
function evaluate_batch!(w::CUDAWorkspace, systems::AbstractVector, p; request=PP.EnergyForcesVirial())
    nsys = length(systems)
    offsets = zeros(Int64, nsys + 1)
    for (s, sys) in enumerate(systems)
        offsets[s+1] = offsets[s] + length(sys)
    end
    n = offsets[end]
    X = Matrix{Float64}(undef, 3, n); H = zeros(9 * nsys); pbc = zeros(UInt8, 3 * nsys)
    ch = Vector{Int32}(undef, n)
    labels = p isa PP.SmoothPair ? p.labels : nothing
    for (s, sys) in enumerate(systems)
        for i = 1:length(sys), a = 1:3
            X[a, offsets[s]+i] = ustrip(u"Å", AtomsBase.position(sys, i)[a])
        end
        cv = AtomsBase.cell_vectors(sys)
        for j = 1:3, a = 1:3
            H[9(s-1)+3(j-1)+a] = ustrip(u"Å", cv[j][a])
        end
        pbc[3(s-1)+1:3s] .= UInt8.(collect(AtomsBase.periodicity(sys)))
        ch[offsets[s]+1:offsets[s+1]] .= isnothing(labels) ? zeros(Int32, length(sys)) : channels_for(sys, labels)
    end
    check(w, ccall((:pfw_set_batch, libpfw), Cint,
                   (Ptr{Cvoid}, Int32, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}, Ptr{UInt8}, Ptr{Int32}),
                   w.handle, nsys, offsets, X, H, pbc, ch))
    bind_model!(w, p)
    E = zeros(nsys); F = zeros(3, n); W = zeros(9, nsys)
    check(w, ccall((:pfw_evaluate_batch, libpfw), Cint,
                   (Ptr{Cvoid}, Int32, UInt32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                   w.handle, 0, request_bits(request), E, F, W, C_NULL))
    map(1:nsys) do s
        (; energy=E[s] * u"eV", forces=F[:, offsets[s]+1:offsets[s+1]] * u"eV/Å",
           virial=reshape(W[:, s], 3, 3) * u"eV")
    end
end

end # module
