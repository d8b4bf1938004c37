# PFWB200.jl — Julia binding of libpfw_b200.so for PotentialFrameWork.jl.
#
# A maintainer adds this module next to the package (or as a package
# extension) to make the B200 library a drop-in behind the reference's own
# API: `evaluate!(::CUDAWorkspace, sys, p; request)` for SmoothPair and
# Lennard-Jones, `neighbour_list(sys, cutoff, ::CUDAWorkspace)`,
# `ace_evaluate!(::CUDAWorkspace, sys, calc::ACECalculator; request)` with
# `site_energies`, `evaluate_batch!` and `set_skin!`.  Units are stripped at the same boundary as
# `NeighbourList/storage.jl:74-78`; species are mapped to channels by strict
# identity as `storage.jl:157-170`.  Not executable in the build container
# (no Julia); the ctypes binding pfw_b200/lib.py exercises the same ABI.
module PFWB200

using AtomsBase, Unitful, StaticArrays, SparseArrays
import AtomsCalculators as AC
using PotentialFrameWork
const PP = PotentialFrameWork.PairPotentials
const NL = PotentialFrameWork.NeighbourList
const ACEM = PotentialFrameWork.ACE

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
    ace_key::Any  # (model, parameters) of the ACE tables on the device, or nothing
    function CUDAWorkspace(; precision=Float64, bruteforce_threshold=32, device=0)
        opt = Ref(Options(precision === Float64 ? 0 : 1, bruteforce_threshold, device, 0))
        h = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:pfw_ws_create, libpfw), Cint, (Ref{Options}, Ref{Ptr{Cvoid}}), opt, h)
        rc == PFW_OK || error("pfw_ws_create failed ($rc): no CUDA device or invalid options")
        w = new(h[], nothing)
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

# ---- ACE ------------------------------------------------------------------
# pfw_radial_family and pfw_ace_tables of include/pfw_b200.h, field for field
# (isbits structs take the C layout).
struct RadialFamilyC
    nchannels::Int32
    nknots::Int32
    lengths::Ptr{Int32}
    nodes::Ptr{Float64}
    coeff::Ptr{Float64}
    transform::Ptr{Float64}
    powers::Ptr{Int32}
    envelope_kind::Ptr{Int32}
    envelope::Ptr{Float64}
end

struct ACETablesC
    nz::Int32
    lmax::Int32
    radial::RadialFamilyC
    pair::RadialFamilyC
    ndensity::Int32
    density::Ptr{Int32}
    nproducts::Int32
    product_offsets::Ptr{Int32}
    product_factors::Ptr{Int32}
    nbasis::Int32
    ncoupling::Int32
    coupling_rows::Ptr{Int32}
    coupling_cols::Ptr{Int32}
    coupling_vals::Ptr{Float64}
    WB::Ptr{Float64}
    Wpair::Ptr{Float64}
    reference::Ptr{Float64}
    pair_allowed::Ptr{UInt8}
    cutoff::Float64
    angular_kind::Int32
end

const ENVELOPE_CODE = Dict(:PolyEnvelope2sX => Int32(1), :ACE1_PolyEnvelope1sR => Int32(2),
                           :PolyEnvelope1sR => Int32(3))

# One radial family (nz × nz RadialChannel, ACE/resolved.jl:11-17) as the C
# row-major arrays of pfw_radial_family: channel pair k = (centre-1)*nz +
# neighbour, nodes padded to the longest list, coefficients
# [pair][interval][channel][power] (the Julia (4, nch, K-1) array per pair),
# the trainable scale[n, centre, neighbour] (ACE/serial.jl:12-17) folded in.
function pack_family(channels::AbstractMatrix, scale)
    all(ch -> ch isa ACEM.RadialChannel, channels) ||
        throw(ArgumentError("custom radial channels are not packed for the device"))
    nz = size(channels, 1)
    nch = size(first(channels).coefficients, 2)
    nk = maximum(ch -> length(ch.nodes), channels)
    lengths = zeros(Int32, nz * nz); nodes = zeros(nk, nz * nz); coeff = zeros(4, nch, nk - 1, nz * nz)
    transform = zeros(6, nz * nz); powers = zeros(Int32, 2, nz * nz)
    kind = zeros(Int32, nz * nz); env = zeros(5, nz * nz); rcut = 0.0
    for ci = 1:nz, ni = 1:nz
        ch = channels[ci, ni]; t = ch.transform; k = (ci - 1) * nz + ni; K = length(ch.nodes)
        haskey(ENVELOPE_CODE, ch.envelope) || throw(ArgumentError("unsupported radial envelope $(ch.envelope)"))
        c = Float64.(ch.coefficients)
        isnothing(scale) || (c = c .* reshape(Float64.(scale[:, ci, ni]), 1, nch, 1))
        lengths[k] = K
        nodes[1:K, k] .= ch.nodes
        coeff[:, :, 1:K-1, k] .= c
        transform[:, k] .= (t.a, t.rin, t.r0, t.yin, t.ycut, t.rcut)
        powers[:, k] .= (t.p, t.q)
        kind[k] = ENVELOPE_CODE[ch.envelope]
        env[1:length(ch.envelope_parameters), k] .= ch.envelope_parameters
        rcut = max(rcut, Float64(t.rcut))
    end
    (; nch, nk, lengths, nodes, coeff, transform, powers, kind, env, rcut)
end

"""pack_ace(model, ps) — a ResolvedModel and its readout as pfw_ace_tables
(the content of pack_model, ACE/adaptation.jl:57-98): 0-based indices, the
invariant mask folded into WB and the coupling (adaptation.jl:84-87,
interface.jl:125), reference energies and pair terms as the policy allows
(interface.jl:123-124).  Returns the struct and the arrays it points into,
which must stay alive across the load."""
function pack_ace(m, ps)
    pol = m.policy
    isempty(pol.species) && isnothing(pol.orders) ||
        throw(ArgumentError("projected species/order policies are not packed for the device"))
    m.angular_kind in (:real_spherical, :real_solid) || throw(ArgumentError("unsupported angular convention"))
    nz = length(m.atomic_numbers)
    rad = pack_family(m.radial, hasproperty(ps, :radial) ? ps.radial.scale : nothing)
    pq = pack_family(m.pair_radial, hasproperty(ps, :pair) ? ps.pair.scale : nothing)
    density = Int32[v[k] - 1 for k = 1:2, v in m.density]  # (2, D): C [D][2]
    offs = Int32.(cumsum([0; length.(m.products)]))
    facs = Int32[a - 1 for p in m.products for a in p]
    mask = collect(Bool, pol.mask)
    C = m.coupling
    rows = Int32[]; cols = Int32[]; vals = Float64[]
    for j = 1:size(C, 2), q in nzrange(C, j)
        r = rowvals(C)[q]
        mask[r] || continue
        push!(rows, r - 1); push!(cols, j - 1); push!(vals, nonzeros(C)[q])
    end
    WB = vec(Float64.(ps.WB) .* mask)  # (nB, nz): C [nz][nB]
    Wpair = vec(Float64.(ps.Wpair))    # (nQ, nz): C [nz][nQ]
    reference = Float64[pol.reference ? m.reference[z] : 0.0 for z = 1:nz]
    pair_allowed = fill(UInt8(pol.pair), nz)
    family(f) = RadialFamilyC(Int32(f.nch), Int32(f.nk), pointer(f.lengths), pointer(f.nodes), pointer(f.coeff),
                              pointer(f.transform), pointer(f.powers), pointer(f.kind), pointer(f.env))
    t = ACETablesC(Int32(nz), Int32(m.lmax), family(rad), family(pq), Int32(length(m.density)), pointer(density),
                   Int32(length(m.products)), pointer(offs), pointer(facs), Int32(size(C, 1)), Int32(length(vals)),
                   pointer(rows), pointer(cols), pointer(vals), pointer(WB), pointer(Wpair), pointer(reference),
                   pointer(pair_allowed), max(rad.rcut, pq.rcut), m.angular_kind === :real_solid ? Int32(1) : Int32(0))
    t, (rad, pq, density, offs, facs, rows, cols, vals, WB, Wpair, reference, pair_allowed)
end

function load_ace!(w::CUDAWorkspace, calc)
    key = (calc.model, calc.parameters)
    w.ace_key === nothing || w.ace_key[1] !== key[1] || w.ace_key[2] != key[2] || return nothing
    t, keep = pack_ace(calc.model, calc.parameters)
    GC.@preserve keep check(w, ccall((:pfw_ace_model_load, libpfw), Cint, (Ptr{Cvoid}, Ref{ACETablesC}),
                                     w.handle, t))
    w.ace_key = (calc.model, deepcopy(calc.parameters))
    nothing
end

"""ace_evaluate!(w, sys, calc; request) — AC.energy_forces_virial(sys, calc)
(ACE/calculators.jl:48-96) for a reference ACECalculator, on the B200:
species mapped to channels by atomic number (ACE/cpu.jl:315), the model
re-packed only when the calculator's model or parameters changed."""
function ace_evaluate!(w::CUDAWorkspace, sys, calc; request=PP.EnergyForcesVirial())
    upload!(w, sys, channels_for(sys, ChemicalSpecies.(calc.model.atomic_numbers)))
    load_ace!(w, calc)
    n = length(sys)
    E = Ref(0.0); F = zeros(3, n); W = zeros(3, 3)
    check(w, ccall((:pfw_evaluate, libpfw), Cint, (Ptr{Cvoid}, Int32, UInt32, Ref{Float64}, Ptr{Float64}, Ptr{Float64}),
                   w.handle, 1, request_bits(request), E, F, W))
    request isa PP.EnergyOnly && return (; energy=E[] * u"eV")
    (; energy=E[] * u"eV", forces=F * u"eV/Å", virial=W * u"eV")
end

"""site_energies(w) — per-site energies (eV, original order) of the last ACE
evaluation (execute_sites!, NeighbourList/execution.jl:153-167)."""
function site_energies(w::CUDAWorkspace, n::Integer)
    e = zeros(n)
    check(w, ccall((:pfw_site_energies, libpfw), Cint, (Ptr{Cvoid}, Ptr{Float64}), w.handle, e))
    e * u"eV"
end

end # module
