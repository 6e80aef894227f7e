#= ================================================================
   Julia package extension binding the B200 CLE library (libscrna_cle.so)
   behind SyntheticscRNAseq's own GPU CLE interface:

     simulate(net, CLE(dt), kin, Val(:gpu); cell_num, T, readout)       ext/SyntheticscRNAseqCUDAExt.jl:48-52
     simulate(net, CLE(dt), kin, Val(:gpu), pop; T, readout)           ext/SyntheticscRNAseqCUDAExt.jl:409-412
     simulate_gpu_batch(networks, CLE(dt), kin; cell_num, T, readout)  ext/SyntheticscRNAseqCUDAExt.jl:132-136
     simulate(net, BinomialTauLeap(dt), kin, Val(:gpu)[, pop]; ...)    ext/SyntheticscRNAseqCUDAExt.jl:215-219, 542-546
     simulate_gpu_batch(networks, BinomialTauLeap(dt), kin[s][, pop])  ext/SyntheticscRNAseqCUDAExt.jl:290-295, 666-671
     apply_capture(X, capture; seed)                                   src/capture.jl:25

   The extension owns only ccalls: every number is computed by the library.
   Keyword additions (seed, stream, capture, partition) have defaults, so
   existing call sites keep working.  Errors raise like the reference's
   @assert / error() (src/network.jl:66-68, src/population.jl:63).
   ================================================================ =#
module SyntheticscRNAseqB200Ext

using SyntheticscRNAseq
using SyntheticscRNAseq: GeneNetwork, CLE, BinomialTauLeap, KineticParams, PopulationConfig, CaptureModel

const LIB = get(ENV, "SCRNA_CLE_LIB", joinpath(@__DIR__, "..", "libscrna_cle.so"))

struct ScrnaKinetics; k_t::Float64; K_d::Float64; n::Float64; mu_m::Float64; mu_p::Float64; dilution::Float64; end
struct ScrnaPopulation
    cell_num::Int64; growth_rate::Float64; V_div::Float64; V_init_lo::Float64; V_init_hi::Float64
    div_check_interval::Int32; partition::Int32; exclude_mother::Int32; reserved::Int32; growth_noise::Float64
end
struct ScrnaCapture; efficiency::Float64; efficiency_std::Float64; readout::Int32; mean_correction::Int32; end
struct ScrnaOpts
    dt::Float64; T::Float64; cell_num::Int64; readout::Int32; precision::Int32; seed::UInt64
    stream::UInt32; path::Int32; n_steps::Int64; cell_offset::Int64
end

readout_code(r::Symbol) = r === :mrna ? Int32(0) : r === :protein ? Int32(1) :
                          r === :both ? Int32(2) : error("readout must be :mrna, :protein or :both")

function check(rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:scrna_last_error, LIB), Cstring, ()))
    error("libscrna_cle: $msg (status $rc)")
end

const CTX = Ref{Ptr{Cvoid}}(C_NULL)
function context()
    if CTX[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:scrna_ctx_create, LIB), Cint, (Cint, Ref{Ptr{Cvoid}}), 0, h))
        CTX[] = h[]
        atexit(() -> ccall((:scrna_ctx_destroy, LIB), Cint, (Ptr{Cvoid},), CTX[]))
    end
    return CTX[]
end

function upload(net::GeneNetwork)
    G = net.G
    flat(edges) = (Int32[e.target for e in edges],
                   Int32[0; cumsum([length(e.sources) for e in edges])],
                   Int32[s for e in edges for s in e.sources],
                   Float64[e.strength for e in edges])
    ct, cp, cs, cw = flat(net.cooperative)
    rt, rp, rs, rw = flat(net.redundant)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:scrna_net_create, LIB), Cint,
                (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64},
                 Int32, Ptr{Int32}, Ptr{Int32}, Ptr{Int32}, Ptr{Float64},
                 Int32, Ptr{Int32}, Ptr{Int32}, Ptr{Int32}, Ptr{Float64},
                 Ptr{Float64}, Ptr{Float64}, Int32, Ref{Ptr{Cvoid}}),
                context(), G, net.basals, Matrix{Float64}(net.interactions),
                length(ct), ct, cp, cs, cw, length(rt), rt, rp, rs, rw,
                net.k_on, net.k_off, Int32(1), h))
    return h[]
end

release(h) = ccall((:scrna_net_destroy, LIB), Cint, (Ptr{Cvoid},), h)

kin_struct(k::KineticParams) = ScrnaKinetics(k.k_t, k.K_d, k.n, k.mu_m, k.mu_p, k.dilution)

pop_struct(p::PopulationConfig; partition::Symbol=:binomial, exclude_mother::Bool=true) =
    ScrnaPopulation(p.cell_num, p.growth_rate, p.V_div, p.V_init[1], p.V_init[2],
                    Int32(p.div_check_interval), partition === :halve ? Int32(1) : Int32(0),
                    Int32(exclude_mother), Int32(0), p.growth_noise)

cap_struct(c::CaptureModel; mean_correction::Bool=true) =
    ScrnaCapture(c.efficiency, c.efficiency_std, readout_code(c.readout), Int32(mean_correction))

# The library's entry point of an algorithm (simulate / simulate_batch), same arguments.
function call_simulate(alg, args...)
    alg isa BinomialTauLeap ?
        ccall((:scrna_tauleap_simulate, LIB), Cint,
              (Ptr{Cvoid}, Ptr{Cvoid}, Ref{ScrnaKinetics}, Ptr{ScrnaPopulation}, Ptr{ScrnaCapture},
               Ref{ScrnaOpts}, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}), args...) :
        ccall((:scrna_cle_simulate, LIB), Cint,
              (Ptr{Cvoid}, Ptr{Cvoid}, Ref{ScrnaKinetics}, Ptr{ScrnaPopulation}, Ptr{ScrnaCapture},
               Ref{ScrnaOpts}, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}), args...)
end

function call_batch(alg, args...)
    alg isa BinomialTauLeap ?
        ccall((:scrna_tauleap_simulate_batch, LIB), Cint,
              (Ptr{Cvoid}, Int32, Ptr{Ptr{Cvoid}}, Ptr{ScrnaKinetics}, Int32, Ptr{Int64},
               Ptr{Ptr{Cvoid}}, Ptr{ScrnaCapture}, Ref{ScrnaOpts}, Ptr{Ptr{Float64}}, Ptr{Ptr{Int32}}), args...) :
        ccall((:scrna_cle_simulate_batch, LIB), Cint,
              (Ptr{Cvoid}, Int32, Ptr{Ptr{Cvoid}}, Ptr{ScrnaKinetics}, Int32, Ptr{Int64},
               Ptr{Ptr{Cvoid}}, Ptr{ScrnaCapture}, Ref{ScrnaOpts}, Ptr{Ptr{Float64}}, Ptr{Ptr{Int32}}), args...)
end

function run_one(net, alg, kin, pop, N; T, readout, seed, stream, capture)
    h = upload(net)
    try
        cols = readout === :both ? 2 * net.G : net.G
        out = Matrix{Float64}(undef, N, cols)
        counts = capture === nothing ? nothing : Matrix{Int32}(undef, N, net.G)
        eff = capture === nothing ? nothing : Vector{Float64}(undef, N)
        opts = ScrnaOpts(alg.dt, T, N, readout_code(readout), Int32(0), UInt64(seed), UInt32(stream),
                         Int32(0), Int64(0), Int64(0))
        k = kin_struct(kin)
        check(call_simulate(alg, context(), h, k,
                            pop === nothing ? C_NULL : Ref(pop),
                            capture === nothing ? C_NULL : Ref(cap_struct(capture)),
                            opts, out,
                            counts === nothing ? C_NULL : counts,
                            eff === nothing ? C_NULL : eff))
        return capture === nothing ? out : (out, counts, eff)
    finally
        release(h)
    end
end

const GpuAlg = Union{CLE, BinomialTauLeap}

function SyntheticscRNAseq.simulate(net::GeneNetwork, alg::GpuAlg, kin::KineticParams, ::Val{:gpu};
                                    cell_num::Int=1000, T::Float64=50.0, readout::Symbol=:protein,
                                    seed::Integer=0, stream::Integer=0, capture=nothing)
    return run_one(net, alg, kin, nothing, cell_num; T, readout, seed, stream, capture)
end

# The reference's CLE population path halves at division and excludes the mother from the
# Moran draw (cle.jl:249-268); its tau-leap path partitions binomially and may replace any
# cell (ext:643-651).  Both are keywords here.
function SyntheticscRNAseq.simulate(net::GeneNetwork, alg::GpuAlg, kin::KineticParams, ::Val{:gpu},
                                    pop::PopulationConfig; T::Float64=50.0, readout::Symbol=:protein,
                                    seed::Integer=0, stream::Integer=0, capture=nothing,
                                    partition::Symbol=:binomial, exclude_mother::Bool=!(alg isa BinomialTauLeap))
    return run_one(net, alg, kin, pop_struct(pop; partition, exclude_mother), pop.cell_num;
                   T, readout, seed, stream, capture)
end

function run_batch(networks, alg, kins::Vector{ScrnaKinetics}, pops, cells; T, readout, seed, stream)
    B = length(networks)
    hs = [upload(n) for n in networks]
    try
        outs = [Matrix{Float64}(undef, cells[b], readout === :both ? 2 * networks[b].G : networks[b].G) for b in 1:B]
        opts = ScrnaOpts(alg.dt, T, 0, readout_code(readout), Int32(0), UInt64(seed), UInt32(stream),
                         Int32(0), Int64(0), Int64(0))
        popref = pops === nothing ? nothing : [Ref(p) for p in pops]
        GC.@preserve popref begin
            pptrs = pops === nothing ? C_NULL :
                    [Base.unsafe_convert(Ptr{ScrnaPopulation}, r) for r in popref]
            check(call_batch(alg, context(), Int32(B), hs, kins, Int32(length(kins)), cells,
                             pptrs, C_NULL, opts, [pointer(o) for o in outs], C_NULL))
        end
        return outs
    finally
        foreach(release, hs)
    end
end

# One KineticParams for all networks, or one per network (ext:689-720).
function SyntheticscRNAseq.simulate_gpu_batch(networks::Vector{GeneNetwork}, alg::GpuAlg,
                                              kin::Union{KineticParams, Vector{<:KineticParams}};
                                              cell_num=1000, T::Float64=50.0,
                                              readout::Symbol=:protein, seed::Integer=0, stream::Integer=0)
    B = length(networks)
    cells = cell_num isa Integer ? fill(Int64(cell_num), B) : Int64.(cell_num)
    kins = kin isa KineticParams ? [kin_struct(kin)] : [kin_struct(k) for k in kin]
    return run_batch(networks, alg, kins, nothing, cells; T, readout, seed, stream)
end

# With one population config for every network (ext:666-671).
function SyntheticscRNAseq.simulate_gpu_batch(networks::Vector{GeneNetwork}, alg::GpuAlg,
                                              kin::Union{KineticParams, Vector{<:KineticParams}},
                                              pop::PopulationConfig; T::Float64=50.0,
                                              readout::Symbol=:protein, seed::Integer=0, stream::Integer=0,
                                              partition::Symbol=:binomial,
                                              exclude_mother::Bool=!(alg isa BinomialTauLeap))
    B = length(networks)
    kins = kin isa KineticParams ? [kin_struct(kin)] : [kin_struct(k) for k in kin]
    ps = [pop_struct(pop; partition, exclude_mother) for _ in 1:B]
    return run_batch(networks, alg, kins, ps, fill(Int64(pop.cell_num), B); T, readout, seed, stream)
end

function SyntheticscRNAseq.apply_capture(X::Matrix{<:Real}, capture::CaptureModel, ::Val{:gpu};
                                         seed::Integer=0, stream::Integer=0)
    N, G = size(X)
    Xd = Matrix{Float64}(X)
    Y = Matrix{Int32}(undef, N, G)
    c = cap_struct(capture)
    check(ccall((:scrna_apply_capture, LIB), Cint,
                (Ptr{Cvoid}, Int64, Int32, Ptr{Float64}, Ref{ScrnaCapture}, UInt64, UInt32, Ptr{Int32}, Ptr{Float64}),
                context(), N, G, Xd, c, UInt64(seed), UInt32(stream), Y, C_NULL))
    return Matrix{Int}(Y)
end

end # module
