// Tensor-core path for large dense networks.
//
// For G in the thousands with ~10 % dense regulation, the additive term
// reg = sum_j A_eff[i,j] act_j (the one-GEMM form of A_pos act + A_neg rep,
// network.jl:206-219, cle.jl:84-86) is a real dense GEMM per Euler step:
//     REG[N x G] = ACT[N x K] * W^T,  W = A_eff as 16-bit [G][K], ACT 16-bit [N][K]
// with FP32 accumulation.  The cooperative / redundant terms (cle.jl:89-106) are extra K
// columns: column G + j of ACT holds the value of term j (the product over its sources,
// from their FP32 activations) and W[target_j][G + j] its coefficient s_j beta_target.
// Each step is a small kernel writing the term columns, the GEMM (cuBLASLt, BF16 or FP16
// inputs) and one fused FP32 kernel that adds the repression constant, applies telegraph
// switching, draws the Philox increments, updates M and P (cle.jl:109-120) and writes the
// next step's 16-bit activations.  State is
// cell-major [N][ld], ld = G rounded up to a whole gene pair, so that both kernels stream
// it with unit stride and the step kernel moves each gene pair with one 8-byte access.
#include <cublasLt.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "capi_internal.h"
#include "cle_device.cuh"
#include "tau_lockstep.cuh"

namespace scrna {

template <class T> __device__ __forceinline__ T to16(float x);
template <> __device__ __forceinline__ __nv_bfloat16 to16<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <> __device__ __forceinline__ __half to16<__half>(float x) { return __float2half_rn(x); }

// Row stride of the cell-major state: G rounded up to a whole gene pair.
inline int tensor_ld(int G) { return (G + 1) & ~1; }

struct TensorArgs {
    int32_t G, ld, Kp, n_src;
    int64_t N, cell_offset;
    int32_t step;
    float k_t, Kn, hill_n, mu_m, mu_p, dt;
    int32_t hill_int;
    uint32_t key0, key1, stream;
    uint32_t rk0[10], rk1[10];   // Philox round keys of (key0, key1)
    const GeneRec* genes;
    const GeneInit* ginit;
    const NonAdd* na;        // sources are compact source indices
    const int32_t* na_src;
    const int32_t* src_of_gene;  // gene -> compact source index or -1
    int32_t n_terms;         // cooperative / redundant terms = extra K columns G .. G + n_terms
    float* reg;              // [N][ld] GEMM output of this step
    float* M;                // [N][ld] (as P, prom, NS)
    float* P;
    uint8_t* prom;
    int2* NS;
    void* act16;             // [N][Kp]
    const float* act32_cur;  // [n_src][N]: source-major, 32 cells of a warp in one 128-byte row piece
    float* act32_next;
    float p_dec_m, p_dec_p;  // binomial tau-leap: decay probabilities 1 - exp(-mu dt)
    // exact regulation (the tau-leap): reg holds the register path's FP32 regulation, cneg
    // included, from the slot-major activations act32 [n_reg][N] (src_of_gene: the slots)
    int32_t exact_reg;
    const float2* in_edge;   // the register path's additive in-edges {w, slot bits}
    const int32_t* na_slot;  // the register path's term sources (regulator slots)
    // population (cle.jl:143-284, ext:409-529, tau-leap ext:531-663); V == nullptr without one.
    // The daughter buffers are cell-major [N][ld] like the state.
    double* V;               // [N] volume at the start of the step
    double growth_factor, V_div, V_lo, V_hi;
    int32_t partition, exclude_mother, tau, epoch;  // tau: Hill of P / V, counts from steady state x V
    unsigned long long* owner;  // [N] epoch << 32 | donor cell of the last claim
    uint8_t* divided;        // [N] the cell divided at this check
    float* dM;
    float* dP;
    uint8_t* dprom;
    int2* dNS;
    double* dV;              // [N] the daughter's volume
    const double* beta64;    // tau-leap initial counts max(1, round(steady state x V)) (ext:560-566)
    double ss_mu_m, ss_mu_p, k_t64;
};

// Initial state (cle.jl:49-53), promoter draws and first activations; thread per (cell, gene).
template <class T>
__global__ void tensor_init_kernel(const TensorArgs a) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.N * a.G) return;
    const int64_t c = idx / a.G;
    const int g = (int)(idx - c * a.G);
    const Key key{a.key0, a.key1};
    const uint32_t gcell = (uint32_t)(a.cell_offset + c);
    const GeneInit gi = a.ginit[g];
    const int64_t sidx = c * a.ld + g;  // state index
    const GeneRec gr = a.genes[g];
    float m0 = gi.m0, p0 = gi.p0;
    double V = 1.0;
    if (a.V) {  // the cell's birth volume (TAG_VOLUME), as the register path draws it
        const uint4 w = philox(gcell, 0u, 0u, tagword(TAG_VOLUME, a.stream), key);
        V = __dadd_rn(a.V_lo, __dmul_rn(__dadd_rn(a.V_hi, -a.V_lo), u53(w.x, w.y)));
        if (g == 0) a.V[c] = V;
        if (a.tau) {
            const double mss = __ddiv_rn(a.beta64[g], a.ss_mu_m);
            const double pss = __ddiv_rn(__dmul_rn(a.k_t64, mss), a.ss_mu_p);
            m0 = (float)fmax(1.0, rint(__dmul_rn(mss, V)));
            p0 = (float)fmax(1.0, rint(__dmul_rn(pss, V)));
        }
    }
    a.M[sidx] = m0;
    a.P[sidx] = p0;
    bool on = true;
    if (gi.init_rand) {
        const uint4 w = philox(gcell, 0u, (uint32_t)(g >> 2), tagword(TAG_PROMOTER, a.stream), key);
        const uint32_t x = (g & 3) == 0 ? w.x : (g & 3) == 1 ? w.y : (g & 3) == 2 ? w.z : w.w;
        on = x < gi.thr_init;
    }
    a.prom[sidx] = on;
    int2 ns = make_int2(kNever, kNever);
    if (gr.inv_off == gr.inv_off) {
        const uint4 w = philox(gcell, 0u, (uint32_t)g, tagword(TAG_SWITCH, a.stream), key);
        ns = fresh_switch(0, w.x, w.y, on, gr.inv_on, gr.inv_off);
    }
    a.NS[sidx] = ns;
    const float act = hill_act(a.V && a.tau ? __fdiv_rn(p0, (float)V) : p0, a.Kn, a.hill_n, a.hill_int);
    if (!a.exact_reg) reinterpret_cast<T*>(a.act16)[c * a.Kp + g] = to16<T>(act);
    const int src = a.src_of_gene[g];
    if (src >= 0) a.act32_next[(size_t)src * a.N + c] = act;
}

// One Euler-Maruyama step after the GEMM.  Thread = one gene pair (blockIdx.y, x) for a chunk
// of kTensorCellsPerThread cells (blockIdx.x); per-gene constants stay in registers across the
// chunk, consecutive threads touch consecutive gene pairs of one cell (unit-stride rows, one
// 8-byte access per pair).  The kernel is bound by HBM: every thread issues the loads of its
// whole chunk (GEMM output, M, P) before computing, so enough bytes are in flight.
constexpr int kTensorCellsPerThread = 8;
constexpr int kTensorPairsPerBlock = 128;

template <class T> struct Pair16;
template <> struct Pair16<__nv_bfloat16> { using type = __nv_bfloat162; };
template <> struct Pair16<__half> { using type = __half2; };

// Term columns of the activation matrix: block = (128 cells, 8 consecutive terms), thread =
// one cell.  The FP32 activations of the terms' compact source genes (written by the previous
// step) are source-major, so a warp reads one 128-byte piece per source; the first 4 sources
// of all 8 terms (32 loads) are in flight together, longer terms loop over the rest.  Each
// cell writes its 8 term columns with one 16-byte store where the row offset allows.
constexpr int kTermsBlock = 128;
constexpr int kTermsGroup = 8;
constexpr int kTermsSrc = 4;
template <class T>
__global__ void __launch_bounds__(kTermsBlock) tensor_terms_kernel(const TensorArgs a) {
    __shared__ int s_src[kTermsGroup][kTermsSrc];  // compact source index or -1
    __shared__ int s_rest[kTermsGroup][2];         // remaining sources [begin, end) of na_src
    __shared__ int s_red[kTermsGroup];             // redundant: 1 - prod(1 - a)
    const int j0 = blockIdx.y * kTermsGroup;
    const int nj = min(kTermsGroup, a.n_terms - j0);
    if (threadIdx.x < kTermsGroup * kTermsSrc) {
        const int k = threadIdx.x / kTermsSrc, q = threadIdx.x % kTermsSrc;
        int v = -1, rb = 0, re = 0, red = 0;
        if (k < nj) {
            const NonAdd na = a.na[j0 + k];
            const int t = na.src_begin + q;
            v = t < na.src_end ? a.na_src[t] : -1;
            rb = na.src_begin + kTermsSrc;
            re = na.src_end;
            red = na.kind != 0;
        }
        s_src[k][q] = v;
        if (q == 0) {
            s_rest[k][0] = rb;
            s_rest[k][1] = re;
            s_red[k] = red;
        }
    }
    __syncthreads();
    const int64_t N = a.N;
    const int64_t c = (int64_t)blockIdx.x * kTermsBlock + threadIdx.x;
    if (c >= N) return;
    const float* act = a.act32_cur + c;
    float x[kTermsGroup][kTermsSrc];
#pragma unroll
    for (int k = 0; k < kTermsGroup; ++k)
#pragma unroll
        for (int q = 0; q < kTermsSrc; ++q) {
            const int si = s_src[k][q];
            x[k][q] = si >= 0 ? act[(size_t)si * (size_t)N] : 0.0f;
        }
    uint16_t v16[kTermsGroup];
#pragma unroll
    for (int k = 0; k < kTermsGroup; ++k) {
        const bool red = s_red[k] != 0;
        float prod = 1.0f;
#pragma unroll
        for (int q = 0; q < kTermsSrc; ++q)
            if (s_src[k][q] >= 0) prod *= red ? 1.0f - x[k][q] : x[k][q];  // uniform per block
        for (int t = s_rest[k][0]; t < s_rest[k][1]; ++t) {
            const float y = act[(size_t)a.na_src[t] * (size_t)N];
            prod *= red ? 1.0f - y : y;
        }
        const T r = to16<T>(red ? 1.0f - prod : prod);
        v16[k] = *reinterpret_cast<const uint16_t*>(&r);
    }
    uint16_t* row = reinterpret_cast<uint16_t*>(a.act16) + (size_t)c * a.Kp + a.G + j0;
    const int off = a.G + j0;  // row offset in elements; rows are 16-byte aligned (Kp % 64 == 0)
    if (nj == kTermsGroup && (off & 7) == 0) {
        uint32_t w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) w[i] = (uint32_t)v16[2 * i] | ((uint32_t)v16[2 * i + 1] << 16);
        *reinterpret_cast<uint4*>(row) = make_uint4(w[0], w[1], w[2], w[3]);
    } else {
        for (int k = 0; k < nj; ++k) row[k] = v16[k];
    }
}

static cudaError_t terms_launch(int dtype, const TensorArgs& a, cudaStream_t st) {
    if (a.N == 0 || a.n_terms == 0) return cudaSuccess;
    const dim3 grid((unsigned)((a.N + kTermsBlock - 1) / kTermsBlock),
                    (unsigned)((a.n_terms + kTermsGroup - 1) / kTermsGroup));
    if (dtype == 0) tensor_terms_kernel<__nv_bfloat16><<<grid, kTermsBlock, 0, st>>>(a);
    else tensor_terms_kernel<__half><<<grid, kTermsBlock, 0, st>>>(a);
    return cudaGetLastError();
}

// Term columns for the fused tcgen05 path (same kernel, its own activation buffer).
cudaError_t tensor_terms_launch(int dtype, int64_t N, int G, int Kp, int n_terms, int n_src, const NonAdd* na,
                                const int32_t* na_src, const float* act32, void* act16, cudaStream_t st) {
    TensorArgs a{};
    a.N = N; a.G = G; a.Kp = Kp; a.n_terms = n_terms; a.n_src = n_src;
    a.na = na; a.na_src = na_src; a.act32_cur = act32; a.act16 = act16;
    return terms_launch(dtype, a, st);
    return cudaGetLastError();
}

template <int HN>
__device__ __forceinline__ float tensor_hill(float p, const TensorArgs& a) {
    if (HN == 2) {
        const float pn = p * p;
        return fminf(pn * frcp_approx(pn + a.Kn), 1.0f);  // as hill_act with hill_int == 2
    }
    return hill_act(p, a.Kn, a.hill_n, a.hill_int);
}

template <class T, bool BURSTY, int HN>
__global__ void __launch_bounds__(kTensorPairsPerBlock) tensor_step_kernel(const TensorArgs a) {
    using T2 = typename Pair16<T>::type;
    const int k = blockIdx.y * kTensorPairsPerBlock + threadIdx.x;
    if (k >= (a.ld >> 1)) return;
    const int g0 = 2 * k;
    const bool has1 = g0 + 1 < a.G;  // the second gene of the pair exists (else: row padding)
    const GeneRec r0 = a.genes[g0];
    const GeneRec r1 = a.genes[has1 ? g0 + 1 : g0];
    const int src0 = a.src_of_gene[g0];
    const int src1 = has1 ? a.src_of_gene[g0 + 1] : -1;
    const uint32_t c3 = tagword(TAG_NORMAL, a.stream);
    const int s = a.step;
    const int64_t c_begin = (int64_t)blockIdx.x * kTensorCellsPerThread;
    const int64_t c_end = c_begin + kTensorCellsPerThread < a.N ? c_begin + kTensorCellsPerThread : a.N;
    const size_t rs = (size_t)(a.ld >> 1);  // row stride in pairs
    const float2* regp = reinterpret_cast<const float2*>(a.reg) + (size_t)c_begin * rs + k;
    float2* Mp = reinterpret_cast<float2*>(a.M) + (size_t)c_begin * rs + k;
    float2* Pp = reinterpret_cast<float2*>(a.P) + (size_t)c_begin * rs + k;
    T2* actp = reinterpret_cast<T2*>(a.act16) + (size_t)c_begin * (a.Kp >> 1) + k;
    constexpr int CPT = kTensorCellsPerThread;
    const int nc = (int)(c_end - c_begin);
    float2 rg[CPT], mm[CPT], pp[CPT];
#pragma unroll
    for (int i = 0; i < CPT; ++i) {
        if (i < nc) {
            rg[i] = regp[i * rs];
            mm[i] = Mp[i * rs];
            pp[i] = Pp[i * rs];
        }
    }
#pragma unroll
    for (int i = 0; i < CPT; ++i) {
        if (i >= nc) break;
        const int64_t c = c_begin + i;
        const uint32_t gcell = (uint32_t)(a.cell_offset + c);
        const uint4 w = philox_rk(gcell, (uint32_t)s, (uint32_t)k, c3, a.rk0, a.rk1);
        float tx0 = (rg[i].x + r0.cneg) + r0.beta, tx1 = (rg[i].y + r1.cneg) + r1.beta;
        if (a.V) {  // population: transcription x V (cle.jl:200-214)
            const float Vf = (float)a.V[c];
            tx0 *= Vf;
            tx1 *= Vf;
        }
        if (BURSTY) {
            const size_t e = (size_t)c * a.ld + g0;
            const uchar2 on = *reinterpret_cast<const uchar2*>(a.prom + e);
            const int4 sw = *reinterpret_cast<const int4*>(a.NS + e);
            bool on0 = on.x, on1 = on.y;
            if (s == sw.x) {  // waiting time from the spare bits of the normal words
                on0 = !on0;
                a.NS[e] = switch_at(s, make_int2(sw.x, sw.y), switch_uniform(w.x, w.y), on0, r0.inv_on, r0.inv_off);
                a.prom[e] = on0;
            }
            if (has1 && s == sw.z) {
                on1 = !on1;
                a.NS[e + 1] = switch_at(s, make_int2(sw.z, sw.w), switch_uniform(w.z, w.w), on1, r1.inv_on, r1.inv_off);
                a.prom[e + 1] = on1;
            }
            if (!on0) tx0 = 0.0f;
            if (!on1) tx1 = 0.0f;
        }
        float2 m2 = mm[i], p2 = pp[i];
        em_update(m2.x, p2.x, tx0, box_muller_parts(w.x, w.y), a.mu_m, a.mu_p, a.k_t, a.dt);
        em_update(m2.y, p2.y, tx1, box_muller_parts(w.z, w.w), a.mu_m, a.mu_p, a.k_t, a.dt);
        Mp[i * rs] = m2;
        Pp[i * rs] = p2;
        const float a0 = tensor_hill<HN>(p2.x, a), a1 = tensor_hill<HN>(p2.y, a);
        T2 act;
        act.x = to16<T>(a0);
        act.y = to16<T>(has1 ? a1 : 0.0f);  // the padding column of the activations stays 0
        actp[(size_t)i * (a.Kp >> 1)] = act;
        if (src0 >= 0) a.act32_next[(size_t)src0 * a.N + c] = a0;
        if (src1 >= 0) a.act32_next[(size_t)src1 * a.N + c] = a1;
    }
}

// Exact regulation of the tau-leap's tensor form: the regulation of gene `gr` in one cell in
// FP32 with the register path's operations in its order (the regulation of cle_fused.cuh: the
// repression constant, the additive in-edges in table order, then the cooperative and
// redundant terms), from the slot-major activations of the step's start (`act`: the cell's
// element of slot 0; lanes over consecutive cells read one 128-byte row piece per slot, each
// edge a broadcast load), so the counts equal the register path's bit for bit.
__device__ __forceinline__ float exact_regulation(const TensorArgs& a, const GeneRec& gr, const float* act) {
    const size_t N = (size_t)a.N;
    float reg = gr.cneg;
    for (int e = gr.in_begin; e < gr.in_end; ++e) {
        const float2 ed = __ldg(a.in_edge + e);
        reg = fmaf(ed.x, act[(size_t)__float_as_int(ed.y) * N], reg);
    }
    const int nab = gr.na_range >> 16, nac = gr.na_range & 0xFFFF;
    for (int e = nab; e < nab + nac; ++e) {
        const NonAdd na = a.na[e];
        float prod = 1.0f;
        if (na.kind == 0) {
            for (int t = na.src_begin; t < na.src_end; ++t) prod *= act[(size_t)__ldg(a.na_slot + t) * N];
            reg = fmaf(na.coef, prod, reg);
        } else {
            for (int t = na.src_begin; t < na.src_end; ++t) prod *= 1.0f - act[(size_t)__ldg(a.na_slot + t) * N];
            reg = fmaf(na.coef, 1.0f - prod, reg);
        }
    }
    return reg;
}

// One binomial tau-leap step, with the regulation computed here (exact_regulation above) or
// taken from the GEMM (ext/SyntheticscRNAseqCUDAExt.jl:215-399 for networks of any size), on
// tiles of 32 cells x 16 gene pairs.  The draws are bound by latency and warp
// divergence, not by HBM: a warp's lanes are the 32 cells of one gene pair, whose Poisson means
// are alike (lanes over different genes would wait for the gene with the longest chains).  The
// tile moves between the cell-major state and shared memory along gene pairs (coalesced), and
// the compute reads it along cells.  Per (cell, gene): the tau-leap's Philox block (tag 9),
// switching from its spare bits, and the pair's draws in lock step (tau_update_unit, the
// register path's arithmetic); with the exact regulation the counts equal the register path's
// bit for bit, and without regulation (the GEMM then gives exactly 0) the oracle's as well.
constexpr int kTauTileCells = 32, kTauTilePairs = 16, kTauTileThreads = 256;

template <class T, bool BURSTY, int HN>
__global__ void __launch_bounds__(kTauTileThreads) tensor_tau_step_kernel(const TensorArgs a) {
    using T2 = typename Pair16<T>::type;
    constexpr int TP = kTauTilePairs + 1;  // padded row: lanes (cells) fall in different banks
    __shared__ float2 s_reg[kTauTileCells][TP], s_m[kTauTileCells][TP], s_p[kTauTileCells][TP];
    __shared__ T2 s_act[kTauTileCells][TP];
    __shared__ int4 s_ns[BURSTY ? kTauTileCells : 1][TP];
    __shared__ uchar2 s_on[BURSTY ? kTauTileCells : 1][TP];
    __shared__ uint8_t s_sw[BURSTY ? kTauTileCells : 1][TP];  // a promoter of the pair switched
    const int t = threadIdx.x;
    const int64_t c0 = (int64_t)blockIdx.x * kTauTileCells;
    const int k0 = blockIdx.y * kTauTilePairs;
    const int pairs = a.ld >> 1;
    const size_t rs = (size_t)pairs;  // state row stride in pairs
    // load along gene pairs
    for (int i = t; i < kTauTileCells * kTauTilePairs; i += kTauTileThreads) {
        const int r = i / kTauTilePairs, q = i - r * kTauTilePairs;
        const int64_t c = c0 + r;
        const int k = k0 + q;
        if (c >= a.N || k >= pairs) continue;
        const size_t e = (size_t)c * rs + k;
        if (!a.exact_reg) s_reg[r][q] = reinterpret_cast<const float2*>(a.reg)[e];
        s_m[r][q] = reinterpret_cast<const float2*>(a.M)[e];
        s_p[r][q] = reinterpret_cast<const float2*>(a.P)[e];
        if (BURSTY) {
            s_on[r][q] = reinterpret_cast<const uchar2*>(a.prom)[e];
            s_ns[r][q] = reinterpret_cast<const int4*>(a.NS)[e];
            s_sw[r][q] = 0;
        }
    }
    __syncthreads();
    // compute along cells: lane = cell, warp = gene pair (and the pair 8 further)
    const int r = t & 31;
    const int64_t c = c0 + r;
    const uint32_t gcell = (uint32_t)(a.cell_offset + c);
    const uint32_t c3 = tagword(TAG_TAU, a.stream);
    const int s = a.step;
    float Vf = 1.0f, Vn = 1.0f;  // the volume now and at the start of the next step (Hill of P / V)
    if (a.V && c < a.N) {
        const double V = a.V[c];
        Vf = (float)V;
        Vn = (float)__dmul_rn(V, a.growth_factor);
    }
    for (int q = t >> 5; q < kTauTilePairs; q += kTauTileThreads / 32) {
        const int k = k0 + q;
        if (c >= a.N || k >= pairs) continue;
        const int g0 = 2 * k;
        const bool has1 = g0 + 1 < a.G;  // the second gene of the pair exists (else: row padding)
        const GeneRec r0 = a.genes[g0];
        const GeneRec r1 = a.genes[has1 ? g0 + 1 : g0];
        uint4 w[2];
        w[0] = philox_rk(gcell, (uint32_t)s, (uint32_t)g0, c3, a.rk0, a.rk1);
        w[1] = has1 ? philox_rk(gcell, (uint32_t)s, (uint32_t)(g0 + 1), c3, a.rk0, a.rk1) : make_uint4(0u, 0u, 0u, 0u);
        float reg0, reg1;
        if (a.exact_reg) {
            const float* act = a.act32_cur + c;
            reg0 = exact_regulation(a, r0, act);
            reg1 = has1 ? exact_regulation(a, r1, act) : 0.0f;
        } else {  // the GEMM's sum, which takes the repression constant afterwards
            const float2 rg = s_reg[r][q];
            reg0 = __fadd_rn(rg.x, r0.cneg);
            reg1 = __fadd_rn(rg.y, r1.cneg);
        }
        float tx0 = fmaxf(__fadd_rn(reg0, r0.beta), 0.0f);
        float tx1 = fmaxf(__fadd_rn(reg1, r1.beta), 0.0f);
        if (a.V) {
            tx0 = __fmul_rn(tx0, Vf);
            tx1 = __fmul_rn(tx1, Vf);
        }
        bool on0 = true, on1 = true;
        if (BURSTY) {  // switching before the transcription update (tauleap_binomial.jl:111-121)
            const uchar2 on = s_on[r][q];
            int4 sw = s_ns[r][q];
            on0 = on.x;
            on1 = on.y;
            bool changed = false;
            if (s == sw.x) {
                on0 = !on0;
                const int2 n0 = switch_at(s, make_int2(sw.x, sw.y), switch_uniform(w[0].x, w[0].y), on0, r0.inv_on,
                                          r0.inv_off);
                sw.x = n0.x;
                sw.y = n0.y;
                changed = true;
            }
            if (has1 && s == sw.z) {
                on1 = !on1;
                const int2 n1 = switch_at(s, make_int2(sw.z, sw.w), switch_uniform(w[1].x, w[1].y), on1, r1.inv_on,
                                          r1.inv_off);
                sw.z = n1.x;
                sw.w = n1.y;
                changed = true;
            }
            if (changed) {
                s_ns[r][q] = sw;
                s_on[r][q] = make_uchar2(on0, on1);
                s_sw[r][q] = 1;
            }
        }
        const float lam[2] = {on0 ? __fmul_rn(tx0, a.dt) : 0.0f, (has1 && on1) ? __fmul_rn(tx1, a.dt) : 0.0f};
        // the padding slot of an odd G holds no state (never initialised): counts 0
        const float2 mm = s_m[r][q], pp = s_p[r][q];
        float m2[2] = {mm.x, has1 ? mm.y : 0.0f}, p2[2] = {pp.x, has1 ? pp.y : 0.0f};
        tau_update_unit<2>(m2, p2, lam, w, has1 ? 2 : 1, true, a.k_t, a.dt, a.p_dec_m, a.p_dec_p);
        s_m[r][q] = make_float2(m2[0], m2[1]);
        s_p[r][q] = make_float2(p2[0], p2[1]);
        const float a0 = tensor_hill<HN>(a.V ? __fdiv_rn(p2[0], Vn) : p2[0], a);
        const float a1 = tensor_hill<HN>(a.V ? __fdiv_rn(p2[1], Vn) : p2[1], a);
        T2 act;
        act.x = to16<T>(a0);
        act.y = to16<T>(has1 ? a1 : 0.0f);  // the padding column of the activations stays 0
        s_act[r][q] = act;
        const int src0 = a.src_of_gene[g0];
        const int src1 = has1 ? a.src_of_gene[g0 + 1] : -1;
        if (src0 >= 0) a.act32_next[(size_t)src0 * a.N + c] = a0;  // lanes: consecutive cells
        if (src1 >= 0) a.act32_next[(size_t)src1 * a.N + c] = a1;
    }
    __syncthreads();
    // store along gene pairs
    for (int i = t; i < kTauTileCells * kTauTilePairs; i += kTauTileThreads) {
        const int rr = i / kTauTilePairs, q = i - rr * kTauTilePairs;
        const int64_t cc = c0 + rr;
        const int k = k0 + q;
        if (cc >= a.N || k >= pairs) continue;
        const size_t e = (size_t)cc * rs + k;
        reinterpret_cast<float2*>(a.M)[e] = s_m[rr][q];
        reinterpret_cast<float2*>(a.P)[e] = s_p[rr][q];
        if (!a.exact_reg) reinterpret_cast<T2*>(a.act16)[(size_t)cc * (a.Kp >> 1) + k] = s_act[rr][q];
        if (BURSTY && s_sw[rr][q]) {
            reinterpret_cast<uchar2*>(a.prom)[e] = s_on[rr][q];
            reinterpret_cast<int4*>(a.NS)[e] = s_ns[rr][q];
        }
    }
}

// ---- population on the tensor path: growth, division checks, Moran replacement ---------------
// The register path's semantics (cle_fused.cuh epilogue, cle.jl:240-273): after each step
// V <- V growth_factor; at a check step a cell with V > V_div halves V, partitions each gene's
// counts (halved, or a binomial split of the rounded counts) into itself and a daughter, and the
// daughter replaces a Moran slot drawn from (cell, step); of several claims on one slot the
// largest donor index wins.  The daughter keeps the mother's promoters and draws fresh waiting
// times.  Three kernels per check: decide and claim (per cell), partition (per cell x gene),
// place daughters and refresh the next step's activations of every changed cell.

__global__ void tensor_growth_kernel(double* V, int64_t N, double growth_factor) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < N) V[c] = __dmul_rn(V[c], growth_factor);
}

__global__ void tensor_divide_kernel(const TensorArgs a) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    double V = a.V[c];
    if (!(V > a.V_div)) {
        a.divided[c] = 0;
        return;
    }
    V = V * 0.5;
    a.V[c] = V;
    a.dV[c] = V;
    a.divided[c] = 1;
    const Key key{a.key0, a.key1};
    const uint4 w = philox((uint32_t)(a.cell_offset + c), (uint32_t)a.step, 0u, tagword(TAG_MORAN, a.stream), key);
    int64_t r;
    if (a.exclude_mother) {
        r = (int64_t)(((uint64_t)w.x * (uint64_t)(a.N - 1)) >> 32);
        if (r >= c) r += 1;
    } else {
        r = (int64_t)(((uint64_t)w.x * (uint64_t)a.N) >> 32);
    }
    atomicMax(&a.owner[r], ((unsigned long long)(uint32_t)(a.epoch + 1) << 32) | (unsigned long long)c);
}

__global__ void tensor_partition_kernel(const TensorArgs a) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.N * a.G) return;
    const int64_t c = idx / a.G;
    const int g = (int)(idx - c * a.G);
    if (!a.divided[c]) return;
    const size_t e = (size_t)c * a.ld + g;
    const uint32_t gcell = (uint32_t)(a.cell_offset + c);
    const Key key{a.key0, a.key1};
    const float m = a.M[e], p = a.P[e];
    float mm, dm, pm, dp;
    if (a.partition == 1) {  // halve
        mm = dm = m * 0.5f;
        pm = dp = p * 0.5f;
    } else {  // binomial split of rounded counts
        const int64_t mi = (int64_t)rintf(m);
        const int64_t pi = (int64_t)rintf(p);
        const int64_t mk = binomial_half(mi, key, a.stream, gcell, (uint32_t)a.step, (uint32_t)g, 0u);
        const int64_t pk = binomial_half(pi, key, a.stream, gcell, (uint32_t)a.step, (uint32_t)g, 1u);
        mm = (float)mk; dm = (float)(mi - mk);
        pm = (float)pk; dp = (float)(pi - pk);
    }
    a.M[e] = mm;
    a.P[e] = pm;
    a.dM[e] = dm;
    a.dP[e] = dp;
    const uint8_t bon = a.prom[e];
    a.dprom[e] = bon;
    int2 dns = make_int2(kNever, kNever);
    const GeneRec gr = a.genes[g];
    if (gr.inv_off == gr.inv_off) {  // the daughter's promoter switches independently of the mother's
        const uint4 w = philox(gcell, (uint32_t)a.step, (uint32_t)g | kDaughterSwitch, tagword(TAG_SWITCH, a.stream), key);
        dns = fresh_switch(a.step, w.x, w.y, bon, gr.inv_on, gr.inv_off);
    }
    a.dNS[e] = dns;
}

template <class T, int HN>
__global__ void tensor_replace_kernel(const TensorArgs a) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.N * a.G) return;
    const int64_t c = idx / a.G;
    const int g = (int)(idx - c * a.G);
    const unsigned long long o = a.owner[c];
    const bool replaced = (uint32_t)(o >> 32) == (uint32_t)(a.epoch + 1);
    if (!replaced && !a.divided[c]) return;
    const size_t e = (size_t)c * a.ld + g;
    float p;
    double V;
    if (replaced) {  // the donor's daughter takes this slot
        const int64_t src = (int64_t)(o & 0xFFFFFFFFull);
        const size_t es = (size_t)src * a.ld + g;
        a.M[e] = a.dM[es];
        p = a.dP[es];
        a.P[e] = p;
        a.prom[e] = a.dprom[es];
        a.NS[e] = a.dNS[es];
        V = a.dV[src];
        if (g == 0) a.V[c] = V;
    } else {  // a mother that kept its slot: its halved counts
        p = a.P[e];
        V = a.V[c];
    }
    const float act = tensor_hill<HN>(a.tau ? __fdiv_rn(p, (float)V) : p, a);
    if (!a.exact_reg) reinterpret_cast<T*>(a.act16)[c * a.Kp + g] = to16<T>(act);
    const int src_idx = a.src_of_gene[g];
    if (src_idx >= 0) a.act32_next[(size_t)src_idx * a.N + c] = act;
}

// The tau-leap's cell-major state [N][ld] into the register path's gene-major [G][N] (counts,
// promoters, switching times), through shared-memory tiles of 32 cells x 32 genes so both
// sides run along their rows.  With exact regulation both forms hold the same state bit for
// bit, so a continuation or a checkpoint takes it as the register path's own.
__global__ void tensor_to_gene_major_kernel(int G, int ld, int64_t N, const float* __restrict__ tM,
                                            const float* __restrict__ tP, const uint8_t* __restrict__ tprom,
                                            const int2* __restrict__ tNS, float* M, float* P, uint8_t* prom, int2* NS) {
    __shared__ float sm[32][33], sp[32][33];
    __shared__ int2 sns[32][33];
    __shared__ uint8_t spr[32][33];
    const int64_t c0 = (int64_t)blockIdx.x * 32;
    const int g0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {  // row r: cell c0 + r, lanes along genes
        const int64_t c = c0 + r;
        const int g = g0 + tx;
        if (c < N && g < G) {
            const size_t e = (size_t)c * ld + g;
            sm[r][tx] = tM[e];
            sp[r][tx] = tP[e];
            spr[r][tx] = tprom[e];
            sns[r][tx] = tNS[e];
        }
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {  // row r: gene g0 + r, lanes along cells
        const int g = g0 + r;
        const int64_t c = c0 + tx;
        if (c < N && g < G) {
            const size_t e = (size_t)g * N + c;
            M[e] = sm[tx][r];
            P[e] = sp[tx][r];
            prom[e] = spr[tx][r];
            NS[e] = sns[tx][r];
        }
    }
}

int tensor_state_to_register(scrna_ctx* ctx, scrna_state* st) {
    if (int r = state_alloc(st, st->last_pop, false)) return r;
    const dim3 grid((unsigned)((st->N + 31) / 32), (unsigned)((st->G + 31) / 32));
    tensor_to_gene_major_kernel<<<grid, dim3(32, 8), 0, ctx->stream>>>(
        st->G, st->t_ld, st->N, st->tM.as<float>(), st->tP.as<float>(), st->tprom.as<uint8_t>(), st->tNS.as<int2>(),
        st->M.as<float>(), st->P.as<float>(), st->prom.as<uint8_t>(), st->NS.as<int2>());
    CU(cudaGetLastError());
    ctx->launches++;
    st->last_cell_major = false;
    return SCRNA_OK;
}

// Readout: cell-major FP32 state -> cells x G (x2) column-major Float64, through a
// shared-memory tile so both the reads and the writes are coalesced.
// With V (a tau-leap population) the readout is the concentrations M / V, P / V (ext:654-661).
__global__ void tensor_readout_kernel(int G, int ld, int64_t N, const float* M, const float* P, int readout,
                                      double* out, const double* V) {
    __shared__ float tile[2][32][33];
    const int64_t c0 = (int64_t)blockIdx.x * 32;
    const int g0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int64_t c = c0 + r;
        const int g = g0 + threadIdx.x;
        const bool ok = c < N && g < G;
        tile[0][r][threadIdx.x] = ok ? M[c * ld + g] : 0.0f;
        tile[1][r][threadIdx.x] = ok ? P[c * ld + g] : 0.0f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int g = g0 + r;
        const int64_t c = c0 + threadIdx.x;
        if (g >= G || c >= N) continue;
        double mv = tile[0][threadIdx.x][r], pv = tile[1][threadIdx.x][r];
        if (V) {
            mv = __ddiv_rn(mv, V[c]);
            pv = __ddiv_rn(pv, V[c]);
        }
        if (readout == 0) out[(size_t)g * N + c] = mv;
        else if (readout == 1) out[(size_t)g * N + c] = pv;
        else { out[(size_t)g * N + c] = mv; out[(size_t)(G + g) * N + c] = pv; }
    }
}

// Capture on the cell-major state (capture.jl:30-44), thread per (cell, gene).
__global__ void tensor_capture_kernel(int G, int ld, int64_t N, int64_t cell_offset, const float* X, double mu_log,
                                      double sigma, uint32_t key0, uint32_t key1, uint32_t stream,
                                      double* eff, int32_t* Y) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= N * G) return;
    const int64_t c = idx / G;
    const int g = (int)(idx - c * G);
    const Key key{key0, key1};
    const uint32_t gcell = (uint32_t)(cell_offset + c);
    const uint4 w = philox(gcell, 0u, 0u, tagword(TAG_EFFICIENCY, stream), key);
    double pe = exp(mu_log + sigma * box_muller_z0_f64(w.x, w.y));
    pe = fmin(fmax(pe, 0.0), 1.0);
    if (g == 0 && eff) eff[c] = pe;
    const double x = rint((double)X[c * ld + g]);
    const int64_t n = x > 0.0 ? (int64_t)x : 0;
    int64_t y = 0;
    if (n > 0 && pe != 0.0) y = binomial_capture(n, pe, key, stream, gcell, (uint32_t)g);
    Y[(size_t)g * N + c] = (int32_t)y;
}

template <class T>
__global__ void tensor_fill_w_kernel(int G, int K, int Kp, const float* w_rowmajor, T* w16) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)G * Kp) return;
    const int i = (int)(idx / Kp), j = (int)(idx - (int64_t)i * Kp);
    w16[idx] = to16<T>(j < K ? w_rowmajor[(size_t)i * K + j] : 0.0f);
}

// ---- host side -------------------------------------------------------------------------------
// Build the 16-bit weight matrix and the compact cooperative/redundant source tables.
int tensor_prepare_net(scrna_net* n, int dtype) {
    if (n->t_dtype == dtype) return SCRNA_OK;
    const int G = n->G;
    const int n_terms = (int)n->na.size();
    if (n_terms > 65535) return fail(SCRNA_ENOTSUP, "the tensor path takes at most 65535 cooperative/redundant terms");
    const int K = G + n_terms;
    const int Kp = (K + 63) / 64 * 64;
    std::vector<float> w((size_t)G * K, 0.0f);
    for (int i = 0; i < G; ++i)
        for (int j = 0; j < G; ++j)
            if (i != j) w[(size_t)i * K + j] = (float)(n->A[(size_t)i * G + j] * n->basals[i]);
    for (int i = 0; i < G; ++i)
        for (int e = n->na_begin[i]; e < n->na_begin[i] + n->na_count[i]; ++e) w[(size_t)i * K + G + e] = n->na[e].coef;
    // compact source indices of the cooperative / redundant edges
    std::vector<int32_t> src_of_gene(G, -1), src_gene;
    std::vector<int32_t> na_src(n->na_src.size());
    for (size_t t = 0; t < n->na_src.size(); ++t) {
        const int gene = n->reg_gene[n->na_src[t]];
        if (src_of_gene[gene] < 0) { src_of_gene[gene] = (int)src_gene.size(); src_gene.push_back(gene); }
        na_src[t] = src_of_gene[gene];
    }
    DevBuf wf;
    CU(wf.ensure(w.size() * 4));
    CU(cudaMemcpy(wf.p, w.data(), w.size() * 4, cudaMemcpyHostToDevice));
    CU(n->t_w16.ensure((size_t)G * Kp * 2));
    const int64_t tot = (int64_t)G * Kp;
    if (dtype == 0) tensor_fill_w_kernel<__nv_bfloat16><<<(unsigned)((tot + 255) / 256), 256>>>(G, K, Kp, wf.as<float>(), n->t_w16.as<__nv_bfloat16>());
    else tensor_fill_w_kernel<__half><<<(unsigned)((tot + 255) / 256), 256>>>(G, K, Kp, wf.as<float>(), n->t_w16.as<__half>());
    CU(cudaGetLastError());
    CU(cudaDeviceSynchronize());
    CU(n->t_na_src.ensure(std::max<size_t>(na_src.size(), 1) * 4));
    if (!na_src.empty()) CU(cudaMemcpy(n->t_na_src.p, na_src.data(), na_src.size() * 4, cudaMemcpyHostToDevice));
    CU(n->t_src_of_gene.ensure((size_t)G * 4));
    CU(cudaMemcpy(n->t_src_of_gene.p, src_of_gene.data(), (size_t)G * 4, cudaMemcpyHostToDevice));
    n->ctx->h2d_bytes += (int64_t)(w.size() * 4 + na_src.size() * 4 + (size_t)G * 4);
    std::vector<int32_t> slot_of_gene(n->reg_slot.begin(), n->reg_slot.end());
    CU(n->t_slot_of_gene.ensure((size_t)G * 4));
    CU(cudaMemcpy(n->t_slot_of_gene.p, slot_of_gene.data(), (size_t)G * 4, cudaMemcpyHostToDevice));
    n->ctx->h2d_bytes += (int64_t)G * 4;
    n->t_kp = Kp;
    n->t_n_src = (int)src_gene.size();
    n->t_dtype = dtype;
    return SCRNA_OK;
}

static int lt_fail(cublasStatus_t st, const char* what) {
    return fail(SCRNA_ECUDA, "%s failed (cuBLAS status %d)", what, (int)st);
}

// REG[N][ld] = ACT[N][Kp] * W[G][Kp]^T in column-major terms: C (G x N, ldc ld) =
// op(A) (G x Kp) * B (Kp x N) with A = W stored as Kp x G (lda Kp) transposed.
struct LtGemm {
    cublasLtMatmulDesc_t op = nullptr;
    cublasLtMatrixLayout_t la = nullptr, lb = nullptr, lc = nullptr;
    cublasLtMatmulAlgo_t algo{};
    bool ok = false;
    ~LtGemm() {
        if (lc) cublasLtMatrixLayoutDestroy(lc);
        if (lb) cublasLtMatrixLayoutDestroy(lb);
        if (la) cublasLtMatrixLayoutDestroy(la);
        if (op) cublasLtMatmulDescDestroy(op);
    }
};

static int lt_setup(scrna_ctx* ctx, LtGemm& g, int dtype, int G, int ld, int Kp, int64_t N) {
    cublasStatus_t st;
    if (!ctx->lt_handle) {
        cublasLtHandle_t h;
        if ((st = cublasLtCreate(&h)) != CUBLAS_STATUS_SUCCESS) return lt_fail(st, "cublasLtCreate");
        ctx->lt_handle = h;
    }
    const size_t ws = 64u << 20;
    CU(ctx->lt_workspace.ensure(ws));
    const cudaDataType_t t16 = dtype == 0 ? CUDA_R_16BF : CUDA_R_16F;
    if ((st = cublasLtMatmulDescCreate(&g.op, CUBLAS_COMPUTE_32F, CUDA_R_32F)) != CUBLAS_STATUS_SUCCESS) return lt_fail(st, "MatmulDescCreate");
    const cublasOperation_t ta = CUBLAS_OP_T, tb = CUBLAS_OP_N;
    cublasLtMatmulDescSetAttribute(g.op, CUBLASLT_MATMUL_DESC_TRANSA, &ta, sizeof ta);
    cublasLtMatmulDescSetAttribute(g.op, CUBLASLT_MATMUL_DESC_TRANSB, &tb, sizeof tb);
    if ((st = cublasLtMatrixLayoutCreate(&g.la, t16, Kp, G, Kp)) != CUBLAS_STATUS_SUCCESS) return lt_fail(st, "LayoutA");
    if ((st = cublasLtMatrixLayoutCreate(&g.lb, t16, Kp, N, Kp)) != CUBLAS_STATUS_SUCCESS) return lt_fail(st, "LayoutB");
    if ((st = cublasLtMatrixLayoutCreate(&g.lc, CUDA_R_32F, G, N, ld)) != CUBLAS_STATUS_SUCCESS) return lt_fail(st, "LayoutC");
    cublasLtMatmulPreference_t pref;
    cublasLtMatmulPreferenceCreate(&pref);
    cublasLtMatmulPreferenceSetAttribute(pref, CUBLASLT_MATMUL_PREF_MAX_WORKSPACE_BYTES, &ws, sizeof ws);
    cublasLtMatmulHeuristicResult_t res{};
    int nres = 0;
    st = cublasLtMatmulAlgoGetHeuristic((cublasLtHandle_t)ctx->lt_handle, g.op, g.la, g.lb, g.lc, g.lc, pref, 1, &res, &nres);
    cublasLtMatmulPreferenceDestroy(pref);
    if (st != CUBLAS_STATUS_SUCCESS || nres == 0) return lt_fail(st, "AlgoGetHeuristic");
    g.algo = res.algo;
    g.ok = true;
    return SCRNA_OK;
}

int64_t run_steps(const scrna_cle_opts* o);

// Whether the tau-leap's tensor form takes the exact FP32 regulation (the register path's
// counts bit for bit) or the 16-bit GEMM (SCRNA_TAU_TENSOR_EXACT=0 or 1 forces one).  At FP32
// precision: exact for every network the register path holds, so the tau-leap's counts are the
// same on either path, and beyond it for sparse networks (at most 8 edge reads a gene); the
// BF16 GEMM for dense networks beyond it, as the CLE.  FP16 inputs: the FP16 GEMM.  Each edge
// of the exact form is one load of a 32-cell activation row, which once a tile's rows outgrow
// L1 come from L2.  ms a step on a B200, exact / GEMM: 300 sampled genes x 20,000 cells
// 0.106 / 0.153; 300 genes at 10 % 0.251 / 0.202; 600 genes at 10 % 0.634 / 0.263; 2,000
// genes at 2 % x 65,536 cells 7.34 / 2.61, at 10 % 24.8 / 3.78.
bool tau_tensor_exact(const scrna_net* n, int dtype) {
    if (const char* e = std::getenv("SCRNA_TAU_TENSOR_EXACT")) return std::atoi(e) != 0;
    if (dtype != 0) return false;
    if (register_path_holds(n->dev)) return true;
    return (int64_t)n->dev.n_in + n->dev.n_na_src <= 8ll * n->G;
}

int tensor_run(scrna_ctx* ctx, scrna_net* n, const scrna_kinetics* kin, const scrna_capture* cap,
               const scrna_cle_opts* o, scrna_state* st, int dtype, bool tau, const scrna_population* pop) {
    if (int r = tensor_prepare_net(n, dtype)) return r;
    const bool exact = tau && tau_tensor_exact(n, dtype);
    const int G = n->G, Kp = n->t_kp, n_src = exact ? n->dev.n_reg : n->t_n_src, ld = tensor_ld(G);
    const int64_t N = st->N;
    const size_t gn = (size_t)G * N, ln = (size_t)ld * N;
    CU(st->tM.ensure(ln * 4));
    CU(st->tP.ensure(ln * 4));
    CU(st->tprom.ensure(ln));
    CU(st->tNS.ensure(ln * sizeof(int2)));
    if (!exact) CU(st->treg.ensure(ln * 4));  // the GEMM's output (the exact form has none)
    st->t_ld = ld;
    if (!exact) CU(st->tact16.ensure((size_t)N * Kp * 2));  // the GEMM's 16-bit activations
    for (int k = 0; k < 2; ++k) CU(st->tact32[k].ensure(std::max<size_t>((size_t)N * n_src, 1) * 4));
    CU(st->out.ensure(gn * (st->readout == SCRNA_READOUT_BOTH ? 2 : 1) * 8));
    if (cap) {
        CU(st->counts.ensure(gn * 4));
        CU(st->eff.ensure((size_t)N * 8));
    }
    cudaStream_t s = ctx->stream;
    if (!exact) CU(cudaMemsetAsync(st->tact16.p, 0, (size_t)N * Kp * 2, s));  // zero K padding
    TensorArgs a{};
    a.G = G; a.ld = ld; a.Kp = Kp; a.n_src = n_src; a.N = N; a.cell_offset = o->cell_offset;
    a.k_t = (float)kin->k_t;
    a.Kn = (float)std::pow(kin->K_d, kin->n);
    a.hill_n = (float)kin->n;
    a.hill_int = (kin->n == std::floor(kin->n) && kin->n >= 1.0 && kin->n <= 16.0) ? (int)kin->n : 0;
    // decay: intrinsic rates with a population (dilution is then the growth), else with dilution
    const double mu_m = pop ? kin->mu_m : kin->mu_m + kin->dilution;
    const double mu_p = pop ? kin->mu_p : kin->mu_p + kin->dilution;
    a.mu_m = (float)mu_m;
    a.mu_p = (float)mu_p;
    a.dt = (float)o->dt;
    a.p_dec_m = (float)(1.0 - std::exp(-mu_m * o->dt));  // as fill_tau_args
    a.p_dec_p = (float)(1.0 - std::exp(-mu_p * o->dt));
    a.key0 = (uint32_t)o->seed; a.key1 = (uint32_t)(o->seed >> 32); a.stream = o->stream & 0xFFFFFFu;
    for (int r = 0; r < 10; ++r) {
        a.rk0[r] = a.key0 + (uint32_t)r * 0x9E3779B9u;
        a.rk1[r] = a.key1 + (uint32_t)r * 0xBB67AE85u;
    }
    a.genes = n->b_genes.as<GeneRec>();
    a.ginit = n->b_ginit.as<GeneInit>();
    a.na = n->dev.na;
    a.na_src = n->t_na_src.as<int32_t>();
    a.src_of_gene = exact ? n->t_slot_of_gene.as<int32_t>() : n->t_src_of_gene.as<int32_t>();
    a.exact_reg = exact ? 1 : 0;
    a.in_edge = n->dev.in_edge;
    a.na_slot = n->dev.na_src;
    a.n_terms = (int)n->na.size();
    a.reg = st->treg.as<float>();
    a.M = st->tM.as<float>(); a.P = st->tP.as<float>();
    a.prom = st->tprom.as<uint8_t>(); a.NS = st->tNS.as<int2>();
    a.act16 = exact ? nullptr : st->tact16.p;
    a.act32_cur = st->tact32[1].as<float>();
    a.act32_next = st->tact32[0].as<float>();
    if (pop) {  // population buffers (the register path's, as cell-major arrays)
        CU(st->V.ensure((size_t)N * 8));
        CU(st->dV[0].ensure((size_t)N * 8));
        CU(st->owner[0].ensure((size_t)N * 8));
        CU(st->dprom[1].ensure((size_t)N));  // division flags
        CU(st->dM[0].ensure(ln * 4));
        CU(st->dP[0].ensure(ln * 4));
        CU(st->dprom[0].ensure(ln));
        CU(st->dNS[0].ensure(ln * sizeof(int2)));
        CU(cudaMemsetAsync(st->owner[0].p, 0, (size_t)N * 8, s));
        a.V = st->V.as<double>();
        a.growth_factor = std::exp(pop->growth_rate * o->dt);
        a.V_div = pop->V_div; a.V_lo = pop->V_init_lo; a.V_hi = pop->V_init_hi;
        a.partition = pop->partition;
        a.exclude_mother = pop->exclude_mother ? 1 : 0;
        a.tau = tau ? 1 : 0;
        a.epoch = 0;
        a.owner = st->owner[0].as<unsigned long long>();
        a.divided = st->dprom[1].as<uint8_t>();
        a.dM = st->dM[0].as<float>(); a.dP = st->dP[0].as<float>();
        a.dprom = st->dprom[0].as<uint8_t>(); a.dNS = st->dNS[0].as<int2>(); a.dV = st->dV[0].as<double>();
        a.beta64 = n->dev.beta64;
        a.ss_mu_m = kin->mu_m + kin->dilution;
        a.ss_mu_p = kin->mu_p + kin->dilution;
        a.k_t64 = kin->k_t;
    }
    const unsigned b_init = (unsigned)((gn + 255) / 256);
    if (dtype == 0) tensor_init_kernel<__nv_bfloat16><<<b_init, 256, 0, s>>>(a);
    else tensor_init_kernel<__half><<<b_init, 256, 0, s>>>(a);
    CU(cudaGetLastError());
    ctx->launches++;

    LtGemm gemm;
    if (!exact)
        if (int r = lt_setup(ctx, gemm, dtype, G, ld, Kp, N)) return r;
    const float alpha = 1.0f, beta = 0.0f;
    const int64_t n_steps = run_steps(o);
    const int pairs = ld / 2;
    using StepFn = void (*)(TensorArgs);
    const bool h2 = a.hill_int == 2, bursty = n->dev.bursty;
    StepFn step_fn;
    if (dtype == 0) step_fn = bursty ? (h2 ? tensor_step_kernel<__nv_bfloat16, true, 2> : tensor_step_kernel<__nv_bfloat16, true, 0>)
                                     : (h2 ? tensor_step_kernel<__nv_bfloat16, false, 2> : tensor_step_kernel<__nv_bfloat16, false, 0>);
    else step_fn = bursty ? (h2 ? tensor_step_kernel<__half, true, 2> : tensor_step_kernel<__half, true, 0>)
                          : (h2 ? tensor_step_kernel<__half, false, 2> : tensor_step_kernel<__half, false, 0>);
    if (tau) {
        if (dtype == 0)
            step_fn = bursty ? (h2 ? tensor_tau_step_kernel<__nv_bfloat16, true, 2> : tensor_tau_step_kernel<__nv_bfloat16, true, 0>)
                             : (h2 ? tensor_tau_step_kernel<__nv_bfloat16, false, 2> : tensor_tau_step_kernel<__nv_bfloat16, false, 0>);
        else
            step_fn = bursty ? (h2 ? tensor_tau_step_kernel<__half, true, 2> : tensor_tau_step_kernel<__half, true, 0>)
                             : (h2 ? tensor_tau_step_kernel<__half, false, 2> : tensor_tau_step_kernel<__half, false, 0>);
    }
    StepFn replace_fn = dtype == 0 ? (h2 ? tensor_replace_kernel<__nv_bfloat16, 2> : tensor_replace_kernel<__nv_bfloat16, 0>)
                                   : (h2 ? tensor_replace_kernel<__half, 2> : tensor_replace_kernel<__half, 0>);
    const dim3 g_step = tau ? dim3((unsigned)((N + kTauTileCells - 1) / kTauTileCells),
                                   (unsigned)((pairs + kTauTilePairs - 1) / kTauTilePairs))
                            : dim3((unsigned)((N + kTensorCellsPerThread - 1) / kTensorCellsPerThread),
                                   (unsigned)((pairs + kTensorPairsPerBlock - 1) / kTensorPairsPerBlock));
    const unsigned step_threads = tau ? kTauTileThreads : kTensorPairsPerBlock;
    if (g_step.y > 65535) return fail(SCRNA_ENOTSUP, "too many genes for the tensor path");
    for (int64_t step = 1; step <= n_steps; ++step) {
        a.step = (int)step;
        a.act32_cur = st->tact32[(step - 1) & 1].as<float>();
        a.act32_next = st->tact32[step & 1].as<float>();
        if (!exact) {  // (the exact form computes its regulation inside the step kernel)
            if (a.n_terms > 0) {  // term columns from the previous step's activations
                CU(terms_launch(dtype, a, s));
                ctx->launches += 1;
            }
            cublasStatus_t stt = cublasLtMatmul((cublasLtHandle_t)ctx->lt_handle, gemm.op, &alpha, n->t_w16.p, gemm.la,
                                                st->tact16.p, gemm.lb, &beta, st->treg.p, gemm.lc, st->treg.p, gemm.lc,
                                                &gemm.algo, ctx->lt_workspace.p, ctx->lt_workspace.n, s);
            if (stt != CUBLAS_STATUS_SUCCESS) return lt_fail(stt, "cublasLtMatmul");
        }
        step_fn<<<g_step, step_threads, 0, s>>>(a);
        CU(cudaGetLastError());
        ctx->launches += 1;  // the library GEMM is not counted as this library's kernel
        if (pop) {
            const unsigned b_cells = (unsigned)((N + 255) / 256);
            tensor_growth_kernel<<<b_cells, 256, 0, s>>>(a.V, N, a.growth_factor);
            CU(cudaGetLastError());
            ctx->launches += 1;
            if (step % pop->div_check_interval == 0) {
                tensor_divide_kernel<<<b_cells, 256, 0, s>>>(a);
                tensor_partition_kernel<<<b_init, 256, 0, s>>>(a);
                replace_fn<<<b_init, 256, 0, s>>>(a);
                CU(cudaGetLastError());
                ctx->launches += 3;
                a.epoch += 1;
            }
        }
    }
    st->epoch = pop ? a.epoch : 0;
    dim3 rgrid((unsigned)((N + 31) / 32), (unsigned)((G + 31) / 32));
    tensor_readout_kernel<<<rgrid, dim3(32, 8), 0, s>>>(G, ld, N, st->tM.as<float>(), st->tP.as<float>(), st->readout,
                                                        st->out.as<double>(), pop && tau ? a.V : nullptr);
    CU(cudaGetLastError());
    ctx->launches++;
    if (cap) {
        const double mu_log = std::log(cap->efficiency) -
                              (cap->mean_correction ? cap->efficiency_std * cap->efficiency_std / 2.0 : 0.0);
        const float* X = cap->readout == SCRNA_READOUT_MRNA ? st->tM.as<float>() : st->tP.as<float>();
        tensor_capture_kernel<<<b_init, 256, 0, s>>>(G, ld, N, o->cell_offset, X, mu_log, cap->efficiency_std, a.key0,
                                                     a.key1, a.stream, st->eff.as<double>(), st->counts.as<int32_t>());
        CU(cudaGetLastError());
        ctx->launches++;
    }
    return SCRNA_OK;
}

}  // namespace scrna
