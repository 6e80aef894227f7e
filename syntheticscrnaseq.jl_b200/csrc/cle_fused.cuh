// Fused FP32 register-path CLE kernel (sm_100a).
//
// One launch advances a tile of cells through a chunk of Euler-Maruyama steps
// (src/algorithms/cle.jl:78-121, population form cle.jl:185-237) with the state
// held in registers for the whole chunk:
//   * lanes are cells (32 per warp), warps are gene quads: thread (lane, warp w)
//     owns genes 4q..4q+3 of one cell for q = w, w+NW, ... (UPT quads);
//   * per step, genes whose protein regulates others publish their Hill
//     activation to a shared-memory slot table (double-buffered, one barrier
//     per step); targets read their sparse in-edges from it;
//   * the additive term uses reg = cneg + sum_j A_eff[g,j] act_j, which equals
//     A_pos act + A_neg rep because rep = 1 - act (network.jl:206-219);
//   * increments come from counter-based Philox keyed by (seed, stream, cell,
//     step, gene), so results do not depend on the tiling;
//   * HBM is touched only at chunk boundaries (state, division buffers) and for
//     the final readout / capture.
#pragma once
#include "launch_attr.h"
#include "cle_device.cuh"
#include "tau_lockstep.cuh"
#include "cle_internal.h"

namespace scrna {

// Shared-memory layout of one block: regulator activations (2 x n_reg x 32 floats),
// then the gene table, the edge tables and the per-quad switching flags.
struct Smem {
    float* act;
    GeneRec* genes;
    float2* in_edge;
    NonAdd* na;
    int32_t* na_src;
    uint8_t* quad_tel;
};

__host__ __device__ inline size_t fused_smem_bytes(int G, int n_reg, int n_in, int n_na,
                                                   int n_na_src, int n_quads) {
    size_t b = (size_t)2 * n_reg * 32 * sizeof(float);
    b += (size_t)G * sizeof(GeneRec);
    b += (size_t)n_in * sizeof(float2);
    b += (size_t)n_na * sizeof(NonAdd);
    b += (size_t)n_na_src * sizeof(int32_t);
    b += (size_t)n_quads;
    return (b + 15) & ~(size_t)15;
}

// One cell tile (32 cells) of one network through the step range of `ctl`.
// TAU: the binomial tau-leap (ext/SyntheticscRNAseqCUDAExt.jl:215-399, population :531-651)
// instead of the CLE step: one Philox block of four uniforms per (cell, step, gene), integer
// counts in FP32, Hill activation of the concentration P / V with a population (whose initial
// counts are max(1, round(steady state x V))) and the concentrations M / V, P / V as readout.
// QG: genes per thread unit, 4 (a quad; the CLE), or 4, 2 or 1 for the tau-leap (any grouping:
// the Philox counters of its draws name genes, and the initial promoter word of gene g is
// word g mod 4 of its quad's block whatever the grouping).
template <int UPT, bool POP, bool TAU = false, int QG = 4>
__device__ __forceinline__ void fused_tile(const FusedArgs& a, int64_t tile, const TileCtl& ctl,
                                           unsigned char* smem_raw) {
    static_assert(QG == 4 || (TAU && (QG == 2 || QG == 1)), "the CLE runs gene quads; the tau-leap quads, pairs or single genes");
    static_assert(UPT * QG <= 32, "one promoter bit per gene of the thread");
    Smem sm;
    {
        unsigned char* p = smem_raw;
        sm.act = reinterpret_cast<float*>(p);       p += (size_t)2 * a.n_reg * 32 * sizeof(float);
        sm.genes = reinterpret_cast<GeneRec*>(p);   p += (size_t)a.G * sizeof(GeneRec);
        sm.in_edge = reinterpret_cast<float2*>(p);  p += (size_t)a.n_in * sizeof(float2);
        sm.na = reinterpret_cast<NonAdd*>(p);       p += (size_t)a.n_na * sizeof(NonAdd);
        sm.na_src = reinterpret_cast<int32_t*>(p);  p += (size_t)a.n_na_src * sizeof(int32_t);
        sm.quad_tel = p;
    }
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;
    for (int i = tid; i < a.G; i += nthr) sm.genes[i] = a.genes[i];
    for (int i = tid; i < a.n_in; i += nthr) sm.in_edge[i] = a.in_edge[i];
    for (int i = tid; i < a.n_na; i += nthr) sm.na[i] = a.na[i];
    for (int i = tid; i < a.n_na_src; i += nthr) sm.na_src[i] = a.na_src[i];
    for (int i = tid; i < a.n_quads; i += nthr) sm.quad_tel[i] = a.quad_tel[i];
    __syncthreads();

    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int NW = nthr >> 5;
    const int64_t N = a.N;
    const int64_t cell = tile * 32 + lane;
    const bool live = cell < N;
    const int64_t cidx = live ? cell : N - 1;  // dead lanes shadow the last cell, never store
    const uint32_t gcell = (uint32_t)(a.cell_offset + cidx);
    const Key key{a.key0, a.key1};
    const int G = a.G;
    const int n_units = (G + QG - 1) / QG;  // thread units of QG genes (the last one may be partial)
    const bool has_reg = a.n_reg > 0;

    float m[UPT][QG], p[UPT][QG];
    int2 ns[UPT][QG];            // switching state of each gene (fresh_switch in cle_device.cuh)
    uint32_t on = 0xFFFFFFFFu;  // bit 4j+i: promoter of gene 4q_j+i is ON
    double V = 0.0;

    // ---- prologue: initial condition or state of the previous chunk -------------
    if (ctl.first) {
#pragma unroll
        for (int j = 0; j < UPT; ++j) {
            const int q = warp + j * NW;
#pragma unroll
            for (int i = 0; i < QG; ++i) {
                const int g = QG * q + i;
                m[j][i] = (q < n_units && g < G) ? a.ginit[g].m0 : 0.0f;
                p[j][i] = (q < n_units && g < G) ? a.ginit[g].p0 : 0.0f;
            }
            if (q < n_units) {
                bool any = false;
#pragma unroll
                for (int i = 0; i < QG; ++i) {
                    const int g = QG * q + i;
                    any |= (g < G) && a.ginit[g].init_rand;
                }
                if (any) {
                    const uint4 w = philox(gcell, 0u, (uint32_t)((QG * q) >> 2), tagword(TAG_PROMOTER, a.stream), key);
                    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                    for (int i = 0; i < QG; ++i) {
                        const int g = QG * q + i;
                        if (g < G && a.ginit[g].init_rand && !(ws[g & 3] < a.ginit[g].thr_init))
                            on &= ~(1u << (QG * j + i));
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < QG; ++i) {  // first waiting times (NaN parameter: gene never switches)
                const int g = QG * q + i;
                ns[j][i] = make_int2(kNever, kNever);
                if (q < n_units && g < G) {
                    const GeneRec gr = sm.genes[g];
                    if (gr.inv_off == gr.inv_off) {
                        const uint4 w = philox(gcell, 0u, (uint32_t)g, tagword(TAG_SWITCH, a.stream), key);
                        ns[j][i] = fresh_switch(0, w.x, w.y, (on >> (QG * j + i)) & 1u, gr.inv_on, gr.inv_off);
                    }
                }
            }
        }
        if (POP) {
            const uint4 w = philox(gcell, 0u, 0u, tagword(TAG_VOLUME, a.stream), key);
            V = __dadd_rn(a.V_lo, __dmul_rn(__dadd_rn(a.V_hi, -a.V_lo), u53(w.x, w.y)));
        }
        if (TAU && POP) {  // counts of a cell of volume V at the steady state (ext:560-566)
#pragma unroll
            for (int j = 0; j < UPT; ++j) {
                const int q = warp + j * NW;
#pragma unroll
                for (int i = 0; i < QG; ++i) {
                    const int g = QG * q + i;
                    if (!(q < n_units && g < G)) continue;
                    const double mss = __ddiv_rn(a.beta64[g], a.ss_mu_m);
                    const double pss = __ddiv_rn(__dmul_rn(a.k_t64, mss), a.ss_mu_p);
                    m[j][i] = (float)fmax(1.0, rint(__dmul_rn(mss, V)));
                    p[j][i] = (float)fmax(1.0, rint(__dmul_rn(pss, V)));
                }
            }
        }
    } else {
        // A cell replaced at the previous division takes the daughter of its new owner.
        int64_t src = cidx;
        bool from_daughter = false;
        const int par = ctl.epoch & 1;
        if (POP && ctl.epoch > 0) {
            const unsigned long long o = a.owner[par][cidx];
            if ((uint32_t)(o >> 32) == (uint32_t)ctl.epoch) {
                src = (int64_t)(o & 0xFFFFFFFFull);
                from_daughter = true;
            }
        }
        const float* Ms = from_daughter ? a.dM[par] : a.M;
        const float* Ps = from_daughter ? a.dP[par] : a.P;
        const uint8_t* Os = from_daughter ? a.dprom[par] : a.prom;
        const int2* Ns = from_daughter ? a.dNS[par] : a.NS;
#pragma unroll
        for (int j = 0; j < UPT; ++j) {
            const int q = warp + j * NW;
#pragma unroll
            for (int i = 0; i < QG; ++i) {
                const int g = QG * q + i;
                const bool ok = q < n_units && g < G;
                m[j][i] = ok ? Ms[(size_t)g * N + src] : 0.0f;
                p[j][i] = ok ? Ps[(size_t)g * N + src] : 0.0f;
                ns[j][i] = ok ? Ns[(size_t)g * N + src] : make_int2(kNever, kNever);
                if (ok && !Os[(size_t)g * N + src]) on &= ~(1u << (QG * j + i));
            }
        }
        if (POP) V = from_daughter ? a.dV[par][src] : a.V[cidx];
    }

    // ---- fused step loop ---------------------------------------------------------
    const float k_t = a.k_t, mu_m = a.mu_m, mu_p = a.mu_p, dt = a.dt;
    // regulation sum of a gene from the step's activation slots: additive in-edges, then the
    // cooperative (product of activations) and redundant (1 - product of 1 - activations) terms
    auto regulation = [&](const GeneRec& gr, const float* act) {
        float reg = gr.cneg;
        for (int e = gr.in_begin; e < gr.in_end; ++e) {
            const float2 ed = sm.in_edge[e];
            reg = fmaf(ed.x, act[__float_as_int(ed.y) * 32 + lane], reg);
        }
        const int nab = gr.na_range >> 16, nac = gr.na_range & 0xFFFF;
        for (int e = nab; e < nab + nac; ++e) {
            const NonAdd na = sm.na[e];
            float prod = 1.0f;
            if (na.kind == 0) {
                for (int t = na.src_begin; t < na.src_end; ++t) prod *= act[sm.na_src[t] * 32 + lane];
                reg = fmaf(na.coef, prod, reg);
            } else {
                for (int t = na.src_begin; t < na.src_end; ++t) prod *= 1.0f - act[sm.na_src[t] * 32 + lane];
                reg = fmaf(na.coef, 1.0f - prod, reg);
            }
        }
        return reg;
    };
    int buf = 0;
    for (int s = ctl.step_begin; s <= ctl.step_end; ++s) {
        // Hill activations of regulator genes -> slot table
        float* act = sm.act + (size_t)buf * a.n_reg * 32;
        const float Vf = POP ? (float)V : 1.0f;
        if (has_reg) {
#pragma unroll
            for (int j = 0; j < UPT; ++j) {
                const int q = warp + j * NW;
                if (q < n_units) {
#pragma unroll
                    for (int i = 0; i < QG; ++i) {
                        const int g = QG * q + i;
                        if (g < G) {
                            const int slot = sm.genes[g].slot;
                            if (slot >= 0)
                                act[slot * 32 + lane] = hill_act(TAU && POP ? __fdiv_rn(p[j][i], Vf) : p[j][i], a.Kn,
                                                                 a.hill_n, a.hill_int);
                        }
                    }
                }
            }
            if (NW > 1) __syncthreads(); else __syncwarp();
        }
#pragma unroll
        for (int j = 0; j < UPT; ++j) {
            const int q = warp + j * NW;
            if (q >= n_units) continue;
            if constexpr (TAU) {
                // the unit's genes: telegraph switching (tauleap_binomial.jl:111-121) from the
                // spare bits of each gene's tau-leap words, transcription propensity, then the
                // draws of the unit (tau_lockstep.cuh)
                float lam[QG];
                uint4 wt[QG];
#pragma unroll
                for (int i = 0; i < QG; ++i) {
                    const int g = QG * q + i;
                    lam[i] = 0.0f;
                    wt[i] = make_uint4(0u, 0u, 0u, 0u);
                    if (g >= G) continue;
                    wt[i] = philox(gcell, (uint32_t)s, (uint32_t)g, tagword(TAG_TAU, a.stream), key);
                    const uint32_t bit = 1u << (QG * j + i);
                    if (s == ns[j][i].x) {
                        on ^= bit;
                        ns[j][i] = switch_at(s, ns[j][i], switch_uniform(wt[i].x, wt[i].y), on & bit,
                                             sm.genes[g].inv_on, sm.genes[g].inv_off);
                    }
                    const GeneRec gr = sm.genes[g];
                    float tx = fmaxf(__fadd_rn(regulation(gr, act), gr.beta), 0.0f);
                    if (POP) tx = __fmul_rn(tx, Vf);
                    lam[i] = (on & bit) ? __fmul_rn(tx, dt) : 0.0f;
                }
                tau_update_unit<QG>(m[j], p[j], lam, wt, min(QG, G - QG * q), a.tau_lockstep != 0, k_t, dt,
                                    a.p_dec_m, a.p_dec_p);
            } else {
#pragma unroll
                for (int h = 0; h < 2; ++h) {  // gene pairs 2q, 2q+1 of this quad
                    const int g0 = 4 * q + 2 * h;
                    if (g0 >= G) continue;
                    const uint4 w = philox(gcell, (uint32_t)s, (uint32_t)(2 * q + h), tagword(TAG_NORMAL, a.stream), key);
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        const int i = 2 * h + k;
                        const int g = g0 + k;
                        if (g >= G) continue;
                        // telegraph switching before the transcription update (tauleap_binomial.jl:111-121):
                        // a gene switches when its waiting time runs out and draws the next one
                        // from the spare bits of its normal words
                        if (s == ns[j][i].x) {
                            const uint32_t bit = 1u << (QG * j + i);
                            on ^= bit;
                            const float us = k == 0 ? switch_uniform(w.x, w.y) : switch_uniform(w.z, w.w);
                            ns[j][i] = switch_at(s, ns[j][i], us, on & bit, sm.genes[g].inv_on, sm.genes[g].inv_off);
                        }
                        const GeneRec gr = sm.genes[g];
                        const float reg = regulation(gr, act);
                        const BM bm = k == 0 ? box_muller_parts(w.x, w.y) : box_muller_parts(w.z, w.w);
                        float tx = reg + gr.beta;
                        if (POP) tx *= Vf;
                        if (!(on & (1u << (QG * j + i)))) tx = 0.0f;
                        em_update(m[j][i], p[j][i], tx, bm, mu_m, mu_p, k_t, dt);
                    }
                }
            }
        }
        if (POP) V = __dmul_rn(V, a.growth_factor);
        buf ^= 1;
    }

    // ---- epilogue --------------------------------------------------------------------
    if (POP && ctl.check) {
        // division (cle.jl:240-273): partition in registers, daughters to the
        // next-epoch buffers, replaced slot claimed with a last-writer-wins max.
        const bool divides = V > a.V_div;
        const int ne = ctl.epoch + 1;
        const int par = ne & 1;
        if (divides) {
            V = V * 0.5;
            if (live && warp == 0) {
                const uint4 w = philox((uint32_t)(a.cell_offset + cidx), (uint32_t)ctl.step_end, 0u,
                                       tagword(TAG_MORAN, a.stream), key);
                int64_t r;
                if (a.exclude_mother) {
                    r = (int64_t)(((uint64_t)w.x * (uint64_t)(N - 1)) >> 32);
                    if (r >= cidx) r += 1;
                } else {
                    r = (int64_t)(((uint64_t)w.x * (uint64_t)N) >> 32);
                }
                a.dV[par][cidx] = V;
                atomicMax(&a.owner[par][r], ((unsigned long long)(uint32_t)ne << 32) | (unsigned long long)cidx);
            }
#pragma unroll
            for (int j = 0; j < UPT; ++j) {
                const int q = warp + j * NW;
#pragma unroll
                for (int i = 0; i < QG; ++i) {
                    const int g = QG * q + i;
                    if (!(live && q < n_units && g < G)) continue;
                    float mm, dm, pm, dp;
                    if (a.partition == 1) {  // halve
                        mm = dm = m[j][i] * 0.5f;
                        pm = dp = p[j][i] * 0.5f;
                    } else {  // binomial split of rounded counts
                        const int64_t mi = (int64_t)rintf(m[j][i]);
                        const int64_t pi = (int64_t)rintf(p[j][i]);
                        const int64_t mk = binomial_half(mi, key, a.stream, gcell, (uint32_t)ctl.step_end, (uint32_t)g, 0u);
                        const int64_t pk = binomial_half(pi, key, a.stream, gcell, (uint32_t)ctl.step_end, (uint32_t)g, 1u);
                        mm = (float)mk; dm = (float)(mi - mk);
                        pm = (float)pk; dp = (float)(pi - pk);
                    }
                    m[j][i] = mm;
                    p[j][i] = pm;
                    const size_t idx = (size_t)g * N + cidx;
                    a.dM[par][idx] = dm;
                    a.dP[par][idx] = dp;
                    const uint32_t bon = (on >> (QG * j + i)) & 1u;
                    a.dprom[par][idx] = bon;
                    // the daughter's promoter switches independently of the mother's
                    int2 dns = make_int2(kNever, kNever);
                    const GeneRec gr = sm.genes[g];
                    if (gr.inv_off == gr.inv_off) {
                        const uint4 w = philox(gcell, (uint32_t)ctl.step_end, (uint32_t)g | kDaughterSwitch,
                                               tagword(TAG_SWITCH, a.stream), key);
                        dns = fresh_switch(ctl.step_end, w.x, w.y, bon, gr.inv_on, gr.inv_off);
                    }
                    a.dNS[par][idx] = dns;
                }
            }
        }
    }
    if (!live) return;
    const bool write_state = !ctl.last || POP;
#pragma unroll
    for (int j = 0; j < UPT; ++j) {
        const int q = warp + j * NW;
#pragma unroll
        for (int i = 0; i < QG; ++i) {
            const int g = QG * q + i;
            if (!(q < n_units && g < G)) continue;
            const size_t idx = (size_t)g * N + cell;
            if (write_state || ctl.last) {
                a.M[idx] = m[j][i];
                a.P[idx] = p[j][i];
                a.prom[idx] = (on >> (QG * j + i)) & 1u;
                a.NS[idx] = ns[j][i];
            }
            if (ctl.last && a.out) {
                // tau-leap populations read out concentrations (ext:654-661)
                const double om = TAU && POP ? __ddiv_rn((double)m[j][i], V) : (double)m[j][i];
                const double op = TAU && POP ? __ddiv_rn((double)p[j][i], V) : (double)p[j][i];
                if (a.readout == 0) a.out[idx] = om;
                else if (a.readout == 1) a.out[idx] = op;
                else { a.out[idx] = om; a.out[(size_t)(G + g) * N + cell] = op; }
            }
        }
    }
    if (POP && warp == 0) a.V[cell] = V;
    if (ctl.last && a.counts) {
        // capture (capture.jl:30-44): per-cell LogNormal efficiency, then inverse-CDF binomials
        const uint4 w = philox(gcell, 0u, 0u, tagword(TAG_EFFICIENCY, a.stream), key);
        const double z = box_muller_z0_f64(w.x, w.y);
        double pe = exp(a.cap_mu_log + a.cap_sigma * z);
        pe = fmin(fmax(pe, 0.0), 1.0);
        if (warp == 0 && a.eff) a.eff[cell] = pe;
#pragma unroll
        for (int j = 0; j < UPT; ++j) {
            const int q = warp + j * NW;
#pragma unroll
            for (int i = 0; i < QG; ++i) {
                const int g = QG * q + i;
                if (!(q < n_units && g < G)) continue;
                const double x = rint((double)(a.capture_species == 0 ? m[j][i] : p[j][i]));
                const int64_t n = x > 0.0 ? (int64_t)x : 0;
                int64_t y = 0;
                if (n > 0 && pe != 0.0) y = binomial_capture(n, pe, key, a.stream, gcell, (uint32_t)g);
                a.counts[(size_t)g * N + cell] = (int32_t)y;
            }
        }
    }
}

template <int UPT, bool POP, bool TAU = false, int QG = 4>
__global__ void __launch_bounds__(UPT <= 2 ? 256 : 512) cle_fused_kernel(const FusedArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const TileCtl ctl{a.step_begin, a.step_end, a.first, a.last, a.check, a.epoch};
    fused_tile<UPT, POP, TAU, QG>(a, blockIdx.x, ctl, smem_raw);
}

// Persistent form: blocks pull (network, tile, step range) items from a device work queue
// until it is empty; items of different networks and sizes share one launch.
template <int UPT, bool POP, bool TAU = false, int QG = 4>
__global__ void __launch_bounds__(UPT <= 2 ? 256 : 512)
cle_fused_queue_kernel(const FusedArgs* args, const TileWork* items, int n_items, int* counter,
                       TileCtl shared_ctl, int use_shared) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int next;
    while (true) {
        if (threadIdx.x == 0) next = atomicAdd(counter, 1);
        __syncthreads();
        const int it = next;
        __syncthreads();
        if (it >= n_items) return;
        const TileWork w = items[it];
        fused_tile<UPT, POP, TAU, QG>(args[w.arg], w.tile, use_shared ? shared_ctl : w.ctl, smem_raw);
        __syncthreads();
    }
}

template <int UPT, bool POP, bool TAU = false, int QG = 4>
cudaError_t fused_launch_t(const FusedArgs& a, int nw, size_t smem, cudaStream_t st) {
    auto k = cle_fused_kernel<UPT, POP, TAU, QG>;
    cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)((a.N + 31) / 32);
    k<<<blocks, nw * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int UPT, bool POP, bool TAU = false, int QG = 4>
cudaError_t fused_queue_launch_t(const FusedArgs* args, const TileWork* items, int n_items, int* counter,
                                 int nw, size_t smem, int grid, TileCtl shared_ctl, int use_shared, cudaStream_t st) {
    auto k = cle_fused_queue_kernel<UPT, POP, TAU, QG>;
    cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    k<<<grid, nw * 32, smem, st>>>(args, items, n_items, counter, shared_ctl, use_shared);
    return cudaGetLastError();
}

}  // namespace scrna
