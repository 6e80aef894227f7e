// Lane-per-gene-unit register-path CLE kernel for networks up to 512 genes (sm_100a).
//
// lane = (cell, unit) where a unit is GPL consecutive genes (a gene pair or a gene quad).
// A cell whose units fit in a warp shares the warp with other cells (no barrier at all);
// a larger cell spans wpc <= 8 warps synchronised by a named barrier of its own.  A cell's regulator
// activations live in one shared-memory row: the regulator slots, the constants 0 and 1,
// a write-only slot, then one slot per cooperative / redundant term holding that term's
// value (the product over its sources), so a term enters its target's regulation as one
// more in-edge.  Each lane keeps in registers its genes' constants and padded lists of
// EMAX in-edges (weight, shared-memory address of the source slot), and the TMAX terms
// of the cell that it evaluates.  Per Euler step:
//   Hill of the lane's genes into the row -> Philox (+ telegraph switch) + Box-Muller
//   -> cell sync -> term values into the row -> cell sync -> reg = cneg + sum of EMAX
//   padded edges -> M, P update -> cell sync.
// No lane branches on the network's structure and there is no block-wide barrier.
// The arithmetic and the Philox streams are those of cle_fused_kernel (same sums in the
// same order: a gene's edges are sorted by slot, so its additive edges come first, then
// its terms in table order; a padded edge has weight 0 and reads the constant-0 slot; a
// padded term source reads the constant 1 (cooperative) or 0 (redundant), which leave
// the product unchanged), so both kernels give identical results.
#pragma once
#include "launch_attr.h"
#include "cle_device.cuh"
#include "cle_internal.h"
#include "philox_hoist.cuh"
#include "switch_table.cuh"

namespace scrna {

constexpr int kWarpcellMaxGenes = 512;

// Launch geometry of a network (host and device agree on it).
__host__ __device__ inline int warpcell_lanes_per_cell(int G, int gpl) { return (G + gpl - 1) / gpl; }
// warps per cell: 1 when a cell fits in a warp (then several cells share it)
__host__ __device__ inline int warpcell_wpc(int G, int gpl) { return (warpcell_lanes_per_cell(G, gpl) + 31) / 32; }
__host__ __device__ inline int warpcell_cells_per_warp(int G, int gpl) {
    const int lpc = warpcell_lanes_per_cell(G, gpl);
    return lpc <= 32 ? 32 / lpc : 1;
}
// warps per block: nw1 (2, 4 or 8; 0 = 4) independent warps of small cells, or whole
// multi-warp cells (<= 8 warps)
__host__ __device__ inline int warpcell_block_warps(int G, int gpl, int nw1 = 0) {
    const int w = warpcell_wpc(G, gpl);
    return w == 1 ? (nw1 > 0 ? nw1 : 4) : w * (8 / w);
}
__host__ __device__ inline int warpcell_cells_per_block(int G, int gpl, int nw1 = 0) {
    const int w = warpcell_wpc(G, gpl);
    const int bw = warpcell_block_warps(G, gpl, nw1);
    return w == 1 ? bw * warpcell_cells_per_warp(G, gpl) : bw / w;
}
// activation rows of a block: one per cell, plus a row per warp for the spare lanes of small cells
__host__ __device__ inline int warpcell_rows_per_block(int G, int gpl, int nw1 = 0) {
    const int w = warpcell_wpc(G, gpl);
    const int bw = warpcell_block_warps(G, gpl, nw1);
    return w == 1 ? bw * (warpcell_cells_per_warp(G, gpl) + 1) : bw / w;
}

// Activation row of one cell: n_reg regulator slots, the constants 0 (slot n_reg) and 1
// (slot n_reg + 1), a write-only slot (n_reg + 2) for values nobody reads, then the
// n_terms term values; odd length so the rows of a warp's cells start in different banks.
__host__ __device__ inline int warpcell_ld(int n_reg, int n_terms) { return (n_reg + 3 + n_terms) | 1; }

__host__ __device__ inline size_t warpcell_smem_bytes(int G, int gpl, int n_reg, int n_terms, int nw1 = 0) {
    const size_t b = (size_t)warpcell_rows_per_block(G, gpl, nw1) * warpcell_ld(n_reg, n_terms) * sizeof(float);
    return (b + 15) & ~(size_t)15;
}

// Barrier of the wpc warps of one cell: named barrier 1 + cell group of the block (a block
// holds at most 4 multi-warp cells).  Literal ids keep the kernel's barrier count at 5.
__device__ __forceinline__ void cell_barrier(int id, int nthreads) {
    switch (id) {
        case 1: asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory"); break;
        case 2: asm volatile("bar.sync 2, %0;" ::"r"(nthreads) : "memory"); break;
        case 3: asm volatile("bar.sync 3, %0;" ::"r"(nthreads) : "memory"); break;
        default: asm volatile("bar.sync 4, %0;" ::"r"(nthreads) : "memory"); break;
    }
}

// Word of gene u*GPL+i in the quad's Philox block (word index (u*GPL+i) mod 4), selected
// without indexing a register array by a runtime value.
template <int GPL>
__device__ __forceinline__ uint32_t quad_word(const uint4& w, int u, int i) {
    if (GPL == 4) return i == 0 ? w.x : i == 1 ? w.y : i == 2 ? w.z : w.w;
    const bool hi = u & 1;
    return i == 0 ? (hi ? w.z : w.x) : (hi ? w.w : w.y);
}

__device__ __forceinline__ float& smem_f32(unsigned char* base, uint32_t off) {
    return *reinterpret_cast<float*>(base + off);
}

// Hill activation p^n / (p^n + K^n); HN == 2 is the square without the exponent dispatch.
template <int HN>
__device__ __forceinline__ float warpcell_hill(float p, const FusedArgs& a) {
    if (HN == 2) {
        const float pn = p * p;
        return fminf(pn * frcp_approx(pn + a.Kn), 1.0f);  // as hill_act with hill_int == 2
    }
    return hill_act(p, a.Kn, a.hill_n, a.hill_int);
}

template <int HN>
__device__ __forceinline__ float2 warpcell_hill2(float2 p, const FusedArgs& a) {
    if (HN == 2) return hill2_n2(p, a.Kn);  // as hill_act with hill_int == 2
    return make_float2(hill_act(p.x, a.Kn, a.hill_n, a.hill_int), hill_act(p.y, a.Kn, a.hill_n, a.hill_int));
}

// One block tile (warpcell_cells_per_block cells) of one network through ctl's step range.
// RK: the Euler-step Philox reads its round keys from rk0 / rk1 (kernel parameter space).
// HN: 2 for a Hill exponent of exactly 2, else 0 (any exponent).
// MW: cells span several warps (warpcell_wpc > 1), else several cells share a warp.
template <int GPL, int EMAX, int TMAX, bool POP, bool RK, int HN, bool MW>
__device__ __forceinline__ void warpcell_tile(const FusedArgs& a, int64_t tile, const TileCtl& ctl,
                                              unsigned char* smem_raw, const uint32_t* rk0, const uint32_t* rk1) {
    static_assert(GPL % 2 == 0, "genes are updated in pairs");
    constexpr int TM = TMAX > 0 ? TMAX : 1;
    const int G = a.G;
    const int lpc = warpcell_lanes_per_cell(G, GPL);
    const int wpc = MW ? warpcell_wpc(G, GPL) : 1;
    const int n_reg = a.n_reg;
    const int n_terms = a.n_na;
    const int ld = warpcell_ld(n_reg, n_terms);

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    int u, row_idx, first_row, n_rows;
    bool lane_ok;
    int64_t cell;
    if (!MW) {  // several cells per warp; spare lanes work on a private dummy row
        const int cpw = 32 / lpc;
        int cl = lane / lpc;
        u = lane - cl * lpc;
        lane_ok = cl < cpw;
        if (!lane_ok) cl = cpw;
        cell = (tile * nwarps + warp) * cpw + (lane_ok ? cl : 0);
        first_row = warp * (cpw + 1);
        n_rows = cpw + 1;
        row_idx = first_row + cl;
    } else {  // one cell per group of wpc warps; spare lanes of its last warp hold no gene
        const int grp = warp / wpc;
        u = (warp - grp * wpc) * 32 + lane;
        lane_ok = u < lpc;
        cell = tile * (nwarps / wpc) + grp;
        first_row = row_idx = grp;
        n_rows = (warp - grp * wpc) == 0 ? 1 : 0;  // the group's first warp sets up the row
    }
    const int bar_id = 1 + warp / wpc, bar_threads = 32 * wpc;
    auto cell_sync = [&]() {
        if (!MW) __syncwarp();
        else cell_barrier(bar_id, bar_threads);
    };
    const int64_t N = a.N;
    const bool live = lane_ok && cell < N;
    const int64_t cidx = cell < N ? cell : N - 1;
    const uint32_t gcell = (uint32_t)(a.cell_offset + cidx);
    const Key key{a.key0, a.key1};

    // constant slots of the rows (written once; Hill stores never touch them)
    float* rows = reinterpret_cast<float*>(smem_raw) + (size_t)first_row * ld;
    for (int r = lane; r < n_rows; r += 32) {
        rows[(size_t)r * ld + n_reg] = 0.0f;
        rows[(size_t)r * ld + n_reg + 1] = 1.0f;
    }
    cell_sync();
    const uint32_t row = (uint32_t)((size_t)row_idx * ld * sizeof(float));
    auto slot_addr = [&](int slot) { return row + (uint32_t)slot * (uint32_t)sizeof(float); };

    // per-lane gene constants
    float beta[GPL], cneg[GPL];
    float inv_on[GPL], inv_off[GPL];
    uint32_t hill_at[GPL];         // where this gene's activation is stored
    float ew[GPL][EMAX];           // padded in-edges: weight, source address
    uint32_t ea[GPL][EMAX];
    // terms this lane evaluates (term u + k lpc): value = off + sgn * prod_q (off + sgn * act[src_q])
    // with (sgn, off) = (1, 0) cooperative, (-1, 1) redundant, stored at tout
    float tsg[TM], tof[TM];
    uint32_t ta[TM][kLaneSrc], tout[TM];
#pragma unroll
    for (int k = 0; k < TMAX; ++k) {
        const int j = u + k * lpc;
        const bool has = lane_ok && j < n_terms;
        const LaneTerm t = a.lane_term[has ? j : 0];
        tsg[k] = t.kind == 0 ? 1.0f : -1.0f;
        tof[k] = t.kind == 0 ? 0.0f : 1.0f;
#pragma unroll
        for (int q = 0; q < kLaneSrc; ++q) ta[k][q] = slot_addr(t.src[q]);
        tout[k] = slot_addr(has ? n_reg + 3 + j : n_reg + 2);
    }
    bool valid[GPL];
#pragma unroll
    for (int i = 0; i < GPL; ++i) {
        const int g = u * GPL + i;
        valid[i] = g < G;
        const int gg = valid[i] ? g : 0;
        const GeneRec gr = a.genes[gg];
        beta[i] = gr.beta;
        cneg[i] = gr.cneg;
        inv_on[i] = gr.inv_on;
        inv_off[i] = valid[i] ? gr.inv_off : __int_as_float(0x7FC00000);  // NaN: never switches
        hill_at[i] = slot_addr(valid[i] && gr.slot >= 0 ? gr.slot : n_reg + 2);
#pragma unroll
        for (int e = 0; e < EMAX; ++e) {
            const int2 ed = a.lane_in[(size_t)gg * kLaneEdges + e];
            ew[i][e] = valid[i] ? __int_as_float(ed.y) : 0.0f;
            ea[i][e] = slot_addr(ed.x);
        }
    }
    const int quad = GPL == 4 ? u : (u >> 1);

    float m[GPL], p[GPL];
    int32_t ns[GPL];  // step of the next promoter switch
    int32_t kn[GPL];  // waiting time after it (fresh_switch); < 0: not drawn yet, -(b + 1) for the
                      // spare bits b of the switch step that created it
    uint32_t on = 0xFFFFFFFFu;  // bit i: promoter of gene u*GPL+i is ON
    double V = 0.0;

    // ---- prologue (as cle_fused_kernel) ----------------------------------------------
    if (ctl.first) {
#pragma unroll
        for (int i = 0; i < GPL; ++i) {
            const int g = u * GPL + i;
            m[i] = valid[i] ? a.ginit[g].m0 : 0.0f;
            p[i] = valid[i] ? a.ginit[g].p0 : 0.0f;
        }
        bool any = false;
#pragma unroll
        for (int i = 0; i < GPL; ++i) any |= valid[i] && a.ginit[u * GPL + i].init_rand;
        if (any) {
            const uint4 w = philox(gcell, 0u, (uint32_t)quad, tagword(TAG_PROMOTER, a.stream), key);
#pragma unroll
            for (int i = 0; i < GPL; ++i) {
                const int g = u * GPL + i;
                if (valid[i] && a.ginit[g].init_rand && !(quad_word<GPL>(w, u, i) < a.ginit[g].thr_init))
                    on &= ~(1u << i);
            }
        }
#pragma unroll
        for (int i = 0; i < GPL; ++i) {
            ns[i] = kn[i] = kNever;
            if (inv_off[i] == inv_off[i]) {
                const uint4 w = philox(gcell, 0u, (uint32_t)(u * GPL + i), tagword(TAG_SWITCH, a.stream), key);
                const int2 f = fresh_switch(0, w.x, w.y, (on >> i) & 1u, inv_on[i], inv_off[i]);
                ns[i] = f.x;
                kn[i] = f.y;
            }
        }
        if (POP) {
            const uint4 w = philox(gcell, 0u, 0u, tagword(TAG_VOLUME, a.stream), key);
            V = __dadd_rn(a.V_lo, __dmul_rn(__dadd_rn(a.V_hi, -a.V_lo), u53(w.x, w.y)));
        }
    } else {
        // The cell's own state and, with a population, its slot's owner word are read together;
        // a cell replaced at the previous division then reads its donor's daughter instead (one
        // memory round trip for the cells that kept their slot instead of two).
        const int par = ctl.epoch & 1;
        const unsigned long long o = POP && ctl.epoch > 0 ? a.owner[par][cidx] : 0ull;
        auto load = [&](const float* Ms, const float* Ps, const uint8_t* Os, const int2* Ns, int64_t src) {
            on = 0xFFFFFFFFu;
#pragma unroll
            for (int i = 0; i < GPL; ++i) {  // cell-major state: a warp's lanes read adjacent entries
                const int g = u * GPL + i;
                const size_t si = (size_t)src * G + g;
                m[i] = valid[i] ? Ms[si] : 0.0f;
                p[i] = valid[i] ? Ps[si] : 0.0f;
                const int2 sw = valid[i] ? Ns[si] : make_int2(kNever, kNever);
                ns[i] = sw.x;
                kn[i] = sw.y;
                if (valid[i] && !Os[si]) on &= ~(1u << i);
            }
        };
        load(a.M, a.P, a.prom, a.NS, cidx);
        if (POP) V = a.V[cidx];
        if (POP && ctl.epoch > 0 && (uint32_t)(o >> 32) == (uint32_t)ctl.epoch) {
            const int64_t src = (int64_t)(o & 0xFFFFFFFFull);
            load(a.dM[par], a.dP[par], a.dprom[par], a.dNS[par], src);
            V = a.dV[par][src];
        }
    }

    // ---- fused step loop --------------------------------------------------------------
    const float k_t = a.k_t, mu_m = a.mu_m, mu_p = a.mu_p, dt = a.dt;
    const float mu_m_neg = -mu_m, mu_p_neg = -mu_p;
    const bool any_reg = n_reg > 0;
    // Draw the pending waiting times of this lane (the state after the next switch is the
    // opposite of the current one, which holds until that switch).
    auto resolve_pending = [&]() {
#pragma unroll
        for (int i = 0; i < GPL; ++i)
            if (kn[i] < 0)
                kn[i] = switch_steps(a.log2_tab, (uint32_t)(-kn[i] - 1), (on >> i) & 1u ? inv_on[i] : inv_off[i]);
    };
    int32_t ns_min = ns[0];  // earliest switch of the lane's genes
#pragma unroll
    for (int i = 1; i < GPL; ++i) ns_min = min(ns_min, ns[i]);
    // Philox blocks of the normals.  AHEAD: drawn one step ahead, step s + 1's rounds issued
    // beside step s's update (two independent dependency chains per lane), where the
    // registers allow it without spilling.
    constexpr bool AHEAD = GPL == 2 && EMAX <= 4 && TMAX <= 1;
    // With the round keys given, the part of the first Philox rounds that does not depend on
    // the step is computed once per lane (philox_hoist.cuh; same bits as philox_rk).
    PhiloxHoist ph[GPL / 2];
    if (RK) {
#pragma unroll
        for (int h = 0; h < GPL / 2; ++h)
            ph[h] = philox_hoist(gcell, (uint32_t)(u * (GPL / 2) + h), tagword(TAG_NORMAL, a.stream), rk0, rk1);
    }
    auto draw = [&](int s, int h) {
        const uint32_t c2 = (uint32_t)(u * (GPL / 2) + h), c3 = tagword(TAG_NORMAL, a.stream);
        return RK ? philox_hoisted(ph[h], (uint32_t)s, rk0, rk1) : philox(gcell, (uint32_t)s, c2, c3, key);
    };
    uint4 wn[GPL / 2];
    if (AHEAD) {
#pragma unroll
        for (int h = 0; h < GPL / 2; ++h) wn[h] = draw(ctl.step_begin, h);
    }
    for (int s = ctl.step_begin; s <= ctl.step_end; ++s) {
        cell_sync();  // every lane has read the row of the previous step
        if (any_reg) {
#pragma unroll
            for (int i = 0; i < GPL; i += 2) {  // gene pairs in packed FP32
                const float2 h = warpcell_hill2<HN>(make_float2(p[i], p[i + 1]), a);
                smem_f32(smem_raw, hill_at[i]) = h.x;
                smem_f32(smem_raw, hill_at[i + 1]) = h.y;
            }
        }
        // telegraph: a promoter switches when its waiting time runs out, and needs the waiting
        // time drawn at its previous switch.  Those draws wait until some switching gene of the
        // warp needs one; then every lane draws all of its pending ones together.
        const bool due = s == ns_min;
        const bool warp_due = __any_sync(0xFFFFFFFFu, due);
        if (warp_due) {
            bool need = false;
#pragma unroll
            for (int i = 0; i < GPL; ++i) need |= s == ns[i] && kn[i] < 0;
            if (__any_sync(0xFFFFFFFFu, need)) resolve_pending();
        }
        BM2 bm[GPL / 2];   // genes 2h, 2h + 1
        uint4 wc[GPL / 2];
#pragma unroll
        for (int h = 0; h < GPL / 2; ++h) {
            wc[h] = AHEAD ? wn[h] : draw(s, h);
            bm[h] = box_muller_parts2(wc[h]);
        }
        if (warp_due) {  // switch_at for the genes due now, with the next draw left pending
#pragma unroll
            for (int i = 0; i < GPL; ++i) {
                const bool sw = s == ns[i];
                on ^= (uint32_t)sw << i;
                // s + kn < 2^32 (both < 2^31): the unsigned sum saturates at kNever
                const int32_t nn = (int32_t)min((uint32_t)s + (uint32_t)kn[i], (uint32_t)kNever);
                // spare bits of the gene's normal words
                const uint32_t sb = (i & 1) ? switch_bits(wc[i / 2].z, wc[i / 2].w) : switch_bits(wc[i / 2].x, wc[i / 2].y);
                ns[i] = sw ? nn : ns[i];
                kn[i] = sw ? -(int32_t)sb - 1 : kn[i];
            }
            ns_min = ns[0];
#pragma unroll
            for (int i = 1; i < GPL; ++i) ns_min = min(ns_min, ns[i]);
        }
        cell_sync();  // the cell's activations are complete
        if (TMAX > 0) {
#pragma unroll
            for (int k = 0; k < TMAX; ++k) {  // x and 1-x are exact as fmaf(+-1, x, 0 or 1)
                float prod = 1.0f;
#pragma unroll
                for (int q = 0; q < kLaneSrc; ++q) prod *= fmaf(tsg[k], smem_f32(smem_raw, ta[k][q]), tof[k]);
                smem_f32(smem_raw, tout[k]) = fmaf(tsg[k], prod, tof[k]);
            }
            cell_sync();  // the cell's term values are complete
        }
        if (AHEAD) {
#pragma unroll
            for (int h = 0; h < GPL / 2; ++h) wn[h] = draw(s + 1, h);
        }
        const float Vf = POP ? (float)V : 1.0f;
#pragma unroll
        for (int i = 0; i < GPL; i += 2) {  // gene pairs in packed FP32 (each half as the scalar form)
            float2 reg = make_float2(cneg[i], cneg[i + 1]);
#pragma unroll
            for (int e = 0; e < EMAX; ++e)
                reg = fma2(make_float2(ew[i][e], ew[i + 1][e]),
                           make_float2(smem_f32(smem_raw, ea[i][e]), smem_f32(smem_raw, ea[i + 1][e])), reg);
            float2 tx = add2(reg, make_float2(beta[i], beta[i + 1]));
            if (POP) tx = mul2(tx, f2(Vf));
            if (!(on & (1u << i))) tx.x = 0.0f;
            if (!(on & (2u << i))) tx.y = 0.0f;
            float2 m2 = make_float2(m[i], m[i + 1]), p2 = make_float2(p[i], p[i + 1]);
            em_update2(m2, p2, tx, bm[i / 2], mu_m, mu_m_neg, mu_p, mu_p_neg, k_t, dt);
            m[i] = m2.x; m[i + 1] = m2.y;
            p[i] = p2.x; p[i + 1] = p2.y;
        }
        if (POP) V = __dmul_rn(V, a.growth_factor);
    }

    // ---- epilogue (as cle_fused_kernel) ------------------------------------------------
    resolve_pending();
    if (POP && ctl.check) {
        const bool divides = V > a.V_div;
        const int ne = ctl.epoch + 1;
        const int par = ne & 1;
        if (divides) {
            V = V * 0.5;
            if (live && u == 0) {
                const uint4 w = philox(gcell, (uint32_t)ctl.step_end, 0u, tagword(TAG_MORAN, a.stream), key);
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
            for (int i = 0; i < GPL; ++i) {
                const int g = u * GPL + i;
                if (!(live && valid[i])) continue;
                float mm, dm, pm, dp;
                if (a.partition == 1) {
                    mm = dm = m[i] * 0.5f;
                    pm = dp = p[i] * 0.5f;
                } else {
                    const int64_t mi = (int64_t)rintf(m[i]);
                    const int64_t pi = (int64_t)rintf(p[i]);
                    const int64_t mk = binomial_half(mi, key, a.stream, gcell, (uint32_t)ctl.step_end, (uint32_t)g, 0u);
                    const int64_t pk = binomial_half(pi, key, a.stream, gcell, (uint32_t)ctl.step_end, (uint32_t)g, 1u);
                    mm = (float)mk; dm = (float)(mi - mk);
                    pm = (float)pk; dp = (float)(pi - pk);
                }
                m[i] = mm;
                p[i] = pm;
                const size_t idx = (size_t)cidx * G + g;
                a.dM[par][idx] = dm;
                a.dP[par][idx] = dp;
                const uint32_t bon = (on >> i) & 1u;
                a.dprom[par][idx] = bon;
                int2 dns = make_int2(kNever, kNever);  // the daughter's promoter switches independently
                if (inv_off[i] == inv_off[i]) {
                    const uint4 w = philox(gcell, (uint32_t)ctl.step_end, (uint32_t)g | kDaughterSwitch,
                                           tagword(TAG_SWITCH, a.stream), key);
                    dns = fresh_switch(ctl.step_end, w.x, w.y, bon, inv_on[i], inv_off[i]);
                }
                a.dNS[par][idx] = dns;
            }
        }
    }
    if (!live) return;
#pragma unroll
    for (int i = 0; i < GPL; ++i) {
        const int g = u * GPL + i;
        if (!valid[i]) continue;
        const size_t si = (size_t)cell * G + g, idx = (size_t)g * N + cell;
        a.M[si] = m[i];
        a.P[si] = p[i];
        a.prom[si] = (on >> i) & 1u;
        a.NS[si] = make_int2(ns[i], kn[i]);
        if (ctl.last && a.out) {
            if (a.readout == 0) a.out[idx] = (double)m[i];
            else if (a.readout == 1) a.out[idx] = (double)p[i];
            else { a.out[idx] = (double)m[i]; a.out[(size_t)(G + g) * N + cell] = (double)p[i]; }
        }
    }
    if (POP && u == 0) a.V[cell] = V;
    if (ctl.last && a.counts) {
        const uint4 w = philox(gcell, 0u, 0u, tagword(TAG_EFFICIENCY, a.stream), key);
        const double z = box_muller_z0_f64(w.x, w.y);
        double pe = exp(a.cap_mu_log + a.cap_sigma * z);
        pe = fmin(fmax(pe, 0.0), 1.0);
        if (u == 0 && a.eff) a.eff[cell] = pe;
#pragma unroll
        for (int i = 0; i < GPL; ++i) {
            const int g = u * GPL + i;
            if (!valid[i]) continue;
            const double x = rint((double)(a.capture_species == 0 ? m[i] : p[i]));
            const int64_t n = x > 0.0 ? (int64_t)x : 0;
            int64_t y = 0;
            if (n > 0 && pe != 0.0) y = binomial_capture(n, pe, key, a.stream, gcell, (uint32_t)g);
            a.counts[(size_t)g * N + cell] = (int32_t)y;
        }
    }
}

template <int GPL, int EMAX, int TMAX, bool POP>
__global__ void __launch_bounds__(256, 3) cle_warpcell_kernel(const FusedArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const TileCtl ctl{a.step_begin, a.step_end, a.first, a.last, a.check, a.epoch};
    const bool mw = warpcell_wpc(a.G, GPL) > 1;
    if (a.hill_int == 2) {
        if (mw) warpcell_tile<GPL, EMAX, TMAX, POP, true, 2, true>(a, blockIdx.x, ctl, smem_raw, a.rk0, a.rk1);
        else warpcell_tile<GPL, EMAX, TMAX, POP, true, 2, false>(a, blockIdx.x, ctl, smem_raw, a.rk0, a.rk1);
    } else {
        if (mw) warpcell_tile<GPL, EMAX, TMAX, POP, true, 0, true>(a, blockIdx.x, ctl, smem_raw, a.rk0, a.rk1);
        else warpcell_tile<GPL, EMAX, TMAX, POP, true, 0, false>(a, blockIdx.x, ctl, smem_raw, a.rk0, a.rk1);
    }
}

template <int GPL, int EMAX, int TMAX, bool POP>
__global__ void __launch_bounds__(256, 3)
cle_warpcell_queue_kernel(const FusedArgs* args, const TileWork* items, int n_items, int* counter,
                       TileCtl shared_ctl, int use_shared, const KeySchedule ks, int use_ks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int next;
    while (true) {
        if (threadIdx.x == 0) next = atomicAdd(counter, 1);
        __syncthreads();
        const int it = next;
        __syncthreads();
        if (it >= n_items) return;
        const TileWork w = items[it];
        const FusedArgs& a = args[w.arg];
        const TileCtl& ctl = use_shared ? shared_ctl : w.ctl;
        const bool mw = warpcell_wpc(a.G, GPL) > 1;
        if (use_ks) {  // one key schedule for the whole launch: round keys from the parameters
            if (a.hill_int == 2) {
                if (mw) warpcell_tile<GPL, EMAX, TMAX, POP, true, 2, true>(a, w.tile, ctl, smem_raw, ks.rk0, ks.rk1);
                else warpcell_tile<GPL, EMAX, TMAX, POP, true, 2, false>(a, w.tile, ctl, smem_raw, ks.rk0, ks.rk1);
            } else {
                if (mw) warpcell_tile<GPL, EMAX, TMAX, POP, true, 0, true>(a, w.tile, ctl, smem_raw, ks.rk0, ks.rk1);
                else warpcell_tile<GPL, EMAX, TMAX, POP, true, 0, false>(a, w.tile, ctl, smem_raw, ks.rk0, ks.rk1);
            }
        } else if (a.hill_int == 2) {
            if (mw) warpcell_tile<GPL, EMAX, TMAX, POP, false, 2, true>(a, w.tile, ctl, smem_raw, nullptr, nullptr);
            else warpcell_tile<GPL, EMAX, TMAX, POP, false, 2, false>(a, w.tile, ctl, smem_raw, nullptr, nullptr);
        } else {
            if (mw) warpcell_tile<GPL, EMAX, TMAX, POP, false, 0, true>(a, w.tile, ctl, smem_raw, nullptr, nullptr);
            else warpcell_tile<GPL, EMAX, TMAX, POP, false, 0, false>(a, w.tile, ctl, smem_raw, nullptr, nullptr);
        }
        __syncthreads();
    }
}

template <int GPL, int EMAX, int TMAX, bool POP>
cudaError_t warpcell_launch_t(const FusedArgs& a, cudaStream_t st) {
    auto k = cle_warpcell_kernel<GPL, EMAX, TMAX, POP>;
    const size_t smem = warpcell_smem_bytes(a.G, GPL, a.n_reg, a.n_na, a.lane_nw1);
    cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    const int64_t cpb = warpcell_cells_per_block(a.G, GPL, a.lane_nw1);
    const unsigned blocks = (unsigned)((a.N + cpb - 1) / cpb);
    k<<<blocks, 32 * warpcell_block_warps(a.G, GPL, a.lane_nw1), smem, st>>>(a);
    return cudaGetLastError();
}

// Every network of one queue launch has the same warps per block (nwarps).
template <int GPL, int EMAX, int TMAX, bool POP>
cudaError_t warpcell_queue_launch_t(const FusedArgs* args, const TileWork* items, int n_items, int* counter,
                                    size_t smem, int grid, int nwarps, TileCtl shared_ctl, int use_shared,
                                    const KeySchedule* ks, cudaStream_t st) {
    auto k = cle_warpcell_queue_kernel<GPL, EMAX, TMAX, POP>;
    cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    const KeySchedule none{};
    k<<<grid, 32 * nwarps, smem, st>>>(args, items, n_items, counter, shared_ctl, use_shared, ks ? *ks : none,
                                       ks ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace scrna

// Explicit instantiation of both launchers of one kernel variant (one .cu file per
// (GPL, EMAX) pair keeps the parallel build balanced).
#define SCRNA_WARPCELL_INSTANTIATE(GPL, EMAX, TMAX, POP)                                                        \
    template cudaError_t scrna::warpcell_launch_t<GPL, EMAX, TMAX, POP>(const FusedArgs&, cudaStream_t);         \
    template cudaError_t scrna::warpcell_queue_launch_t<GPL, EMAX, TMAX, POP>(                                   \
        const FusedArgs*, const TileWork*, int, int*, size_t, int, int, TileCtl, int, const KeySchedule*,        \
        cudaStream_t);
#define SCRNA_WARPCELL_INSTANTIATE_ALL(GPL, EMAX)       \
    SCRNA_WARPCELL_INSTANTIATE(GPL, EMAX, 0, false)     \
    SCRNA_WARPCELL_INSTANTIATE(GPL, EMAX, 0, true)      \
    SCRNA_WARPCELL_INSTANTIATE(GPL, EMAX, 1, false)     \
    SCRNA_WARPCELL_INSTANTIATE(GPL, EMAX, 1, true)      \
    SCRNA_WARPCELL_INSTANTIATE(GPL, EMAX, 2, false)     \
    SCRNA_WARPCELL_INSTANTIATE(GPL, EMAX, 2, true)
