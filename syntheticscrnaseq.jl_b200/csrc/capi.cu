// C ABI of libscrna_cle.so: contexts, network upload, run planning and the
// reference-facing simulate / simulate_gpu_batch / apply_capture entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/scrna_cle.h"
#include "capi_internal.h"
#include "nvtx_range.h"
#include "cle_internal.h"

namespace scrna {
FusedLaunch fused_plan(int G, int n_reg, int n_in, int n_na, int n_na_src, int n_quads);
int fused_max_quads();
cudaError_t fused_launch(const FusedArgs& a, const FusedLaunch& L, bool pop, cudaStream_t st);
cudaError_t tau_launch(const FusedArgs& a, const FusedLaunch& L, bool pop, cudaStream_t st);
int warpcell_max_genes();
int warpcell_emax_class(int max_in);
int warpcell_pick_gpl(int G, bool bursty, int emax);
cudaError_t warpcell_launch(const FusedArgs& a, int gpl, int emax, int tmax, bool pop, cudaStream_t st);
cudaError_t plain_step_launch(const PlainArgs& a, cudaStream_t st);
cudaError_t plain_init_launch(int G, int64_t N, int64_t cell_offset, const GeneInit* gi,
                              const GeneRec* gr, uint32_t key0, uint32_t key1, uint32_t stream,
                              double* M, double* P, uint8_t* prom, int2* NS, cudaStream_t st);
cudaError_t plain_readout_launch(int G, int64_t N, const double* M, const double* P, int readout,
                                 double* out, cudaStream_t st);
cudaError_t capture_launch(int G, int64_t N, int64_t cell_offset, const double* X, double mu_log,
                           double sigma, uint32_t key0, uint32_t key1, uint32_t stream, double* eff,
                           int32_t* Y, cudaStream_t st);
cudaError_t philox_check_launch(int n, const uint32_t* d_ctr, uint32_t k0, uint32_t k1,
                                uint32_t* d_out, cudaStream_t st);
cudaError_t peak_launch(int which, int blocks, int iters, float* sink, cudaStream_t st);
cudaError_t peak_philox_launch(int blocks, int iters, float* sink, cudaStream_t st);
cudaError_t switch_log2_init_launch(float* tab, uint32_t n, cudaStream_t st);
int tensor_run(scrna_ctx* ctx, scrna_net* n, const scrna_kinetics* kin, const scrna_capture* cap,
               const scrna_cle_opts* o, scrna_state* st, int dtype, bool tau,
               const scrna_population* pop);
}  // namespace scrna

using namespace scrna;

// ---- errors ------------------------------------------------------------------------------------
static thread_local std::string g_err;

int scrna::fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

// ---- helpers ----------------------------------------------------------------------------------
static constexpr double kLn2 = 0.69314718055994530942;

static uint32_t prob_threshold(double p) {
    if (!(p > 0.0)) return 0u;
    double t = std::floor(p * 4294967296.0);
    if (t >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)t;
}

static int check_ctx(scrna_ctx* ctx) {
    if (!ctx) return fail(SCRNA_EINVAL, "context is NULL");
    return SCRNA_OK;
}

int scrna::set_device(scrna_ctx* ctx) {
    CU(cudaSetDevice(ctx->device));
    return SCRNA_OK;
}

extern "C" const char* scrna_last_error(void) { return g_err.c_str(); }
extern "C" int scrna_version(void) { return SCRNA_ABI_VERSION; }

extern "C" int scrna_ctx_create(int device, scrna_ctx** out) {
    if (!out) return fail(SCRNA_EINVAL, "out is NULL");
    *out = nullptr;
    int n = 0;
    CU(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(SCRNA_EINVAL, "device %d out of range (%d devices)", device, n);
    CU(cudaSetDevice(device));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(SCRNA_ENOTSUP, "device %d is sm_%d%d; this build targets sm_100a", device, prop.major, prop.minor);
    auto* c = new scrna_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete c; return fail(SCRNA_ECUDA, "cudaStreamCreate: %s", cudaGetErrorString(e)); }
    c->own_stream = true;
    tune_init_ctx(c);
    *out = c;
    return SCRNA_OK;
}

extern "C" int scrna_state_destroy(scrna_state* st);

extern "C" int scrna_ctx_destroy(scrna_ctx* ctx) {
    if (!ctx) return SCRNA_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (scrna_state* st : ctx->state_cache) scrna_state_destroy(st);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SCRNA_OK;
}

extern "C" int scrna_ctx_set_stream(scrna_ctx* ctx, void* s) {
    if (int r = check_ctx(ctx)) return r;
    if (ctx->own_stream && ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    ctx->stream = static_cast<cudaStream_t>(s);
    ctx->own_stream = false;
    return SCRNA_OK;
}

extern "C" int scrna_ctx_synchronize(scrna_ctx* ctx) {
    if (int r = check_ctx(ctx)) return r;
    if (int r = set_device(ctx)) return r;
    CU(cudaStreamSynchronize(ctx->stream));
    return SCRNA_OK;
}

extern "C" int64_t scrna_ctx_launch_count(const scrna_ctx* ctx) { return ctx ? ctx->launches.load() : -1; }

extern "C" int scrna_ctx_transfer_bytes(const scrna_ctx* ctx, int64_t* h2d, int64_t* d2h) {
    if (!ctx) return fail(SCRNA_EINVAL, "context is NULL");
    if (h2d) *h2d = ctx->h2d_bytes.load();
    if (d2h) *d2h = ctx->d2h_bytes.load();
    return SCRNA_OK;
}

// ---- networks ---------------------------------------------------------------------------------
static int build_edges(scrna_net* n, int32_t n_e, const int32_t* tgt, const int32_t* ptr,
                       const int32_t* src, const double* str, int base, int kind,
                       std::vector<std::vector<std::pair<NonAdd, std::vector<int32_t>>>>& per_target,
                       std::vector<std::vector<double>>& coef64) {
    const int G = n->G;
    if (n_e < 0) return fail(SCRNA_EINVAL, "negative edge count");
    if (n_e == 0) return SCRNA_OK;
    if (!tgt || !ptr || !src || !str) return fail(SCRNA_EINVAL, "edge arrays are NULL");
    if (ptr[0] != 0) return fail(SCRNA_EINVAL, "edge pointer array must start at 0");
    for (int e = 0; e < n_e; ++e) {
        const int t = tgt[e] - base;
        if (t < 0 || t >= G) return fail(SCRNA_EINVAL, "edge %d target %d out of range", e, tgt[e]);
        if (ptr[e + 1] < ptr[e]) return fail(SCRNA_EINVAL, "edge pointers not monotone");
        if (ptr[e + 1] == ptr[e]) return fail(SCRNA_EINVAL, "edge %d has no sources", e);
        std::vector<int32_t> s;
        for (int k = ptr[e]; k < ptr[e + 1]; ++k) {
            const int j = src[k] - base;
            if (j < 0 || j >= G) return fail(SCRNA_EINVAL, "edge %d source %d out of range", e, src[k]);
            s.push_back(j);
        }
        NonAdd na{};
        na.kind = kind;
        na.coef = (float)(str[e] * n->basals[t]);
        per_target[t].push_back({na, s});
        coef64[t].push_back(str[e] * n->basals[t]);
    }
    return SCRNA_OK;
}

extern "C" int scrna_net_create(scrna_ctx* ctx, int32_t G, const double* basals, const double* A_colmajor,
                                int32_t n_coop, const int32_t* coop_target, const int32_t* coop_ptr,
                                const int32_t* coop_src, const double* coop_strength,
                                int32_t n_redun, const int32_t* redun_target, const int32_t* redun_ptr,
                                const int32_t* redun_src, const double* redun_strength,
                                const double* k_on, const double* k_off, int32_t index_base,
                                scrna_net** out) {
    if (int r = check_ctx(ctx)) return r;
    if (!out) return fail(SCRNA_EINVAL, "out is NULL");
    *out = nullptr;
    if (G <= 0) return fail(SCRNA_EINVAL, "G must be positive (got %d)", G);
    if (!basals) return fail(SCRNA_EINVAL, "basals is NULL");
    if (index_base != 0 && index_base != 1) return fail(SCRNA_EINVAL, "index_base must be 0 or 1");
    auto n = std::make_unique<scrna_net>();
    n->ctx = ctx;
    n->G = G;
    n->basals.assign(basals, basals + G);
    n->A.assign((size_t)G * G, 0.0);
    if (A_colmajor)
        for (int i = 0; i < G; ++i)
            for (int j = 0; j < G; ++j) n->A[(size_t)i * G + j] = A_colmajor[i + (size_t)j * G];
    for (int i = 0; i < G; ++i)
        if (n->A[(size_t)i * G + i] != 0.0) return fail(SCRNA_EINVAL, "interaction diagonal must be zero (gene %d)", i + index_base);
    for (int i = 0; i < G; ++i)
        if (!std::isfinite(n->basals[i])) return fail(SCRNA_EINVAL, "basal %d is not finite", i + index_base);
    n->k_on.assign(G, INFINITY);
    n->k_off.assign(G, INFINITY);
    if (k_on) n->k_on.assign(k_on, k_on + G);
    if (k_off) n->k_off.assign(k_off, k_off + G);
    for (int i = 0; i < G; ++i)
        if (n->k_on[i] < 0 || n->k_off[i] < 0 || std::isnan(n->k_on[i]) || std::isnan(n->k_off[i]))
            return fail(SCRNA_EINVAL, "switching rates of gene %d must be >= 0", i + index_base);

    std::vector<std::vector<std::pair<NonAdd, std::vector<int32_t>>>> per_t(G);
    std::vector<std::vector<double>> coef64(G);
    if (int r = build_edges(n.get(), n_coop, coop_target, coop_ptr, coop_src, coop_strength, index_base, 0, per_t, coef64)) return r;
    if (int r = build_edges(n.get(), n_redun, redun_target, redun_ptr, redun_src, redun_strength, index_base, 1, per_t, coef64)) return r;

    // regulator slots: genes whose protein enters any additive, cooperative or redundant term
    std::vector<char> is_reg(G, 0);
    for (int i = 0; i < G; ++i)
        for (int j = 0; j < G; ++j)
            if (i != j && n->A[(size_t)i * G + j] * n->basals[i] != 0.0) is_reg[j] = 1;
    for (int t = 0; t < G; ++t)
        for (auto& pr : per_t[t])
            for (int j : pr.second) is_reg[j] = 1;
    n->reg_slot.assign(G, -1);
    for (int j = 0; j < G; ++j)
        if (is_reg[j]) { n->reg_slot[j] = (int)n->reg_gene.size(); n->reg_gene.push_back(j); }

    // additive in-edges per target (A_eff = A[i,j] beta_i, network.jl:206-219), sorted by source gene
    n->in_begin.resize(G); n->in_end.resize(G); n->cneg64.assign(G, 0.0);
    for (int i = 0; i < G; ++i) {
        n->in_begin[i] = (int)n->in_edge.size();
        for (int j = 0; j < G; ++j) {
            if (i == j) continue;
            const double w = n->A[(size_t)i * G + j] * n->basals[i];
            if (w == 0.0) continue;
            float2 e;
            e.x = (float)w;
            int32_t slot = n->reg_slot[j];
            std::memcpy(&e.y, &slot, 4);
            n->in_edge.push_back(e);
            n->in_w64.push_back(w);
            if (w < 0.0) n->cneg64[i] += -w;
        }
        n->in_end[i] = (int)n->in_edge.size();
    }
    n->na_begin.resize(G); n->na_count.resize(G);
    for (int t = 0; t < G; ++t) {
        n->na_begin[t] = (int)n->na.size();
        n->na_count[t] = (int)per_t[t].size();
        for (size_t k = 0; k < per_t[t].size(); ++k) {
            NonAdd na = per_t[t][k].first;
            na.src_begin = (int)n->na_src.size();
            for (int j : per_t[t][k].second) n->na_src.push_back(n->reg_slot[j]);
            na.src_end = (int)n->na_src.size();
            n->na.push_back(na);
            n->na_coef64.push_back(coef64[t][k]);
        }
    }
    if (n->na.size() >= 65536) return fail(SCRNA_ENOTSUP, "more than 65535 cooperative/redundant edges");

    if (int r = set_device(ctx)) return r;
    NetDev& d = n->dev;
    d.G = G;
    d.n_reg = (int)n->reg_gene.size();
    d.n_in = (int)n->in_edge.size();
    d.n_na = (int)n->na.size();
    d.n_na_src = (int)n->na_src.size();
    d.n_quads = (G + 3) / 4;
    for (int g = 0; g < G; ++g) d.bursty = d.bursty || std::isfinite(n->k_on[g]);
    // tables of the warp-per-cell-group kernel (small networks): per gene its additive
    // edges then one edge per term targeting it (term j's value sits in slot n_reg+3+j)
    bool lane_ok = G <= warpcell_max_genes();
    int max_in = 0;
    for (int g = 0; g < G && lane_ok; ++g) {
        max_in = std::max(max_in, n->in_end[g] - n->in_begin[g] + n->na_count[g]);
        for (int e = n->na_begin[g]; e < n->na_begin[g] + n->na_count[g]; ++e)
            lane_ok = lane_ok && n->na[e].src_end - n->na[e].src_begin <= kLaneSrc;
    }
    lane_ok = lane_ok && max_in <= kLaneEdges;
    const int emax = warpcell_emax_class(max_in);
    // genes per lane: the cheaper of 2 and 4 that leaves <= kLaneTerms terms per lane
    auto terms_per_lane = [&](int g) { const int lpc = (G + g - 1) / g; return (d.n_na + lpc - 1) / lpc; };
    int gpl = warpcell_pick_gpl(G, d.bursty, emax);
    if (terms_per_lane(gpl) > kLaneTerms && gpl == 4) gpl = 2;
    const int tmax = terms_per_lane(gpl);
    lane_ok = lane_ok && tmax <= kLaneTerms;
    std::vector<int2> li;
    std::vector<LaneTerm> lt;
    if (lane_ok) {
        const int zero_slot = d.n_reg, one_slot = d.n_reg + 1;  // constant slots of the kernel's rows
        li.assign((size_t)G * kLaneEdges, make_int2(zero_slot, 0));
        for (int g = 0; g < G; ++g) {
            int k = 0;
            for (int e = n->in_begin[g]; e < n->in_end[g]; ++e, ++k) {
                int32_t slot, wbits;
                std::memcpy(&slot, &n->in_edge[e].y, 4);
                std::memcpy(&wbits, &n->in_edge[e].x, 4);
                li[(size_t)g * kLaneEdges + k] = make_int2(slot, wbits);
            }
            for (int e = n->na_begin[g]; e < n->na_begin[g] + n->na_count[g]; ++e, ++k) {
                int32_t wbits;
                std::memcpy(&wbits, &n->na[e].coef, 4);
                li[(size_t)g * kLaneEdges + k] = make_int2(d.n_reg + 3 + e, wbits);
            }
        }
        lt.assign(std::max<size_t>(n->na.size(), 1), LaneTerm{});
        for (size_t e = 0; e < n->na.size(); ++e) {
            const NonAdd& na = n->na[e];
            LaneTerm t{};
            t.coef = na.coef;
            t.kind = na.kind;
            for (int q = 0; q < kLaneSrc; ++q) {
                const int si = na.src_begin + q;
                t.src[q] = si < na.src_end ? n->na_src[si] : (na.kind == 0 ? one_slot : zero_slot);
            }
            lt[e] = t;
        }
    }
    // every table in one device allocation and one copy (parts 256-byte aligned)
    struct Part { const void* src; size_t bytes; size_t off; };
    std::vector<Part> parts;
    size_t total = 0, payload = 0;
    auto add = [&](const void* src, size_t bytes) {
        parts.push_back(Part{src, bytes, total});
        total += (bytes + 255) & ~(size_t)255;
        payload += bytes;
        return parts.size() - 1;
    };
    const size_t p_in = add(n->in_edge.data(), n->in_edge.size() * sizeof(float2));
    const size_t p_na = add(n->na.data(), n->na.size() * sizeof(NonAdd));
    const size_t p_na_src = add(n->na_src.data(), n->na_src.size() * sizeof(int32_t));
    const size_t p_reg = add(n->reg_gene.data(), n->reg_gene.size() * sizeof(int32_t));
    const size_t p_w64 = add(n->in_w64.data(), n->in_w64.size() * sizeof(double));
    const size_t p_coef64 = add(n->na_coef64.data(), n->na_coef64.size() * sizeof(double));
    const size_t p_beta64 = add(n->basals.data(), n->basals.size() * sizeof(double));
    const size_t p_li = lane_ok ? add(li.data(), li.size() * sizeof(int2)) : 0;
    const size_t p_lt = lane_ok ? add(lt.data(), lt.size() * sizeof(LaneTerm)) : 0;
    std::vector<unsigned char> staging(std::max<size_t>(total, 16), 0);
    for (const Part& pt : parts)
        if (pt.bytes) std::memcpy(staging.data() + pt.off, pt.src, pt.bytes);
    CU(n->b_tables.ensure(staging.size()));
    CU(cudaMemcpy(n->b_tables.p, staging.data(), staging.size(), cudaMemcpyHostToDevice));
    ctx->h2d_bytes += (int64_t)payload;
    unsigned char* base = n->b_tables.as<unsigned char>();
    d.in_edge = reinterpret_cast<float2*>(base + parts[p_in].off);
    d.na = reinterpret_cast<NonAdd*>(base + parts[p_na].off);
    d.na_src = reinterpret_cast<int32_t*>(base + parts[p_na_src].off);
    d.reg_gene = reinterpret_cast<int32_t*>(base + parts[p_reg].off);
    d.in_w64 = reinterpret_cast<double*>(base + parts[p_w64].off);
    d.na_coef64 = reinterpret_cast<double*>(base + parts[p_coef64].off);
    d.beta64 = reinterpret_cast<double*>(base + parts[p_beta64].off);
    if (lane_ok) {
        d.lane_in = reinterpret_cast<int2*>(base + parts[p_li].off);
        d.lane_term = reinterpret_cast<LaneTerm*>(base + parts[p_lt].off);
        d.lane_gpl = gpl;
        d.lane_emax = emax;
        d.lane_tmax = tmax;
    }
    *out = n.release();
    return SCRNA_OK;
}

extern "C" int scrna_net_destroy(scrna_net* net) {
    if (!net) return SCRNA_OK;
    cudaSetDevice(net->ctx->device);
    cudaStreamSynchronize(net->ctx->stream);
    delete net;
    return SCRNA_OK;
}

extern "C" int32_t scrna_net_genes(const scrna_net* net) { return net ? net->G : -1; }

// Per-run gene tables (thresholds depend on dt, initial values on the kinetics).
int scrna::ensure_gene_tables(scrna_net* n, const scrna_kinetics* kin, double dt, bool pop) {
    const double kv[6] = {kin->k_t, kin->K_d, kin->n, kin->mu_m, kin->mu_p, kin->dilution};
    if (n->cache_valid && n->c_dt == dt && n->c_pop == pop && std::memcmp(kv, n->c_kin, sizeof kv) == 0)
        return SCRNA_OK;
    const int G = n->G;
    std::vector<GeneRec> gr(G);
    std::vector<GeneInit> gi(G);
    const int nq = (G + 3) / 4;
    std::vector<uint8_t> qt(nq, 0);
    for (int g = 0; g < G; ++g) {
        GeneRec& r = gr[g];
        r.beta = (float)n->basals[g];
        r.cneg = (float)n->cneg64[g];
        const double kon = n->k_on[g], koff = n->k_off[g];
        const bool tel = std::isfinite(kon);
        if (tel) {
            // waiting-time parameters -ln2/(k dt): k = inf -> -0 (switch at once), k = 0 -> -inf (never)
            r.inv_on = (float)(-kLn2 / (kon * dt));
            r.inv_off = (float)(-kLn2 / (koff * dt));
            qt[g >> 2] = 1;
        } else {
            r.inv_on = r.inv_off = std::nanf("");  // never switches
        }
        r.slot = n->reg_slot[g];
        r.in_begin = n->in_begin[g];
        r.in_end = n->in_end[g];
        r.na_range = (n->na_begin[g] << 16) | n->na_count[g];
        // initial condition: ceil of the deterministic steady state (kinetics.jl:65-70)
        const double mss = n->basals[g] / (kin->mu_m + kin->dilution);
        const double pss = kin->k_t * mss / (kin->mu_p + kin->dilution);
        gi[g].m0 = (float)std::ceil(mss);
        gi[g].p0 = (float)std::ceil(pss);
        gi[g].init_rand = (std::isfinite(kon) && std::isfinite(koff)) ? 1 : 0;
        gi[g].thr_init = gi[g].init_rand ? prob_threshold(kon / (kon + koff)) : 0u;
    }
    if (int r = set_device(n->ctx)) return r;
    CU(cudaStreamSynchronize(n->ctx->stream));
    CU(n->b_genes.ensure(G * sizeof(GeneRec)));
    CU(n->b_ginit.ensure(G * sizeof(GeneInit)));
    CU(n->b_quad_tel.ensure(nq));
    CU(cudaMemcpy(n->b_genes.p, gr.data(), G * sizeof(GeneRec), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(n->b_ginit.p, gi.data(), G * sizeof(GeneInit), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(n->b_quad_tel.p, qt.data(), nq, cudaMemcpyHostToDevice));
    n->ctx->h2d_bytes += (int64_t)(G * (sizeof(GeneRec) + sizeof(GeneInit)) + nq);
    n->cache_valid = true;
    n->c_dt = dt;
    n->c_pop = pop;
    std::memcpy(n->c_kin, kv, sizeof kv);
    return SCRNA_OK;
}

// ---- states ------------------------------------------------------------------------------------
int scrna::state_alloc(scrna_state* st, bool pop, bool plain) {
    const size_t gn = (size_t)st->G * st->N;
    const int outcols = st->readout == SCRNA_READOUT_BOTH ? 2 : 1;
    CU(st->M.ensure(gn * 4));
    CU(st->P.ensure(gn * 4));
    CU(st->prom.ensure(gn));
    CU(st->NS.ensure(gn * sizeof(int2)));
    CU(st->out.ensure(gn * outcols * 8));
    if (st->capture) {
        CU(st->counts.ensure(gn * 4));
        CU(st->eff.ensure((size_t)st->N * 8));
    }
    if (pop) {
        CU(st->V.ensure((size_t)st->N * 8));
        for (int k = 0; k < 2; ++k) {
            CU(st->dM[k].ensure(gn * 4));
            CU(st->dP[k].ensure(gn * 4));
            CU(st->dprom[k].ensure(gn));
            CU(st->dNS[k].ensure(gn * sizeof(int2)));
            CU(st->dV[k].ensure((size_t)st->N * 8));
            CU(st->owner[k].ensure((size_t)st->N * 8));
        }
    }
    if (plain) {
        CU(st->M64.ensure(gn * 8));
        CU(st->P64a.ensure(gn * 8));
        CU(st->P64b.ensure(gn * 8));
    }
    return SCRNA_OK;
}

extern "C" int scrna_state_create(scrna_ctx* ctx, const scrna_net* net, int64_t cell_num, int32_t readout,
                                  int32_t with_capture, scrna_state** out) {
    if (int r = check_ctx(ctx)) return r;
    if (!net || !out) return fail(SCRNA_EINVAL, "net/out is NULL");
    if (cell_num <= 0) return fail(SCRNA_EINVAL, "cell_num must be positive");
    if (readout < 0 || readout > 2) return fail(SCRNA_EINVAL, "readout must be 0 (mrna), 1 (protein) or 2 (both)");
    auto* st = new scrna_state();
    st->ctx = ctx;
    st->G = net->G;
    st->N = cell_num;
    st->readout = readout;
    st->capture = with_capture != 0;
    *out = st;
    return SCRNA_OK;
}

extern "C" int scrna_state_destroy(scrna_state* st) {
    if (!st) return SCRNA_OK;
    cudaSetDevice(st->ctx->device);
    cudaStreamSynchronize(st->ctx->stream);
    delete st;
    return SCRNA_OK;
}

extern "C" int scrna_state_device_ptrs(scrna_state* st, void** m, void** p) {
    if (!st) return fail(SCRNA_EINVAL, "state is NULL");
    if (m) *m = st->M.p;
    if (p) *p = st->P.p;
    return SCRNA_OK;
}

// ---- run planning ---------------------------------------------------------------------------
int scrna::validate_run(const scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                        const scrna_capture* cap, const scrna_cle_opts* o) {
    if (!net || !kin || !o) return fail(SCRNA_EINVAL, "net, kinetics and opts are required");
    if (!(o->dt > 0.0) || !std::isfinite(o->dt)) return fail(SCRNA_EINVAL, "dt must be positive and finite");
    if (o->n_steps <= 0 && !(o->T >= 0.0)) return fail(SCRNA_EINVAL, "T must be >= 0");
    if (o->readout < 0 || o->readout > 2) return fail(SCRNA_EINVAL, "readout must be 0, 1 or 2");
    if (!(kin->K_d > 0.0) || !(kin->n > 0.0)) return fail(SCRNA_EINVAL, "K_d and n must be positive");
    if (!(kin->mu_m + kin->dilution > 0.0) || !(kin->mu_p + kin->dilution > 0.0))
        return fail(SCRNA_EINVAL, "decay rates must be positive");
    if (pop) {
        if (pop->cell_num < 2) return fail(SCRNA_EINVAL, "population needs at least 2 cells");
        if (pop->div_check_interval <= 0) return fail(SCRNA_EINVAL, "div_check_interval must be positive");
        if (!(pop->V_div > 0.0) || !(pop->V_init_hi >= pop->V_init_lo)) return fail(SCRNA_EINVAL, "bad volume config");
        if (pop->partition != SCRNA_PARTITION_BINOMIAL && pop->partition != SCRNA_PARTITION_HALVE)
            return fail(SCRNA_EINVAL, "partition must be 0 (binomial) or 1 (halve)");
    }
    if (cap) {
        if (!(cap->efficiency > 0.0) || !(cap->efficiency_std >= 0.0)) return fail(SCRNA_EINVAL, "capture efficiency must be > 0 and std >= 0");
        if (cap->readout != SCRNA_READOUT_MRNA && cap->readout != SCRNA_READOUT_PROTEIN)
            return fail(SCRNA_EINVAL, "readout must be :mrna or :protein");  // population.jl:63
    }
    return SCRNA_OK;
}

int64_t scrna::n_steps_of(const scrna_cle_opts* o) {
    if (o->n_steps > 0) return o->n_steps;
    return (int64_t)std::ceil(o->T / o->dt);  // cle.jl:56
}

// Kernel arguments of one network's run (everything but the step range and flags).
void scrna::fill_fused_args(scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                            const scrna_capture* cap, const scrna_cle_opts* o, scrna_state* st, FusedArgs* out) {
    const NetDev& d = net->dev;
    FusedArgs a{};
    a.G = d.G; a.n_quads = d.n_quads; a.n_reg = d.n_reg; a.n_in = d.n_in; a.n_na = d.n_na; a.n_na_src = d.n_na_src;
    a.N = st->N;
    a.cell_offset = o->cell_offset;
    a.k_t = (float)kin->k_t;
    a.Kn = (float)std::pow(kin->K_d, kin->n);
    a.hill_n = (float)kin->n;
    a.hill_int = (kin->n == std::floor(kin->n) && kin->n >= 1.0 && kin->n <= 16.0) ? (int)kin->n : 0;
    a.mu_m = (float)(pop ? kin->mu_m : kin->mu_m + kin->dilution);
    a.mu_p = (float)(pop ? kin->mu_p : kin->mu_p + kin->dilution);
    a.dt = (float)o->dt;
    a.key0 = (uint32_t)o->seed; a.key1 = (uint32_t)(o->seed >> 32); a.stream = o->stream & 0xFFFFFFu;
    if (pop) {
        a.growth_factor = std::exp(pop->growth_rate * o->dt);
        a.V_div = pop->V_div; a.V_lo = pop->V_init_lo; a.V_hi = pop->V_init_hi;
        a.partition = pop->partition; a.exclude_mother = pop->exclude_mother ? 1 : 0;
    }
    a.genes = net->b_genes.as<GeneRec>();
    a.ginit = net->b_ginit.as<GeneInit>();
    a.in_edge = d.in_edge; a.na = d.na; a.na_src = d.na_src;
    a.quad_tel = net->b_quad_tel.as<uint8_t>();
    a.M = st->M.as<float>(); a.P = st->P.as<float>(); a.prom = st->prom.as<uint8_t>();
    a.NS = st->NS.as<int2>();
    if (pop) {
        a.V = st->V.as<double>();
        for (int k = 0; k < 2; ++k) {
            a.dM[k] = st->dM[k].as<float>(); a.dP[k] = st->dP[k].as<float>();
            a.dprom[k] = st->dprom[k].as<uint8_t>(); a.dV[k] = st->dV[k].as<double>();
            a.dNS[k] = st->dNS[k].as<int2>();
            a.owner[k] = st->owner[k].as<unsigned long long>();
        }
    }
    a.out = st->out.as<double>();
    a.readout = st->readout;
    if (cap) {
        a.counts = st->counts.as<int32_t>();
        a.eff = st->eff.as<double>();
        a.capture_species = cap->readout == SCRNA_READOUT_MRNA ? 0 : 1;
        a.cap_mu_log = std::log(cap->efficiency) - (cap->mean_correction ? cap->efficiency_std * cap->efficiency_std / 2.0 : 0.0);
        a.cap_sigma = cap->efficiency_std;
    }
    a.lane_in = d.lane_in;
    a.lane_term = d.lane_term;
    a.log2_tab = d.bursty ? switch_log2_table(net->ctx) : nullptr;
    for (int r = 0; r < 10; ++r) {
        a.rk0[r] = a.key0 + (uint32_t)r * 0x9E3779B9u;
        a.rk1[r] = a.key1 + (uint32_t)r * 0xBB67AE85u;
    }
    *out = a;
}

// The tau-leap's additions to the kernel arguments: FP32 decay probabilities 1 - exp(-mu dt)
// (with dilution unless a population makes it emergent, ext:240-241 and ext:574-575), FP64
// basals and steady-state denominators for a population's initial counts (ext:560-566).
void scrna::fill_tau_args(const scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                          const scrna_cle_opts* o, FusedArgs* a) {
    const double mu_m = pop ? kin->mu_m : kin->mu_m + kin->dilution;
    const double mu_p = pop ? kin->mu_p : kin->mu_p + kin->dilution;
    a->p_dec_m = (float)(1.0 - std::exp(-mu_m * o->dt));
    a->p_dec_p = (float)(1.0 - std::exp(-mu_p * o->dt));
    a->beta64 = net->dev.beta64;
    a->ss_mu_m = kin->mu_m + kin->dilution;
    a->ss_mu_p = kin->mu_p + kin->dilution;
    a->k_t64 = kin->k_t;
    a->tau_lockstep = tau_lockstep_default();
}

// The tau-leap's draw schedule: in lock step (measured faster on every workload tried: the
// 5-gene constitutive case, 10 telegraph genes, 100 regulated genes at 2,000 and 20,000
// cells), unless SCRNA_TAU_LOCKSTEP=0 asks for one draw after another; both give the same counts.
int scrna::tau_lockstep_default() {
    if (const char* e = std::getenv("SCRNA_TAU_LOCKSTEP")) return std::atoi(e) != 0 ? 1 : 0;
    return 1;
}

const float* scrna::switch_log2_table(scrna_ctx* ctx) {
    // built once per context, under a lock: a server's worker shares its caller's context
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (ctx->log2_tab_ready) return ctx->log2_tab.as<float>();
    const uint32_t n = 1u << 18;
    if (ctx->log2_tab.ensure((size_t)n * 4) != cudaSuccess) return nullptr;
    if (switch_log2_init_launch(ctx->log2_tab.as<float>(), n, ctx->stream) != cudaSuccess) return nullptr;
    ctx->launches++;
    // once per context: wait for the table, so kernels on any stream (batch groups, the
    // server's) read it filled
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return nullptr;
    ctx->log2_tab_ready = true;
    return ctx->log2_tab.as<float>();
}

// Whether the automatic path runs a network of N cells on the tensor path: always when the
// register path cannot hold it; the tau-leap beyond 128 genes, where the register path's
// threads hold pairs or quads of genes at its register limit and fit one block an SM, while
// the tensor form keeps the state in HBM at full occupancy with the same counts (exact
// regulation; ms a step, register / tensor: 129 sampled genes 0.027 / 0.009 at 1,000 cells
// and 0.144 / 0.051 at 20,000, 300 genes 0.055 / 0.012 and 0.281 / 0.107; 128 genes 0.009 /
// 0.008 and 0.040 / 0.047);
// the CLE and its populations for regulation of at least 5 % density over 256 genes or
// more, where the register path's in-edge loops cost more than the contraction.  The tensor
// path's step has a floor of about 20 us (its launches) whatever N; the register path's
// step at small N is one cell tile's latency, which for up to 64 gene quads (4 a thread) the
// CLE keeps below that floor.  Measured on a B200 (ms a step, register / tensor, 256 genes
// at 5 %): CLE 0.012 / 0.025 at 1,000 and 4,000 cells, 0.062 / 0.050 at 20,000, with a
// population 0.020 / 0.027 at 4,000 and 0.102 / 0.050 at 20,000; 400 genes at 5 %: CLE
// 0.047 / 0.026 at 1,000 cells, with a population 0.063 / 0.022.
bool scrna::auto_tensor(const scrna_net* net, bool tau, int64_t N) {
    const NetDev& d = net->dev;
    if (!register_path_holds(d)) return true;
    if (tau) return net->G > 128;
    const double density = (double)d.n_in / ((double)net->G * net->G);
    if (net->G < 256 || density < 0.05) return false;
    return d.n_quads > 64 || N >= 8192;
}

// Register-path kernel of a network: warp-per-cell-group (genes per lane, in-edges and
// terms per gene) or block tiles.
scrna::KernelChoice scrna::choose_kernel(const scrna_net* net, int path) {
    const NetDev& d = net->dev;
    KernelChoice k{};
    const bool warp_ok = d.lane_in != nullptr;
    k.warp = path == SCRNA_PATH_BLOCK ? false : warp_ok;
    k.gpl = d.lane_gpl;
    k.emax = d.lane_emax;
    k.tmax = d.lane_tmax;
    k.nw1 = 0;
    k.nwarps = warp_ok ? warpcell_block_warps_host(d.G, d.lane_gpl, 0) : 0;
    k.block = fused_plan(d.G, d.n_reg, d.n_in, d.n_na, d.n_na_src, d.n_quads);
    k.smem = k.warp ? warpcell_smem(d.G, k.gpl, d.n_reg, d.n_na, 0) : k.block.smem;
    return k;
}

// A register-path run of `st` from step start + 1 to the run's total step count.  start = 0:
// a new run from the initial state; start > 0: the continuation of the state's previous run
// (its state and `start_epoch` divisions), bit for bit the same as one run of the total
// length.  A continuation measures no kernel variants (that would overwrite the state) and
// converts the state to the layout of the kernel it runs.
static int run_fused(scrna_ctx* ctx, scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                     const scrna_capture* cap, const scrna_cle_opts* o, scrna_state* st, bool tau,
                     int64_t start = 0, int start_epoch = 0) {
    const NetDev& d = net->dev;
    if (d.n_quads > fused_max_quads())
        return fail(SCRNA_ENOTSUP, "G=%d exceeds the register path limit of %d genes", d.G, 4 * fused_max_quads());
    const int64_t n_steps = n_steps_of(o);
    if (n_steps >= (1ll << 31)) return fail(SCRNA_EINVAL, "too many steps");
    const FusedLaunch L = fused_plan(d.G, d.n_reg, d.n_in, d.n_na, d.n_na_src, d.n_quads);
    if (L.smem > kMaxDynamicSmem) return fail(SCRNA_ENOTSUP, "network tables need %zu bytes of shared memory", L.smem);
    cudaStream_t s = ctx->stream;
    // kernel choice: the lane kernel for small networks, block tiles otherwise (or as tuned)
    const bool warp_ok = d.lane_in != nullptr;
    if (o->path == SCRNA_PATH_WARP && !warp_ok)
        return fail(SCRNA_ENOTSUP, "the warp kernel needs G <= %d, <= %d in-edges (additive and cooperative/redundant) "
                    "per gene, terms of <= %d sources and <= %d terms per lane", warpcell_max_genes(), kLaneEdges,
                    kLaneSrc, kLaneTerms);
    KernelChoice kc{};
    if (tau) {  // the tau-leap runs on block tiles, in gene pairs or quads per thread unit
        kc = choose_kernel(net, SCRNA_PATH_BLOCK);
        kc.block = tau_plan(d.G, d.n_reg, d.n_in, d.n_na, d.n_na_src,
                            tau_genes_per_unit(d.G, d.n_reg, d.n_in, d.n_na, d.n_na_src, st->N));
        kc.smem = kc.block.smem;
        if (kc.block.smem > kMaxDynamicSmem)
            return fail(SCRNA_ENOTSUP, "network tables need %zu bytes of shared memory", kc.block.smem);
    }
    else if (int r = choose_kernel_tuned(ctx, net, kin, o, st, &kc, nullptr, nullptr, start == 0)) return r;
    if (start > 0 && st->last_cell_major != kc.warp)
        if (int r = state_relayout(ctx, st, kc.warp)) return r;
    FusedArgs a{};
    fill_fused_args(net, kin, pop, cap, o, st, &a);
    if (tau) fill_tau_args(net, kin, pop, o, &a);
    a.lane_nw1 = kc.nw1;
    auto launch = [&](bool is_pop) -> cudaError_t {
        if (tau) return tau_launch(a, kc.block, is_pop, s);
        return kc.warp ? warpcell_launch(a, kc.gpl, kc.emax, kc.tmax, is_pop, s) : fused_launch(a, kc.block, is_pop, s);
    };
    st->last_cell_major = kc.warp;  // the lane kernel keeps M, P, prom, NS cell-major
    st->steps_done = std::max(n_steps, start);
    st->last_tau = tau;
    if (!pop) {
        a.step_begin = (int)start + 1; a.step_end = (int)n_steps; a.first = start == 0 ? 1 : 0; a.last = 1;
        a.check = 0; a.epoch = 0;
        CU(launch(false));
        ctx->launches++;
        st->epoch = 0;
        return SCRNA_OK;
    }
    // Moran slot owners start empty; a continuation's previous placements are already in its state
    for (int k = 0; k < 2; ++k) CU(cudaMemsetAsync(st->owner[k].p, 0, (size_t)st->N * 8, s));
    const int64_t I = pop->div_check_interval;
    int64_t s0 = start + 1;
    int epoch = start_epoch;
    bool first = start == 0;
    if (s0 > n_steps && start > 0) {  // nothing left to run: read out the state as it is
        a.step_begin = (int)s0; a.step_end = (int)s0 - 1; a.first = 0; a.epoch = epoch; a.check = 0; a.last = 1;
        CU(launch(true));
        ctx->launches++;
        st->epoch = epoch;
        return SCRNA_OK;
    }
    while (true) {
        int64_t s1 = std::min(n_steps, ((s0 - 1) / I + 1) * I);
        if (n_steps == 0) s1 = 0;
        const bool check = s1 >= s0 && (s1 % I == 0);
        const bool final_chunk = s1 >= n_steps;
        a.step_begin = (int)s0; a.step_end = (int)s1;
        a.first = first ? 1 : 0;
        a.epoch = epoch;
        a.check = check ? 1 : 0;
        a.last = (final_chunk && !check) ? 1 : 0;
        CU(launch(true));
        ctx->launches++;
        first = false;
        if (check) epoch += 1;
        if (final_chunk) {
            if (check) {  // apply the last division's placements, then read out
                a.step_begin = (int)s1 + 1; a.step_end = (int)s1;
                a.first = 0; a.epoch = epoch; a.check = 0; a.last = 1;
                CU(launch(true));
                ctx->launches++;
            }
            break;
        }
        s0 = s1 + 1;
    }
    st->epoch = epoch;
    return SCRNA_OK;
}

// Continuation of a register-path run (scrna_cle_resume / scrna_tauleap_resume).
int scrna::resume_register_run(scrna_ctx* ctx, scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                               const scrna_capture* cap, const scrna_cle_opts* o, scrna_state* st, bool tau) {
    if (int r = validate_run(net, kin, pop, cap, o)) return r;
    if (!st->has_register_state) return fail(SCRNA_EINVAL, "the state holds no register-path run to continue");
    if (st->last_tau != tau) return fail(SCRNA_EINVAL, "the state was run by the other algorithm");
    if (st->G != net->G) return fail(SCRNA_EINVAL, "state was created for G=%d, network has G=%d", st->G, net->G);
    const int64_t N = pop ? pop->cell_num : o->cell_num;
    if (N != st->N) return fail(SCRNA_EINVAL, "state holds %lld cells, run asks for %lld", (long long)st->N, (long long)N);
    if ((pop != nullptr) != st->last_pop) return fail(SCRNA_EINVAL, "population mode differs from the state's run");
    if (cap && !st->capture) return fail(SCRNA_EINVAL, "state was created without capture buffers");
    if (o->readout != st->readout) return fail(SCRNA_EINVAL, "readout differs from the state's readout");
    if (o->precision != SCRNA_PRECISION_FP32) return fail(SCRNA_ENOTSUP, "continuations run the FP32 register path");
    // (a tau-leap run of the tensor path continues on the register path, with the same counts)
    const bool tensor_tau = tau && (o->path == SCRNA_PATH_TENSOR || o->path == SCRNA_PATH_TENSOR_LIBRARY);
    if (!tensor_tau && o->path != SCRNA_PATH_AUTO && o->path != SCRNA_PATH_REGISTER && o->path != SCRNA_PATH_BLOCK &&
        o->path != SCRNA_PATH_WARP)
        return fail(SCRNA_ENOTSUP, "continuations run the register path");
    const int64_t total = n_steps_of(o);
    if (total < st->steps_done)
        return fail(SCRNA_EINVAL, "the run asks for %lld steps in total, the state has done %lld",
                    (long long)total, (long long)st->steps_done);
    if (int r = set_device(ctx)) return r;
    if (int r = ensure_gene_tables(net, kin, o->dt, pop != nullptr)) return r;
    if (int r = state_alloc(st, pop != nullptr, false)) return r;
    st->have_counts = cap != nullptr;
    st->last_tensor = false;  // (a tensor-form tau-leap run left its state in the register layout)
    return run_fused(ctx, net, kin, pop, cap, o, st, tau, st->steps_done, st->epoch);
}

static int run_plain(scrna_ctx* ctx, scrna_net* net, const scrna_kinetics* kin, const scrna_capture* cap,
                     const scrna_cle_opts* o, scrna_state* st) {
    const NetDev& d = net->dev;
    const int64_t n_steps = n_steps_of(o);
    const uint32_t k0 = (uint32_t)o->seed, k1 = (uint32_t)(o->seed >> 32), sid = o->stream & 0xFFFFFFu;
    cudaStream_t s = ctx->stream;
    double* M = st->M64.as<double>();
    double* Pa = st->P64a.as<double>();
    double* Pb = st->P64b.as<double>();
    CU(plain_init_launch(d.G, st->N, o->cell_offset, net->b_ginit.as<GeneInit>(), net->b_genes.as<GeneRec>(),
                         k0, k1, sid, M, Pa, st->prom.as<uint8_t>(), st->NS.as<int2>(), s));
    ctx->launches++;
    PlainArgs a{};
    a.G = d.G; a.n_quads = d.n_quads; a.N = st->N; a.cell_offset = o->cell_offset;
    a.k_t = kin->k_t; a.Kn = std::pow(kin->K_d, kin->n); a.hill_n = kin->n;
    a.mu_m = kin->mu_m + kin->dilution; a.mu_p = kin->mu_p + kin->dilution;
    a.dt = o->dt; a.sqrt_dt = std::sqrt(o->dt);
    a.key0 = k0; a.key1 = k1; a.stream = sid;
    a.genes = net->b_genes.as<GeneRec>();
    a.in_edge = d.in_edge; a.in_w64 = d.in_w64; a.na = d.na; a.na_coef64 = d.na_coef64;
    a.na_src = d.na_src; a.reg_gene = d.reg_gene; a.quad_tel = net->b_quad_tel.as<uint8_t>();
    a.beta64 = d.beta64;
    a.M = M; a.prom = st->prom.as<uint8_t>(); a.NS = st->NS.as<int2>();
    for (int64_t step = 1; step <= n_steps; ++step) {
        a.step = (int)step;
        a.Pold = (step & 1) ? Pa : Pb;
        a.Pnew = (step & 1) ? Pb : Pa;
        CU(plain_step_launch(a, s));
        ctx->launches++;
    }
    const double* Pfinal = (n_steps & 1) ? Pb : Pa;
    st->p64_final = Pfinal;
    CU(plain_readout_launch(d.G, st->N, M, Pfinal, st->readout, st->out.as<double>(), s));
    ctx->launches++;
    if (cap) {
        const double mu_log = std::log(cap->efficiency) -
                              (cap->mean_correction ? cap->efficiency_std * cap->efficiency_std / 2.0 : 0.0);
        const double* X = cap->readout == SCRNA_READOUT_MRNA ? M : Pfinal;
        CU(capture_launch(d.G, st->N, o->cell_offset, X, mu_log, cap->efficiency_std, k0, k1, sid,
                          st->eff.as<double>(), st->counts.as<int32_t>(), s));
        ctx->launches += 2;
    }
    return SCRNA_OK;
}

static int run_device(scrna_ctx* ctx, const scrna_net* cnet, const scrna_kinetics* kin, const scrna_population* pop,
                      const scrna_capture* cap, const scrna_cle_opts* o, scrna_state* st, bool tau) {
    if (int r = check_ctx(ctx)) return r;
    if (int r = validate_run(cnet, kin, pop, cap, o)) return r;
    if (!st) return fail(SCRNA_EINVAL, "state is NULL");
    scrna_net* net = const_cast<scrna_net*>(cnet);
    if (st->G != net->G) return fail(SCRNA_EINVAL, "state was created for G=%d, network has G=%d", st->G, net->G);
    const int64_t N = pop ? pop->cell_num : o->cell_num;
    if (N != st->N) return fail(SCRNA_EINVAL, "state holds %lld cells, run asks for %lld", (long long)st->N, (long long)N);
    if (cap && !st->capture) return fail(SCRNA_EINVAL, "state was created without capture buffers");
    if (o->readout != st->readout) return fail(SCRNA_EINVAL, "readout differs from the state's readout");
    if (o->cell_offset < 0 || o->cell_offset + N > (1ll << 32)) return fail(SCRNA_EINVAL, "cell indices must fit 32 bits");
    const bool plain = o->precision == SCRNA_PRECISION_FP64_PLAIN;
    if (tau) {
        if (o->precision != SCRNA_PRECISION_FP32 && o->precision != SCRNA_PRECISION_FP32_F16)
            return fail(SCRNA_ENOTSUP, "the binomial tau-leap runs in FP32 (counts) only");
        if (o->path == SCRNA_PATH_WARP)
            return fail(SCRNA_ENOTSUP, "the binomial tau-leap runs on the block-tile kernel or the tensor path");
        if ((o->path == SCRNA_PATH_REGISTER || o->path == SCRNA_PATH_BLOCK) && net->dev.n_quads > fused_max_quads())
            return fail(SCRNA_ENOTSUP, "the register-path tau-leap takes G <= %d", 4 * fused_max_quads());
    }
    if (plain && pop) return fail(SCRNA_ENOTSUP, "the FP64 baseline path has no population dynamics");
    if (o->precision != SCRNA_PRECISION_FP32 && o->precision != SCRNA_PRECISION_FP32_F16 && !plain)
        return fail(SCRNA_EINVAL, "unknown precision");
    if (int r = set_device(ctx)) return r;
    if (int r = ensure_gene_tables(net, kin, o->dt, pop != nullptr)) return r;
    // kernel family: tensor cores for large dense networks (or when asked), else the register path
    const bool tensor = !plain && (o->path == SCRNA_PATH_TENSOR || o->path == SCRNA_PATH_TENSOR_LIBRARY ||
                                   (o->path == SCRNA_PATH_AUTO && auto_tensor(net, tau, N)));
    if (tensor) {
        st->has_register_state = false;
        st->have_counts = cap != nullptr;
        st->last_plain = false;
        st->last_pop = pop != nullptr;
        const int dtype = o->precision == SCRNA_PRECISION_FP32_F16 ? 1 : 0;
        // library-GEMM variant, cell-major state (the only tensor form of the tau-leap and of populations)
        if (tau || pop || o->path == SCRNA_PATH_TENSOR_LIBRARY || net->G > 4096) {
            st->last_tensor = true;
            st->last_tau = tau;
            if (int r = tensor_run(ctx, net, kin, cap, o, st, dtype, tau, pop)) return r;
            // an exact tau-leap state is the register path's: where that path holds the
            // network, the state continues and checkpoints as one of its runs
            if (tau && tau_tensor_exact(net, dtype) && register_path_holds(net->dev)) {
                if (int r = tensor_state_to_register(ctx, st)) return r;
                st->steps_done = n_steps_of(o);
                st->has_register_state = true;
            }
            return SCRNA_OK;
        }
        st->last_tensor = false;  // the fused kernel keeps the register path's gene-major state
        st->last_cell_major = false;
        return tc_run(ctx, net, kin, cap, o, st, dtype);
    }
    st->last_tensor = false;
    st->last_cell_major = false;
    if (int r = state_alloc(st, pop != nullptr, plain)) return r;
    st->have_counts = cap != nullptr;
    st->last_plain = plain;
    st->last_pop = pop != nullptr;
    st->has_register_state = false;
    if (plain) return run_plain(ctx, net, kin, cap, o, st);
    const int r = run_fused(ctx, net, kin, pop, cap, o, st, tau);
    st->has_register_state = r == SCRNA_OK;
    return r;
}

extern "C" int scrna_cle_run_device(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                                    const scrna_population* pop, const scrna_capture* cap,
                                    const scrna_cle_opts* o, scrna_state* st) {
    NvtxRange nvtx_range_("scrna_cle_run_device");
    return run_device(ctx, net, kin, pop, cap, o, st, false);
}

extern "C" int scrna_tauleap_run_device(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                                        const scrna_population* pop, const scrna_capture* cap,
                                        const scrna_cle_opts* o, scrna_state* st) {
    NvtxRange nvtx_range_("scrna_tauleap_run_device");
    return run_device(ctx, net, kin, pop, cap, o, st, true);
}

extern "C" int scrna_state_read(scrna_ctx* ctx, scrna_state* st, double* out, int32_t* counts, double* eff) {
    NvtxRange nvtx_range_("scrna_state_read");
    if (int r = check_ctx(ctx)) return r;
    if (!st) return fail(SCRNA_EINVAL, "state is NULL");
    if (int r = set_device(ctx)) return r;
    const size_t gn = (size_t)st->G * st->N;
    const int outcols = st->readout == SCRNA_READOUT_BOTH ? 2 : 1;
    if (out) CU(cudaMemcpyAsync(out, st->out.p, gn * outcols * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if ((counts || eff) && !st->have_counts) return fail(SCRNA_EINVAL, "the last run had no capture");
    if (counts) CU(cudaMemcpyAsync(counts, st->counts.p, gn * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (eff) CU(cudaMemcpyAsync(eff, st->eff.p, (size_t)st->N * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->d2h_bytes += (int64_t)((out ? gn * outcols * 8 : 0) + (counts ? gn * 4 : 0) + (eff ? (size_t)st->N * 8 : 0));
    return SCRNA_OK;
}

extern "C" int scrna_state_read_raw(scrna_ctx* ctx, scrna_state* st, void* mrna, void* protein,
                                    uint8_t* promoter, double* volume) {
    if (int r = check_ctx(ctx)) return r;
    if (!st) return fail(SCRNA_EINVAL, "state is NULL");
    if (int r = set_device(ctx)) return r;
    const size_t gn = (size_t)st->G * st->N;
    if (st->last_tensor) {  // cell-major state [N][t_ld]: transpose to [G][N] on the host
        const size_t ln = (size_t)st->t_ld * st->N;
        std::vector<float> tm(ln), tp(ln);
        std::vector<uint8_t> tpr(ln);
        CU(cudaMemcpyAsync(tm.data(), st->tM.p, ln * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaMemcpyAsync(tp.data(), st->tP.p, ln * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaMemcpyAsync(tpr.data(), st->tprom.p, ln, cudaMemcpyDeviceToHost, ctx->stream));
        if (volume) {
            if (!st->last_pop) return fail(SCRNA_EINVAL, "the last run had no population");
            CU(cudaMemcpyAsync(volume, st->V.p, (size_t)st->N * 8, cudaMemcpyDeviceToHost, ctx->stream));
        }
        CU(cudaStreamSynchronize(ctx->stream));
        for (int64_t c = 0; c < st->N; ++c)
            for (int g = 0; g < st->G; ++g) {
                const size_t src = (size_t)c * st->t_ld + g, dst = (size_t)g * st->N + c;
                if (mrna) static_cast<float*>(mrna)[dst] = tm[src];
                if (protein) static_cast<float*>(protein)[dst] = tp[src];
                if (promoter) promoter[dst] = tpr[src];
            }
        return SCRNA_OK;
    }
    if (st->last_cell_major) {  // lane-kernel state [N][G]: transpose to [G][N] on the host
        std::vector<float> tm(gn), tp(gn);
        std::vector<uint8_t> tpr(gn);
        if (!st->M.p || !st->P.p) return fail(SCRNA_EINVAL, "the state has not been run");
        CU(cudaMemcpyAsync(tm.data(), st->M.p, gn * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaMemcpyAsync(tp.data(), st->P.p, gn * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaMemcpyAsync(tpr.data(), st->prom.p, gn, cudaMemcpyDeviceToHost, ctx->stream));
        if (volume) {
            if (!st->last_pop) return fail(SCRNA_EINVAL, "the last run had no population");
            CU(cudaMemcpyAsync(volume, st->V.p, (size_t)st->N * 8, cudaMemcpyDeviceToHost, ctx->stream));
        }
        CU(cudaStreamSynchronize(ctx->stream));
        for (int64_t c = 0; c < st->N; ++c)
            for (int g = 0; g < st->G; ++g) {
                const size_t src = (size_t)c * st->G + g, dst = (size_t)g * st->N + c;
                if (mrna) static_cast<float*>(mrna)[dst] = tm[src];
                if (protein) static_cast<float*>(protein)[dst] = tp[src];
                if (promoter) promoter[dst] = tpr[src];
            }
        return SCRNA_OK;
    }
    const size_t esz = st->last_plain ? 8 : 4;
    const void* dm = st->last_plain ? st->M64.p : st->M.p;
    const void* dp = st->last_plain ? (const void*)st->p64_final : st->P.p;
    if (!dm || !dp) return fail(SCRNA_EINVAL, "the state has not been run");
    if (mrna) CU(cudaMemcpyAsync(mrna, dm, gn * esz, cudaMemcpyDeviceToHost, ctx->stream));
    if (protein) CU(cudaMemcpyAsync(protein, dp, gn * esz, cudaMemcpyDeviceToHost, ctx->stream));
    if (promoter) CU(cudaMemcpyAsync(promoter, st->prom.p, gn, cudaMemcpyDeviceToHost, ctx->stream));
    if (volume) {
        if (!st->last_pop) return fail(SCRNA_EINVAL, "the last run had no population");
        CU(cudaMemcpyAsync(volume, st->V.p, (size_t)st->N * 8, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CU(cudaStreamSynchronize(ctx->stream));
    return SCRNA_OK;
}

static int simulate(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                    const scrna_capture* cap, const scrna_cle_opts* o, double* out, int32_t* counts, double* eff,
                    bool tau) {
    if (int r = check_ctx(ctx)) return r;
    if (int r = validate_run(net, kin, pop, cap, o)) return r;
    if (!out) return fail(SCRNA_EINVAL, "out is NULL");
    if (cap && !counts) return fail(SCRNA_EINVAL, "counts is NULL but capture was requested");
    const int64_t N = pop ? pop->cell_num : o->cell_num;
    if (N <= 0) return fail(SCRNA_EINVAL, "cell_num must be positive");
    // reuse a cached state of the same shape, so repeated calls allocate nothing
    scrna_state* st = nullptr;
    auto& cache = ctx->state_cache;
    for (size_t i = 0; i < cache.size(); ++i) {
        scrna_state* c = cache[i];
        if (c->G == net->G && c->N == N && c->readout == o->readout && c->capture == (cap != nullptr)) {
            st = c;
            cache.erase(cache.begin() + i);
            cache.push_back(st);
            break;
        }
    }
    if (!st) {
        if (int r = scrna_state_create(ctx, net, N, o->readout, cap != nullptr, &st)) return r;
        if (cache.size() >= 4) {
            scrna_state_destroy(cache.front());
            cache.erase(cache.begin());
        }
        cache.push_back(st);
    }
    if (int r = run_device(ctx, net, kin, pop, cap, o, st, tau)) return r;
    return scrna_state_read(ctx, st, out, cap ? counts : nullptr, cap ? eff : nullptr);
}

extern "C" int scrna_cle_simulate(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                                  const scrna_population* pop, const scrna_capture* cap,
                                  const scrna_cle_opts* o, double* out, int32_t* counts, double* eff) {
    NvtxRange nvtx_range_("scrna_cle_simulate");
    return simulate(ctx, net, kin, pop, cap, o, out, counts, eff, false);
}

extern "C" int scrna_tauleap_simulate(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                                      const scrna_population* pop, const scrna_capture* cap,
                                      const scrna_cle_opts* o, double* out, int32_t* counts, double* eff) {
    NvtxRange nvtx_range_("scrna_tauleap_simulate");
    return simulate(ctx, net, kin, pop, cap, o, out, counts, eff, true);
}

extern "C" int scrna_cle_simulate_batch(scrna_ctx* ctx, int32_t B, const scrna_net* const* nets,
                                        const scrna_kinetics* kins, int32_t n_kins, const int64_t* cell_nums,
                                        const scrna_population* const* pops, const scrna_capture* cap,
                                        const scrna_cle_opts* opts, double* const* outs, int32_t* const* counts) {
    NvtxRange nvtx_range_("scrna_cle_simulate_batch");
    if (int r = check_ctx(ctx)) return r;
    if (B <= 0 || !nets || !kins || !opts || !outs) return fail(SCRNA_EINVAL, "bad batch arguments");
    if (n_kins != 1 && n_kins != B) return fail(SCRNA_EINVAL, "n_kins must be 1 or B");
    if (opts->precision != SCRNA_PRECISION_FP32) return fail(SCRNA_ENOTSUP, "batches run the FP32 path");
    if (int r = set_device(ctx)) return r;
    return batch_simulate(ctx, B, nets, kins, n_kins, cell_nums, pops, cap, opts, outs, counts, false);
}

extern "C" int scrna_tauleap_simulate_batch(scrna_ctx* ctx, int32_t B, const scrna_net* const* nets,
                                            const scrna_kinetics* kins, int32_t n_kins, const int64_t* cell_nums,
                                            const scrna_population* const* pops, const scrna_capture* cap,
                                            const scrna_cle_opts* opts, double* const* outs, int32_t* const* counts) {
    NvtxRange nvtx_range_("scrna_tauleap_simulate_batch");
    if (int r = check_ctx(ctx)) return r;
    if (B <= 0 || !nets || !kins || !opts || !outs) return fail(SCRNA_EINVAL, "bad batch arguments");
    if (n_kins != 1 && n_kins != B) return fail(SCRNA_EINVAL, "n_kins must be 1 or B");
    if (opts->precision != SCRNA_PRECISION_FP32) return fail(SCRNA_ENOTSUP, "the binomial tau-leap runs in FP32 only");
    if (int r = set_device(ctx)) return r;
    return batch_simulate(ctx, B, nets, kins, n_kins, cell_nums, pops, cap, opts, outs, counts, true);
}

extern "C" int scrna_apply_capture(scrna_ctx* ctx, int64_t N, int32_t G, const double* X, const scrna_capture* cap,
                                   uint64_t seed, uint32_t stream, int32_t* Y, double* eff) {
    NvtxRange nvtx_range_("scrna_apply_capture");
    if (int r = check_ctx(ctx)) return r;
    if (N <= 0 || G <= 0 || !X || !cap || !Y) return fail(SCRNA_EINVAL, "bad capture arguments");
    if (!(cap->efficiency > 0.0) || !(cap->efficiency_std >= 0.0)) return fail(SCRNA_EINVAL, "capture efficiency must be > 0 and std >= 0");
    if (int r = set_device(ctx)) return r;
    const size_t gn = (size_t)G * N;
    DevBuf dX, dY, dE;
    CU(dX.ensure(gn * 8));
    CU(dY.ensure(gn * 4));
    CU(dE.ensure((size_t)N * 8));
    CU(cudaMemcpyAsync(dX.p, X, gn * 8, cudaMemcpyHostToDevice, ctx->stream));
    const double mu_log = std::log(cap->efficiency) -
                          (cap->mean_correction ? cap->efficiency_std * cap->efficiency_std / 2.0 : 0.0);
    CU(capture_launch(G, N, 0, dX.as<double>(), mu_log, cap->efficiency_std, (uint32_t)seed,
                      (uint32_t)(seed >> 32), stream & 0xFFFFFFu, dE.as<double>(), dY.as<int32_t>(), ctx->stream));
    ctx->launches += 2;
    CU(cudaMemcpyAsync(Y, dY.p, gn * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (eff) CU(cudaMemcpyAsync(eff, dE.p, (size_t)N * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return SCRNA_OK;
}

extern "C" int scrna_debug_philox(scrna_ctx* ctx, int32_t n, const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
    if (int r = check_ctx(ctx)) return r;
    if (n <= 0 || !ctr || !key || !out) return fail(SCRNA_EINVAL, "bad arguments");
    if (int r = set_device(ctx)) return r;
    DevBuf dc, dout;
    CU(dc.ensure((size_t)n * 16));
    CU(dout.ensure((size_t)n * 16));
    CU(cudaMemcpyAsync(dc.p, ctr, (size_t)n * 16, cudaMemcpyHostToDevice, ctx->stream));
    CU(philox_check_launch(n, dc.as<uint32_t>(), key[0], key[1], dout.as<uint32_t>(), ctx->stream));
    ctx->launches++;
    CU(cudaMemcpyAsync(out, dout.p, (size_t)n * 16, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return SCRNA_OK;
}

extern "C" int scrna_host_alloc(size_t bytes, void** p) {
    if (!p) return fail(SCRNA_EINVAL, "NULL argument");
    *p = nullptr;
    CU(cudaHostAlloc(p, bytes ? bytes : 16, cudaHostAllocPortable));
    return SCRNA_OK;
}

extern "C" int scrna_host_free(void* p) {
    if (p) CU(cudaFreeHost(p));
    return SCRNA_OK;
}

extern "C" int scrna_measure_pipe_peaks(scrna_ctx* ctx, double* fma, double* sfu, double* iops) {
    if (int r = check_ctx(ctx)) return r;
    if (int r = set_device(ctx)) return r;
    DevBuf sink;
    CU(sink.ensure(256 * 4));
    const int blocks = ctx->sm_count * 8;
    const int iters[3] = {4096, 1024, 2048};
    double res[3];
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    for (int w = 0; w < 3; ++w) {
        CU(peak_launch(w, blocks, iters[w] / 8, sink.as<float>(), ctx->stream));  // warm-up
        CU(cudaEventRecord(e0, ctx->stream));
        CU(peak_launch(w, blocks, iters[w], sink.as<float>(), ctx->stream));
        CU(cudaEventRecord(e1, ctx->stream));
        CU(cudaEventSynchronize(e1));
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, e0, e1));
        ctx->launches += 2;
        res[w] = (double)blocks * 256.0 * iters[w] * 16.0 * 8.0 / (ms * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (fma) *fma = res[0];
    if (sfu) *sfu = res[1];
    if (iops) *iops = res[2];
    return SCRNA_OK;
}

extern "C" int scrna_measure_philox_rate(scrna_ctx* ctx, double* calls_per_s) {
    if (int r = check_ctx(ctx)) return r;
    if (!calls_per_s) return fail(SCRNA_EINVAL, "calls_per_s is NULL");
    if (int r = set_device(ctx)) return r;
    DevBuf sink;
    CU(sink.ensure(256 * 4));
    const int blocks = ctx->sm_count * 8, iters = 2048;
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    CU(peak_philox_launch(blocks, iters / 8, sink.as<float>(), ctx->stream));  // warm-up
    CU(cudaEventRecord(e0, ctx->stream));
    CU(peak_philox_launch(blocks, iters, sink.as<float>(), ctx->stream));
    CU(cudaEventRecord(e1, ctx->stream));
    CU(cudaEventSynchronize(e1));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->launches += 2;
    *calls_per_s = (double)blocks * 256.0 * 4.0 * iters / (ms * 1e-3);
    return SCRNA_OK;
}

// ---- internal views for other translation units of the library ----------------------------------
namespace scrna {

int set_error(int code, const char* msg) { return fail(code, "%s", msg); }

int check_run_args(const scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                   const scrna_capture* cap, const scrna_cle_opts* o) {
    return validate_run(net, kin, pop, cap, o);
}

int64_t run_steps(const scrna_cle_opts* o) { return n_steps_of(o); }

cudaStream_t ctx_stream(scrna_ctx* ctx) { return ctx->stream; }
int ctx_device(scrna_ctx* ctx) { return ctx->device; }
void ctx_add_launches(scrna_ctx* ctx, int n) { ctx->launches += n; }
const NetDev& net_dev(const scrna_net* n) { return n->dev; }

// Per-run gene tables of `n` written into caller-provided host arrays (G, G and
// (G+3)/4 entries); same contents as the tables the regular path uploads.
void gene_tables_host(const scrna_net* n, const scrna_kinetics* kin, double dt, GeneRec* gr,
                      GeneInit* gi, uint8_t* qt) {
    const int G = n->G;
    for (int q = 0; q < (G + 3) / 4; ++q) qt[q] = 0;
    for (int g = 0; g < G; ++g) {
        GeneRec& r = gr[g];
        r.beta = (float)n->basals[g];
        r.cneg = (float)n->cneg64[g];
        const double kon = n->k_on[g], koff = n->k_off[g];
        if (std::isfinite(kon)) {
            r.inv_on = (float)(-kLn2 / (kon * dt));
            r.inv_off = (float)(-kLn2 / (koff * dt));
            qt[g >> 2] = 1;
        } else {
            r.inv_on = r.inv_off = std::nanf("");
        }
        r.slot = n->reg_slot[g];
        r.in_begin = n->in_begin[g];
        r.in_end = n->in_end[g];
        r.na_range = (n->na_begin[g] << 16) | n->na_count[g];
        const double mss = n->basals[g] / (kin->mu_m + kin->dilution);
        const double pss = kin->k_t * mss / (kin->mu_p + kin->dilution);
        gi[g].m0 = (float)std::ceil(mss);
        gi[g].p0 = (float)std::ceil(pss);
        gi[g].init_rand = (std::isfinite(kon) && std::isfinite(koff)) ? 1 : 0;
        gi[g].thr_init = gi[g].init_rand ? prob_threshold(kon / (kon + koff)) : 0u;
    }
}

}  // namespace scrna
