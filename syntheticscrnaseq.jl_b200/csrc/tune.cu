// Autotuner of the register-path kernels: per network shape it measures the kernel
// variants that compute the same sums in the same order (block tiles; the lane kernel with
// 2 or 4 genes per lane and 2, 4 or 8 warps per block) and keeps the fastest, in memory and
// in a JSON file shared by processes.  Every candidate gives bit-identical results, so a
// tuned run equals an untuned one.
//
// Key: device (compute capability and SM count), G, padded in-edges per gene, the number of
// cooperative / redundant terms, telegraph genes present, Hill exponent 2, and the cell
// count's power-of-two bucket.  A measurement runs the candidates without population for a
// short step range on the run's own state buffers (the run then starts from its initial
// state), a warm-up and three timed launches each, and takes the fastest launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

#include "capi_internal.h"
#include "nvtx_range.h"

namespace scrna {

FusedLaunch fused_plan(int G, int n_reg, int n_in, int n_na, int n_na_src, int n_quads);
int fused_max_quads();
cudaError_t fused_launch(const FusedArgs& a, const FusedLaunch& L, bool pop, cudaStream_t st);
cudaError_t warpcell_launch(const FusedArgs& a, int gpl, int emax, int tmax, bool pop, cudaStream_t st);

namespace {

std::mutex g_mu;
std::map<std::string, std::map<std::string, scrna_tune_choice>> g_files;  // path -> key -> choice

// ---- the cache file ----------------------------------------------------------------------
// {"version": 1, "entries": {"<key>": {"kernel": 1, "genes_per_lane": 2, "block_warps": 4,
//  "us_per_step": 0.71}, ...}}

struct Parser {
    const char* p;
    const char* e;
    void ws() { while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p; }
    bool eat(char c) { ws(); if (p < e && *p == c) { ++p; return true; } return false; }
    bool str(std::string* out) {
        ws();
        if (p >= e || *p != '"') return false;
        ++p;
        out->clear();
        while (p < e && *p != '"') {
            if (*p == '\\' && p + 1 < e) ++p;
            out->push_back(*p++);
        }
        if (p >= e) return false;
        ++p;
        return true;
    }
    bool num(double* out) {
        ws();
        char* end = nullptr;
        *out = std::strtod(p, &end);
        if (end == p || end > e) return false;
        p = end;
        return true;
    }
};

// Parses the file's entries; a missing, empty or malformed file gives an empty map.
std::map<std::string, scrna_tune_choice> read_file(const std::string& path) {
    std::map<std::string, scrna_tune_choice> out;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return out;
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    std::fclose(f);
    Parser ps{text.data(), text.data() + text.size()};
    std::map<std::string, scrna_tune_choice> tmp;
    std::string k;
    double v;
    if (!ps.eat('{')) return out;
    bool have_entries = false;
    while (!ps.eat('}')) {
        if (!ps.str(&k) || !ps.eat(':')) return out;
        if (k == "version") {
            if (!ps.num(&v) || v != 1.0) return out;
        } else if (k == "entries") {
            if (!ps.eat('{')) return out;
            while (!ps.eat('}')) {
                std::string key;
                if (!ps.str(&key) || !ps.eat(':') || !ps.eat('{')) return out;
                scrna_tune_choice c{};
                while (!ps.eat('}')) {
                    std::string field;
                    if (!ps.str(&field) || !ps.eat(':') || !ps.num(&v)) return out;
                    if (field == "kernel") c.kernel = (int32_t)v;
                    else if (field == "genes_per_lane") c.genes_per_lane = (int32_t)v;
                    else if (field == "block_warps") c.block_warps = (int32_t)v;
                    else if (field == "us_per_step") c.us_per_step = v;
                    ps.eat(',');
                }
                c.found = 1;
                tmp[key] = c;
                ps.eat(',');
            }
            have_entries = true;
        } else {
            return out;
        }
        ps.eat(',');
    }
    if (have_entries) out.swap(tmp);
    return out;
}

int mkdirs_for(const std::string& path) {
    for (size_t i = 1; i < path.size(); ++i)
        if (path[i] == '/') {
            const std::string d = path.substr(0, i);
            if (::mkdir(d.c_str(), 0755) != 0 && errno != EEXIST) return -1;
        }
    return 0;
}

// Writes the entries to a temporary file next to `path` and renames it over `path`, so a
// reader sees the old or the new file, never a partial one.
int write_file(const std::string& path, const std::map<std::string, scrna_tune_choice>& entries) {
    if (mkdirs_for(path) != 0) return -1;
    char tmp_name[64];
    std::snprintf(tmp_name, sizeof tmp_name, ".tmp.%d", (int)::getpid());
    const std::string tmp = path + tmp_name;
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return -1;
    std::fprintf(f, "{\"version\": 1, \"entries\": {");
    bool first = true;
    for (const auto& kv : entries) {
        std::fprintf(f, "%s\n  \"%s\": {\"kernel\": %d, \"genes_per_lane\": %d, \"block_warps\": %d, \"us_per_step\": %.6g}",
                     first ? "" : ",", kv.first.c_str(), kv.second.kernel, kv.second.genes_per_lane,
                     kv.second.block_warps, kv.second.us_per_step);
        first = false;
    }
    std::fprintf(f, "\n}}\n");
    const bool ok = std::fflush(f) == 0;
    std::fclose(f);
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        return -1;
    }
    return 0;
}

std::map<std::string, scrna_tune_choice>& file_entries(const std::string& path) {
    auto it = g_files.find(path);
    if (it == g_files.end()) it = g_files.emplace(path, read_file(path)).first;
    return it->second;
}

int lookup(const std::string& path, const std::string& key, scrna_tune_choice* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto& m = file_entries(path);
    auto it = m.find(key);
    if (it == m.end()) {
        // another process may have written it since this one read the file
        m = read_file(path);
        it = m.find(key);
    }
    if (it == m.end()) { *out = scrna_tune_choice{}; return SCRNA_OK; }
    *out = it->second;
    out->found = 1;
    return SCRNA_OK;
}

int store(const std::string& path, const std::string& key, const scrna_tune_choice& c) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto merged = read_file(path);  // keep entries other processes added
    merged[key] = c;
    merged[key].found = 1;
    g_files[path] = merged;
    if (write_file(path, merged) != 0) return fail(SCRNA_EINVAL, "cannot write the autotune cache %s", path.c_str());
    return SCRNA_OK;
}

std::string default_cache_path() {
    if (const char* p = std::getenv("SCRNA_AUTOTUNE_CACHE")) return p;
    if (const char* x = std::getenv("XDG_CACHE_HOME")) return std::string(x) + "/scrna_b200/autotune.json";
    if (const char* h = std::getenv("HOME")) return std::string(h) + "/.cache/scrna_b200/autotune.json";
    return "";
}

int floor_log2(int64_t n) {
    int b = 0;
    while (n > 1) { n >>= 1; ++b; }
    return b;
}

std::string make_key(const char* arch, int G, int emax, int n_terms, int bursty, int hill2, int64_t N) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "%s|G%d|e%d|t%d|b%d|h%d|N%d", arch, G, emax, n_terms, bursty ? 1 : 0,
                  hill2 ? 1 : 0, floor_log2(std::max<int64_t>(N, 1)));
    return buf;
}

}  // namespace

void tune_init_ctx(scrna_ctx* ctx) {
    int mode = 1;
    if (const char* m = std::getenv("SCRNA_AUTOTUNE")) mode = std::atoi(m);
    ctx->tune_mode = std::min(std::max(mode, 0), 2);
    ctx->tune_path = default_cache_path();
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ctx->device) == cudaSuccess)
        std::snprintf(ctx->tune_arch, sizeof ctx->tune_arch, "sm%d%dx%d", prop.major, prop.minor,
                      prop.multiProcessorCount);
}

// Lane-kernel terms evaluated per lane for a genes-per-lane choice.
static int terms_per_lane(int G, int n_terms, int gpl) {
    const int lpc = (G + gpl - 1) / gpl;
    return (n_terms + lpc - 1) / lpc;
}

KernelChoice choice_from(const scrna_net* net, const scrna_tune_choice& c) {
    const NetDev& d = net->dev;
    KernelChoice k{};
    k.warp = c.kernel == 1;
    k.block = fused_plan(d.G, d.n_reg, d.n_in, d.n_na, d.n_na_src, d.n_quads);
    if (k.warp) {
        k.gpl = c.genes_per_lane;
        k.emax = d.lane_emax;
        k.tmax = terms_per_lane(d.G, d.n_na, k.gpl);
        k.nw1 = warpcell_wpc_host(d.G, k.gpl) == 1 ? c.block_warps : 0;
        k.nwarps = warpcell_block_warps_host(d.G, k.gpl, k.nw1);
        k.smem = warpcell_smem(d.G, k.gpl, d.n_reg, d.n_na, k.nw1);
    } else {
        k.smem = k.block.smem;
    }
    return k;
}

// Candidates of a network for a path (AUTO / REGISTER: both families, WARP: lane kernel only).
static std::vector<scrna_tune_choice> candidates(const scrna_net* net, int path) {
    const NetDev& d = net->dev;
    std::vector<scrna_tune_choice> out;
    const bool block_ok = path != SCRNA_PATH_WARP && register_path_holds(d);
    if (block_ok) out.push_back(scrna_tune_choice{0, 0, 0, 0, 0.0});
    if (d.lane_in && path != SCRNA_PATH_BLOCK)
        for (int gpl : {2, 4}) {
            if (gpl == 4 && d.lane_emax > 4) continue;
            if (terms_per_lane(d.G, d.n_na, gpl) > kLaneTerms) continue;
            if (warpcell_wpc_host(d.G, gpl) == 1) {
                for (int nw1 : {2, 4, 8}) out.push_back(scrna_tune_choice{1, gpl, nw1, 0, 0.0});
            } else {
                out.push_back(scrna_tune_choice{1, gpl, 0, 0, 0.0});
            }
        }
    return out;
}

// Measures the candidates on the state buffers of `st` (allocated for `N` cells) with the
// kernel arguments `base` (its tables; state, step range and outputs are set here), on
// `stream`, and returns the fastest; SCRNA_OK with c->found = 0 when there is nothing to
// choose or the arguments lack a table.
static int measure(scrna_ctx* ctx, scrna_net* net, const FusedArgs& base, scrna_state* st, int path,
                   cudaStream_t stream, scrna_tune_choice* best) {
    const auto cands = candidates(net, path);
    *best = scrna_tune_choice{};
    if (cands.size() < 2) return SCRNA_OK;
    if (!base.genes || !base.ginit || !base.quad_tel || !st->M.p || !st->P.p || !st->prom.p || !st->NS.p)
        return SCRNA_OK;
    FusedArgs a = base;
    a.M = st->M.as<float>(); a.P = st->P.as<float>(); a.prom = st->prom.as<uint8_t>(); a.NS = st->NS.as<int2>();
    a.N = st->N;
    a.V = nullptr;
    a.out = nullptr;
    a.counts = nullptr;
    a.eff = nullptr;
    a.first = 1; a.last = 0; a.check = 0; a.epoch = 0;
    const double units_per_step = (double)st->N * net->G;
    const int steps = (int)std::min(512.0, std::max(8.0, 1.0e8 / std::max(units_per_step, 1.0)));
    a.step_begin = 1;
    a.step_end = steps;
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    double best_ms = 1e30;
    int err = SCRNA_OK;
    for (const auto& c : cands) {
        const KernelChoice k = choice_from(net, c);
        a.lane_nw1 = k.nw1;
        auto launch = [&]() {
            return k.warp ? warpcell_launch(a, k.gpl, k.emax, k.tmax, false, stream)
                          : fused_launch(a, k.block, false, stream);
        };
        double ms_min = 1e30;
        for (int rep = 0; rep < 4 && err == SCRNA_OK; ++rep) {
            cudaError_t e = cudaEventRecord(e0, stream);
            if (e == cudaSuccess) e = launch();
            if (e == cudaSuccess) e = cudaEventRecord(e1, stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) { err = fail(SCRNA_ECUDA, "autotune launch: %s", cudaGetErrorString(e)); break; }
            ctx->launches++;
            if (rep > 0) ms_min = std::min(ms_min, (double)ms);  // the first launch warms up
        }
        if (err != SCRNA_OK) break;
        if (ms_min < best_ms) {
            best_ms = ms_min;
            *best = c;
            best->us_per_step = 1e3 * ms_min / steps;
            best->found = 1;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return err;
}

// The last choice of a context (reported by scrna_autotune_last_choice), written under the tuner's
// lock: a server's worker and its caller may choose kernels on one context at once.
static void set_last(scrna_ctx* ctx, const scrna_tune_choice& c) {
    std::lock_guard<std::mutex> lk(g_mu);
    ctx->tune_last = c;
}

constexpr double kTuneMinUnits = 5e8;  // cell-gene-steps of a run worth measuring for (~2.5 ms)

// The register-path kernel of a run: the static choice (choose_kernel), or with autotuning on
// the cached or measured fastest variant for the network's shape.  A measurement runs on
// `st`'s state buffers (state_alloc for N cells) with the kernel arguments `base` (NULL:
// those of fill_fused_args, whose gene tables ensure_gene_tables has uploaded) on `stream`
// (NULL: the context's).
int choose_kernel_tuned(scrna_ctx* ctx, scrna_net* net, const scrna_kinetics* kin, const scrna_cle_opts* o,
                        scrna_state* st, KernelChoice* out, const FusedArgs* base, cudaStream_t stream,
                        bool may_measure) {
    *out = choose_kernel(net, o->path);
    set_last(ctx, scrna_tune_choice{out->warp ? 1 : 0, out->warp ? out->gpl : 0, out->warp ? out->nw1 : 0, 0, 0.0});
    const int path = o->path;
    if (ctx->tune_mode == 0 || (path != SCRNA_PATH_AUTO && path != SCRNA_PATH_REGISTER && path != SCRNA_PATH_WARP))
        return SCRNA_OK;
    const NetDev& d = net->dev;
    const int hill2 = kin->n == 2.0;
    const std::string key = make_key(ctx->tune_arch, d.G, d.lane_in ? d.lane_emax : 0, d.n_na, d.bursty, hill2, st->N) +
                            (path == SCRNA_PATH_WARP ? "|lane" : "");
    scrna_tune_choice c{};
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = ctx->tune_mem.find(key);
        if (it != ctx->tune_mem.end()) c = it->second;
    }
    if (!c.found && !ctx->tune_path.empty())
        if (int r = lookup(ctx->tune_path, key, &c)) return r;
    // A run shorter than kTuneMinUnits takes the static choice and leaves the cache alone: measuring
    // the candidates (and loading their modules on first launch) would cost more than it can save.
    const double run_units = (double)st->N * net->G * (double)n_steps_of(o);
    if (!c.found && ctx->tune_mode == 1 && may_measure && run_units >= kTuneMinUnits) {
        NvtxRange nvtx_range_("scrna_autotune_measure");
        FusedArgs a{};
        if (base) a = *base;
        else fill_fused_args(net, kin, nullptr, nullptr, o, st, &a);
        if (int r = measure(ctx, net, a, st, path, stream ? stream : ctx->stream, &c)) return r;
        if (c.found && !ctx->tune_path.empty()) store(ctx->tune_path, key, c);  // unwritable: keep it in memory
    }
    if (!c.found) return SCRNA_OK;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        ctx->tune_mem[key] = c;
    }
    // a cached choice must still fit this network (a file written for another build is ignored)
    for (const auto& cand : candidates(net, path))
        if (cand.kernel == c.kernel && cand.genes_per_lane == c.genes_per_lane && cand.block_warps == c.block_warps) {
            *out = choice_from(net, c);
            set_last(ctx, c);
            return SCRNA_OK;
        }
    return SCRNA_OK;
}

int tc_choose_slices(scrna_ctx* ctx, int G, int64_t N, bool bursty, int dtype, bool hill2,
                     const std::function<int(int, double*)>& measure, int* S, bool* measured) {
    *S = 7;
    *measured = false;
    set_last(ctx, scrna_tune_choice{2, 224, 0, 0, 0.0});
    if (ctx->tune_mode == 0) return SCRNA_OK;
    char buf[160];
    std::snprintf(buf, sizeof buf, "%s|tc|G%d|d%d|b%d|h%d|N%d", ctx->tune_arch, G, dtype, bursty ? 1 : 0,
                  hill2 ? 1 : 0, floor_log2(std::max<int64_t>(N, 1)));
    const std::string key = buf;
    scrna_tune_choice c{};
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = ctx->tune_mem.find(key);
        if (it != ctx->tune_mem.end()) c = it->second;
    }
    if (!c.found && !ctx->tune_path.empty())
        if (int r = lookup(ctx->tune_path, key, &c)) return r;
    if (!c.found && ctx->tune_mode == 1) {
        double best = 1e30;
        for (int s : {5, 6, 7}) {
            double us = 0;
            if (int r = measure(s, &us)) return r;
            *measured = true;
            if (us < best) { best = us; c = scrna_tune_choice{2, 32 * s, 0, 1, us}; }
        }
        if (c.found && !ctx->tune_path.empty()) store(ctx->tune_path, key, c);
    }
    if (!c.found || c.kernel != 2 || (c.genes_per_lane != 160 && c.genes_per_lane != 192 && c.genes_per_lane != 224))
        return SCRNA_OK;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        ctx->tune_mem[key] = c;
    }
    *S = c.genes_per_lane / 32;
    set_last(ctx, c);
    return SCRNA_OK;
}

}  // namespace scrna

using namespace scrna;

extern "C" int scrna_ctx_set_autotune(scrna_ctx* ctx, int32_t mode, const char* cache_path) {
    if (!ctx) return fail(SCRNA_EINVAL, "context is NULL");
    if (mode < 0 || mode > 2) return fail(SCRNA_EINVAL, "autotune mode must be 0 (off), 1 (on) or 2 (cache only)");
    ctx->tune_mode = mode;
    if (cache_path) ctx->tune_path = cache_path;
    std::lock_guard<std::mutex> lk(g_mu);
    ctx->tune_mem.clear();
    return SCRNA_OK;
}

extern "C" int scrna_autotune_last_choice(const scrna_ctx* ctx, scrna_tune_choice* out) {
    if (!ctx || !out) return fail(SCRNA_EINVAL, "NULL argument");
    {
        std::lock_guard<std::mutex> lk(g_mu);
        *out = ctx->tune_last;
    }
    return SCRNA_OK;
}

extern "C" int scrna_autotune_key(const char* device, int32_t G, int32_t in_edges, int32_t n_terms, int32_t bursty,
                                  int32_t hill2, int64_t cell_num, char* out, int32_t out_len) {
    if (!device || !out || out_len <= 0 || G <= 0) return fail(SCRNA_EINVAL, "bad autotune key arguments");
    const std::string k = make_key(device, G, in_edges, n_terms, bursty, hill2, cell_num);
    if ((int)k.size() + 1 > out_len) return fail(SCRNA_EINVAL, "key buffer too small");
    std::memcpy(out, k.c_str(), k.size() + 1);
    return SCRNA_OK;
}

extern "C" int scrna_autotune_cache_lookup(const char* path, const char* key, scrna_tune_choice* out) {
    if (!path || !key || !out) return fail(SCRNA_EINVAL, "NULL argument");
    return lookup(path, key, out);
}

extern "C" int scrna_autotune_cache_store(const char* path, const char* key, const scrna_tune_choice* c) {
    if (!path || !key || !c) return fail(SCRNA_EINVAL, "NULL argument");
    if (c->kernel < 0 || c->kernel > 2)
        return fail(SCRNA_EINVAL, "kernel must be 0 (block tiles), 1 (lane) or 2 (tensor-core step)");
    return store(path, key, *c);
}
