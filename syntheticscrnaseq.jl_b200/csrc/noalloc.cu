// Scratch-free CLE entry point: scrna_cle_simulate_noalloc.
//
// Some callers cannot allocate device memory at the moment they want a
// simulation: code that runs while another component owns the allocator (a
// framework's caching allocator or a fixed memory pool that forbids cudaMalloc),
// code inside a latency-critical serving loop where cudaMalloc/cudaFree would
// synchronise the device, or host programs embedding the library under a strict
// device-memory budget decided at start-up.  This entry point runs the block-tile
// FP32 register kernel of scrna_cle_run_device but takes all of its working memory
// from one file-scope device array.  The caller passes the network (created
// earlier) and device pointers for the outputs.
//
// The array belongs to this file's device-code module.  Under CUDA's default lazy
// module loading that module, and the array's memory with it, is loaded onto a
// device by the first call on that device (the call looks up the array's device
// address), so the first call per device maps the array and may synchronise the
// device; later calls allocate nothing.  Callers make that first call during their
// set-up, before the point from which they cannot allocate.
//
// Limits: at most kMaxCells cells, kMaxGenes genes and kMaxCellGenes cell-genes
// per call.  The array (kScratchBytes, about 16.0 MB) stays on every device it was
// loaded on until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/scrna_cle.h"
#include "cle_internal.h"

namespace scrna {
FusedLaunch fused_plan(int G, int n_reg, int n_in, int n_na, int n_na_src, int n_quads);
int fused_max_quads();
cudaError_t fused_launch(const FusedArgs& a, const FusedLaunch& L, bool pop, cudaStream_t st);
int set_error(int code, const char* msg);
int check_run_args(const scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                   const scrna_capture* cap, const scrna_cle_opts* o);
int64_t run_steps(const scrna_cle_opts* o);
cudaStream_t ctx_stream(scrna_ctx* ctx);
int ctx_device(scrna_ctx* ctx);
void ctx_add_launches(scrna_ctx* ctx, int n);
const NetDev& net_dev(const scrna_net* n);
void gene_tables_host(const scrna_net* n, const scrna_kinetics* kin, double dt, GeneRec* gr,
                      GeneInit* gi, uint8_t* qt);
}  // namespace scrna

using namespace scrna;

namespace {

constexpr int64_t kMaxCells = 1 << 16;       // 65,536 cells
constexpr int32_t kMaxGenes = 512;
constexpr int64_t kMaxCellGenes = 1 << 18;   // 262,144 cell-genes

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Fixed layout of the scratch array (offsets for the maximum sizes).
constexpr size_t kOffM = 0;
constexpr size_t kOffP = kOffM + align256(4 * kMaxCellGenes);
constexpr size_t kOffProm = kOffP + align256(4 * kMaxCellGenes);
constexpr size_t kOffNS = kOffProm + align256(kMaxCellGenes);
constexpr size_t kOffV = kOffNS + align256(8 * kMaxCellGenes);
constexpr size_t kOffDM = kOffV + align256(8 * kMaxCells);            // two parities each below
constexpr size_t kOffDP = kOffDM + 2 * align256(4 * kMaxCellGenes);
constexpr size_t kOffDProm = kOffDP + 2 * align256(4 * kMaxCellGenes);
constexpr size_t kOffDNS = kOffDProm + 2 * align256(kMaxCellGenes);
constexpr size_t kOffDV = kOffDNS + 2 * align256(8 * kMaxCellGenes);
constexpr size_t kOffOwner = kOffDV + 2 * align256(8 * kMaxCells);
constexpr size_t kOffGenes = kOffOwner + 2 * align256(8 * kMaxCells);
constexpr size_t kOffGinit = kOffGenes + align256(sizeof(GeneRec) * kMaxGenes);
constexpr size_t kOffQuad = kOffGinit + align256(sizeof(GeneInit) * kMaxGenes);
constexpr size_t kScratchBytes = kOffQuad + align256(kMaxGenes / 4);

// The working memory of every call on this device.  Host code must not take
// its address directly (that is a host-side stand-in); it uses the address
// returned by cudaGetSymbolAddress for the current device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Once per device, with that device current: look up the device address of the array.
int scratch_for_device(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return set_error(SCRNA_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            char msg[256];
            snprintf(msg, sizeof msg, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
            return set_error(SCRNA_ECUDA, msg);
        }
        g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[dev];
    return SCRNA_OK;
}

// Host staging for the per-run gene tables (fixed size, no allocation), laid out as
// the tables sit in the scratch array from kOffGenes on.
constexpr size_t kTablesBytes = kScratchBytes - kOffGenes;
alignas(16) thread_local unsigned char t_tables[kTablesBytes];

// The tables reach the device as the by-value parameter of a small copy kernel, one
// chunk per launch: the launch copies its parameters, so no host memory is read later
// and no copy engine call is made.
constexpr uint32_t kStageChunk = 3968;
struct StageChunk {
    uint32_t offset;  // from kOffGenes
    uint32_t bytes;
    unsigned char data[kStageChunk];
};

__global__ void noalloc_stage_kernel(unsigned char* dst, const StageChunk c) {
    for (uint32_t i = threadIdx.x; i < c.bytes; i += blockDim.x) dst[c.offset + i] = c.data[i];
}

int cuda_fail(const char* what, cudaError_t e) {
    char msg[256];
    snprintf(msg, sizeof msg, "%s failed: %s", what, cudaGetErrorString(e));
    return set_error(SCRNA_ECUDA, msg);
}

// Restores the caller's current device when the call returns.
struct DeviceGuard {
    int prev = -1;
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

}  // namespace

extern "C" int scrna_cle_simulate_noalloc(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                                          const scrna_population* pop, const scrna_capture* cap,
                                          const scrna_cle_opts* o, double* d_out, int32_t* d_counts,
                                          double* d_eff) {
    if (!ctx) return set_error(SCRNA_EINVAL, "context is NULL");
    if (int r = check_run_args(net, kin, pop, cap, o)) return r;
    if (!d_out) return set_error(SCRNA_EINVAL, "d_out is NULL");
    if (cap && (!d_counts || !d_eff)) return set_error(SCRNA_EINVAL, "capture needs d_counts and d_eff");
    if (o->precision != SCRNA_PRECISION_FP32)
        return set_error(SCRNA_ENOTSUP, "the scratch-free entry point runs the FP32 path only");
    if (o->path != SCRNA_PATH_AUTO && o->path != SCRNA_PATH_REGISTER && o->path != SCRNA_PATH_BLOCK)
        return set_error(SCRNA_ENOTSUP, "the scratch-free entry point runs the block-tile register kernel only");
    const NetDev& d = net_dev(net);
    const int64_t N = pop ? pop->cell_num : o->cell_num;
    if (N <= 0) return set_error(SCRNA_EINVAL, "cell_num must be positive");
    if (N > kMaxCells || d.G > kMaxGenes || (int64_t)d.G * N > kMaxCellGenes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "scratch-free run too large: %lld cells x %d genes (limits: %lld cells, %d genes, %lld cell-genes)",
                 (long long)N, d.G, (long long)kMaxCells, kMaxGenes, (long long)kMaxCellGenes);
        return set_error(SCRNA_EINVAL, msg);
    }
    if (d.n_quads > fused_max_quads()) return set_error(SCRNA_ENOTSUP, "network too large for the register path");
    if (o->cell_offset < 0 || o->cell_offset + N > (1ll << 32)) return set_error(SCRNA_EINVAL, "cell indices must fit 32 bits");
    const int64_t n_steps = run_steps(o);
    if (n_steps >= (1ll << 31)) return set_error(SCRNA_EINVAL, "too many steps");

    DeviceGuard guard;
    cudaError_t e = cudaGetDevice(&guard.prev);
    if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
    if ((e = cudaSetDevice(ctx_device(ctx))) != cudaSuccess) return cuda_fail("cudaSetDevice", e);
    unsigned char* s = nullptr;
    if (int r = scratch_for_device(ctx_device(ctx), &s)) return r;
    cudaStream_t st = ctx_stream(ctx);

    GeneRec* genes = reinterpret_cast<GeneRec*>(t_tables);
    GeneInit* ginit = reinterpret_cast<GeneInit*>(t_tables + (kOffGinit - kOffGenes));
    uint8_t* quad = t_tables + (kOffQuad - kOffGenes);
    gene_tables_host(net, kin, o->dt, genes, ginit, quad);
    const int nq = (d.G + 3) / 4;
    const size_t ranges[3][2] = {{0, sizeof(GeneRec) * d.G},
                                 {kOffGinit - kOffGenes, sizeof(GeneInit) * d.G},
                                 {kOffQuad - kOffGenes, (size_t)nq}};
    for (const auto& r : ranges)
        for (size_t off = r[0]; off < r[0] + r[1]; off += kStageChunk) {
            StageChunk c;
            c.offset = (uint32_t)off;
            c.bytes = (uint32_t)std::min<size_t>(kStageChunk, r[0] + r[1] - off);
            std::memcpy(c.data, t_tables + off, c.bytes);
            noalloc_stage_kernel<<<1, 256, 0, st>>>(s + kOffGenes, c);
            if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail("table staging launch", e);
            ctx_add_launches(ctx, 1);
        }

    FusedArgs a{};
    a.G = d.G; a.n_quads = d.n_quads; a.n_reg = d.n_reg; a.n_in = d.n_in; a.n_na = d.n_na; a.n_na_src = d.n_na_src;
    a.N = N;
    a.cell_offset = o->cell_offset;
    a.k_t = (float)kin->k_t;
    a.Kn = (float)std::pow(kin->K_d, kin->n);
    a.hill_n = (float)kin->n;
    a.hill_int = (kin->n == std::floor(kin->n) && kin->n >= 1.0 && kin->n <= 16.0) ? (int)kin->n : 0;
    a.mu_m = (float)(pop ? kin->mu_m : kin->mu_m + kin->dilution);
    a.mu_p = (float)(pop ? kin->mu_p : kin->mu_p + kin->dilution);
    a.dt = (float)o->dt;
    a.key0 = (uint32_t)o->seed; a.key1 = (uint32_t)(o->seed >> 32); a.stream = o->stream & 0xFFFFFFu;
    a.genes = reinterpret_cast<const GeneRec*>(s + kOffGenes);
    a.ginit = reinterpret_cast<const GeneInit*>(s + kOffGinit);
    a.in_edge = d.in_edge; a.na = d.na; a.na_src = d.na_src;
    a.quad_tel = s + kOffQuad;
    a.M = reinterpret_cast<float*>(s + kOffM);
    a.P = reinterpret_cast<float*>(s + kOffP);
    a.prom = s + kOffProm;
    a.NS = reinterpret_cast<int2*>(s + kOffNS);
    if (pop) {
        a.growth_factor = std::exp(pop->growth_rate * o->dt);
        a.V_div = pop->V_div; a.V_lo = pop->V_init_lo; a.V_hi = pop->V_init_hi;
        a.partition = pop->partition; a.exclude_mother = pop->exclude_mother ? 1 : 0;
        a.V = reinterpret_cast<double*>(s + kOffV);
        for (int k = 0; k < 2; ++k) {
            a.dM[k] = reinterpret_cast<float*>(s + kOffDM + k * align256(4 * kMaxCellGenes));
            a.dP[k] = reinterpret_cast<float*>(s + kOffDP + k * align256(4 * kMaxCellGenes));
            a.dprom[k] = s + kOffDProm + k * align256(kMaxCellGenes);
            a.dNS[k] = reinterpret_cast<int2*>(s + kOffDNS + k * align256(8 * kMaxCellGenes));
            a.dV[k] = reinterpret_cast<double*>(s + kOffDV + k * align256(8 * kMaxCells));
            a.owner[k] = reinterpret_cast<unsigned long long*>(s + kOffOwner + k * align256(8 * kMaxCells));
        }
        // The array keeps the previous call's contents: the Moran slot owners must start at zero.
        if ((e = cudaMemsetAsync(s + kOffOwner, 0, 2 * align256(8 * kMaxCells), st)) != cudaSuccess)
            return cuda_fail("cudaMemsetAsync(owner)", e);
    }
    a.out = d_out;
    a.readout = o->readout;
    if (cap) {
        a.counts = d_counts;
        a.eff = d_eff;
        a.capture_species = cap->readout == SCRNA_READOUT_MRNA ? 0 : 1;
        a.cap_mu_log = std::log(cap->efficiency) - (cap->mean_correction ? cap->efficiency_std * cap->efficiency_std / 2.0 : 0.0);
        a.cap_sigma = cap->efficiency_std;
    }
    const FusedLaunch L = fused_plan(d.G, d.n_reg, d.n_in, d.n_na, d.n_na_src, d.n_quads);
    if (L.smem > 227 * 1024) return set_error(SCRNA_ENOTSUP, "network tables exceed shared memory");

    if (!pop) {
        a.step_begin = 1; a.step_end = (int)n_steps; a.first = 1; a.last = 1; a.check = 0; a.epoch = 0;
        if ((e = fused_launch(a, L, false, st)) != cudaSuccess) return cuda_fail("fused kernel launch", e);
        ctx_add_launches(ctx, 1);
        return SCRNA_OK;
    }
    const int64_t I = pop->div_check_interval;
    int64_t s0 = 1;
    int epoch = 0;
    bool first = true;
    while (true) {
        int64_t s1 = n_steps == 0 ? 0 : std::min(n_steps, ((s0 - 1) / I + 1) * I);
        const bool check = s1 >= s0 && (s1 % I == 0);
        const bool final_chunk = s1 >= n_steps;
        a.step_begin = (int)s0; a.step_end = (int)s1;
        a.first = first ? 1 : 0; a.epoch = epoch; a.check = check ? 1 : 0;
        a.last = (final_chunk && !check) ? 1 : 0;
        if ((e = fused_launch(a, L, true, st)) != cudaSuccess) return cuda_fail("fused kernel launch", e);
        ctx_add_launches(ctx, 1);
        first = false;
        if (check) epoch += 1;
        if (final_chunk) {
            if (check) {
                a.step_begin = (int)s1 + 1; a.step_end = (int)s1;
                a.first = 0; a.epoch = epoch; a.check = 0; a.last = 1;
                if ((e = fused_launch(a, L, true, st)) != cudaSuccess) return cuda_fail("fused kernel launch", e);
                ctx_add_launches(ctx, 1);
            }
            break;
        }
        s0 = s1 + 1;
    }
    return SCRNA_OK;
}
