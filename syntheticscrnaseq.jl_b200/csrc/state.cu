// Continuation and checkpoints of register-path runs.
//
// A run is a pure function of its inputs and of the counter-based increments keyed by
// (seed, stream, cell, step, gene), and its state between launches is exact (FP32 counts,
// FP64 volumes, promoter bits, switching times), so a run of T1 steps continued to T2
// equals one run of T2 steps bit for bit.  scrna_cle_resume / scrna_tauleap_resume continue
// the run a state holds; scrna_state_checkpoint / scrna_state_restore move that state
// through host memory (another process, or a later job), in a fixed little-endian format
// with the arrays gene-major [G][N] whatever the layout of the kernel that wrote them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "capi_internal.h"
#include "nvtx_range.h"

namespace scrna {
namespace {

// out[c * G + g] = in[g * N + c] (to cell-major) or out[g * N + c] = in[c * G + g].
template <class T>
__global__ void relayout_kernel(const T* in, T* out, int G, int64_t N, int to_cell_major) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)G * N) return;
    if (to_cell_major) {  // k = g * N + c: coalesced reads
        const int64_t g = k / N, c = k - g * N;
        out[c * G + g] = in[k];
    } else {  // k = c * G + g: coalesced reads
        const int64_t c = k / G, g = k - c * G;
        out[g * N + c] = in[k];
    }
}

template <class T>
int relayout(scrna_ctx* ctx, DevBuf& buf, int G, int64_t N, bool to_cell_major) {
    const size_t bytes = (size_t)G * N * sizeof(T);
    DevBuf tmp;
    CU(tmp.ensure(bytes));
    CU(cudaMemcpyAsync(tmp.p, buf.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    const int64_t n = (int64_t)G * N;
    relayout_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(tmp.as<T>(), buf.as<T>(), G, N,
                                                                             to_cell_major ? 1 : 0);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(ctx->stream));  // tmp goes out of scope
    ctx->launches++;
    return SCRNA_OK;
}

struct CheckpointHeader {
    char magic[8];       // "SCRNACK1"
    int32_t G;
    int32_t flags;       // bit 0 population, bit 1 tau-leap
    int64_t N;
    int64_t steps_done;
    int32_t epoch;
    int32_t reserved;
};
static_assert(sizeof(CheckpointHeader) == 40, "checkpoint header layout");

size_t checkpoint_bytes(int G, int64_t N, bool pop) {
    const size_t gn = (size_t)G * N;
    return sizeof(CheckpointHeader) + gn * (4 + 4 + 1 + 8) + (pop ? (size_t)N * 8 : 0);
}

}  // namespace

int state_relayout(scrna_ctx* ctx, scrna_state* st, bool to_cell_major) {
    if (st->last_cell_major == to_cell_major) return SCRNA_OK;
    if (int r = relayout<float>(ctx, st->M, st->G, st->N, to_cell_major)) return r;
    if (int r = relayout<float>(ctx, st->P, st->G, st->N, to_cell_major)) return r;
    if (int r = relayout<uint8_t>(ctx, st->prom, st->G, st->N, to_cell_major)) return r;
    if (int r = relayout<int2>(ctx, st->NS, st->G, st->N, to_cell_major)) return r;
    st->last_cell_major = to_cell_major;
    return SCRNA_OK;
}

}  // namespace scrna

using namespace scrna;

extern "C" int scrna_cle_resume(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                                const scrna_population* pop, const scrna_capture* cap, const scrna_cle_opts* opts,
                                scrna_state* st) {
    NvtxRange nvtx_range_("scrna_cle_resume");
    if (!ctx || !net || !st) return fail(SCRNA_EINVAL, "NULL argument");
    return resume_register_run(ctx, const_cast<scrna_net*>(net), kin, pop, cap, opts, st, false);
}

extern "C" int scrna_tauleap_resume(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                                    const scrna_population* pop, const scrna_capture* cap, const scrna_cle_opts* opts,
                                    scrna_state* st) {
    NvtxRange nvtx_range_("scrna_tauleap_resume");
    if (!ctx || !net || !st) return fail(SCRNA_EINVAL, "NULL argument");
    return resume_register_run(ctx, const_cast<scrna_net*>(net), kin, pop, cap, opts, st, true);
}

extern "C" int scrna_state_steps_done(const scrna_state* st, int64_t* steps) {
    if (!st || !steps) return fail(SCRNA_EINVAL, "NULL argument");
    *steps = st->has_register_state ? st->steps_done : 0;
    return SCRNA_OK;
}

extern "C" int scrna_state_checkpoint(scrna_ctx* ctx, scrna_state* st, void* buf, size_t capacity, size_t* bytes) {
    NvtxRange nvtx_range_("scrna_state_checkpoint");
    if (!ctx || !st || !bytes) return fail(SCRNA_EINVAL, "NULL argument");
    if (!st->has_register_state) return fail(SCRNA_EINVAL, "the state holds no register-path run");
    const size_t need = checkpoint_bytes(st->G, st->N, st->last_pop);
    *bytes = need;
    if (!buf) return SCRNA_OK;
    if (capacity < need) return fail(SCRNA_EINVAL, "checkpoint needs %zu bytes, the buffer has %zu", need, capacity);
    if (int r = set_device(ctx)) return r;
    if (int r = state_relayout(ctx, st, false)) return r;  // gene-major in the file
    CheckpointHeader h{};
    std::memcpy(h.magic, "SCRNACK1", 8);
    h.G = st->G;
    h.flags = (st->last_pop ? 1 : 0) | (st->last_tau ? 2 : 0);
    h.N = st->N;
    h.steps_done = st->steps_done;
    h.epoch = st->epoch;
    unsigned char* p = static_cast<unsigned char*>(buf);
    std::memcpy(p, &h, sizeof h);
    p += sizeof h;
    const size_t gn = (size_t)st->G * st->N;
    CU(cudaMemcpyAsync(p, st->M.p, gn * 4, cudaMemcpyDeviceToHost, ctx->stream)); p += gn * 4;
    CU(cudaMemcpyAsync(p, st->P.p, gn * 4, cudaMemcpyDeviceToHost, ctx->stream)); p += gn * 4;
    CU(cudaMemcpyAsync(p, st->prom.p, gn, cudaMemcpyDeviceToHost, ctx->stream)); p += gn;
    CU(cudaMemcpyAsync(p, st->NS.p, gn * 8, cudaMemcpyDeviceToHost, ctx->stream)); p += gn * 8;
    if (st->last_pop) CU(cudaMemcpyAsync(p, st->V.p, (size_t)st->N * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->d2h_bytes += (int64_t)(need - sizeof h);
    return SCRNA_OK;
}

extern "C" int scrna_state_restore(scrna_ctx* ctx, scrna_state* st, const void* buf, size_t bytes) {
    NvtxRange nvtx_range_("scrna_state_restore");
    if (!ctx || !st || !buf) return fail(SCRNA_EINVAL, "NULL argument");
    if (bytes < sizeof(CheckpointHeader)) return fail(SCRNA_EINVAL, "not a checkpoint (too short)");
    CheckpointHeader h;
    std::memcpy(&h, buf, sizeof h);
    if (std::memcmp(h.magic, "SCRNACK1", 8) != 0) return fail(SCRNA_EINVAL, "not a checkpoint of this library");
    if (h.G != st->G || h.N != st->N)
        return fail(SCRNA_EINVAL, "checkpoint of %d genes x %lld cells, state of %d x %lld", h.G, (long long)h.N,
                    st->G, (long long)st->N);
    const bool pop = (h.flags & 1) != 0;
    if (bytes != checkpoint_bytes(h.G, h.N, pop) || h.steps_done < 0 || h.epoch < 0)
        return fail(SCRNA_EINVAL, "damaged checkpoint");
    if (int r = set_device(ctx)) return r;
    if (int r = state_alloc(st, pop, false)) return r;
    const unsigned char* p = static_cast<const unsigned char*>(buf) + sizeof h;
    const size_t gn = (size_t)st->G * st->N;
    CU(cudaMemcpyAsync(st->M.p, p, gn * 4, cudaMemcpyHostToDevice, ctx->stream)); p += gn * 4;
    CU(cudaMemcpyAsync(st->P.p, p, gn * 4, cudaMemcpyHostToDevice, ctx->stream)); p += gn * 4;
    CU(cudaMemcpyAsync(st->prom.p, p, gn, cudaMemcpyHostToDevice, ctx->stream)); p += gn;
    CU(cudaMemcpyAsync(st->NS.p, p, gn * 8, cudaMemcpyHostToDevice, ctx->stream)); p += gn * 8;
    if (pop) CU(cudaMemcpyAsync(st->V.p, p, (size_t)st->N * 8, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->h2d_bytes += (int64_t)(bytes - sizeof h);
    st->last_cell_major = false;
    st->last_tensor = false;
    st->last_plain = false;
    st->last_pop = pop;
    st->last_tau = (h.flags & 2) != 0;
    st->steps_done = h.steps_done;
    st->epoch = h.epoch;
    st->has_register_state = true;
    st->have_counts = false;
    return SCRNA_OK;
}
