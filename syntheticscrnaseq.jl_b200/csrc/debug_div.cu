// Exhaustive check of the branch-free quotient of the Poisson inverse CDF (small_div.cuh)
// against IEEE division: every float lam with bit pattern in [lo, hi), every k = 1..50.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/scrna_cle.h"
#include "capi_internal.h"
#include "small_div.cuh"

namespace scrna {
namespace {

__global__ void small_div_check_kernel(uint32_t lo, uint32_t hi, unsigned long long* mismatches,
                                       unsigned long long* first_bad) {
    const uint64_t n = (uint64_t)(hi - lo);
    unsigned long long bad = 0;
    unsigned long long first = ~0ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t bits = lo + (uint32_t)i;
        const float lam = __uint_as_float(bits);
        if (!small_div_ok(lam)) continue;
        for (int k = 1; k <= 50; ++k) {
            const float kf = (float)k;
            const float q = small_div(lam, kf, kRecipSmall[k]);
            const float ref = __fdiv_rn(lam, kf);
            if (__float_as_uint(q) != __float_as_uint(ref)) {
                ++bad;
                const unsigned long long key = ((unsigned long long)bits << 8) | (unsigned long long)k;
                first = key < first ? key : first;
            }
        }
    }
    if (bad) {
        atomicAdd(mismatches, bad);
        atomicMin(first_bad, first);
    }
}

}  // namespace
}  // namespace scrna

using namespace scrna;

extern "C" int scrna_debug_small_div_check(scrna_ctx* ctx, uint32_t lo, uint32_t hi, int64_t* mismatches,
                                           uint32_t* first_bad_lam, int32_t* first_bad_k) {
    if (!ctx) return fail(SCRNA_EINVAL, "context is NULL");
    if (!mismatches || hi < lo) return fail(SCRNA_EINVAL, "bad arguments");
    if (int r = set_device(ctx)) return r;
    DevBuf d;
    CU(d.ensure(16));
    unsigned long long init[2] = {0ull, ~0ull};
    CU(cudaMemcpyAsync(d.p, init, 16, cudaMemcpyHostToDevice, ctx->stream));
    int dev = 0, sms = 148;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    unsigned long long* p = d.as<unsigned long long>();
    small_div_check_kernel<<<sms * 8, 256, 0, ctx->stream>>>(lo, hi, p, p + 1);
    CU(cudaGetLastError());
    ctx->launches++;
    unsigned long long out[2];
    CU(cudaMemcpyAsync(out, d.p, 16, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    *mismatches = (int64_t)out[0];
    if (first_bad_lam) *first_bad_lam = out[0] ? (uint32_t)(out[1] >> 8) : 0u;
    if (first_bad_k) *first_bad_k = out[0] ? (int32_t)(out[1] & 0xFF) : 0;
    return SCRNA_OK;
}
