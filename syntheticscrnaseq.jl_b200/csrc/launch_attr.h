// The dynamic shared-memory limit of a kernel, raised and never lowered.
//
// cudaFuncAttributeMaxDynamicSharedMemorySize belongs to the kernel in the device's context,
// which every context of this library on that device shares (the runtime's primary context).
// A launch that set the limit to its own size could lower it just before another thread
// launches the same kernel with a larger size (a server worker beside a user's call, two
// contexts on one GPU), and that launch would fail.  Raising it to the largest size asked
// for so far, under a lock, keeps every launch within the limit; the limit does not change
// the shared memory a launch actually gets.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

namespace scrna {

inline cudaError_t ensure_dynamic_smem(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> raised;  // (kernel, device) -> limit set
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = raised[{kernel, dev}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

}  // namespace scrna
