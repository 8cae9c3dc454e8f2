// Per-device, thread-safe one-time set-up of a kernel (its dynamic
// shared-memory limit, its occupancy) before the first launch on a device.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <utility>

namespace marl {

constexpr int kSetupDevices = 64;

// `slots` is one kernel's per-device record (static storage, so zero at
// start): 0 = not set up on that device, otherwise the set-up's result + 1.
// `setup(&value)` runs on the current device until it succeeds once; its int
// result (for example resident blocks per SM) is kept and returned in *value
// by later calls.  When two host threads make their first launches on one
// device at the same time, both may run `setup`; it only sets attributes and
// queries occupancy, so running it twice is harmless, and no thread launches
// before its own set-up (or an earlier completed one) has finished.
template <class F>
cudaError_t setup_once(std::atomic<int>* slots, int* value, F setup) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kSetupDevices) return setup(value);  // no record kept
    const int v = slots[dev].load(std::memory_order_acquire);
    if (v > 0) {
        *value = v - 1;
        return cudaSuccess;
    }
    int got = 0;
    e = setup(&got);
    if (e != cudaSuccess) return e;
    slots[dev].store(got + 1, std::memory_order_release);
    *value = got;
    return cudaSuccess;
}

// The common case: raise the dynamic shared-memory limit of `kernel` to
// `bytes` once per device.
template <class K>
cudaError_t set_smem_once(std::atomic<int>* slots, K kernel, int bytes) {
    int unused = 0;
    return setup_once(slots, &unused, [&](int* v) {
        *v = 0;
        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    });
}

// Launch with programmatic stream serialization: the kernel may be scheduled
// while the previous kernel of the stream drains, so it must call
// griddep_wait (common.cuh) before it touches global memory that an earlier
// launch writes or reads.
template <class... KArgs, class... Args>
cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                             Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace marl
