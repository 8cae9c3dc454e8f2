// marl_diffuse_device_noalloc: the device-pointer diffusion tick with its
// scratch memory held in a fixed, file-scope device array instead of being
// allocated per call.
//
// Who needs it: callers that must not allocate device memory while they run.
// Examples are code whose device memory belongs to another allocator (a
// framework's caching allocator or a fixed pool it may not grow), and
// latency-critical loops where a cudaMalloc/cudaFree, and the device-wide
// synchronisation it can imply, is not acceptable.  marl_diffuse_device
// allocates a pitched occupancy mask and an error word on every call; this
// variant allocates nothing.
//
// Scratch: one array, g_noalloc_scratch, holding (1) the ping-pong copy of the
// field, (2) the occupancy mask with rows padded to 16 bytes (the TMA stride
// rule), (3) the error word.  Limits: at most kNoAllocMaxVoxels voxels, and
// Y * Z * (X rounded up to 16) <= kNoAllocMaskBytes.  Every GPU that loads the
// library holds the array (about 13 MiB) until the process exits.
//
// Host code cannot use the array's name as a device address (it is a host-side
// stand-in).  Every call looks the address up with cudaGetSymbolAddress, with
// the caller's device current, before it launches anything: the lookup is
// cheap and allocates nothing, and a cached address would go stale if the
// application reset the device (the module, and with it the array, is then
// loaded again at a new address).  The first call on a device also loads the
// module, which reserves the array; that first call should come before any
// stream capture.  All calls share the array and it keeps the last call's
// contents: the mask is rewritten and the error word cleared at the start of
// every call, and the scratch field is fully written by the first substep
// before it is read.  Calls that overlap on the GPU (for example on two
// streams at once) race on the array and must not be issued.
#include <cuda_runtime.h>

#include "../../include/marl_cuda.h"
#include "common.cuh"
#include "internal.h"

namespace marl {
marl_status fail(marl_status st, const char* fmt, ...);
marl_status cuda_fail(cudaError_t e, const char* where);
void derive_consts(const marl_sim_params& p, FieldConsts* fk, CellConsts* ck);
marl_status check_device(int* dev, int* sms);
}  // namespace marl

namespace {

constexpr size_t kNoAllocMaxVoxels = size_t(1) << 18;              // 262,144 voxels (e.g. 64 x 64 x 64)
constexpr size_t kNoAllocFieldBytes = kNoAllocMaxVoxels * 48;      // 12 MiB
constexpr size_t kNoAllocMaskBytes = kNoAllocMaxVoxels * 4;        // 1 MiB
constexpr size_t kNoAllocBytes = kNoAllocFieldBytes + kNoAllocMaskBytes + 256;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of the scratch array on the current device.
marl_status scratch_for_current_device(unsigned char** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return marl::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    *out = static_cast<unsigned char*>(p);
    return MARL_OK;
}

}  // namespace

extern "C" marl_status marl_diffuse_device_noalloc(float* field_dev, const uint8_t* occupancy_dev, int32_t gx,
                                                   int32_t gy, int32_t gz, const marl_sim_params* sim,
                                                   uint32_t substeps, void* cuda_stream) {
    using namespace marl;
    if (!field_dev || !occupancy_dev || !sim) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (gx < 1 || gy < 1 || gz < 1 || gx > kMaxXY || gy > kMaxXY || gz > kMaxZ)
        return fail(MARL_ERR_INVALID_INPUT, "grid %dx%dx%d outside 1..%d x 1..%d x 1..%d", gx, gy, gz, kMaxXY,
                    kMaxXY, kMaxZ);
    const Grid g{gx, gy, gz};
    const size_t mask_bytes = (size_t)gz * gy * mask_pitch(gx);
    if (g.V() > kNoAllocMaxVoxels || mask_bytes > kNoAllocMaskBytes)
        return fail(MARL_ERR_INVALID_INPUT,
                    "grid %dx%dx%d exceeds the allocation-free scratch (at most %zu voxels and %zu padded mask bytes)",
                    gx, gy, gz, kNoAllocMaxVoxels, kNoAllocMaskBytes);
    if ((uintptr_t)field_dev & 15) return fail(MARL_ERR_INVALID_INPUT, "field must be 16-byte aligned");
    if (substeps == 0) return MARL_OK;
    if (sim->diffusion_substeps == 0) return fail(MARL_ERR_INVALID_INPUT, "sim.diffusion_substeps == 0");

    int dev = 0, sms = 0;
    marl_status st = check_device(&dev, &sms);  // MARL_ERR_NO_DEVICE without an sm_100 device
    if (st) return st;
    unsigned char* base = nullptr;
    if ((st = scratch_for_current_device(&base))) return st;
    float* scratch = reinterpret_cast<float*>(base);
    uint8_t* mask = base + kNoAllocFieldBytes;
    uint32_t* err = reinterpret_cast<uint32_t*>(base + kNoAllocFieldBytes + kNoAllocMaskBytes);

    cudaStream_t s = (cudaStream_t)cuda_stream;
    FieldConsts fk;
    CellConsts ck;
    derive_consts(*sim, &fk, &ck);
    cudaError_t e = cudaMemsetAsync(err, 0, 4, s);
    if (e != cudaSuccess) return cuda_fail(e, "clear error word");
    if ((e = launch_repack_mask(occupancy_dev, mask, g, s)) != cudaSuccess) return cuda_fail(e, "repack occupancy");
    DiffusionPlan plan;
    if (!plan_diffusion(&plan, field_dev, scratch, mask, g, 0, 16))
        return fail(MARL_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    int cur = 0;  // 0: field_dev holds the live state, 1: the scratch copy does
    for (uint32_t i = 0; i < substeps; ++i) {
        if ((e = launch_diffuse(plan, cur, g, fk, 0, nullptr, err, s)) != cudaSuccess)
            return cuda_fail(e, "diffusion substep");
        cur ^= 1;
    }
    if (cur != 0 && (e = cudaMemcpyAsync(field_dev, scratch, g.V() * 48, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
        return cuda_fail(e, "copy result");
    uint32_t h_err = 0;
    if ((e = cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_fail(e, "read error word");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "synchronize");
    if (h_err) return fail(MARL_ERR_TIMEOUT, "device wait gave up (error bits 0x%x)", h_err);
    return MARL_OK;
}
