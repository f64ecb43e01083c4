// max |u|, |v|, |v| a of a caller-owned streamfunction, computed without allocating device
// memory. Written for this project; the reference has no such entry point.
//
// Who needs it: a caller that already holds psi and the a_node metric on the device but may
// not allocate, either because its device memory is carved up in advance by its own pool (a
// solver embedded in a larger code that owns all of HBM), or because it runs under a
// memory budget where a cudaMalloc/cudaFree pair would synchronise the device and stall
// its other streams. The context API cannot serve it: nse2d_create allocates the fields and
// the workspace of the whole time step.
//
// How: the reduction kernel is the time step's own k_maxuv_dt (the CTAs combine their maxima
// by atomic max in a control block, and the last CTA reads them). That control block lives in
// g_maxuv_scratch, a fixed file-scope device variable, instead of the context's. The first call
// on a device, with that device current, looks up its address with cudaGetSymbolAddress and
// caches it. CUDA loads a library's kernels onto a device when they are first used (lazy
// module loading, the default since CUDA 12.2), so that first call is also where the driver
// places this file's code and the static scratch on the device: a one-time placement of a few
// kilobytes by the driver, not an allocation of this entry point. A caller that must see no
// change of free device memory after its set-up makes one call during set-up, on any grid.
// Every call clears the control block (the maxima, the last-CTA counter and the non-finite
// flag must start at zero) with cudaMemsetAsync. One scratch array serves every caller on a
// device, so calls that overlap in time on one device, from two streams or two host threads,
// race. Each call ends with a copy to pageable host memory and a stream synchronisation, so it
// must not be called while any stream of the device is being captured into a CUDA graph.
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "nse2d_internal.h"
#include "step_kernels.cuh"
#include "../../include/nse2d.h"

namespace nse2d {

namespace {
constexpr int kMaxUvNoAllocBlocks = NSE2D_MAXUV_NOALLOC_MAX_BLOCKS;
struct MaxUvScratch {
    Ctl ctl;                                     // atomic maxima, last-CTA counter, non-finite flag, results
};
constexpr int kMaxDevices = 64;

struct DeviceSlot {
    MaxUvScratch* scratch = nullptr;
    int num_sms = 0;
    int per_sm = 0;          // resident CTAs of the reduction kernel per SM
};
std::mutex g_slot_mutex;
DeviceSlot g_slots[kMaxDevices];
}  // namespace

static __device__ __align__(256) MaxUvScratch g_maxuv_scratch;

// Address of this device's scratch, its SM count and the reduction's occupancy, looked up once
// per device.
static int device_slot(DeviceSlot& out) {
    int dev = -1;
    NSE_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("nse2d_max_uv_noalloc: device %d outside the %d devices this entry point serves",
                  dev, kMaxDevices);
        return -1;
    }
    std::lock_guard<std::mutex> lock(g_slot_mutex);
    DeviceSlot& slot = g_slots[dev];
    if (!slot.scratch) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_maxuv_scratch);
        if (e != cudaSuccess || !ptr) {
            set_error("nse2d_max_uv_noalloc: cudaGetSymbolAddress of the scratch failed on device %d: %s",
                      dev, cudaGetErrorString(e));
            return -1;
        }
        int sms = 0;
        NSE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        int per_sm = 0;
        NSE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_maxuv_dt<false>, 256, 0));
        slot.num_sms = sms > 0 ? sms : 1;
        slot.per_sm = per_sm > 0 ? per_sm : 1;
        slot.scratch = static_cast<MaxUvScratch*>(ptr);
    }
    out = slot;
    return 0;
}

}  // namespace nse2d

extern "C" int nse2d_max_uv_noalloc(const double* d_psi, const double* d_a_node, int Nx, int Ny,
                                    double inv_dx, double inv_deta, double* out3, cudaStream_t s) {
    using namespace nse2d;
    if (!d_psi || !d_a_node || !out3) {
        set_error("nse2d_max_uv_noalloc: null pointer argument");
        return -1;
    }
    if (Nx < 2 || Ny < 3) {
        set_error("nse2d_max_uv_noalloc: grid %d x %d too small (need Nx >= 2, Ny >= 3)", Nx, Ny);
        return -1;
    }
    if (reinterpret_cast<uintptr_t>(d_psi) % 8 != 0 || reinterpret_cast<uintptr_t>(d_a_node) % 8 != 0) {
        set_error("nse2d_max_uv_noalloc: psi and a_node must be 8-byte aligned device pointers");
        return -1;
    }
    if (Nx > (1 << 30)) {
        set_error("nse2d_max_uv_noalloc: Nx = %d exceeds the maximum %d (32-bit column index)", Nx, 1 << 30);
        return -1;
    }
    DeviceSlot slot;
    if (device_slot(slot)) return -1;
    MaxUvScratch* sc = slot.scratch;
    NSE_CUDA_TRY(cudaMemsetAsync(&sc->ctl, 0, sizeof(Ctl), s));
    MaxParams p{};
    p.psi = d_psi; p.a_node = d_a_node; p.ctl = &sc->ctl;
    p.Nx = Nx; p.Ny = Ny; p.adapt = 0; p.set_dt = 0;
    p.inv_dx = inv_dx; p.inv_deta = inv_deta;
    // At most NSE2D_MAXUV_NOALLOC_MAX_BLOCKS CTAs; they stride over the (column strip, row band)
    // items, so every grid is covered, and combine their maxima atomically in the control block.
    int grid = 1;
    maxuv_plan(p, slot.per_sm * slot.num_sms, kMaxUvNoAllocBlocks, grid);
    // 16-byte loads only where every row and column pair is 16-byte aligned; a caller's psi may
    // be any 8-byte-aligned pointer and Nx any size from 2
    const bool vec = (Nx % 2 == 0) && (reinterpret_cast<uintptr_t>(d_psi) % 16 == 0);
    if (vec) k_maxuv_dt<true><<<grid, 256, 0, s>>>(p);
    else k_maxuv_dt<false><<<grid, 256, 0, s>>>(p);
    NSE_CUDA_TRY(cudaGetLastError());
    Ctl h{};
    NSE_CUDA_TRY(cudaMemcpyAsync(&h, &sc->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    out3[0] = h.umax; out3[1] = h.vmax; out3[2] = h.vmaxm;
    if (h.nonfinite & 1) {
        // the maxima skip NaN, so out3 alone would not show it
        set_error("nse2d_max_uv_noalloc: psi holds NaN or Inf (out3 holds the maxima of the finite differences)");
        return NSE2D_STATUS_NONFINITE;
    }
    return 0;
}
