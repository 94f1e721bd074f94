// ne2b_noalloc.cu — spike_counts for callers that cannot allocate.
//
// ne2b_spike_counts computes its per-neuron counts into a temporary device
// buffer it allocates and frees on every call.  Some callers must not do
// that: a serving thread that runs under a fixed device-memory budget (every
// byte already handed to its own arena, so any allocation fails), or one that
// must not stall, since cudaMalloc and cudaFree synchronise the whole device
// and a stream-ordered pool may have to grow.  ne2b_spike_counts_noalloc is
// the same computation with its scratch in the file-scope array below: it
// allocates nothing and frees nothing.
//
// The array holds kNoAllocMaxNeurons u32 counts (4 MiB) on every GPU that
// loads this library, until the process exits.  Its device address is looked
// up once per device, with that device current, when the first engine on the
// device is created (noalloc_setup, called from Engine::init), so the entry
// point itself does no set-up.  A failed look-up (or a device ordinal past
// kNoAllocMaxDevices) leaves the address unset: engine creation goes on, and
// only this entry point reports the missing scratch.  Every call shares the one array and leaves
// the last call's counts in it; each call overwrites entries [0, n) before
// reading them, so nothing has to start at zero.  Calls whose kernels overlap
// on the GPU (two host threads, two sims on one device) race on the array.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "../../include/ne2b.h"
#include "ne2b_handles.h"

namespace ne2b {

constexpr uint32_t kNoAllocMaxNeurons = 1u << 20;  // 1,048,576 neurons, 4 MiB
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) uint32_t g_noalloc_counts[kNoAllocMaxNeurons];

// Device address of g_noalloc_counts per device ordinal.  In host code the
// array's name is only a host-side stand-in, so the address must come from
// cudaGetSymbolAddress with the device current.
static uint32_t *g_noalloc_ptr[kNoAllocMaxDevices] = {};
static std::mutex g_noalloc_mu;

// Returns NE2B_OK or the look-up's error; the caller may ignore it, since a
// device without the address only refuses ne2b_spike_counts_noalloc.
ne2b_status noalloc_setup(int device) {
    if (device < 0 || device >= kNoAllocMaxDevices) return NE2B_OK;  // entry point unavailable there
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (g_noalloc_ptr[device]) return NE2B_OK;
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_counts);
    if (e != cudaSuccess) {
        cudaGetLastError();  // clear the (non-sticky) error so that the engine's next runtime call does not return it
        return cuda_error(e, "cudaGetSymbolAddress(spike-count scratch)");
    }
    g_noalloc_ptr[device] = (uint32_t *)p;
    return NE2B_OK;
}

// Same counts as window_count_kernel / pn_total_kernel, written to `scratch`.
__global__ void noalloc_window_count_kernel(const uint32_t *rec_bits, uint32_t rec_rows, uint32_t n_pad, uint32_t n,
                                            unsigned long long t, uint32_t rows, uint32_t *scratch) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t words32 = n_pad >> 5;
    uint32_t c = 0;
    for (uint32_t b = 0; b < rows; ++b) {
        const uint32_t row = (uint32_t)((t - 1 - b) % rec_rows);
        c += (rec_bits[(size_t)row * words32 + (i >> 5)] >> (i & 31)) & 1u;
    }
    scratch[i] = c;
}

__global__ void noalloc_pn_total_kernel(const unsigned long long *pn, uint32_t n, uint32_t *scratch) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long c = pn[i];
    scratch[i] = c > 0xffffffffull ? 0xffffffffu : (uint32_t)c;
}

}  // namespace ne2b

extern "C" ne2b_status ne2b_spike_counts_noalloc(ne2b_sim *sim, uint64_t rows, uint32_t *out) {
    using namespace ne2b;
    if (!sim) return set_error(NE2B_EINVAL, "null sim handle");
    NetHost *h = sim->eng.net(sim->slot);
    if (!h) return set_error(NE2B_EINVAL, "sim has no network");
    const uint32_t n = h->n;
    if (!out && n) return set_error(NE2B_EINVAL, "null out");
    // window rules of Backend::spike_counts (sim/src/cpu.rs:424-458), in the
    // order Engine::spike_counts applies them: no recording or no step yet
    // gives zeros at any size
    if (!h->dev.rec_rows || h->t == 0) {
        if (n) memset(out, 0, sizeof(uint32_t) * n);
        return NE2B_OK;
    }
    if (rows < h->t && rows > h->dev.rec_rows)
        return set_error(NE2B_EWINDOW, "spike_counts window %llu exceeds the recorded %u steps",
                         (unsigned long long)rows, h->dev.rec_rows);
    if (n == 0) return NE2B_OK;
    if (n > kNoAllocMaxNeurons)
        return set_error(NE2B_EINVAL, "spike_counts_noalloc: %u neurons exceed the %u-neuron scratch array", n,
                         kNoAllocMaxNeurons);
    const int device = sim->eng.device();
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    uint32_t *scratch = (device >= 0 && device < kNoAllocMaxDevices) ? g_noalloc_ptr[device] : nullptr;
    if (!scratch) return set_error(NE2B_ECUDA, "spike-count scratch not set up on device %d", device);
    cudaStream_t st = sim->eng.stream();
    const uint32_t grid = (n + 255) / 256;
    if (rows >= h->t) noalloc_pn_total_kernel<<<grid, 256, 0, st>>>(h->dev.pn_total, n, scratch);
    else noalloc_window_count_kernel<<<grid, 256, 0, st>>>(h->dev.rec_bits, h->dev.rec_rows, h->n_pad, n, h->t,
                                                              (uint32_t)rows, scratch);
    e = cudaGetLastError();
    sim->eng.count_launches(1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, scratch, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return cuda_error(e, "spike_counts_noalloc");
}
