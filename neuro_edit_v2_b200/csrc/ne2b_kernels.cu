// ne2b_kernels.cu — the helper kernels (advance, reset, trace and window
// readouts) and the host launchers; the step kernels themselves are in
// ne2b_step.cuh, instantiated per kind in ne2b_step_k*.cu.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ne2b_kernels.h"
#include "ne2b_step.cuh"

namespace ne2b {

// Advance every active net by `steps` after a launch group (t and t % D).
__global__ void advance_kernel(NetDev *nets, uint32_t n_nets, uint32_t steps) {
    pdl_enter();
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_nets) return;
    NetDev &nd = nets[j];
    if (!(nd.flags & kNetActive)) return;
    unsigned long long t = nd.t + steps;
    if (t > nd.t_end) t = nd.t_end;
    set_step(nd, t);
}

// reset_state for one net (cpu.rs:158-183): state rows from v0/u0, zeros.
__global__ void reset_neurons_kernel(NetDev nd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd.n_pad) return;
    nd.v[i] = nd.v0[i];
    nd.u[i] = nd.u0[i];
    nd.s[i] = 0.0f;
    nd.tk[i] = kTraceZero;
    nd.pn_total[i] = 0ull;
    if (nd.wcount) nd.wcount[i] = 0u;
}

// Backend::trace (lib.rs:137): trace_tab[tk], 0 for kTraceZero.
__global__ void trace_kernel(const uint16_t *tk, const float *tab, uint32_t n, float *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint16_t k = tk[i];
    out[i] = k == kTraceZero ? 0.0f : tab[k];
}

// spike_counts over the last `rows` record rows (cpu.rs:424-458): thread per
// neuron; the 32 lanes of a warp share each record word.
__global__ void window_count_kernel(const uint32_t *rec_bits, uint32_t rec_rows, uint32_t n_pad, uint32_t n,
                                    unsigned long long t, uint32_t rows, uint32_t *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t words32 = n_pad >> 5;
    uint32_t c = 0;
    for (uint32_t b = 0; b < rows; ++b) {
        const uint32_t row = (uint32_t)((t - 1 - b) % rec_rows);
        c += (rec_bits[(size_t)row * words32 + (i >> 5)] >> (i & 31)) & 1u;
    }
    out[i] = c;
}

// pn_total saturated to u32 (cpu.rs:432-436).
__global__ void pn_total_kernel(const unsigned long long *pn, uint32_t n, uint32_t *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long c = pn[i];
    out[i] = c > 0xffffffffull ? 0xffffffffu : (uint32_t)c;
}

// Self-test of the bounded grid barrier: every block but `absent` arrives,
// so the others give up after `limit_ns`, set the error flag and return
// (a wait that cannot end, ended by its limit, with no fault).
__global__ void barrier_selftest_kernel(unsigned int *counter, unsigned int *err, uint32_t absent,
                                        unsigned long long limit_ns) {
    __shared__ unsigned int s_flag;
    if (blockIdx.x == absent) return;
    grid_barrier(counter, gridDim.x, err, &s_flag, limit_ns);
}

// ------------------------------------------------------------- launchers
bool shape_supported(uint32_t block, uint32_t npt) {
#define X(B, P) if (block == B && npt == P) return true;
    NE2B_SHAPES(X)
#undef X
    return false;
}

bool ws_shape_supported(uint32_t block, uint32_t npt) {
#define X(B, P) if (block == B && npt == P) return true;
    NE2B_WS_SHAPES(X)
#undef X
    return false;
}

void shape_list(uint32_t *blocks, uint32_t *npts, uint32_t *count) {
    uint32_t c = 0;
#define X(B, P) blocks[c] = B; npts[c] = P; ++c;
    NE2B_SHAPES(X)
#undef X
    *count = c;
}

static bool g_pdl = true;
void set_pdl(bool on) { g_pdl = on; }
bool pdl_enabled() { return g_pdl; }

// Kernel variants: INT (int32 fixed-point ring) x ADEX (AdEx rows present;
// an all-Izhikevich engine runs the instance without the AdEx path).
#define NE2B_KIND(int_ring, adex, call)                                  \
    ((int_ring) ? ((adex) ? StepKind<true, true>::call : StepKind<true, false>::call) \
                : ((adex) ? StepKind<false, true>::call : StepKind<false, false>::call))

int step_occupancy(bool int_ring, bool adex, int variant, uint32_t block, uint32_t npt) {
    return NE2B_KIND(int_ring, adex, occupancy(block, npt, variant));
}

cudaError_t launch_step(bool int_ring, bool adex, int variant, uint32_t block, uint32_t npt, const EngineDev *eng,
                        uint32_t k_step, uint32_t grid, cudaStream_t st) {
    return NE2B_KIND(int_ring, adex, launch(block, npt, variant, eng, k_step, grid, st));
}

uint32_t resident_head(uint32_t block, uint32_t npt) {
#define X(B, P) if (block == B && npt == P) return resident_head_bytes<B, P>();
    NE2B_SHAPES(X)
#undef X
    return 0;
}

int resident_occupancy(bool int_ring, bool adex, uint32_t block, uint32_t npt, size_t smem) {
    return NE2B_KIND(int_ring, adex, resident_occupancy(block, npt, smem));
}

cudaError_t launch_resident(bool int_ring, bool adex, uint32_t block, uint32_t npt, const EngineDev *eng,
                            uint32_t k0, uint32_t nsteps, uint32_t grid, size_t smem, cudaStream_t st) {
    return NE2B_KIND(int_ring, adex, launch_resident(block, npt, eng, k0, nsteps, grid, smem, st));
}

cudaError_t launch_barrier_selftest(unsigned int *counter, unsigned int *err, uint32_t blocks, uint32_t absent,
                                    unsigned long long limit_ns, cudaStream_t st) {
    void *args[] = {(void *)&counter, (void *)&err, (void *)&absent, (void *)&limit_ns};
    return cudaLaunchCooperativeKernel((const void *)barrier_selftest_kernel, dim3(blocks), dim3(32), args, 0, st);
}

cudaError_t launch_advance(NetDev *nets, uint32_t n_nets, uint32_t steps, cudaStream_t st) {
    if (n_nets == 0) return cudaSuccess;
    return launch_pdl(advance_kernel, (n_nets + 127) / 128, 128, st, true, nets, n_nets, steps);
}

cudaError_t launch_reset_neurons(const NetDev &nd, cudaStream_t st) {
    if (nd.n_pad == 0) return cudaSuccess;
    reset_neurons_kernel<<<(nd.n_pad + 255) / 256, 256, 0, st>>>(nd);
    return cudaGetLastError();
}

cudaError_t launch_trace(const uint16_t *tk, const float *tab, uint32_t n, float *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    trace_kernel<<<(n + 255) / 256, 256, 0, st>>>(tk, tab, n, out);
    return cudaGetLastError();
}

cudaError_t launch_window_count(const uint32_t *rec_bits, uint32_t rec_rows, uint32_t n_pad, uint32_t n,
                                unsigned long long t, uint32_t rows, uint32_t *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    window_count_kernel<<<(n + 255) / 256, 256, 0, st>>>(rec_bits, rec_rows, n_pad, n, t, rows, out);
    return cudaGetLastError();
}

cudaError_t launch_pn_total(const unsigned long long *pn, uint32_t n, uint32_t *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    pn_total_kernel<<<(n + 255) / 256, 256, 0, st>>>(pn, n, out);
    return cudaGetLastError();
}

}  // namespace ne2b
