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

// Split delivery, the second launch of a step: one warp per tile delivers
// the spikes the step kernel listed for it (ids in the tile's range of
// spk_ids, count in spk_cnt, emptied here).  For each spike the warp loads
// the row bounds and strides the row, U synapses per lane and pass with all
// their CSR loads issued before any add; an arrival goes into
// ring[(t + d) % D][tgt] by a no-return atomic, or, with event queues and
// d >= 2, is appended to the tile's segment of its bucket (cpu.rs:264-278,
// kernels.rs:174-204).  `tile` is the tile size of the step kernel.
template <bool INT>
__global__ void __launch_bounds__(256) deliver_kernel(const EngineDev *__restrict__ eng, uint32_t k_step,
                                                      uint32_t tile_size) {
    pdl_trigger();
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t n_tiles = eng->n_tiles;
    pdl_wait();  // the step kernel's lists are complete
    for (uint32_t tix = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); tix < n_tiles; tix += warps) {
        const Tile tile = eng->tiles[tix];
        const NetDev &nd = eng->nets[tile.net];
        uint32_t *const cntp = nd.spk_cnt;
        if (!cntp) continue;  // a custom-tau net: delivered by the step kernel
        const uint32_t k = tile.start / tile_size;
        const uint32_t cnt = cntp[k];
        if (cnt == 0u) continue;
        __syncwarp();
        if (lane == 0) cntp[k] = 0u;
        const uint32_t D = nd.D, n_pad = nd.n_pad;
        uint32_t tmod = nd.tmod + k_step;
        if (tmod >= D) tmod %= D;
        const uint32_t b1 = tmod + 1u == D ? 0u : tmod + 1u;
        const bool evq = (nd.flags & kNetEvq) != 0u;
        const bool d16 = (nd.flags & kNetDelay16) != 0u;
        const uint32_t *__restrict__ rowptr = nd.rowptr;
        const uint32_t *__restrict__ tgt = nd.tgt;
        const uint32_t *__restrict__ wbits = (const uint32_t *)nd.w;
        uint32_t *__restrict__ ringw = (uint32_t *)nd.ring;
        for (uint32_t b0 = 0; b0 < cnt; b0 += 32) {
            uint32_t lo = 0, hi = 0;
            if (b0 + lane < cnt) {
                const uint32_t id = nd.spk_ids[tile.start + b0 + lane];
                lo = rowptr[id];
                hi = rowptr[id + 1];
            }
            const uint32_t m = cnt - b0 < 32u ? cnt - b0 : 32u;
            for (uint32_t r = 0; r < m; ++r) {
                const uint32_t rl = __shfl_sync(0xffffffffu, lo, r), rh = __shfl_sync(0xffffffffu, hi, r);
                constexpr int U = 4;
                for (uint32_t j0 = rl; j0 < rh; j0 += 32u * U) {
                    uint32_t tg[U], sl_[U], wb[U];
#pragma unroll
                    for (int q = 0; q < U; ++q) {
                        const uint32_t j0q = j0 + 32u * q + lane;
                        const uint32_t j = j0q < rh ? j0q : rl;  // past the end: the row's first synapse again
                        tg[q] = tgt[j];
                        const uint32_t d = d16 ? (uint32_t)((const uint16_t *)nd.delay)[j]
                                               : (uint32_t)((const uint8_t *)nd.delay)[j];
                        sl_[q] = tmod + d >= D ? tmod + d - D : tmod + d;
                        wb[q] = wbits[j];
                    }
#pragma unroll
                    for (int q = 0; q < U; ++q) {
                        if (j0 + 32u * q + lane >= rh) continue;
                        if (evq && sl_[q] != b1) {
                            const uint32_t pos = atomicAdd(nd.evq_cnt + (size_t)sl_[q] * nd.evq_nseg + k, 1u);
                            if (pos < tile.count) {
                                nd.evq[(size_t)sl_[q] * n_pad + tile.start + pos] = make_uint2(tg[q], wb[q]);
                                continue;
                            }
                        }
                        const size_t idx = (size_t)sl_[q] * n_pad + tg[q];
                        if (INT) atomicAdd((int *)ringw + idx, (int)wb[q]);
                        else atomicAdd((float *)ringw + idx, __uint_as_float(wb[q]));
                    }
                }
            }
        }
    }
}

// Event queues: add every segment of every pending bucket into its ring slot
// and empty it (the segments of tile size `tile`), so the queues can be
// refilled under another tile size.  Pending arrivals reach their slots
// early, which changes nothing: the slot of bucket b is next read at the
// step they are due.  Bucket tmod (the next step's) was added into its slot
// during the last step and only awaits its counter reset: it is emptied
// without adding.
template <bool INT>
__global__ void evq_flush_kernel(NetDev nd, uint32_t tile) {
    const uint32_t nseg = (nd.n_pad + tile - 1) / tile;
    for (uint32_t s = blockIdx.x; s < nseg * nd.D; s += gridDim.x) {
        const uint32_t b = s / nseg, k = s - b * nseg;
        const uint32_t cnt = b == nd.tmod ? 0u : nd.evq_cnt[(size_t)b * nd.evq_nseg + k];
        const uint32_t size = nd.n_pad - k * tile < tile ? nd.n_pad - k * tile : tile;
        const uint32_t ne = cnt < size ? cnt : size;
        const uint2 *q = nd.evq + (size_t)b * nd.n_pad + (size_t)k * tile;
        for (uint32_t e = threadIdx.x; e < ne; e += blockDim.x) {
            const size_t idx = (size_t)b * nd.n_pad + q[e].x;
            if (INT) atomicAdd((int *)nd.ring + idx, (int)q[e].y);
            else atomicAdd((float *)nd.ring + idx, __uint_as_float(q[e].y));
        }
        __syncthreads();
        if (threadIdx.x == 0) nd.evq_cnt[(size_t)b * nd.evq_nseg + k] = 0u;
    }
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

cudaError_t launch_deliver(bool int_ring, const EngineDev *eng, uint32_t n_tiles, uint32_t k_step, uint32_t tile,
                           uint32_t max_blocks, cudaStream_t st) {
    uint32_t grid = (n_tiles + 7) / 8;  // 8 warps per block, one tile per warp
    if (grid > max_blocks) grid = max_blocks;
    if (grid == 0) grid = 1;
    return int_ring ? launch_pdl(deliver_kernel<true>, grid, 256, st, true, eng, k_step, tile)
                    : launch_pdl(deliver_kernel<false>, grid, 256, st, true, eng, k_step, tile);
}

cudaError_t launch_evq_flush(const NetDev &nd, bool int_ring, uint32_t tile, cudaStream_t st) {
    if (!nd.evq || tile == 0) return cudaSuccess;
    const uint32_t segs = (nd.n_pad + tile - 1) / tile * nd.D;
    const uint32_t grid = segs < 4096 ? segs : 4096;
    if (int_ring) evq_flush_kernel<true><<<grid, 256, 0, st>>>(nd, tile);
    else evq_flush_kernel<false><<<grid, 256, 0, st>>>(nd, tile);
    return cudaGetLastError();
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
