// ne2b_kernels.cu — the per-step kernel and its helpers.
//
// One launch = one dt step of every active network in the engine.  The grid
// is persistent (a multiple of the SM count) and strides over tiles; a tile
// is `count` consecutive neurons of one network.  Per tile the block:
//
//   1. streams the neurons' state (SoA, coalesced) and the ring slot of this
//      step, zeroing the slot words that held arrivals
//        (sim/src/cpu.rs:218-222, kernels.rs:104-107);
//   2. assembles the input current s + ext (+ stimulus) (+ noise) in the
//      reference order and runs the model step (cpu.rs:223-250);
//   3. updates trace and s with the host-computed decays (cpu.rs:252-260);
//   4. compacts the tile's spikes with warp ballots and a block prefix sum
//      into shared memory, writing the spike-record words straight from the
//      ballots (replaces the global atomicAdd slot of kernels.rs:150-156);
//   5. delivers its own spikes: one warp per spiking neuron, lanes striding
//      the neuron's source-major CSR row, a no-return atomic add into
//      ring[(t + delay) % D][tgt] (cpu.rs:264-278, kernels.rs:174-204).
//
// No cross-block ordering is needed inside a step: step t reads ring slot
// t % D and every delivery of step t lands in slot (t + d) % D with
// 1 <= d < D, a different slot.  The kernel boundary orders step t's
// deliveries before step t+1's reads.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ne2b_device.cuh"
#include "ne2b_kernels.h"

namespace ne2b {

template <bool INT, int BLOCK, int NPT>
__global__ void __launch_bounds__(BLOCK) step_kernel(const EngineDev *__restrict__ eng, uint32_t k_step) {
    constexpr int NW = BLOCK / 32;
    constexpr int TILE = BLOCK * NPT;
    __shared__ uint32_t s_list[TILE];
    __shared__ uint32_t s_woff[NW];
    __shared__ uint32_t s_total;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t n_tiles = eng->n_tiles;
    const Tile *__restrict__ tiles = eng->tiles;
    NetDev *__restrict__ nets = eng->nets;
    const ParamRow *__restrict__ ptab = eng->ptab;

    for (uint32_t tix = blockIdx.x; tix < n_tiles; tix += gridDim.x) {
        const Tile tile = tiles[tix];
        const NetDev &nd = nets[tile.net];
        const uint32_t flags = nd.flags;
        if (!(flags & kNetActive)) continue;
        const uint64_t t = nd.t + k_step;
        if (t >= nd.t_end) continue;

        const uint32_t n = nd.n, n_pad = nd.n_pad, D = nd.D;
        const uint32_t tmod = (nd.tmod + k_step) % D;
        const size_t slot_off = (size_t)tmod * n_pad;
        const float dt = nd.dt, decay_s = nd.decay_s, decay_t = nd.decay_t;
        const float pkick = nd.pkick, kick = nd.kick, gauss_k = nd.gauss_k;
        const uint64_t seed = nd.seed;
        uint32_t *__restrict__ ringw = (uint32_t *)nd.ring;
        float *__restrict__ va = nd.v;
        float *__restrict__ ua = nd.u;
        float *__restrict__ sa = nd.s;
        float *__restrict__ ta = nd.trace;
        const bool has_ext = flags & kNetHasExt;
        const bool has_stim = tile.flags & kTileHasStim;
        const bool windows = flags & kNetWindows;
        bool win_end = false;
        uint32_t widx = 0;
        if (windows) {
            win_end = ((t + 1) % nd.win_steps) == 0;
            widx = (uint32_t)((t + 1) / nd.win_steps) - 1u;
        }

        uint32_t li[NPT];
        bool valid[NPT];
        float v[NPT], u[NPT], s[NPT], tr[NPT], ex[NPT];
        uint32_t rw[NPT];
        uint32_t pi[NPT];
#pragma unroll
        for (int q = 0; q < NPT; ++q) {
            const uint32_t off = q * BLOCK + threadIdx.x;
            li[q] = tile.start + off;
            valid[q] = off < tile.count && li[q] < n;
            if (valid[q]) {
                rw[q] = ringw[slot_off + li[q]];
                v[q] = va[li[q]];
                u[q] = ua[li[q]];
                s[q] = sa[li[q]];
                tr[q] = ta[li[q]];
                pi[q] = nd.pidx[li[q]];
                ex[q] = has_ext ? nd.ext[li[q]] : 0.0f;
            }
        }

        bool spk[NPT];
#pragma unroll
        for (int q = 0; q < NPT; ++q) {
            spk[q] = false;
            if (!valid[q]) continue;
            const uint32_t i = li[q];
            float arr;
            if (INT) {
                arr = __fmul_rn(__int2float_rn((int)rw[q]), 0x1p-12f);  // rt_get, kernels.rs:60
            } else {
                arr = __uint_as_float(rw[q]);
            }
            if (rw[q] != 0u) ringw[slot_off + i] = 0u;
            const float sv = __fadd_rn(s[q], arr);
            float I = __fadd_rn(sv, ex[q]);
            if (has_stim) {
                // the host uploads the [steps x inputs] values covering every
                // launched step; the range check only guards the read
                const long long rel = (long long)t - nd.stim_t0;
                const float *row = (rel >= 0 && rel < (long long)nd.stim_len) ? nd.stim_buf + (size_t)rel * nd.n_inputs : nullptr;
                const uint32_t lo = nd.stim_ptr[i], hi = nd.stim_ptr[i + 1];
                if (row)
                    for (uint32_t j = lo; j < hi; ++j) I = __fadd_rn(I, __fmul_rn(nd.stim_w[j], row[nd.stim_in[j]]));
            }
            const ParamRow &pr = ptab[pi[q]];
            float p[10];
            const float4 p0 = *reinterpret_cast<const float4 *>(&pr.p[0]);
            const float4 p1 = *reinterpret_cast<const float4 *>(&pr.p[4]);
            const float4 p2 = *reinterpret_cast<const float4 *>(&pr.p[8]);
            p[0] = p0.x; p[1] = p0.y; p[2] = p0.z; p[3] = p0.w;
            p[4] = p1.x; p[5] = p1.y; p[6] = p1.z; p[7] = p1.w;
            p[8] = p2.x; p[9] = p2.y;
            const uint32_t model = pr.model;
            const float gain = model == 1u ? p[0] : 1.0f;  // model/mod.rs:104-106, adex.rs:189-191
            if (pkick > 0.0f || gauss_k != 0.0f) {
                const uint64_t base = noise_base(i, t, seed);
                if (pkick > 0.0f && noise_fires(base, pkick)) I = __fadd_rn(I, __fmul_rn(kick, gain));
                if (gauss_k != 0.0f)
                    I = __fadd_rn(I, __fmul_rn(__int2float_rn(gauss_numer(base)), __fmul_rn(gauss_k, gain)));
            }
            bool sp = model == 1u ? adex_step(p, v[q], u[q], I, dt) : izh_step(p, v[q], u[q], I, dt);
            tr[q] = sp ? 1.0f : __fmul_rn(tr[q], decay_t);
            va[i] = v[q];
            ua[i] = u[q];
            sa[i] = __fmul_rn(sv, decay_s);
            ta[i] = tr[q];
            if (sp) nd.pn_total[i] += 1ull;
            if (windows) {
                if (win_end) {
                    const uint32_t c = nd.wcount[i] + (sp ? 1u : 0u);
                    if (widx < nd.max_windows) nd.win_out[(size_t)widx * n_pad + i] = (uint16_t)(c > 65535u ? 65535u : c);
                    nd.wcount[i] = 0u;
                } else if (sp) {
                    nd.wcount[i] += 1u;
                }
            }
            spk[q] = sp;
        }

        // ---- compaction: warp ballots -> record words + block prefix sum
        uint32_t mask[NPT];
        uint32_t wcnt = 0;
#pragma unroll
        for (int q = 0; q < NPT; ++q) {
            mask[q] = __ballot_sync(0xffffffffu, spk[q]);
            wcnt += __popc(mask[q]);
        }
        if (flags & kNetRecord) {
            const uint32_t row = (uint32_t)(t % nd.rec_rows);
            const uint32_t words32 = n_pad >> 5;
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < NPT; ++q) {
                    const uint32_t off = q * BLOCK + warp * 32;
                    if (off < tile.count) nd.rec_bits[(size_t)row * words32 + ((tile.start + off) >> 5)] = mask[q];
                }
            }
        }
        if (lane == 0) s_woff[warp] = wcnt;
        __syncthreads();
        if (warp == 0) {
            uint32_t c = lane < NW ? s_woff[lane] : 0u;
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane < NW) s_woff[lane] = incl - c;
            if (lane == 31) s_total = incl;
        }
        __syncthreads();
        {
            uint32_t pos = s_woff[warp];
            const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
            for (int q = 0; q < NPT; ++q) {
                if (spk[q]) s_list[pos + __popc(mask[q] & lt)] = li[q];
                pos += __popc(mask[q]);
            }
        }
        __syncthreads();
        const uint32_t total = s_total;
        if (total) {
            if (threadIdx.x == 0) atomicAdd(&eng->counters[tile.net].spikes_total, (unsigned long long)total);
            const uint32_t *__restrict__ rowptr = nd.rowptr;
            const uint32_t *__restrict__ tgt = nd.tgt;
            const bool d16 = flags & kNetDelay16;
            for (uint32_t si = warp; si < total; si += NW) {
                const uint32_t i = s_list[si];
                const uint32_t lo = rowptr[i], hi = rowptr[i + 1];
                for (uint32_t j = lo + lane; j < hi; j += 32) {
                    const uint32_t tg = tgt[j];
                    const uint32_t d = d16 ? (uint32_t)((const uint16_t *)nd.delay)[j] : (uint32_t)((const uint8_t *)nd.delay)[j];
                    uint32_t sl = tmod + d;
                    if (sl >= D) sl -= D;
                    const size_t idx = (size_t)sl * n_pad + tg;
                    if (INT) {
                        atomicAdd((int *)ringw + idx, ((const int *)nd.w)[j]);
                    } else {
                        atomicAdd((float *)ringw + idx, ((const float *)nd.w)[j]);
                    }
                }
            }
        }
        __syncthreads();
    }
}

// Advance every active net by `steps` after a launch group (t and t % D).
__global__ void advance_kernel(NetDev *nets, uint32_t n_nets, uint32_t steps) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_nets) return;
    NetDev &nd = nets[j];
    if (!(nd.flags & kNetActive)) return;
    unsigned long long t = nd.t + steps;
    if (t > nd.t_end) t = nd.t_end;
    nd.t = t;
    nd.tmod = (uint32_t)(t % nd.D);
}

// reset_state for one net (cpu.rs:158-183): state rows from v0/u0, zeros.
__global__ void reset_neurons_kernel(NetDev nd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd.n_pad) return;
    nd.v[i] = nd.v0[i];
    nd.u[i] = nd.u0[i];
    nd.s[i] = 0.0f;
    nd.trace[i] = 0.0f;
    nd.pn_total[i] = 0ull;
    if (nd.wcount) nd.wcount[i] = 0u;
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

// L2 flush helper for timing hygiene: writes a buffer larger than L2.
__global__ void scrub_kernel(uint4 *buf, size_t n16) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n16; k += (size_t)gridDim.x * blockDim.x)
        buf[k] = make_uint4((uint32_t)k, 0u, 0u, 0u);
}

// ------------------------------------------------------------- launchers
template <bool INT, int BLOCK, int NPT>
static cudaError_t launch_step_t(const EngineDev *eng, uint32_t k_step, uint32_t grid, cudaStream_t st) {
    step_kernel<INT, BLOCK, NPT><<<grid, BLOCK, 0, st>>>(eng, k_step);
    return cudaGetLastError();
}

template <bool INT, int BLOCK, int NPT>
static int occupancy_t() {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, step_kernel<INT, BLOCK, NPT>, BLOCK, 0);
    return b;
}

#define NE2B_SHAPES(X) \
    X(128, 1) X(128, 2) X(128, 4) X(256, 1) X(256, 2) X(256, 4) X(512, 1) X(512, 2)

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

cudaError_t launch_step(bool int_ring, uint32_t block, uint32_t npt, const EngineDev *eng, uint32_t k_step,
                        uint32_t grid, cudaStream_t st) {
#define X(B, P)                                                                         \
    if (block == B && npt == P)                                                         \
        return int_ring ? launch_step_t<true, B, P>(eng, k_step, grid, st)              \
                        : launch_step_t<false, B, P>(eng, k_step, grid, st);
    NE2B_SHAPES(X)
#undef X
    return cudaErrorInvalidValue;
}

int step_occupancy(bool int_ring, uint32_t block, uint32_t npt) {
#define X(B, P) \
    if (block == B && npt == P) return int_ring ? occupancy_t<true, B, P>() : occupancy_t<false, B, P>();
    NE2B_SHAPES(X)
#undef X
    return 0;
}

cudaError_t launch_advance(NetDev *nets, uint32_t n_nets, uint32_t steps, cudaStream_t st) {
    if (n_nets == 0) return cudaSuccess;
    advance_kernel<<<(n_nets + 127) / 128, 128, 0, st>>>(nets, n_nets, steps);
    return cudaGetLastError();
}

cudaError_t launch_reset_neurons(const NetDev &nd, cudaStream_t st) {
    if (nd.n_pad == 0) return cudaSuccess;
    reset_neurons_kernel<<<(nd.n_pad + 255) / 256, 256, 0, st>>>(nd);
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

cudaError_t launch_scrub(void *buf, size_t bytes, cudaStream_t st) {
    scrub_kernel<<<1184, 256, 0, st>>>((uint4 *)buf, bytes / 16);
    return cudaGetLastError();
}

}  // namespace ne2b
