// ne2b_csr.cu — Network::synapse_csr (net-format/src/network.rs:654-692) on
// the device, for sims created from a plain synapse list.
//
//   1. prepass: every synapse's references are checked (the first bad index
//      is kept), its delay rounded to steps (max(1, roundf(ms / dt)), at most
//      65535: network.rs:660-666), the largest delay found, and the synapses
//      counted per source;
//   2. the counts are scanned into the row pointers, and a copy of them
//      becomes the per-source fill cursor;
//   3. stable scatter: block c takes synapses [8192 c, 8192 (c + 1)) of the
//      list and sorts them by (source, position) in shared memory (bitonic),
//      which makes each source's synapses one run in list order.  The blocks
//      then claim their runs' places in list order: block c waits until
//      block c - 1 has added its run lengths to the cursors, adds its own
//      (one atomic per run) and releases block c + 1, so the synapses of a
//      source land in list order across blocks as well.  Blocks take their
//      chunk index from a ticket when they start, so the block waited on has
//      always started; each wait is bounded by %globaltimer and a timeout is
//      reported, never spun forever.  Finally each synapse is written to its
//      place: target, Dale-signed weight (network.rs:668-672; quantised as
//      kernels.rs:61 rt_put for the fixed-point ring) and delay, packed in
//      one 8-byte record (target | delay << 24, weight bits), or the bare
//      target and a separate u16 delay for a wide net (kNetDelayWide).
//
// The result equals the host build (ne2b_net_from_synapses, a stable
// counting sort) bit for bit.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ne2b_csr.h"

namespace ne2b {

namespace {

constexpr uint32_t kChunk = 8192;   // synapses per scatter block
constexpr uint32_t kThreads = 1024; // scatter block size
constexpr uint32_t kPer = kChunk / kThreads;
// dynamic shared memory of a scatter block: keys, run starts (u16), run bases
constexpr size_t kScatterSmem = kChunk * (sizeof(unsigned long long) + sizeof(uint16_t) + sizeof(uint32_t));
constexpr uint32_t kScan = 4096;    // counts per scan block (1024 threads x 4)

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__global__ void csr_prepass_kernel(const uint32_t *__restrict__ src, const uint32_t *__restrict__ tgt,
                                   const float *__restrict__ dly, uint64_t E, uint32_t n, float dt,
                                   uint32_t *__restrict__ counts, uint16_t *__restrict__ steps, CsrScalars *sc) {
    uint32_t mx = 1;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < E; j += stride) {
        const uint32_t s = src[j], t = tgt[j];
        if (s >= n || t >= n) {
            atomicMin(&sc->bad_ref, (unsigned long long)j);
            continue;
        }
        atomicAdd(&counts[s], 1u);
        float st = roundf(__fdiv_rn(dly[j], dt));
        if (st < 1.0f) st = 1.0f;
        if (!(st <= 65535.0f)) {
            atomicMin(&sc->bad_delay, (unsigned long long)j);
            continue;
        }
        const uint32_t k = (uint32_t)st;
        steps[j] = (uint16_t)k;
        mx = k > mx ? k : mx;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31u) == 0u) atomicMax(&sc->max_delay, mx);
}

// Block-wide exclusive sum of one value per thread (1024 threads); the
// block total goes to *total.
__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t *warp_sums, uint32_t *total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31u) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = warp_sums[lane];
        uint32_t z = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= (uint32_t)o) z += y;
        }
        warp_sums[lane] = z - w;
        if (lane == 31u) *total = z;
    }
    __syncthreads();
    const uint32_t r = warp_sums[warp] + x - v;
    __syncthreads();  // warp_sums may be reused by the caller
    return r;
}

// rowptr[i] = sum of counts[0..i) within the block's 4096 counts; the
// block's total to sums[blockIdx.x].
__global__ void __launch_bounds__(1024) csr_scan_blocks_kernel(const uint32_t *__restrict__ counts, uint32_t n,
                                                               uint32_t *__restrict__ rowptr, uint32_t *sums) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t total;
    const uint64_t base = (uint64_t)blockIdx.x * kScan + (uint64_t)threadIdx.x * 4u;
    uint32_t c[4], s = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        c[e] = base + e < n ? counts[base + e] : 0u;
        s += c[e];
    }
    uint32_t run = block_exclusive_sum(s, warp_sums, &total);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        if (base + e < n) rowptr[base + e] = run;
        run += c[e];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Exclusive scan of the block totals in place (one block, any count).
__global__ void __launch_bounds__(1024) csr_scan_sums_kernel(uint32_t *sums, uint32_t nb) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t total;
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < nb; b0 += 1024) {
        const uint32_t b = b0 + threadIdx.x;
        const uint32_t v = b < nb ? sums[b] : 0u;
        const uint32_t x = block_exclusive_sum(v, warp_sums, &total);
        if (b < nb) sums[b] = carry + x;
        carry += total;
    }
}

// Adds each block's offset; cursor = rowptr; rowptr[n] = the synapse count.
__global__ void __launch_bounds__(1024) csr_scan_add_kernel(uint32_t *__restrict__ rowptr, const uint32_t *sums,
                                                            uint32_t n, uint32_t e, uint32_t *__restrict__ cursor) {
    const uint64_t base = (uint64_t)blockIdx.x * kScan + (uint64_t)threadIdx.x * 4u;
    const uint32_t off = sums[blockIdx.x];
#pragma unroll
    for (int e4 = 0; e4 < 4; ++e4)
        if (base + e4 < n) {
            const uint32_t r = rowptr[base + e4] + off;
            rowptr[base + e4] = r;
            cursor[base + e4] = r;
        }
    if (blockIdx.x == 0 && threadIdx.x == 0) rowptr[n] = e;
}

__global__ void __launch_bounds__(kThreads) csr_scatter_kernel(const uint32_t *__restrict__ src,
                                                               const uint32_t *__restrict__ tgt,
                                                               const float *__restrict__ w,
                                                               const uint16_t *__restrict__ steps,
                                                               const uint8_t *__restrict__ kind, uint64_t E,
                                                               uint32_t *cursor, SynRec *__restrict__ syn_out,
                                                               uint16_t *__restrict__ delay16_out,
                                                               bool int_w, bool wide, uint32_t *ticket, uint32_t *done,
                                                               CsrScalars *sc, unsigned long long limit_ns) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long *key = (unsigned long long *)smem;         // (source << 32) | position in the chunk
    uint32_t *run_base = (uint32_t *)(key + kChunk);              // at a run's start: its length, then its place
    uint16_t *run_start = (uint16_t *)(run_base + kChunk);        // sorted position of the run's first synapse
    __shared__ uint32_t warp_max[32];
    __shared__ uint32_t s_chunk, s_fail;
    if (threadIdx.x == 0) {
        s_chunk = atomicAdd(ticket, 1u);
        s_fail = 0u;
    }
    __syncthreads();
    const uint32_t c = s_chunk;
    const uint64_t j0 = (uint64_t)c * kChunk;
    const uint32_t nvalid = j0 >= E ? 0u : (uint32_t)(E - j0 < kChunk ? E - j0 : kChunk);
    for (uint32_t i = threadIdx.x; i < kChunk; i += kThreads)
        key[i] = i < nvalid ? ((unsigned long long)src[j0 + i] << 32) | i : ~0ull;
    __syncthreads();
    // bitonic sort, ascending (the padding keys sort last)
    for (uint32_t k = 2; k <= kChunk; k <<= 1)
        for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
            for (uint32_t i = threadIdx.x; i < kChunk; i += kThreads) {
                const uint32_t l = i ^ jj;
                if (l > i) {
                    const unsigned long long a = key[i], b = key[l];
                    if ((a > b) == ((i & k) == 0u)) {
                        key[i] = b;
                        key[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    // run starts: inclusive max-scan of (p if a run starts at p else 0) over
    // the sorted positions, 4 consecutive positions per thread
    {
        const uint32_t p0 = threadIdx.x * kPer;
        uint32_t loc[kPer], m = 0;
#pragma unroll
        for (uint32_t e = 0; e < kPer; ++e) {
            const uint32_t p = p0 + e;
            const bool head = p == 0u || (key[p] >> 32) != (key[p - 1] >> 32);
            m = max(m, head ? p : 0u);
            loc[e] = m;
        }
        const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
        uint32_t x = m;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x = max(x, y);
        }
        if (lane == 31u) warp_max[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t z = warp_max[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
                if (lane >= (uint32_t)o) z = max(z, y);
            }
            warp_max[lane] = z;
        }
        __syncthreads();
        uint32_t before = __shfl_up_sync(0xffffffffu, x, 1);
        if (lane == 0u) before = 0u;
        if (warp > 0) before = max(before, warp_max[warp - 1]);
#pragma unroll
        for (uint32_t e = 0; e < kPer; ++e) run_start[p0 + e] = (uint16_t)max(before, loc[e]);
    }
    __syncthreads();
    // run lengths, stored at each run's start by its last synapse
    for (uint32_t p = threadIdx.x; p < nvalid; p += kThreads)
        if (p + 1u == nvalid || (key[p + 1] >> 32) != (key[p] >> 32)) run_base[run_start[p]] = p - run_start[p] + 1u;
    // wait for the previous chunk's claims (bounded)
    if (threadIdx.x == 0 && c > 0) {
        const unsigned long long t0 = globaltimer_ns();
        while (ld_acquire(&done[c - 1]) == 0u) {
            if (globaltimer_ns() - t0 > limit_ns) {
                atomicExch(&sc->timeout, 1u);
                s_fail = 1u;
                break;
            }
            __nanosleep(100);
        }
    }
    __syncthreads();
    if (!s_fail)
        for (uint32_t p = threadIdx.x; p < nvalid; p += kThreads)
            if (run_start[p] == p) run_base[p] = atomicAdd(&cursor[(uint32_t)(key[p] >> 32)], run_base[p]);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release(&done[c], 1u);
    }
    if (s_fail) return;
    for (uint32_t p = threadIdx.x; p < nvalid; p += kThreads) {
        const unsigned long long kv = key[p];
        const uint32_t s = (uint32_t)(kv >> 32);
        const uint64_t j = j0 + (uint32_t)kv;
        const uint32_t pos = run_base[run_start[p]] + (p - run_start[p]);
        const float m = fabsf(w[j]);
        const float ws = kind[s] == 1u ? -m : m;
        const uint32_t wb = int_w ? (uint32_t)__float2int_rn(__fmul_rn(ws, 4096.0f)) : __float_as_uint(ws);
        const uint32_t td = wide ? tgt[j] : tgt[j] | ((uint32_t)steps[j] << kSynTgtBits);
        *reinterpret_cast<uint2 *>(syn_out + pos) = make_uint2(td, wb);
        if (wide) delay16_out[pos] = steps[j];
    }
}

}  // namespace

cudaError_t csr_prepass(const DevSynapses &ds, uint32_t *counts, uint16_t *steps, CsrScalars *sc, cudaStream_t st) {
    if (ds.n_syn == 0) return cudaSuccess;
    uint64_t blocks = (ds.n_syn + 255) / 256;
    if (blocks > 148ull * 32) blocks = 148ull * 32;
    csr_prepass_kernel<<<(unsigned)blocks, 256, 0, st>>>(ds.src, ds.tgt, ds.delay_ms, ds.n_syn, ds.n, ds.dt_ms,
                                                         counts, steps, sc);
    return cudaGetLastError();
}

cudaError_t csr_scan(const uint32_t *counts, uint32_t n, uint32_t e, uint32_t *rowptr, uint32_t *cursor,
                     uint32_t *sums, cudaStream_t st) {
    if (n == 0) return cudaMemsetAsync(rowptr, 0, sizeof(uint32_t), st);
    const uint32_t nb = (n + kScan - 1) / kScan;
    csr_scan_blocks_kernel<<<nb, 1024, 0, st>>>(counts, n, rowptr, sums);
    csr_scan_sums_kernel<<<1, 1024, 0, st>>>(sums, nb);
    csr_scan_add_kernel<<<nb, 1024, 0, st>>>(rowptr, sums, n, e, cursor);
    return cudaGetLastError();
}

uint32_t csr_scan_blocks(uint32_t n) { return (n + kScan - 1) / kScan; }
uint64_t csr_chunks(uint64_t n_syn) { return (n_syn + kChunk - 1) / kChunk; }

cudaError_t csr_scatter(const DevSynapses &ds, const uint16_t *steps, uint32_t *cursor, SynRec *syn_out,
                        uint16_t *delay16_out, bool int_w, bool wide, uint32_t *ticket, uint32_t *done,
                        CsrScalars *sc, unsigned long long limit_ns, cudaStream_t st) {
    const uint64_t chunks = csr_chunks(ds.n_syn);
    if (chunks == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(csr_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kScatterSmem);
    if (e != cudaSuccess) return e;
    csr_scatter_kernel<<<(unsigned)chunks, kThreads, kScatterSmem, st>>>(ds.src, ds.tgt, ds.w, steps, ds.kind, ds.n_syn, cursor,
                                                              syn_out, delay16_out, int_w, wide, ticket, done, sc,
                                                              limit_ns);
    return cudaGetLastError();
}

}  // namespace ne2b
