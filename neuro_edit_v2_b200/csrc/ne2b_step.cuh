// ne2b_step.cuh — the step kernels (streaming and resident), included by the
// four translation units that instantiate them, one per kernel kind.
//
// A tile is `count` consecutive neurons of one network.  Processing one tile
// for one dt step (process_tile):
//
//   1. read the tile's state and its ring slot for this step, zeroing the slot
//      words that held arrivals (sim/src/cpu.rs:218-222, kernels.rs:104-107);
//   2. assemble the input current s + ext (+ stimulus) (+ noise) in the
//      reference order and run the model step (cpu.rs:223-250);
//   3. update s and the trace with the host-computed decays (cpu.rs:252-260);
//      the trace is kept as "steps since the last spike" into a table of the
//      exact f32 products 1.0 * decay_t * decay_t ..., which reproduces the
//      reference's repeated multiply bit-for-bit at 2 bytes per neuron;
//   4. write the spike-record words straight from warp ballots, and compact
//      the tile's spikes by their CSR rows with block prefix sums over
//      (spikes, synapses) into shared memory (replaces the global atomicAdd
//      slot of kernels.rs:150-156);
//   5. deliver its own spikes: the block strides the flat range of all its
//      spikes' synapses, a no-return atomic add into
//      ring[(t + delay) % D][tgt] per synapse (cpu.rs:264-278,
//      kernels.rs:174-204).
//
// Within a step no cross-block ordering is needed: step t reads slot t % D and
// every delivery of step t lands in slot (t + d) % D, 1 <= d < D.  Between
// steps, step t's deliveries must land before step t+1 reads:
//   * step_kernel (streaming): one launch per step, the kernel boundary orders
//     the steps; state is streamed from HBM every step.
//   * resident_kernel (persistent, cooperative): each block owns a fixed set
//     of tiles whose state stays in shared memory for the whole launch; steps
//     are separated by a grid barrier whose wait is bounded by %globaltimer
//     (2 s, then the launch stops and reports an error flag).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ne2b_device.cuh"
#include "ne2b_step_kind.h"

namespace ne2b {

// Synapses a thread delivers per pass of the flat range, their CSR loads in
// flight together: four with the int32 ring (against one: -20% per step at
// ~22 Hz on the 100k net; eight was slower), two with the f32 ring, where
// four makes the compiler spill in the 64 x 2 and 128 x 2 instances.
template <bool INT>
constexpr int kDeliverUnroll = INT ? 4 : 2;

// Shared memory of the delivery phase.  The tile's spiking neurons are
// listed by their CSR rows: lo[k] is row k's first synapse and off[k] the
// number of synapses in rows 0..k-1 (off[total] = all of them), so the
// block can stride one flat range of synapse indices.
struct SmemLists {
    uint32_t *lo;     // [tile size]
    uint32_t *off;    // [tile size + 1]
    uint32_t *woff;   // [warps] spike prefix per warp
    uint32_t *wsyn;   // [warps] synapse prefix per warp
    uint32_t *total;  // [2] spikes, synapses
};
__device__ __forceinline__ SmemLists smem_lists(uint32_t *base, uint32_t tile, uint32_t nw) {
    return SmemLists{base, base + tile, base + 2 * tile + 1, base + 2 * tile + 1 + nw, base + 2 * tile + 1 + 2 * nw};
}

// Delivery queue of the warp-specialised streaming kernel (step_kernel_ws):
// the tile warps push one cell per spiking neuron with synapses, and the
// block's delivery warps take the cells and deliver their rows, so a tile's
// delivery overlaps the next tiles' neuron passes.  A bounded multi-producer
// multi-consumer ring in shared memory: cell c holds {turn, row start, row
// end}; position p (claimed with an atomic counter) uses cell p % kWsCells,
// whose producer waits for turn == p, writes the row, then publishes turn =
// p + 1 (release); its consumer waits for turn == p + 1 (acquire), reads the
// row and hands the cell on with turn = p + kWsCells.  Every wait is bounded
// by %globaltimer (kWsWaitLimitNs), after which the kernel raises the engine
// error flag (kErrDeliveryQueue) and stops waiting.
constexpr uint32_t kWsCells = 256;
constexpr unsigned long long kWsWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ uint32_t ld_acquire_cta(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.cta.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_cta(uint32_t *p, uint32_t v) {
    asm volatile("st.release.cta.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct WsQueue {
    uint4 *cell;     // [kWsCells] {turn, rlo, rhi, -}
    uint32_t *ctr;   // [0] positions claimed by producers, [1] by consumers,
                     // [2] tile warps finished, [3] spikes counted
};

// Wait (bounded) until cell `turn` reads `want`; false when the wait gave up
// (the error flag is then set) or another wait of the launch already did.
__device__ __forceinline__ bool ws_wait_turn(const uint32_t *turn, uint32_t want, unsigned int *err) {
    unsigned long long t0 = 0;
    for (uint32_t polls = 1; ld_acquire_cta(turn) != want; ++polls) {
        if ((polls & 63u) == 0u) {
            const unsigned long long now = globaltimer_ns();
            if (t0 == 0) t0 = now;
            else if (now - t0 > kWsWaitLimitNs || *(volatile unsigned int *)err != 0u) {
                atomicCAS(err, 0u, kErrDeliveryQueue);
                return false;
            }
        }
        __nanosleep(32);
    }
    return true;
}

// `nd` is the tile's net descriptor (global memory, or a shared-memory copy
// staged before the launch's dependency wait); `t` is the absolute step,
// `tmod` = t % D and `k` = t - nd.t (the step within the launch group).
// PHASES: the record row and the window come from the phases the
// descriptor keeps beside its t, with a division only when a phase wraps
// within the group (else t % rec_rows and (t + 1) / win_steps directly).  ADEX: the net holds AdEx rows (else the Izhikevich path is
// the only one compiled into this instance).
// `ptab` is the parameter table (a shared-memory copy when it is small).
// LEAN: no net of the engine uses record rows, custom-tau synapses, the f32
// trace or watches; NOIO: nor an external current, a stimulus or windows.
// Their code is compiled out (the engine launches such an instance only
// then).
// A ring arrival: a no-return add whose L2 line is marked evict-first, so
// the random ring lines of a large net do not push the neuron state (read
// and written every step) out of L2.
__device__ __forceinline__ uint64_t ring_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
template <bool INT>
__device__ __forceinline__ void ring_add(uint32_t *word, uint32_t wb, uint64_t pol) {
    if (INT) asm volatile("red.global.add.L2::cache_hint.s32 [%0], %1, %2;" ::"l"(word), "r"(wb), "l"(pol) : "memory");
    else asm volatile("red.global.add.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(word), "f"(__uint_as_float(wb)), "l"(pol)
                      : "memory");
}

// WSQ (step_kernel_ws): the tile's threads are the producer warps of a
// delivery queue; they push their spiking neurons' rows into `wq` and count
// their spikes into *nspk (per warp) instead of compacting and delivering.
template <bool INT, int BLOCK, int NPT, bool RES, bool ADEX, bool PHASES, bool LEAN = false, bool NOIO = false,
          bool WSQ = false>
__device__ __forceinline__ void process_tile(const EngineDev *__restrict__ eng, const ParamRow *ptab, const NetDev &nd,
                                             const Tile &tile, uint64_t t, uint32_t tmod, uint32_t k, float *vs, float *us,
                                             float *ss, uint16_t *tks, const uint16_t *pis, const SmemLists &sl,
                                             const WsQueue *wq = nullptr, uint32_t *nspk = nullptr) {
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t flags = nd.flags;
    if (!(flags & kNetActive)) return;  // uniform across the block
    if (t >= nd.t_end) return;  // uniform across the block

    const uint32_t n = nd.n, n_pad = nd.n_pad, D = nd.D;
    const size_t slot_off = (size_t)tmod * n_pad;
    const float dt = nd.dt, decay_s = nd.decay_s;
    const float pkick = nd.pkick, kick = nd.kick, gauss_k = nd.gauss_k;
    const uint64_t nbase = nd.noise_step + (uint64_t)k * kNoiseStepMul;  // = noise_base_step(t, seed)
    const uint32_t tlast = nd.trace_last;
    uint32_t *__restrict__ ringw = (uint32_t *)nd.ring;
    const bool has_ext = !NOIO && (flags & kNetHasExt);
    const bool has_stim = !NOIO && (tile.flags & kTileHasStim);
    const bool windows = !NOIO && (flags & kNetWindows);
    const bool xsyn_on = !LEAN && (flags & kNetXsyn);
    bool win_end = false;
    uint32_t widx = 0;
    if (windows) {
        if constexpr (PHASES) {
            uint32_t ph = nd.wphase + k, wi = nd.widx0;
            if (ph >= nd.win_steps) {
                wi += ph / nd.win_steps;
                ph %= nd.win_steps;
            }
            win_end = ph == 0u;
            widx = wi - 1u;
        } else {
            win_end = mod_steps(t + 1, nd.win_steps) == 0u;
            widx = (uint32_t)div_steps(t + 1, nd.win_steps) - 1u;
        }
    }

    uint32_t li[NPT];
    bool valid[NPT];
    float v[NPT], u[NPT], s[NPT], ex[NPT];
    uint32_t rw[NPT], tk[NPT], pi[NPT];
#pragma unroll
    for (int q = 0; q < NPT; ++q) {
        const uint32_t off = q * BLOCK + threadIdx.x;
        li[q] = tile.start + off;
        valid[q] = off < tile.count && li[q] < n;
        if (valid[q]) {
            rw[q] = RES ? __ldcg(ringw + slot_off + li[q]) : ringw[slot_off + li[q]];
            v[q] = vs[off];
            u[q] = us[off];
            s[q] = ss[off];
            tk[q] = tks[off];
            pi[q] = pis[off];
            ex[q] = has_ext ? nd.ext[li[q]] : 0.0f;
        }
    }
    // warm L2 with the next step's ring slot (one prefetch per 32-byte
    // sector): in a quiet net that slot was last touched D steps ago and
    // would otherwise come from DRAM on the next step's critical path
    {
        const uint32_t nslot = tmod + 1u == D ? 0u : tmod + 1u;
        const uint32_t *nrow = ringw + (size_t)nslot * n_pad;
#pragma unroll
        for (int q = 0; q < NPT; ++q)
            if (valid[q] && (lane & 7) == 0) asm volatile("prefetch.global.L2 [%0];" ::"l"(nrow + li[q]));
        // and the next step's input values: a new row every step, which
        // would otherwise be a DRAM miss in the stimulated tiles
        if (has_stim) {
            const long long rel = (long long)t + 1 - nd.stim_t0;
            if (rel >= 0 && rel < (long long)nd.stim_len)
                for (uint32_t c = threadIdx.x * 8u; c < nd.n_inputs; c += BLOCK * 8u)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(nd.stim_buf + (size_t)rel * nd.n_inputs + c));
        }
    }

    bool spk[NPT];
    uint32_t rlo[NPT], rhi[NPT];  // CSR row of a spiking neuron, loaded as soon as it spikes
    const uint32_t *__restrict__ rowptr = nd.rowptr;
#pragma unroll
    for (int q = 0; q < NPT; ++q) {
        spk[q] = false;
        rlo[q] = rhi[q] = 0u;
        if (!valid[q]) continue;
        const uint32_t i = li[q];
        const uint32_t off = q * BLOCK + threadIdx.x;
        const float arr = INT ? __fmul_rn(__int2float_rn((int)rw[q]), 0x1p-12f)  // rt_get, kernels.rs:60
                              : __uint_as_float(rw[q]);
        if (rw[q] != 0u) ringw[slot_off + i] = 0u;
        const float sv = __fadd_rn(s[q], arr);
        float I = __fadd_rn(sv, ex[q]);
        if (xsyn_on) {
            // synapses with their own tau (cpu.rs:206-228): an arrival due
            // this step (its bit in this slot's words) adds w, then the
            // current joins the input and decays; a synapse arrives at most
            // once per step, so arrivals commute and fold into this loop
            uint32_t *pend = nd.xpend + (size_t)tmod * nd.xwords;
            for (uint32_t j = nd.xt_ptr[i], je = nd.xt_ptr[i + 1]; j < je; ++j) {
                const uint32_t k = nd.xt_idx[j];
                const uint32_t bit = 1u << (k & 31u);
                float x = nd.xsyn[k];
                const uint32_t word = RES ? __ldcg(pend + (k >> 5)) : pend[k >> 5];
                if (word & bit) {
                    x = __fadd_rn(x, nd.xw[k]);
                    atomicAnd(pend + (k >> 5), ~bit);  // other bits of the word belong to other targets
                }
                I = __fadd_rn(I, x);
                nd.xsyn[k] = __fmul_rn(x, nd.xdecay[k]);
            }
        }
        if (has_stim) {
            // the host provides the [steps x inputs] values covering every
            // launched step; the range check only guards the read
            const long long rel = (long long)t - nd.stim_t0;
            const float *row = (rel >= 0 && rel < (long long)nd.stim_len) ? nd.stim_buf + (size_t)rel * nd.n_inputs
                                                                          : nullptr;
            const uint32_t lo = nd.stim_ptr[i], hi = nd.stim_ptr[i + 1];
            if (row)
                for (uint32_t j = lo; j < hi; ++j) I = __fadd_rn(I, __fmul_rn(nd.stim_w[j], row[nd.stim_in[j]]));
        }
        // pidx bit 15 marks an AdEx row: an Izhikevich neuron reads only the
        // first 16 bytes of its parameter row
        const bool adex = ADEX && (pi[q] & kParamAdexBit) != 0u;
        const ParamRow &pr = ptab[pi[q] & ~kParamAdexBit];
        float p[10];
        const float4 p0 = *reinterpret_cast<const float4 *>(&pr.p[0]);
        p[0] = p0.x; p[1] = p0.y; p[2] = p0.z; p[3] = p0.w;
        if (ADEX && adex) {
            const float4 p1 = *reinterpret_cast<const float4 *>(&pr.p[4]);
            const float4 p2 = *reinterpret_cast<const float4 *>(&pr.p[8]);
            p[4] = p1.x; p[5] = p1.y; p[6] = p1.z; p[7] = p1.w;
            p[8] = p2.x; p[9] = p2.y;
        }
        const float gain = (ADEX && adex) ? p[0] : 1.0f;  // model/mod.rs:104-106, adex.rs:189-191
        if (pkick > 0.0f && noise_fires(noise_base_at(i, nbase), pkick)) I = __fadd_rn(I, __fmul_rn(kick, gain));
        if (gauss_k != 0.0f)
            I = __fadd_rn(I, __fmul_rn(__int2float_rn(gauss_numer(i, nbase)), __fmul_rn(gauss_k, gain)));
        bool sp;
        if (ADEX && adex) sp = adex_step(p, v[q], u[q], I, dt);
        else sp = izh_step(p, v[q], u[q], I, dt);
        // trace: 1 on spike, else one more multiply by decay_t (saturating at
        // the table's last entry, 0 or the subnormal fixed point)
        const uint32_t k0 = tk[q];
        uint32_t k = sp ? 0u : (k0 == kTraceZero ? k0 : (k0 < tlast ? k0 + 1u : tlast));
        if (!LEAN && (flags & kNetTraceF32)) {  // a readout tau too long for the step table: the f32 trace
            const float tr = nd.trace_f[i];
            const float tn = sp ? 1.0f : __fmul_rn(tr, nd.decay_t);  // cpu.rs:252-260
            if (__float_as_uint(tn) != __float_as_uint(tr)) nd.trace_f[i] = tn;
            k = k0;
        }
        const float snew = __fmul_rn(sv, decay_s);
        vs[off] = v[q];
        us[off] = u[q];
        // s and tk are written only when they change (quiet neurons keep s = 0
        // and a zero trace step after step)
        if (__float_as_uint(snew) != __float_as_uint(s[q])) ss[off] = snew;
        if (k != k0) tks[off] = (uint16_t)k;
        if (sp) {
            rlo[q] = rowptr[i];
            rhi[q] = rowptr[i + 1];
            nd.pn_total[i] += 1ull;
            if (!LEAN && (flags & kNetGridWatch)) {  // cpu.rs:293-304
                const uint32_t t32 = t < 0xFFFFFFFEull ? (uint32_t)t : 0xFFFFFFFEu;
                for (uint32_t g = 0; g < nd.gw_n; ++g) {
                    const int32_t k = nd.gw_map[(size_t)g * n_pad + i];
                    if (k >= 0) nd.gw_ls[nd.gw_off[g] + (uint32_t)k] = t32;
                }
            }
        }
        if (!LEAN && (flags & kNetWatch)) {  // state after the step, cpu.rs:311-324
            const uint32_t w = nd.watch_idx[i];
            if (w != kNoWatch) {
                const size_t pos = (size_t)(t & (kWatchCap - 1u));
                nd.watch_ring[(size_t)w * kWatchCap + pos] = v[q];
                nd.watch_ring[((size_t)nd.watch_n + w) * kWatchCap + pos] = u[q];
            }
        }
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

    // ---- spike record: one ballot word per warp and q
    if (!LEAN && (flags & kNetRecord)) {
        uint32_t row;
        if constexpr (PHASES) {
            row = nd.rphase + k;
            if (row >= nd.rec_rows) row %= nd.rec_rows;
        } else {
            row = mod_steps(t, nd.rec_rows);
        }
        const uint32_t words32 = n_pad >> 5;
#pragma unroll
        for (int q = 0; q < NPT; ++q) {
            const uint32_t mask = __ballot_sync(0xffffffffu, spk[q]);
            const uint32_t off = q * BLOCK + warp * 32;
            if (lane == 0 && off < tile.count) nd.rec_bits[(size_t)row * words32 + ((tile.start + off) >> 5)] = mask;
        }
    }
    if constexpr (WSQ) {
        // ---- push each spiking neuron's CSR row to the block's delivery
        // warps: one position claim per warp and q, then each spiking lane
        // fills its cell in turn (no block barrier)
        const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
        for (int q = 0; q < NPT; ++q) {
            *nspk += __popc(__ballot_sync(0xffffffffu, spk[q]));
            const bool has = spk[q] && rhi[q] > rlo[q];
            const uint32_t m = __ballot_sync(0xffffffffu, has);
            if (m == 0u) continue;
            const int leader = __ffs(m) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&wq->ctr[0], (uint32_t)__popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (has) {
                const uint32_t pos = base + __popc(m & lt);
                uint4 *c = wq->cell + (pos & (kWsCells - 1u));
                if (ws_wait_turn(&c->x, pos, eng->err)) {
                    c->y = rlo[q];
                    c->z = rhi[q];
                    st_release_cta(&c->x, pos + 1u);
                }
            }
        }
        return;
    }
    // ---- compaction: per-thread (spikes, synapses), block prefix sums
    uint32_t cnt = 0, syn = 0;
#pragma unroll
    for (int q = 0; q < NPT; ++q)
        if (spk[q]) {
            ++cnt;
            syn += rhi[q] - rlo[q];
        }
    // quiet tile: one block barrier, no scan, no delivery
    if (!__syncthreads_or(cnt != 0u)) return;
    uint32_t ic = cnt, is = syn;  // inclusive warp scans
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t yc = __shfl_up_sync(0xffffffffu, ic, o);
        const uint32_t ys = __shfl_up_sync(0xffffffffu, is, o);
        if (lane >= o) {
            ic += yc;
            is += ys;
        }
    }
    if (lane == 31) {
        sl.woff[warp] = ic;
        sl.wsyn[warp] = is;
    }
    __syncthreads();
    if (warp == 0) {
        uint32_t c = lane < NW ? sl.woff[lane] : 0u, y = lane < NW ? sl.wsyn[lane] : 0u;
        uint32_t jc = c, js = y;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t a = __shfl_up_sync(0xffffffffu, jc, o);
            const uint32_t b = __shfl_up_sync(0xffffffffu, js, o);
            if (lane >= o) {
                jc += a;
                js += b;
            }
        }
        if (lane < NW) {
            sl.woff[lane] = jc - c;
            sl.wsyn[lane] = js - y;
        }
        if (lane == 31) {
            sl.total[0] = jc;
            sl.total[1] = js;
        }
    }
    __syncthreads();
    {
        uint32_t pos = sl.woff[warp] + ic - cnt;
        uint32_t so = sl.wsyn[warp] + is - syn;
#pragma unroll
        for (int q = 0; q < NPT; ++q)
            if (spk[q]) {
                sl.lo[pos] = rlo[q];
                sl.off[pos] = so;
                ++pos;
                so += rhi[q] - rlo[q];
            }
    }
    const uint32_t total = sl.total[0], nsyn = sl.total[1];
    if (threadIdx.x == 0) sl.off[total] = nsyn;
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&eng->counters[tile.net].spikes_total, (unsigned long long)total);
    // ---- delivery: the block strides the flat synapse range; a thread
    // finds its row by binary search over off[], loads the synapse's 8-byte
    // record (target | delay << 24, weight bits), then adds the weight into
    // ring[(t + d) % D][tgt] with a no-return atomic
    const SynRec *__restrict__ csr = nd.syn;
    const bool wide = flags & kNetDelayWide;
    auto syn_at = [&](uint32_t f) {
        uint32_t lo = 0, hi = total;  // off[lo] <= f < off[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sl.off[mid] <= f) lo = mid;
            else hi = mid;
        }
        return sl.lo[lo] + (f - sl.off[lo]);
    };
    // the record's target and arrival slot
    auto unpack = [&](uint32_t j, const uint2 r, uint32_t &tg, uint32_t &slot) {
        const uint32_t d = wide ? (uint32_t)nd.delay16[j] : r.x >> kSynTgtBits;
        tg = wide ? r.x : r.x & kSynTgtMask;
        slot = tmod + d;
        if (slot >= D) slot -= D;
    };
    const uint64_t pol = ring_policy();
    auto add = [&](uint32_t slot, uint32_t tg, uint32_t wb) {
        const size_t idx = (size_t)slot * n_pad + tg;
        ring_add<INT>(ringw + idx, wb, pol);
    };
    if (!xsyn_on) {
        // U synapses per thread and pass, all their loads issued before any
        // add, so a tile with more synapses than threads pays one round trip
        // to the CSR per U block-widths
        constexpr int U = kDeliverUnroll<INT>;
        for (uint32_t f = threadIdx.x; f < nsyn; f += U * BLOCK) {
            // a thread past the end repeats its first synapse's loads (same
            // lines; cheaper in registers than predicated loads) and skips
            // the add
            uint32_t j[U], tg[U], sl_[U], wb[U];
            j[0] = syn_at(f);
#pragma unroll
            for (int q = 1; q < U; ++q) j[q] = f + q * BLOCK < nsyn ? syn_at(f + q * BLOCK) : j[0];
#pragma unroll
            for (int q = 0; q < U; ++q) {
                const uint2 r = *reinterpret_cast<const uint2 *>(csr + j[q]);
                unpack(j[q], r, tg[q], sl_[q]);
                wb[q] = r.y;
            }
#pragma unroll
            for (int q = 0; q < U; ++q)
                if (f + q * BLOCK < nsyn) add(sl_[q], tg[q], wb[q]);
        }
        __syncthreads();  // the next tile reuses the shared lists
        return;
    }
    for (uint32_t f = threadIdx.x; f < nsyn; f += BLOCK) {
        const uint32_t j = syn_at(f);
        const uint2 r = *reinterpret_cast<const uint2 *>(csr + j);
        uint32_t tg, slot;
        unpack(j, r, tg, slot);
        {
            const uint32_t k = nd.xmap[j];
            if (k != kNoXsyn) {  // its own current: mark the arrival (cpu.rs:270-273)
                atomicOr(nd.xpend + (size_t)slot * nd.xwords + (k >> 5), 1u << (k & 31u));
                continue;
            }
        }
        add(slot, tg, r.y);
    }
    // the next tile reuses the shared lists
    __syncthreads();
}

// Programmatic dependent launch: let the next kernel of the stream be
// scheduled now (griddepcontrol.launch_dependents), and wait until the
// previous one has completed and its memory is visible (griddepcontrol.wait).
// Both are no-ops for a kernel launched without the programmatic-serialization
// attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_enter() {
    pdl_trigger();
    pdl_wait();
}

// Copy the parameter table into shared memory when it has at most
// kSmemParamRows rows; returns the table the block reads from.
template <int BLOCK>
__device__ __forceinline__ const ParamRow *stage_params(const EngineDev *__restrict__ eng, ParamRow *s_ptab) {
    const uint32_t np = eng->n_params;
    if (np > kSmemParamRows) return eng->ptab;
    constexpr uint32_t kWords = sizeof(ParamRow) / 16;
    for (uint32_t w = threadIdx.x; w < np * kWords; w += BLOCK)
        reinterpret_cast<uint4 *>(s_ptab)[w] = reinterpret_cast<const uint4 *>(eng->ptab)[w];
    return s_ptab;
}

// Copy net descriptor `net` into shared memory (16-byte words, one per
// thread).
__device__ __forceinline__ void stage_net(const EngineDev *__restrict__ eng, uint32_t net, NetDev *s_nd) {
    constexpr uint32_t kNetWords = sizeof(NetDev) / 16;
    if (threadIdx.x < kNetWords)
        reinterpret_cast<uint4 *>(s_nd)[threadIdx.x] = reinterpret_cast<const uint4 *>(eng->nets + net)[threadIdx.x];
}

// ------------------------------------------------------ streaming kernel
// Block b processes tiles b, b + G, b + 2G, ... (G = gridDim.x).  The tile
// list and the net descriptors are written by host copies, which a launch
// always follows in full, and by advance_kernel (`t` and its phases), after
// which the next step launch is never programmatic (launch_step gives
// k_step = 0 a plain stream dependency).  So every block reads its first
// tile and stages the net descriptor, t included, before the dependency
// wait, overlapping the previous step's tail; after the wait only the
// step's own data is read.
//
// MULTI (engines of many nets: batches, the server): the block's tiles
// mostly belong to different nets, so it stages the records of its first
// kStageTiles tiles, and the descriptor of each net among them, before the
// wait as well: after the wait a tile costs one dependent round trip (its
// state) instead of three (record, descriptor, state).  The tile being
// processed reads its descriptor from one fixed shared-memory copy, refilled
// from the staged one when the net changes; tiles past the staged ones load
// their record and descriptor as they come.  Single-net engines restage the
// descriptor only when the net changes, which it never does.
constexpr uint32_t kStageTiles = 16;

// PLAIN: the lean instance; single-net, it also drops the input features
// (LEAN and NOIO), many-net only the others (LEAN).
template <bool INT, int BLOCK, int NPT, bool ADEX, bool MULTI, bool PLAIN>
__device__ __forceinline__ void step_body(const EngineDev *__restrict__ eng, uint32_t k_step) {
    pdl_trigger();
    constexpr uint32_t kNetWords = sizeof(NetDev) / 16;
    __shared__ uint32_t s_lists[smem_lists_words<BLOCK, NPT>()];
    __shared__ __align__(16) NetDev s_nd;
    __shared__ __align__(16) ParamRow s_ptab[kSmemParamRows];
    static_assert(sizeof(NetDev) % 16 == 0 && sizeof(ParamRow) % 16 == 0, "16-byte staging");
    static_assert(kNetWords <= BLOCK && kStageTiles <= BLOCK, "one 16-byte word per thread");
    const SmemLists sl = smem_lists(s_lists, BLOCK * NPT, BLOCK / 32);
    const uint32_t n_tiles = eng->n_tiles;
    if constexpr (!MULTI) {
        uint32_t tix = blockIdx.x;
        if (tix >= n_tiles) return;  // a fixed grid larger than the tile list
        Tile tile = eng->tiles[tix];
        stage_net(eng, tile.net, &s_nd);
        const ParamRow *ptab = stage_params<BLOCK>(eng, s_ptab);
        __syncthreads();
        pdl_wait();
        for (;;) {
            const uint32_t nx = tix + gridDim.x;
            const uint64_t t = s_nd.t + k_step;
            uint32_t tmod = s_nd.tmod + k_step;
            if (tmod >= s_nd.D) tmod %= s_nd.D;
            process_tile<INT, BLOCK, NPT, false, ADEX, false, PLAIN, PLAIN>(eng, ptab, s_nd, tile, t, tmod, k_step,
                                                             s_nd.v + tile.start, s_nd.u + tile.start,
                                                             s_nd.s + tile.start, s_nd.tk + tile.start,
                                                             s_nd.pidx + tile.start, sl);
            if (nx >= n_tiles) break;
            const Tile next = eng->tiles[nx];
            if (next.net != tile.net) {
                __syncthreads();  // every thread is done with the staged descriptor
                stage_net(eng, next.net, &s_nd);
                __syncthreads();
            }
            tix = nx;
            tile = next;
        }
    } else {
        __shared__ __align__(16) NetDev s_stage[kStageTiles];  // slot j: tile j's net, where it changes
        __shared__ __align__(16) Tile s_tile[kStageTiles];
        const uint32_t G = gridDim.x, b = blockIdx.x;
        if (b >= n_tiles) return;  // a fixed grid larger than the tile list
        const uint32_t m = (n_tiles - b + G - 1) / G;  // this block's tiles
        const uint32_t ms = m < kStageTiles ? m : kStageTiles;
        if (threadIdx.x < ms) s_tile[threadIdx.x] = eng->tiles[b + threadIdx.x * G];
        const ParamRow *ptab = stage_params<BLOCK>(eng, s_ptab);
        __syncthreads();
        for (uint32_t w = threadIdx.x; w < ms * kNetWords; w += BLOCK) {
            const uint32_t j = w / kNetWords, q = w - j * kNetWords;
            const uint32_t net = s_tile[j].net;
            const uint4 word = reinterpret_cast<const uint4 *>(eng->nets + net)[q];
            if (j == 0) reinterpret_cast<uint4 *>(&s_nd)[q] = word;
            else if (net != s_tile[j - 1].net) reinterpret_cast<uint4 *>(&s_stage[j])[q] = word;
        }
        __syncthreads();
        pdl_wait();
        uint32_t net = s_tile[0].net;
        for (uint32_t j = 0; j < m; ++j) {
            const Tile tile = j < kStageTiles ? s_tile[j] : eng->tiles[b + j * G];
            if (tile.net != net) {
                __syncthreads();  // every thread is done with the current descriptor
                if (j < kStageTiles) {
                    if (threadIdx.x < kNetWords)
                        reinterpret_cast<uint4 *>(&s_nd)[threadIdx.x] =
                            reinterpret_cast<const uint4 *>(&s_stage[j])[threadIdx.x];
                } else {
                    stage_net(eng, tile.net, &s_nd);
                }
                __syncthreads();
                net = tile.net;
            }
            const uint64_t t = s_nd.t + k_step;
            uint32_t tmod = s_nd.tmod + k_step;
            if (tmod >= s_nd.D) tmod %= s_nd.D;
            process_tile<INT, BLOCK, NPT, false, ADEX, true, PLAIN>(eng, ptab, s_nd, tile, t, tmod, k_step,
                                                            s_nd.v + tile.start, s_nd.u + tile.start,
                                                            s_nd.s + tile.start, s_nd.tk + tile.start,
                                                            s_nd.pidx + tile.start, sl);
        }
    }
}

template <bool INT, int BLOCK, int NPT, bool ADEX, bool MULTI, bool PLAIN>
__global__ void __launch_bounds__(BLOCK) step_kernel(const EngineDev *__restrict__ eng, uint32_t k_step) {
    step_body<INT, BLOCK, NPT, ADEX, MULTI, PLAIN>(eng, k_step);
}

// The plain single-net instance at one neuron per thread, held to 64
// registers (1,024 resident threads per SM), which its code fits without
// spilling.  Left to its own heuristic the compiler chose 56 registers and
// a spill on the critical path of the 100k step (128 x 1: 2.28 against
// 1.94 us per step, one box).  The other instances keep the compiler's
// choice: the same cap made them spill or run slower.
template <bool INT, int BLOCK, bool ADEX>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) step_kernel_r64(const EngineDev *__restrict__ eng,
                                                                       uint32_t k_step) {
    step_body<INT, BLOCK, 1, ADEX, false, true>(eng, k_step);
}

// ------------------------------------------- warp-specialised streaming kernel
// One net (single-net engines only).  Warps 0 .. BLOCK/32 - 1 are the tile
// warps: they stride the block's tiles (b, b + G, ...) doing the neuron pass
// and push each spiking neuron's CSR row into the block's delivery queue,
// never waiting on a block barrier.  The ws_warps(BLOCK) warps after them
// take the queued rows one per warp (lanes stride the row, U synapses per
// lane and pass, all their CSR loads in flight before the adds) and deliver
// them into the ring, so a tile's delivery overlaps the neuron passes of the
// block's later tiles.  They stop when every tile warp has finished and the
// queue is drained.  The last tile warp to finish adds the block's spike
// count to the net's total.
template <int BLOCK>
__host__ __device__ constexpr int ws_warps() {
    return BLOCK <= 128 ? 2 : 4;
}

template <bool INT, int BLOCK, int NPT, bool ADEX, bool PLAIN>
__global__ void __launch_bounds__(BLOCK + 32 * ws_warps<BLOCK>()) step_kernel_ws(const EngineDev *__restrict__ eng,
                                                                               uint32_t k_step) {
    pdl_trigger();
    constexpr int THREADS = BLOCK + 32 * ws_warps<BLOCK>();
    constexpr uint32_t P = BLOCK / 32;  // tile warps
    __shared__ __align__(16) NetDev s_nd;
    __shared__ __align__(16) ParamRow s_ptab[kSmemParamRows];
    __shared__ __align__(16) uint4 s_cell[kWsCells];
    __shared__ uint32_t s_ctr[4];
    static_assert(sizeof(NetDev) / 16 <= BLOCK, "one 16-byte word per thread");
    const uint32_t n_tiles = eng->n_tiles;
    uint32_t tix = blockIdx.x;
    if (tix >= n_tiles) return;  // a fixed grid larger than the tile list
    Tile tile = eng->tiles[tix];
    stage_net(eng, tile.net, &s_nd);
    const ParamRow *ptab = stage_params<THREADS>(eng, s_ptab);
    for (uint32_t c = threadIdx.x; c < kWsCells; c += THREADS) s_cell[c] = make_uint4(c, 0u, 0u, 0u);
    if (threadIdx.x < 4) s_ctr[threadIdx.x] = 0u;
    __syncthreads();
    pdl_wait();
    const WsQueue wq{s_cell, s_ctr};
    const uint64_t t = s_nd.t + k_step;
    uint32_t tmod = s_nd.tmod + k_step;
    if (tmod >= s_nd.D) tmod %= s_nd.D;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < BLOCK) {
        uint32_t nspk = 0;  // this warp's spikes (warp-uniform)
        const SmemLists none{};
        for (;;) {
            process_tile<INT, BLOCK, NPT, false, ADEX, false, PLAIN, PLAIN, true>(
                eng, ptab, s_nd, tile, t, tmod, k_step, s_nd.v + tile.start, s_nd.u + tile.start, s_nd.s + tile.start,
                s_nd.tk + tile.start, s_nd.pidx + tile.start, none, &wq, &nspk);
            tix += gridDim.x;
            if (tix >= n_tiles) break;
            tile = eng->tiles[tix];
        }
        if (lane == 0) {
            if (nspk) atomicAdd(&s_ctr[3], nspk);
            __threadfence_block();
            if (atomicAdd(&s_ctr[2], 1u) == P - 1u) {  // the last tile warp: the block's spike count
                __threadfence_block();
                const uint32_t total = *(volatile uint32_t *)&s_ctr[3];
                if (total) atomicAdd(&eng->counters[tile.net].spikes_total, (unsigned long long)total);
            }
        }
        return;
    }
    // ---- delivery warps
    constexpr int U = kDeliverUnroll<INT>;
    uint32_t *__restrict__ ringw = (uint32_t *)s_nd.ring;
    const SynRec *__restrict__ syn = s_nd.syn;
    const uint16_t *__restrict__ delay16 = s_nd.delay16;
    const uint32_t n_pad = s_nd.n_pad, D = s_nd.D;
    const bool wide = s_nd.flags & kNetDelayWide;
    const bool xsyn_on = !PLAIN && (s_nd.flags & kNetXsyn);
    const uint32_t e_total = s_nd.rowptr[s_nd.n];  // a queued row must lie inside the CSR
    const uint64_t pol = ring_policy();
    for (;;) {
        uint32_t pos = 0;
        if (lane == 0) pos = atomicAdd(&s_ctr[1], 1u);
        pos = __shfl_sync(0xffffffffu, pos, 0);
        const uint4 *c = s_cell + (pos & (kWsCells - 1u));
        // lane 0 waits for the row at `pos` (1), or for the end: every tile
        // warp finished and `pos` lies past the last claimed position (2),
        // or gives up (3); the warp follows its decision
        uint32_t st = 0;
        if (lane == 0) {
            unsigned long long t0 = 0;
            for (uint32_t polls = 1; st == 0u; ++polls) {
                if (ld_acquire_cta(&c->x) == pos + 1u) st = 1u;
                else if (ld_acquire_cta(&s_ctr[2]) == P && pos >= *(volatile uint32_t *)&s_ctr[0]) st = 2u;
                else if ((polls & 63u) == 0u) {
                    const unsigned long long now = globaltimer_ns();
                    if (t0 == 0) t0 = now;
                    else if (now - t0 > kWsWaitLimitNs || *(volatile unsigned int *)eng->err != 0u) {
                        atomicCAS(eng->err, 0u, kErrDeliveryQueue);
                        st = 3u;
                    }
                }
                if (st == 0u) __nanosleep(20);
            }
        }
        st = __shfl_sync(0xffffffffu, st, 0);
        if (st != 1u) break;
        __syncwarp();  // orders lane 0's acquire before the other lanes' reads
        const uint32_t rlo = c->y, rhi = c->z;
        __syncwarp();  // every lane has read the cell before lane 0 hands it on
        if (lane == 0) st_release_cta((uint32_t *)&c->x, pos + kWsCells);
        if (rlo > rhi || rhi > e_total) {  // never expected: report it rather than read outside the CSR
            if (lane == 0) atomicCAS(eng->err, 0u, kErrDeliveryQueue);
            continue;
        }
        const uint32_t cnt = rhi - rlo;
        for (uint32_t f = lane; f < cnt; f += 32u * U) {
            // a lane past the row's end repeats its first synapse's loads and
            // skips the add
            uint32_t j[U], tg[U], sl_[U], wb[U];
            j[0] = rlo + f;
#pragma unroll
            for (int q = 1; q < U; ++q) j[q] = f + 32u * q < cnt ? rlo + f + 32u * q : j[0];
#pragma unroll
            for (int q = 0; q < U; ++q) {
                const uint2 r = *reinterpret_cast<const uint2 *>(syn + j[q]);  // target | delay << 24, weight
                const uint32_t d = wide ? (uint32_t)delay16[j[q]] : r.x >> kSynTgtBits;
                tg[q] = wide ? r.x : r.x & kSynTgtMask;
                const uint32_t slot = tmod + d;
                sl_[q] = slot >= D ? slot - D : slot;
                wb[q] = r.y;
            }
#pragma unroll
            for (int q = 0; q < U; ++q) {
                if (f + 32u * q >= cnt) continue;
                if (xsyn_on) {
                    const uint32_t k = s_nd.xmap[j[q]];
                    if (k != kNoXsyn) {  // its own current: mark the arrival (cpu.rs:270-273)
                        atomicOr(s_nd.xpend + (size_t)sl_[q] * s_nd.xwords + (k >> 5), 1u << (k & 31u));
                        continue;
                    }
                }
                const size_t idx = (size_t)sl_[q] * n_pad + tg[q];
                ring_add<INT>(ringw + idx, wb[q], pol);
            }
        }
    }
}

// ------------------------------------------------------- resident kernel

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

constexpr unsigned long long kBarrierLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned int atom_add_release_gpu(unsigned int *p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Grid barrier for a cooperative launch.  Arrival: block-wide barrier, then
// thread 0 publishes the block's ring deliveries (gpu-scope fence) and
// increments the counter with a release atomic; the last block to arrive
// sees target - 1 and does not wait.  The others poll the counter with
// acquire loads; every 64 polls they check the error flag (another block
// gave up) and the %globaltimer limit, after which they flag the error and
// stop.  Returns false (for every thread of the block) when the launch must
// stop.
__device__ __forceinline__ bool grid_barrier(unsigned int *counter, unsigned int target, unsigned int *err,
                                             unsigned int *s_flag,
                                             unsigned long long limit_ns = kBarrierLimitNs) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int ok = 1u;
        if (atom_add_release_gpu(counter, 1u) + 1u < target) {
            const unsigned long long t0 = globaltimer_ns();
            for (uint32_t polls = 1;; ++polls) {
                if (ld_acquire_gpu(counter) >= target) break;
                if ((polls & 63u) == 0u) {
                    if (ld_acquire_gpu(err) != 0u) {
                        ok = 0u;
                        break;
                    }
                    if (globaltimer_ns() - t0 > limit_ns) {
                        atomicExch(err, kErrBarrier);
                        ok = 0u;
                        break;
                    }
                }
            }
        }
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0u;
}


template <bool INT, int BLOCK, int NPT, bool ADEX>
__global__ void __launch_bounds__(BLOCK) resident_kernel(const EngineDev *__restrict__ eng, uint32_t k0,
                                                         uint32_t nsteps) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int TILE = BLOCK * NPT;
    uint32_t *head = reinterpret_cast<uint32_t *>(smem);
    const SmemLists sl = smem_lists(head, TILE, BLOCK / 32);
    unsigned int *s_flag = head + smem_lists_words<BLOCK, NPT>();
    const uint32_t M = eng->block_neurons;
    float *sv = reinterpret_cast<float *>(smem + resident_head_bytes<BLOCK, NPT>());
    float *su = sv + M;
    float *ss = su + M;
    uint16_t *stk = reinterpret_cast<uint16_t *>(ss + M);
    uint16_t *spi = stk + M;
    __shared__ __align__(16) ParamRow s_ptab[kSmemParamRows];
    const ParamRow *ptab = stage_params<BLOCK>(eng, s_ptab);
    const uint32_t t_lo = eng->block_tiles[blockIdx.x], t_hi = eng->block_tiles[blockIdx.x + 1];

    for (uint32_t tix = t_lo; tix < t_hi; ++tix) {
        const Tile tile = eng->tiles[tix];
        const NetDev &nd = eng->nets[tile.net];
        for (uint32_t j = threadIdx.x; j < tile.count; j += BLOCK) {
            const uint32_t i = tile.start + j, o = tile.smem_off + j;
            sv[o] = nd.v[i];
            su[o] = nd.u[i];
            ss[o] = nd.s[i];
            stk[o] = nd.tk[i];
            spi[o] = nd.pidx[i];
        }
    }
    __syncthreads();

    for (uint32_t k = 0; k < nsteps; ++k) {
        for (uint32_t tix = t_lo; tix < t_hi; ++tix) {
            const Tile tile = eng->tiles[tix];
            const uint32_t o = tile.smem_off;
            const NetDev &nd = eng->nets[tile.net];
            const uint64_t t = nd.t + k0 + k;
            uint32_t tmod = nd.tmod + k0 + k;
            if (tmod >= nd.D) tmod %= nd.D;
            process_tile<INT, BLOCK, NPT, true, ADEX, false>(eng, ptab, nd, tile, t, tmod, k0 + k, sv + o, su + o,
                                                             ss + o, stk + o, spi + o, sl);
        }
        if (k + 1 < nsteps && !grid_barrier(eng->barrier, (k + 1) * gridDim.x, eng->err, s_flag)) break;
    }
    __syncthreads();

    for (uint32_t tix = t_lo; tix < t_hi; ++tix) {
        const Tile tile = eng->tiles[tix];
        const NetDev &nd = eng->nets[tile.net];
        for (uint32_t j = threadIdx.x; j < tile.count; j += BLOCK) {
            const uint32_t i = tile.start + j, o = tile.smem_off + j;
            nd.v[i] = sv[o];
            nd.u[i] = su[o];
            nd.s[i] = ss[o];
            nd.tk[i] = stk[o];
        }
    }
}

// ------------------------------------------------ per-kind launchers
template <typename... Args>
static cudaError_t launch_pdl(void (*kernel)(Args...), uint32_t grid, uint32_t block, cudaStream_t st, bool pdl,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = (pdl_enabled() && pdl) ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <bool INT, bool ADEX>
int StepKind<INT, ADEX>::occupancy(uint32_t block, uint32_t npt, int variant) {
    if (variant & kStepWS) {
#define X(B, P)                                                                                                 \
        if (block == B && npt == P) {                                                                           \
            int b = 0;                                                                                          \
            if ((variant & ~kStepWS) == kStepPlain)                                                             \
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, step_kernel_ws<INT, B, P, ADEX, true>,        \
                                                              B + 32 * ws_warps<B>(), 0);                       \
            else                                                                                                \
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, step_kernel_ws<INT, B, P, ADEX, false>,       \
                                                              B + 32 * ws_warps<B>(), 0);                       \
            return b;                                                                                           \
        }
        NE2B_WS_SHAPES(X)
#undef X
        return 0;
    }
#define X(B, P)                                                                                                 \
    if (block == B && npt == P) {                                                                               \
        int b = 0;                                                                                              \
        if (variant == kStepMulti)                                                                              \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, step_kernel<INT, B, P, ADEX, true, false>, B, 0);  \
        else if (variant == kStepMultiLean)                                                                     \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, step_kernel<INT, B, P, ADEX, true, true>, B, 0);   \
        else if (variant == kStepPlain && P == 1)                                                               \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, step_kernel_r64<INT, B, ADEX>, B, 0);              \
        else if (variant == kStepPlain)                                                                         \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, step_kernel<INT, B, P, ADEX, false, true>, B, 0);  \
        else                                                                                                    \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, step_kernel<INT, B, P, ADEX, false, false>, B, 0); \
        return b;                                                                                               \
    }
    NE2B_SHAPES(X)
#undef X
    return 0;
}

template <bool INT, bool ADEX>
cudaError_t StepKind<INT, ADEX>::launch(uint32_t block, uint32_t npt, int variant, const EngineDev *eng,
                                        uint32_t k_step, uint32_t grid, cudaStream_t st) {
    if (variant & kStepWS) {
#define X(B, P)                                                                                                    \
        if (block == B && npt == P)                                                                                \
            return (variant & ~kStepWS) == kStepPlain                                                              \
                       ? launch_pdl(step_kernel_ws<INT, B, P, ADEX, true>, grid, B + 32 * ws_warps<B>(), st,       \
                                    k_step > 0, eng, k_step)                                                       \
                       : launch_pdl(step_kernel_ws<INT, B, P, ADEX, false>, grid, B + 32 * ws_warps<B>(), st,      \
                                    k_step > 0, eng, k_step);
        NE2B_WS_SHAPES(X)
#undef X
        return cudaErrorInvalidValue;
    }
#define X(B, P)                                                                                                   \
    if (block == B && npt == P)                                                                                   \
        return variant == kStepMulti                                                                              \
                   ? launch_pdl(step_kernel<INT, B, P, ADEX, true, false>, grid, B, st, k_step > 0, eng, k_step)  \
               : variant == kStepMultiLean                                                                        \
                   ? launch_pdl(step_kernel<INT, B, P, ADEX, true, true>, grid, B, st, k_step > 0, eng, k_step)   \
               : variant == kStepPlain && P == 1                                                                  \
                   ? launch_pdl(step_kernel_r64<INT, B, ADEX>, grid, B, st, k_step > 0, eng, k_step)              \
               : variant == kStepPlain                                                                            \
                   ? launch_pdl(step_kernel<INT, B, P, ADEX, false, true>, grid, B, st, k_step > 0, eng, k_step)  \
                   : launch_pdl(step_kernel<INT, B, P, ADEX, false, false>, grid, B, st, k_step > 0, eng, k_step);
    NE2B_SHAPES(X)
#undef X
    return cudaErrorInvalidValue;
}

template <bool INT, bool ADEX>
int StepKind<INT, ADEX>::resident_occupancy(uint32_t block, uint32_t npt, size_t smem) {
#define X(B, P)                                                                                            \
    if (block == B && npt == P) {                                                                          \
        auto *k = resident_kernel<INT, B, P, ADEX>;                                                        \
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) \
            return 0;                                                                                      \
        int b = 0;                                                                                         \
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, B, smem) != cudaSuccess) return 0;        \
        return b;                                                                                          \
    }
    NE2B_SHAPES(X)
#undef X
    return 0;
}

template <bool INT, bool ADEX>
cudaError_t StepKind<INT, ADEX>::launch_resident(uint32_t block, uint32_t npt, const EngineDev *eng, uint32_t k0,
                                                 uint32_t nsteps, uint32_t grid, size_t smem, cudaStream_t st) {
#define X(B, P)                                                                                              \
    if (block == B && npt == P) {                                                                            \
        auto *k = resident_kernel<INT, B, P, ADEX>;                                                          \
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
        if (e != cudaSuccess) return e;                                                                      \
        void *args[] = {(void *)&eng, (void *)&k0, (void *)&nsteps};                                         \
        return cudaLaunchCooperativeKernel((const void *)k, dim3(grid), dim3(B), args, smem, st);            \
    }
    NE2B_SHAPES(X)
#undef X
    return cudaErrorInvalidValue;
}

}  // namespace ne2b
