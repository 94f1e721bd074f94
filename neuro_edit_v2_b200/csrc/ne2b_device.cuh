// ne2b_device.cuh — per-neuron arithmetic of the B200 step kernel.
//
// Every float operation that the reference performs in f32 is written with an
// explicit round-to-nearest intrinsic (__fadd_rn, __fmul_rn, __fdiv_rn), so the
// compiler cannot contract it into an FMA or reorder it: the kernel computes
// exactly the IEEE-754 sequence of the reference CPU step (sim/src/cpu.rs:
// 216-261, sim/src/model/izh.rs:184-192, sim/src/model/adex.rs:163-176).
#pragma once
#include <stdint.h>

namespace ne2b {

// Counter-hash base of (neuron, step, seed): sim/src/state.rs:285-288.
__device__ __forceinline__ uint64_t noise_base(uint32_t i, uint64_t t, uint64_t seed) {
    return (uint64_t)i * 0x9E3779B97F4A7C15ull + t * 0xBF58476D1CE4E5B9ull + seed * 0x94D049BB133111EBull;
}
// The same base split into its step part (one per tile) and its neuron part:
// the sum is taken mod 2^64, so the grouping does not change the value.
__device__ __forceinline__ uint64_t noise_base_step(uint64_t t, uint64_t seed) {
    return t * 0xBF58476D1CE4E5B9ull + seed * 0x94D049BB133111EBull;
}
__device__ __forceinline__ uint64_t noise_base_at(uint32_t i, uint64_t step_part) {
    return (uint64_t)i * 0x9E3779B97F4A7C15ull + step_part;
}

// x mod m for the step counters: x < 2^32 in every run shorter than 5 days
// of 0.1 ms steps, where 32-bit division is used.
__device__ __forceinline__ uint32_t mod_steps(uint64_t x, uint32_t m) {
    return x <= 0xffffffffull ? (uint32_t)x % m : (uint32_t)(x % m);
}
__device__ __forceinline__ uint64_t div_steps(uint64_t x, uint32_t m) {
    return x <= 0xffffffffull ? (uint64_t)((uint32_t)x / m) : x / m;
}

// splitmix64 finaliser: sim/src/state.rs:289-293.
__device__ __forceinline__ uint64_t mix64(uint64_t h) {
    h ^= h >> 30;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 27;
    h *= 0x94D049BB133111EBull;
    h ^= h >> 31;
    return h;
}

// Poisson kick flag: state.rs:299-301, kernels.rs:128-130.
__device__ __forceinline__ bool noise_fires(uint64_t base, float p) {
    uint32_t h = (uint32_t)(mix64(base) >> 32);
    return __fmul_rn(__uint2float_rn(h), 2.3283064e-10f) < p;
}

// Gaussian current numerator for neuron i at the step whose noise step part
// (noise_base_step) is `step`: one 32-bit hash, x = i XOR the step part's
// low half through the lowbias32 mixer (C. Wellons' hash-prospector), then
// its high half folded in by one multiply-xorshift round; the four bytes of
// x summed (Irwin-Hall, 4 uniforms on [0, 255]) minus the mean 510.
// Multiplied by sd*sqrt(3)/256 it has mean 0 and variance 1 - 2^-16; tails
// end at +-3.45 sd.  32-bit integer operations only (the 64-bit splitmix64
// draw it replaces cost the 1M step 15% of its time), integer-exact, so CPU
// and GPU agree bit for bit.
__device__ __forceinline__ int32_t gauss_numer(uint32_t i, uint64_t step) {
    uint32_t x = i ^ (uint32_t)step;
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    x ^= (uint32_t)(step >> 32);
    x *= 0x9e3779b1u;
    x ^= x >> 16;
    const uint32_t pairs = (x & 0x00ff00ffu) + ((x >> 8) & 0x00ff00ffu);  // two 16-bit byte-pair sums
    return (int32_t)((pairs & 0xffffu) + (pairs >> 16)) - 510;
}

// Deterministic exp(x) for the AdEx step, in single precision: Cody-Waite
// reduction x = k*ln2 + r with fdlibm's split of ln2 (a 15-bit head, so
// k*head is exact for every k reached here, and a tail), the degree-7
// Taylor polynomial of e^r (coefficients 1/i! rounded to float) by Horner
// with fused multiply-adds, and the scale 2^k applied as two exact powers
// of two (so neither factor underflows before the last rounding).  Only
// rounded IEEE single operations, so the host copy (ne2b_expf) and the
// parity oracle reproduce it bit for bit; within 2 ulp of the correctly
// rounded exp on [-104, 88.8].
__device__ __forceinline__ float det_expf(float x) {
    if (x != x) return x;
    if (x > 88.8f) return __int_as_float(0x7f800000);
    if (x < -104.0f) return 0.0f;
    const float k = rintf(__fmul_rn(x, 0x1.715476p+0f));
    float r = __fmaf_rn(-k, 0x1.62e4p-1f, x);
    r = __fmaf_rn(-k, 0x1.7f7d1cp-20f, r);
    float p = 0x1.a01a02p-13f;
    p = __fmaf_rn(p, r, 0x1.6c16c2p-10f);
    p = __fmaf_rn(p, r, 0x1.111112p-7f);
    p = __fmaf_rn(p, r, 0x1.555556p-5f);
    p = __fmaf_rn(p, r, 0x1.555556p-3f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    const int ki = (int)k, k1 = ki / 2, k2 = ki - k1;  // both in [-75, 64]
    p = __fmul_rn(p, __int_as_float((k1 + 127) << 23));
    return __fmul_rn(p, __int_as_float((k2 + 127) << 23));
}

// Izhikevich step, sim/src/model/izh.rs:184-192 (CUDA text izh.rs:194-199):
// reset for last step's crossing, v with the old u, u with the new v.
__device__ __forceinline__ bool izh_step(const float *p, float &v, float &u, float I, float dt) {
    if (v >= 30.0f) {
        v = p[2];
        u = __fadd_rn(u, p[3]);
    }
    float a = __fmul_rn(__fmul_rn(0.04f, v), v);
    float b = __fmul_rn(5.0f, v);
    float sum = __fadd_rn(__fsub_rn(__fadd_rn(__fadd_rn(a, b), 140.0f), u), I);
    v = __fadd_rn(v, __fmul_rn(dt, sum));
    u = __fadd_rn(u, __fmul_rn(__fmul_rn(dt, p[0]), __fsub_rn(__fmul_rn(p[1], v), u)));
    return v >= 30.0f;
}

// AdEx step, sim/src/model/adex.rs:163-176 (CUDA text adex.rs:178-185):
// p = [C, gL, EL, VT, dT, a, tau_w, b, Vr, Vpeak].
__device__ __forceinline__ bool adex_step(const float *p, float &v, float &w, float I, float dt) {
    if (v >= p[9]) {
        v = p[8];
        w = __fadd_rn(w, p[7]);
    }
    const float arg = fminf(__fdiv_rn(__fsub_rn(v, p[3]), p[4]), 10.0f);
    const float ex = det_expf(arg);
    // -p1*(v-p2) + p1*p4*ex - w + I
    float acc = __fmul_rn(-p[1], __fsub_rn(v, p[2]));
    acc = __fadd_rn(acc, __fmul_rn(__fmul_rn(p[1], p[4]), ex));
    acc = __fadd_rn(__fsub_rn(acc, w), I);
    v = __fadd_rn(v, __fdiv_rn(__fmul_rn(dt, acc), p[0]));
    float accw = __fsub_rn(__fmul_rn(p[5], __fsub_rn(v, p[2])), w);
    w = __fadd_rn(w, __fdiv_rn(__fmul_rn(dt, accw), p[6]));
    const bool spiked = v >= p[9];
    if (v > p[9]) v = p[9];
    return spiked;
}

}  // namespace ne2b
