// probe_floors.cu — measured floors that bound the step kernel on this GPU,
// printed as JSON lines (run by `python bench.py --floors`):
//   * launch: an empty kernel replayed from a CUDA graph of 64 launches,
//     with and without programmatic dependent launch (the per-step floor);
//   * stream: a grid-stride kernel that reads the 20 B per neuron a quiet
//     step reads (v, u, s f32; tk, pidx u16; one ring slot u32) and writes
//     v and u, at 100k and 1M neurons (the neuron-pass floor);
//   * atomics: no-return int32 atomic adds at hashed indices into a 64 MiB
//     (L2-resident) and a 2 GiB (HBM-sized) array, bare and with the target
//     and weight read from CSR-like arrays (the delivery floor).
// Standalone: no library code, sizes fixed below (about 2.8 GB of device
// memory at most), every index masked to its array.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#define CK(x)                                                                          \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "%s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            return 1;                                                                  \
        }                                                                              \
    } while (0)

__device__ __forceinline__ void pdl() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__global__ void empty_kernel(int *x) {
    pdl();
    if (threadIdx.x == 0 && blockIdx.x == 0xffffffu) x[0] = 1;  // never true; keeps the kernel alive
}

__global__ void stream_kernel(float *v, float *u, const float *s, const uint16_t *tk, const uint16_t *pi,
                              const uint32_t *ring, uint32_t n, uint32_t depth, uint32_t k) {
    pdl();
    const size_t slot = (size_t)(k % depth) * n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float a = v[i], b = u[i];
        const float c = s[i];
        const uint32_t r = ring[slot + i];
        const uint32_t q = (uint32_t)tk[i] + pi[i];
        a = a + 0.001f * (b + c + (float)r + (float)q);
        b = b * 0.999f;
        v[i] = a;
        u[i] = b;
    }
}

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__global__ void atomic_kernel(int *a, uint32_t mask, uint32_t per, uint32_t seed) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t k = 0; k < per; ++k) atomicAdd(a + (hash32(t * per + k + seed) & mask), 1);
}

__global__ void csr_atomic_kernel(int *a, const uint32_t *tgt, const int *w, uint64_t n) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(a + tgt[j], w[j]);
}

__global__ void fill_targets(uint32_t *tgt, int *w, uint64_t n, uint32_t mask) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        tgt[j] = hash32((uint32_t)j * 2654435761u) & mask;
        w[j] = 1;
    }
}

// Mean microseconds per launch of `launch(k)` replayed from a graph of
// `steps` launches, `reps` replays after 20 warm-up replays.
template <typename F>
static float graph_us(cudaStream_t st, F launch, int steps, int reps) {
    cudaGraph_t g;
    cudaGraphExec_t ge;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1.0f;
    for (int k = 0; k < steps; ++k) launch(k);
    if (cudaStreamEndCapture(st, &g) != cudaSuccess) return -1.0f;
    if (cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) return -1.0f;
    for (int w = 0; w < 20; ++w) cudaGraphLaunch(ge, st);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) cudaGraphLaunch(ge, st);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    return ms * 1000.0f / (float)(steps * reps);
}

static cudaLaunchConfig_t config(uint32_t grid, uint32_t block, cudaStream_t st, cudaLaunchAttribute *attr, int pdl_on) {
    cudaLaunchConfig_t c = {};
    c.gridDim = dim3(grid);
    c.blockDim = dim3(block);
    c.stream = st;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = pdl_on;
    c.attrs = attr;
    c.numAttrs = 1;
    return c;
}

int main() {
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    cudaStream_t st;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int *flag;
    CK(cudaMalloc(&flag, sizeof(int)));
    cudaLaunchAttribute attr[1];

    for (int pdl_on = 0; pdl_on < 2; ++pdl_on)
        for (int mult : {1, 2}) {
            cudaLaunchConfig_t c = config(sms * mult, 256, st, attr, pdl_on);
            const float us = graph_us(st, [&](int) { cudaLaunchKernelEx(&c, empty_kernel, flag); }, 64, 200);
            printf("{\"probe\": \"launch\", \"pdl\": %d, \"grid\": %d, \"us_per_launch\": %.3f}\n", pdl_on,
                   sms * mult, us);
        }

    for (uint32_t n : {100000u, 1000000u}) {
        const uint32_t depth = 170;
        float *v, *u, *s;
        uint16_t *tk, *pi;
        uint32_t *ring;
        CK(cudaMalloc(&v, 4ull * n));
        CK(cudaMalloc(&u, 4ull * n));
        CK(cudaMalloc(&s, 4ull * n));
        CK(cudaMalloc(&tk, 2ull * n));
        CK(cudaMalloc(&pi, 2ull * n));
        CK(cudaMalloc(&ring, 4ull * n * depth));
        CK(cudaMemset(v, 0, 4ull * n));
        CK(cudaMemset(u, 0, 4ull * n));
        CK(cudaMemset(s, 0, 4ull * n));
        CK(cudaMemset(tk, 0, 2ull * n));
        CK(cudaMemset(pi, 0, 2ull * n));
        CK(cudaMemset(ring, 0, 4ull * n * depth));
        float best = 1e30f;
        int best_grid = 0;
        for (int mult : {1, 2, 4, 8}) {
            cudaLaunchConfig_t c = config(sms * mult, 256, st, attr, 1);
            const float us = graph_us(
                st,
                [&](int k) {
                    cudaLaunchKernelEx(&c, stream_kernel, v, u, (const float *)s, (const uint16_t *)tk,
                                       (const uint16_t *)pi, (const uint32_t *)ring, n, depth, (uint32_t)k);
                },
                64, 50);
            if (us > 0.0f && us < best) {
                best = us;
                best_grid = sms * mult;
            }
        }
        printf("{\"probe\": \"stream\", \"neurons\": %u, \"bytes_per_neuron\": 20, \"grid\": %d, \"us_per_launch\": %.3f, "
               "\"gbs\": %.1f}\n",
               n, best_grid, best, 20.0 * n / best / 1e3);
        CK(cudaGetLastError());
        cudaFree(v);
        cudaFree(u);
        cudaFree(s);
        cudaFree(tk);
        cudaFree(pi);
        cudaFree(ring);
    }

    const uint64_t max_words = 1ull << 29;  // 2 GiB of int32
    const uint64_t events = 1ull << 26;     // 64 M per pass
    int *a;
    uint32_t *tgt;
    int *w;
    CK(cudaMalloc(&a, 4 * max_words));
    CK(cudaMemset(a, 0, 4 * max_words));
    CK(cudaMalloc(&tgt, 4 * events));
    CK(cudaMalloc(&w, 4 * events));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (uint64_t words : {(uint64_t)1 << 24, max_words}) {
        const uint32_t mask = (uint32_t)(words - 1);
        const uint32_t grid = sms * 8, block = 256;
        const uint32_t per = (uint32_t)(events / ((uint64_t)grid * block));
        atomic_kernel<<<grid, block, 0, st>>>(a, mask, per, 1);
        CK(cudaEventRecord(e0, st));
        for (int r = 0; r < 3; ++r) atomic_kernel<<<grid, block, 0, st>>>(a, mask, per, 7 + r);
        CK(cudaEventRecord(e1, st));
        CK(cudaEventSynchronize(e1));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        printf("{\"probe\": \"atomics\", \"array_mib\": %llu, \"kind\": \"hashed index\", \"g_per_s\": %.2f}\n",
               (unsigned long long)(words * 4 >> 20), 3.0 * grid * block * per / (ms * 1e6));
        fill_targets<<<grid, block, 0, st>>>(tgt, w, events, mask);
        csr_atomic_kernel<<<grid, block, 0, st>>>(a, tgt, w, events);
        CK(cudaEventRecord(e0, st));
        for (int r = 0; r < 3; ++r) csr_atomic_kernel<<<grid, block, 0, st>>>(a, tgt, w, events);
        CK(cudaEventRecord(e1, st));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(&ms, e0, e1));
        printf("{\"probe\": \"atomics\", \"array_mib\": %llu, \"kind\": \"target and weight read from arrays\", "
               "\"g_per_s\": %.2f}\n",
               (unsigned long long)(words * 4 >> 20), 3.0 * events / (ms * 1e6));
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    return 0;
}
