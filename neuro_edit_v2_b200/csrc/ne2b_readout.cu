// ne2b_readout.cu — readout training on the GPU, from features that are
// already on the device (a batch's per-window spike counts) or that the
// caller passes: the multi-class ridge of sim/src/readout.rs:190-252
// (`fit_ridge_multi`), solved in the dual.
//
//   1. column means mu (f64, rows summed in order) and the centred design
//      Xc = x - mu (f64);
//   2. the Gram matrix G = Xc Xc^T + lambda I: tiled in shared memory, each
//      thread owning 2 x 2 entries and summing each dot product exactly as
//      the reference does (four accumulators by column mod 4, the tail
//      apart, then tail + ((a0 + a1) + a2) + a3);
//   3. Cholesky G = L L^T in place, right-looking: column j is divided by
//      sqrt(G[j][j]), then the trailing lower triangle loses
//      L[i][j] L[k][j] — every entry meets its subtractions in the same
//      order k = 0, 1, ... as the reference's left-looking loop;
//   4. per class, L z = y and L^T a = z on the host (T^2 work), in the
//      reference's loop order;
//   5. w = Xc^T a on the device (rows summed in order), bias on the host.
//
// Every f64 operation is an explicit round-to-nearest intrinsic, so nothing
// is contracted into an FMA: the weights equal the reference's bit for bit.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "ne2b_engine.h"
#include "ne2b_handles.h"

#define NE2B_CUDA(call)                                      \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) return cuda_error(_e, #call); \
    } while (0)
#define NE2B_TRY(call)                 \
    do {                               \
        ne2b_status _s = (call);       \
        if (_s != NE2B_OK) return _s;  \
    } while (0)

namespace ne2b {
namespace {

constexpr uint32_t kGramTile = 32;  // 32 x 32 Gram entries per block, 16 x 16 threads
constexpr uint32_t kGramK = 32;     // columns staged per pass (a multiple of 4)

__global__ void col_mean_kernel(const float *__restrict__ x, uint32_t t, uint32_t f, double *__restrict__ mu) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= f) return;
    double s = 0.0;
    for (uint32_t r = 0; r < t; ++r) s = __dadd_rn(s, (double)x[(size_t)r * f + c]);
    mu[c] = __ddiv_rn(s, (double)t);
}

__global__ void center_kernel(const float *__restrict__ x, uint64_t n, uint32_t f, const double *__restrict__ mu,
                              double *__restrict__ xc) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        xc[i] = __dsub_rn((double)x[i], mu[i % f]);
}

// Lower-triangle tiles (bi >= bj) of G = Xc Xc^T; the diagonal gets lambda;
// both halves are written.
__global__ void __launch_bounds__(256) gram_kernel(const double *__restrict__ xc, uint32_t t, uint32_t f,
                                                   double lambda, double *__restrict__ g) {
    __shared__ double sa[kGramTile][kGramK + 1];
    __shared__ double sb[kGramTile][kGramK + 1];
    // linear block id -> (bi, bj), bj <= bi
    const uint32_t id = blockIdx.x;
    uint32_t bi = (uint32_t)((sqrt(8.0 * id + 1.0) - 1.0) / 2.0);
    while ((bi + 1) * (bi + 2) / 2 <= id) ++bi;
    while (bi * (bi + 1) / 2 > id) --bi;
    const uint32_t bj = id - bi * (bi + 1) / 2;
    const uint32_t i0 = bi * kGramTile, j0 = bj * kGramTile;
    const uint32_t tx = threadIdx.x & 15u, ty = threadIdx.x >> 4;
    double acc[2][2][4] = {};
    double tail[2][2] = {};
    const uint32_t f4 = f / 4u * 4u;
    for (uint32_t k0 = 0; k0 < f; k0 += kGramK) {
        for (uint32_t e = threadIdx.x; e < kGramTile * kGramK; e += 256) {
            const uint32_t r = e / kGramK, c = e % kGramK;
            const bool in_c = k0 + c < f;
            sa[r][c] = (i0 + r < t && in_c) ? xc[(size_t)(i0 + r) * f + k0 + c] : 0.0;
            sb[r][c] = (j0 + r < t && in_c) ? xc[(size_t)(j0 + r) * f + k0 + c] : 0.0;
        }
        __syncthreads();
        const uint32_t kn = min(kGramK, f - k0);
        uint32_t c = 0;
        // k0 and f4 are multiples of 4: whole groups of four below f4, each
        // column into its accumulator (static indices keep them in registers)
        for (; c + 4u <= kn && k0 + c + 4u <= f4; c += 4u)
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        acc[a][b][q] = __dadd_rn(acc[a][b][q], __dmul_rn(sa[ty * 2 + a][c + q], sb[tx * 2 + b][c + q]));
        for (; c < kn; ++c)  // the columns from f4 on
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
                    tail[a][b] = __dadd_rn(tail[a][b], __dmul_rn(sa[ty * 2 + a][c], sb[tx * 2 + b][c]));
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const uint32_t i = i0 + ty * 2 + a, j = j0 + tx * 2 + b;
            if (i >= t || j >= t || j > i) continue;
            const double *q = acc[a][b];
            double s = __dadd_rn(tail[a][b], __dadd_rn(__dadd_rn(__dadd_rn(q[0], q[1]), q[2]), q[3]));
            if (i == j) s = __dadd_rn(s, lambda);
            g[(size_t)i * t + j] = s;
            g[(size_t)j * t + i] = s;
        }
}

// Column j below the diagonal divided by sqrt(G[j][j]); a non-positive
// pivot raises *bad (the matrix is not positive definite).
__global__ void chol_column_kernel(double *g, uint32_t t, uint32_t j, unsigned int *bad) {
    const double d = g[(size_t)j * t + j];
    if (d <= 0.0) {  // the reference's test (readout.rs:155): a NaN pivot carries on
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(bad, 1u);
        return;
    }
    const double ljj = __dsqrt_rn(d);
    const uint32_t i = j + 1u + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < t) g[(size_t)i * t + j] = __ddiv_rn(g[(size_t)i * t + j], ljj);
}

// G[i][k] -= L[i][j] L[k][j] for j < k <= i; G[j][j] becomes sqrt(G[j][j]).
__global__ void chol_update_kernel(double *g, uint32_t t, uint32_t j, const unsigned int *bad) {
    if (*bad) return;
    const uint32_t k = j + 1u + blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = j + 1u + blockIdx.y * blockDim.y + threadIdx.y;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0)
        g[(size_t)j * t + j] = __dsqrt_rn(g[(size_t)j * t + j]);
    if (i >= t || k > i) return;
    g[(size_t)i * t + k] = __dsub_rn(g[(size_t)i * t + k], __dmul_rn(g[(size_t)i * t + j], g[(size_t)k * t + j]));
}

// w[c][q] = sum over rows r (in order) of a[c][r] xc[r][q].
__global__ void weights_kernel(const double *__restrict__ xc, const double *__restrict__ a, uint32_t t, uint32_t f,
                               uint32_t k, double *__restrict__ w) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t c = blockIdx.y;
    if (q >= f) return;
    double s = 0.0;
    for (uint32_t r = 0; r < t; ++r) s = __dadd_rn(s, __dmul_rn(a[(size_t)c * t + r], xc[(size_t)r * f + q]));
    w[(size_t)c * f + q] = s;
}

// trial r's features: window counts [windows][n] of one net (u16 -> f32)
__global__ void gather_counts_kernel(const uint16_t *const *__restrict__ win, uint32_t n, uint32_t n_pad,
                                     uint32_t windows, float *__restrict__ x) {
    const uint32_t r = blockIdx.y;
    const uint32_t f = windows * n;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < f; q += gridDim.x * blockDim.x) {
        const uint32_t wdx = q / n, i = q - wdx * n;
        x[(size_t)r * f + q] = (float)win[r][(size_t)wdx * n_pad + i];
    }
}

struct DevBuf {
    std::vector<void *> ps;
    cudaStream_t st;
    explicit DevBuf(cudaStream_t s) : st(s) {}
    ~DevBuf() {
        for (void *p : ps) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
    }
    template <class T>
    ne2b_status get(T **p, size_t count) {
        void *q = nullptr;
        const cudaError_t e = cudaMallocAsync(&q, sizeof(T) * (count ? count : 1), st);
        if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync (readout)");
        ps.push_back(q);
        *p = (T *)q;
        return NE2B_OK;
    }
};

ne2b_status check_labels(const uint32_t *labels, uint32_t t, uint32_t f, uint32_t k) {
    if (t < 2 || k < 2 || f == 0)
        return set_error(NE2B_EINVAL, "fit_ridge_multi: need T >= 2, K >= 2, F >= 1 (T=%u F=%u K=%u)", t, f, k);
    if (t > 32768) return set_error(NE2B_UNSUPPORTED, "fit_ridge_multi: at most 32768 rows (T=%u)", t);
    for (uint32_t r = 0; r < t; ++r)
        if (labels[r] >= k) return set_error(NE2B_EINVAL, "fit_ridge_multi: label %u outside 0..%u", labels[r], k);
    return NE2B_OK;
}

// The fit on a device design x[T x F] (f32) on stream `st`.
ne2b_status fit_on_device(const float *x, uint32_t t, uint32_t f, const uint32_t *labels, uint32_t k, double lambda,
                          cudaStream_t st, double *w_out) {
    DevBuf buf(st);
    double *mu = nullptr, *xc = nullptr, *g = nullptr, *a = nullptr, *w = nullptr;
    unsigned int *bad = nullptr;
    NE2B_TRY(buf.get(&mu, f));
    NE2B_TRY(buf.get(&xc, (size_t)t * f));
    NE2B_TRY(buf.get(&g, (size_t)t * t));
    NE2B_TRY(buf.get(&a, (size_t)t * k));
    NE2B_TRY(buf.get(&w, (size_t)f * k));
    NE2B_TRY(buf.get(&bad, 1));
    NE2B_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned int), st));
    col_mean_kernel<<<(f + 255) / 256, 256, 0, st>>>(x, t, f, mu);
    const uint64_t n = (uint64_t)t * f;
    center_kernel<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 64), 256, 0, st>>>(x, n, f, mu, xc);
    const uint32_t nt = (t + kGramTile - 1) / kGramTile;
    gram_kernel<<<nt * (nt + 1) / 2, 256, 0, st>>>(xc, t, f, lambda, g);
    for (uint32_t j = 0; j < t; ++j) {
        const uint32_t below = t - j - 1u;
        chol_column_kernel<<<(below + 255) / 256 + (below == 0), 256, 0, st>>>(g, t, j, bad);
        const dim3 blk(16, 16), grd((below + 15) / 16 + (below == 0), (below + 15) / 16 + (below == 0));
        chol_update_kernel<<<grd, blk, 0, st>>>(g, t, j, bad);
    }
    NE2B_CUDA(cudaGetLastError());
    // the triangular solves on the host, in the reference's order
    std::vector<double> L((size_t)t * t), mu_h(f);
    unsigned int bad_h = 0;
    NE2B_CUDA(cudaMemcpyAsync(L.data(), g, sizeof(double) * L.size(), cudaMemcpyDeviceToHost, st));
    NE2B_CUDA(cudaMemcpyAsync(mu_h.data(), mu, sizeof(double) * f, cudaMemcpyDeviceToHost, st));
    NE2B_CUDA(cudaMemcpyAsync(&bad_h, bad, sizeof bad_h, cudaMemcpyDeviceToHost, st));
    NE2B_CUDA(cudaStreamSynchronize(st));
    std::vector<double> ybar(k, 0.0), ah((size_t)t * k, 0.0), z(t);
    for (uint32_t r = 0; r < t; ++r) ybar[labels[r]] += 1.0 / (double)t;
    if (!bad_h)
        for (uint32_t c = 0; c < k; ++c) {
            double *ac = ah.data() + (size_t)c * t;
            for (uint32_t i = 0; i < t; ++i) {
                double s = (labels[i] == c ? 1.0 : 0.0) - ybar[c];
                for (uint32_t q = 0; q < i; ++q) s -= L[(size_t)i * t + q] * z[q];
                z[i] = s / L[(size_t)i * t + i];
            }
            for (uint32_t i = t; i-- > 0;) {
                double s = z[i];
                for (uint32_t q = i + 1; q < t; ++q) s -= L[(size_t)q * t + i] * ac[q];
                ac[i] = s / L[(size_t)i * t + i];
            }
        }
    NE2B_CUDA(cudaMemcpyAsync(a, ah.data(), sizeof(double) * ah.size(), cudaMemcpyHostToDevice, st));
    weights_kernel<<<dim3((f + 255) / 256, k), 256, 0, st>>>(xc, a, t, f, k, w);
    NE2B_CUDA(cudaGetLastError());
    std::vector<double> wh((size_t)f * k);
    NE2B_CUDA(cudaMemcpyAsync(wh.data(), w, sizeof(double) * wh.size(), cudaMemcpyDeviceToHost, st));
    NE2B_CUDA(cudaStreamSynchronize(st));
    for (uint32_t c = 0; c < k; ++c) {
        double *wc = w_out + (size_t)c * (f + 1);
        memcpy(wc, wh.data() + (size_t)c * f, sizeof(double) * f);
        double dot = 0.0;
        for (uint32_t q = 0; q < f; ++q) dot += wc[q] * mu_h[q];
        wc[f] = ybar[c] - dot;
    }
    return NE2B_OK;
}

}  // namespace
}  // namespace ne2b

using ne2b::cuda_error;
using ne2b::set_error;

extern "C" {

ne2b_status ne2b_fit_ridge_multi(const float *x, uint32_t t, uint32_t f, const uint32_t *labels, uint32_t k,
                                 double lambda, int device, double *w) {
    if (!x || !labels || !w) return set_error(NE2B_EINVAL, "ne2b_fit_ridge_multi: null argument");
    const ne2b_status cs = ne2b::check_labels(labels, t, f, k);
    if (cs != NE2B_OK) return cs;
    try {
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) return ne2b::cuda_error(e, "cudaSetDevice");
        cudaPointerAttributes attr{};
        const bool on_device = cudaPointerGetAttributes(&attr, x) == cudaSuccess && attr.type == cudaMemoryTypeDevice;
        cudaGetLastError();  // a host pointer may leave a benign error behind
        cudaStream_t st = nullptr;
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e != cudaSuccess) return ne2b::cuda_error(e, "cudaStreamCreate");
        ne2b_status r = NE2B_OK;
        {
            ne2b::DevBuf buf(st);
            const float *xd = x;
            if (!on_device) {
                float *p = nullptr;
                r = buf.get(&p, (size_t)t * f);
                if (r == NE2B_OK)
                    r = ne2b::cuda_error(cudaMemcpyAsync(p, x, sizeof(float) * (size_t)t * f, cudaMemcpyHostToDevice, st),
                                         "design upload");
                xd = p;
            }
            if (r == NE2B_OK) r = ne2b::fit_on_device(xd, t, f, labels, k, lambda, st, w);
        }
        cudaStreamDestroy(st);
        return r;
    } catch (const std::bad_alloc &) {
        return set_error(NE2B_ENOMEM, "host allocation failed");
    }
}

ne2b_status ne2b_batch_fit_ridge_multi(ne2b_batch *b, const uint32_t *nets, uint32_t t, uint32_t windows,
                                       const uint32_t *labels, uint32_t k, double lambda, uint32_t *n_features,
                                       double *w) {
    if (!b || !nets || !labels || !w) return set_error(NE2B_EINVAL, "ne2b_batch_fit_ridge_multi: null argument");
    if (t == 0 || windows == 0) return set_error(NE2B_EINVAL, "ne2b_batch_fit_ridge_multi: no trials or no windows");
    try {
        std::vector<const uint16_t *> win(t);
        uint32_t n = 0, n_pad = 0;
        for (uint32_t r = 0; r < t; ++r) {
            if (nets[r] >= b->slots.size()) return set_error(NE2B_EINVAL, "net %u out of range", nets[r]);
            ne2b::NetHost *h = b->eng.net(b->slots[nets[r]]);
            if (!h) return set_error(NE2B_EINVAL, "net %u has no network", nets[r]);
            if (r == 0) {
                n = h->n;
                n_pad = h->n_pad;
            } else if (h->n != n) {
                return set_error(NE2B_EINVAL, "the trials' nets differ in size (%u and %u neurons)", n, h->n);
            }
            const uint64_t done = h->dev.win_steps ? h->t / h->dev.win_steps : 0;
            if (!h->dev.win_out || done < windows || windows > h->dev.max_windows)
                return set_error(NE2B_EINVAL, "net %u has %llu of the %u windows asked for", nets[r],
                                 (unsigned long long)done, windows);
            win[r] = h->dev.win_out;
        }
        const uint64_t f64 = (uint64_t)windows * n;
        if (f64 > 0xffffffffull) return set_error(NE2B_UNSUPPORTED, "more than 2^32-1 features");
        const uint32_t f = (uint32_t)f64;
        const ne2b_status cs = ne2b::check_labels(labels, t, f, k);
        if (cs != NE2B_OK) return cs;
        if (n_features) *n_features = f;
        cudaStream_t st = b->eng.stream();  // after the batch's queued steps
        ne2b::DevBuf buf(st);
        const uint16_t **wd = nullptr;
        float *x = nullptr;
        NE2B_TRY(buf.get(&wd, t));
        NE2B_TRY(buf.get(&x, (size_t)t * f));
        NE2B_CUDA(cudaMemcpyAsync(wd, win.data(), sizeof(void *) * t, cudaMemcpyHostToDevice, st));
        ne2b::gather_counts_kernel<<<dim3((f + 255) / 256 < 1024 ? (f + 255) / 256 : 1024, t), 256, 0, st>>>(
            wd, n, n_pad, windows, x);
        NE2B_CUDA(cudaGetLastError());
        return ne2b::fit_on_device(x, t, f, labels, k, lambda, st, w);
    } catch (const std::bad_alloc &) {
        return set_error(NE2B_ENOMEM, "host allocation failed");
    }
}

}  // extern "C"
