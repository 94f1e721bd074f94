// ne2b_readout.cu — readout training on the GPU, from features that are
// already on the device (a batch's per-window spike counts) or that the
// caller passes: the multi-class ridge of sim/src/readout.rs:190-252
// (`fit_ridge_multi`), solved in the dual, and the binary ridge of
// readout.rs:103-141 (`fit_ridge`), solved in the primal.
//
// fit_ridge_multi:
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
// fit_ridge: the (F + 1) x (F + 1) normal matrix, each entry summed over the
// rows in order as the reference accumulates it, the bias column, lambda on
// the diagonal and off the bias again ((s + lambda) - lambda, as there), the
// same Cholesky, and the solve on the host; a matrix that is not positive
// definite is refactored with 1e-3 + lambda more on the diagonal (from a
// copy kept on the device), then gives zeros.
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

// Upper-triangle tiles (bi <= bj) of the normal matrix: a[i][j] = sum over
// rows r, in order, of x[r][i] x[r][j] (f32 read as f64); both halves of
// the (F + 1)-wide matrix are written.
__global__ void __launch_bounds__(256) normal_kernel(const float *__restrict__ x, uint32_t t, uint32_t f,
                                                     double *__restrict__ a) {
    __shared__ double si[kGramK][kGramTile + 1];
    __shared__ double sj[kGramK][kGramTile + 1];
    const uint32_t id = blockIdx.x;
    uint32_t bj = (uint32_t)((sqrt(8.0 * id + 1.0) - 1.0) / 2.0);
    while ((bj + 1) * (bj + 2) / 2 <= id) ++bj;
    while (bj * (bj + 1) / 2 > id) --bj;
    const uint32_t bi = id - bj * (bj + 1) / 2;  // bi <= bj
    const uint32_t i0 = bi * kGramTile, j0 = bj * kGramTile, nf = f + 1u;
    const uint32_t tx = threadIdx.x & 15u, ty = threadIdx.x >> 4;
    double acc[2][2] = {};
    for (uint32_t r0 = 0; r0 < t; r0 += kGramK) {
        for (uint32_t e = threadIdx.x; e < kGramK * kGramTile; e += 256) {
            const uint32_t r = e / kGramTile, c = e % kGramTile;
            const bool in_r = r0 + r < t;
            si[r][c] = (in_r && i0 + c < f) ? (double)x[(size_t)(r0 + r) * f + i0 + c] : 0.0;
            sj[r][c] = (in_r && j0 + c < f) ? (double)x[(size_t)(r0 + r) * f + j0 + c] : 0.0;
        }
        __syncthreads();
        const uint32_t rn = min(kGramK, t - r0);
        for (uint32_t r = 0; r < rn; ++r)
#pragma unroll
            for (int p = 0; p < 2; ++p)
#pragma unroll
                for (int q = 0; q < 2; ++q)
                    acc[p][q] = __dadd_rn(acc[p][q], __dmul_rn(si[r][ty * 2 + p], sj[r][tx * 2 + q]));
        __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const uint32_t i = i0 + ty * 2 + p, j = j0 + tx * 2 + q;
            if (i >= f || j >= f || i > j) continue;
            a[(size_t)i * nf + j] = acc[p][q];
            a[(size_t)j * nf + i] = acc[p][q];
        }
}

// The bias column (sum of each feature over the rows, in order), the
// right-hand side b[i] = sum of x[r][i] y[r], and b[f] = sum of y.
__global__ void bias_rhs_kernel(const float *__restrict__ x, const float *__restrict__ y, uint32_t t, uint32_t f,
                                double *__restrict__ a, double *__restrict__ b) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nf = f + 1u;
    if (j > f) return;
    double s = 0.0, sb = 0.0;
    for (uint32_t r = 0; r < t; ++r) {
        const double yr = (double)y[r];
        if (j < f) {
            const double xv = (double)x[(size_t)r * f + j];
            s = __dadd_rn(s, xv);
            sb = __dadd_rn(sb, __dmul_rn(xv, yr));
        } else {
            sb = __dadd_rn(sb, yr);
        }
    }
    b[j] = sb;
    if (j < f) {
        a[(size_t)j * nf + f] = s;
        a[(size_t)f * nf + j] = s;
    } else {
        double ones = 0.0;
        for (uint32_t r = 0; r < t; ++r) ones = __dadd_rn(ones, 1.0);
        a[(size_t)f * nf + f] = ones;
    }
}

// a[i][i] += add for every i; with `unbias`, a[f][f] then loses lambda again.
__global__ void diag_kernel(double *a, uint32_t n, double add, bool unbias, double lambda) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = __dadd_rn(a[(size_t)i * n + i], add);
    if (unbias && i + 1u == n) v = __dsub_rn(v, lambda);
    a[(size_t)i * n + i] = v;
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

// G = L L^T in place (lower triangle; n launches of two kernels); true when
// G is positive definite.
ne2b_status cholesky(double *g, uint32_t n, unsigned int *bad, cudaStream_t st, bool *pd) {
    NE2B_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned int), st));
    for (uint32_t j = 0; j < n; ++j) {
        const uint32_t below = n - j - 1u;
        chol_column_kernel<<<(below + 255) / 256 + (below == 0), 256, 0, st>>>(g, n, j, bad);
        const dim3 blk(16, 16), grd((below + 15) / 16 + (below == 0), (below + 15) / 16 + (below == 0));
        chol_update_kernel<<<grd, blk, 0, st>>>(g, n, j, bad);
    }
    NE2B_CUDA(cudaGetLastError());
    unsigned int bad_h = 0;
    NE2B_CUDA(cudaMemcpyAsync(&bad_h, bad, sizeof bad_h, cudaMemcpyDeviceToHost, st));
    NE2B_CUDA(cudaStreamSynchronize(st));
    *pd = bad_h == 0;
    return NE2B_OK;
}

// L z = b, L^T w = z with L the lower triangle of l (readout.rs:170-186 order).
void host_solve(const std::vector<double> &l, const double *b, uint32_t n, double *w) {
    std::vector<double> z(n);
    for (uint32_t i = 0; i < n; ++i) {
        double s = b[i];
        for (uint32_t q = 0; q < i; ++q) s -= l[(size_t)i * n + q] * z[q];
        z[i] = s / l[(size_t)i * n + i];
    }
    for (uint32_t i = n; i-- > 0;) {
        double s = z[i];
        for (uint32_t q = i + 1; q < n; ++q) s -= l[(size_t)q * n + i] * w[q];
        w[i] = s / l[(size_t)i * n + i];
    }
}

// fit_ridge on a device design x[T x F] and host targets y[T].
ne2b_status fit_binary_on_device(const float *x, uint32_t t, uint32_t f, const float *y_host, float lambda,
                                 cudaStream_t st, double *w_out) {
    const uint32_t nf = f + 1u;
    DevBuf buf(st);
    double *a = nullptr, *a0 = nullptr, *b = nullptr;
    float *y = nullptr;
    unsigned int *bad = nullptr;
    NE2B_TRY(buf.get(&a, (size_t)nf * nf));
    NE2B_TRY(buf.get(&a0, (size_t)nf * nf));
    NE2B_TRY(buf.get(&b, nf));
    NE2B_TRY(buf.get(&y, t));
    NE2B_TRY(buf.get(&bad, 1));
    NE2B_CUDA(cudaMemcpyAsync(y, y_host, sizeof(float) * t, cudaMemcpyHostToDevice, st));
    const uint32_t nt = (f + kGramTile - 1) / kGramTile;
    normal_kernel<<<nt * (nt + 1) / 2, 256, 0, st>>>(x, t, f, a);
    bias_rhs_kernel<<<(nf + 255) / 256, 256, 0, st>>>(x, y, t, f, a, b);
    const double lam = (double)lambda;
    diag_kernel<<<(nf + 255) / 256, 256, 0, st>>>(a, nf, lam, true, lam);
    NE2B_CUDA(cudaMemcpyAsync(a0, a, sizeof(double) * nf * nf, cudaMemcpyDeviceToDevice, st));
    bool pd = false;
    NE2B_TRY(cholesky(a, nf, bad, st, &pd));
    if (!pd) {  // readout.rs:131-139: more regularisation, once
        NE2B_CUDA(cudaMemcpyAsync(a, a0, sizeof(double) * nf * nf, cudaMemcpyDeviceToDevice, st));
        diag_kernel<<<(nf + 255) / 256, 256, 0, st>>>(a, nf, 1e-3 + lam, false, 0.0);
        NE2B_TRY(cholesky(a, nf, bad, st, &pd));
    }
    if (!pd) {
        for (uint32_t i = 0; i < nf; ++i) w_out[i] = 0.0;
        return NE2B_OK;
    }
    std::vector<double> l((size_t)nf * nf), bh(nf);
    NE2B_CUDA(cudaMemcpyAsync(l.data(), a, sizeof(double) * l.size(), cudaMemcpyDeviceToHost, st));
    NE2B_CUDA(cudaMemcpyAsync(bh.data(), b, sizeof(double) * nf, cudaMemcpyDeviceToHost, st));
    NE2B_CUDA(cudaStreamSynchronize(st));
    host_solve(l, bh.data(), nf, w_out);
    return NE2B_OK;
}

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
    col_mean_kernel<<<(f + 255) / 256, 256, 0, st>>>(x, t, f, mu);
    const uint64_t n = (uint64_t)t * f;
    center_kernel<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 64), 256, 0, st>>>(x, n, f, mu, xc);
    const uint32_t nt = (t + kGramTile - 1) / kGramTile;
    gram_kernel<<<nt * (nt + 1) / 2, 256, 0, st>>>(xc, t, f, lambda, g);
    bool pd = false;
    NE2B_TRY(cholesky(g, t, bad, st, &pd));
    // the triangular solves on the host, in the reference's order
    std::vector<double> L((size_t)t * t), mu_h(f);
    NE2B_CUDA(cudaMemcpyAsync(L.data(), g, sizeof(double) * L.size(), cudaMemcpyDeviceToHost, st));
    NE2B_CUDA(cudaMemcpyAsync(mu_h.data(), mu, sizeof(double) * f, cudaMemcpyDeviceToHost, st));
    NE2B_CUDA(cudaStreamSynchronize(st));
    std::vector<double> ybar(k, 0.0), ah((size_t)t * k, 0.0), yc(t);
    for (uint32_t r = 0; r < t; ++r) ybar[labels[r]] += 1.0 / (double)t;
    if (pd)
        for (uint32_t c = 0; c < k; ++c) {
            for (uint32_t i = 0; i < t; ++i) yc[i] = (labels[i] == c ? 1.0 : 0.0) - ybar[c];
            host_solve(L, yc.data(), t, ah.data() + (size_t)c * t);
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

}  // extern "C"

// A batch's window counts as a [t x windows*n] design on its stream.
static ne2b_status gather_batch(ne2b_batch *b, const uint32_t *nets, uint32_t t, uint32_t windows,
                                ne2b::DevBuf &buf, float **x, uint32_t *f_out) {
    if (t == 0 || windows == 0) return set_error(NE2B_EINVAL, "batch readout: no trials or no windows");
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
    if (f64 == 0 || f64 > 0xffffffffull) return set_error(NE2B_UNSUPPORTED, "%llu features", (unsigned long long)f64);
    const uint32_t f = (uint32_t)f64;
    cudaStream_t st = b->eng.stream();  // after the batch's queued steps
    const uint16_t **wd = nullptr;
    NE2B_TRY(buf.get(&wd, t));
    NE2B_TRY(buf.get(x, (size_t)t * f));
    NE2B_CUDA(cudaMemcpyAsync(wd, win.data(), sizeof(void *) * t, cudaMemcpyHostToDevice, st));
    ne2b::gather_counts_kernel<<<dim3((f + 255) / 256 < 1024 ? (f + 255) / 256 : 1024, t), 256, 0, st>>>(
        wd, n, n_pad, windows, *x);
    NE2B_CUDA(cudaGetLastError());
    *f_out = f;
    return NE2B_OK;
}

extern "C" {

ne2b_status ne2b_batch_fit_ridge_multi(ne2b_batch *b, const uint32_t *nets, uint32_t t, uint32_t windows,
                                       const uint32_t *labels, uint32_t k, double lambda, uint32_t *n_features,
                                       double *w) {
    if (!b || !nets || !labels || !w) return set_error(NE2B_EINVAL, "ne2b_batch_fit_ridge_multi: null argument");
    try {
        ne2b::DevBuf buf(b->eng.stream());
        float *x = nullptr;
        uint32_t f = 0;
        NE2B_TRY(gather_batch(b, nets, t, windows, buf, &x, &f));
        const ne2b_status cs = ne2b::check_labels(labels, t, f, k);
        if (cs != NE2B_OK) return cs;
        if (n_features) *n_features = f;
        return ne2b::fit_on_device(x, t, f, labels, k, lambda, b->eng.stream(), w);
    } catch (const std::bad_alloc &) {
        return set_error(NE2B_ENOMEM, "host allocation failed");
    }
}

ne2b_status ne2b_fit_ridge(const float *x, uint32_t t, uint32_t f, const float *y, float lambda, int device,
                           double *w) {
    if (!x || !y || !w) return set_error(NE2B_EINVAL, "ne2b_fit_ridge: null argument");
    if (t == 0 || f == 0) return set_error(NE2B_EINVAL, "fit_ridge: need T >= 1, F >= 1 (T=%u F=%u)", t, f);
    if (f >= 32768) return set_error(NE2B_UNSUPPORTED, "fit_ridge: at most 32767 features (F=%u)", f);
    try {
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) return ne2b::cuda_error(e, "cudaSetDevice");
        cudaPointerAttributes attr{};
        const bool on_device = cudaPointerGetAttributes(&attr, x) == cudaSuccess && attr.type == cudaMemoryTypeDevice;
        cudaGetLastError();
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
            if (r == NE2B_OK) r = ne2b::fit_binary_on_device(xd, t, f, y, lambda, st, w);
        }
        cudaStreamDestroy(st);
        return r;
    } catch (const std::bad_alloc &) {
        return set_error(NE2B_ENOMEM, "host allocation failed");
    }
}

ne2b_status ne2b_batch_fit_ridge(ne2b_batch *b, const uint32_t *nets, uint32_t t, uint32_t windows, const float *y,
                                 float lambda, uint32_t *n_features, double *w) {
    if (!b || !nets || !y || !w) return set_error(NE2B_EINVAL, "ne2b_batch_fit_ridge: null argument");
    try {
        ne2b::DevBuf buf(b->eng.stream());
        float *x = nullptr;
        uint32_t f = 0;
        NE2B_TRY(gather_batch(b, nets, t, windows, buf, &x, &f));
        if (f >= 32768) return set_error(NE2B_UNSUPPORTED, "fit_ridge: at most 32767 features (F=%u)", f);
        if (n_features) *n_features = f;
        return ne2b::fit_binary_on_device(x, t, f, y, lambda, b->eng.stream(), w);
    } catch (const std::bad_alloc &) {
        return set_error(NE2B_ENOMEM, "host allocation failed");
    }
}

}  // extern "C"
