// Training of the learned preconditioner's MLP on the device.
//
// Network (same as the inference kernel in mlp.cu): o = W3 relu(W2 relu(W1 x + b1)
// + b2) + b3 with the weight matrices rounded to BF16 (round to nearest even) and
// FP32 accumulation; factor = exp(o).  Loss over a batch of B rows with sample
// weights w, in log space: L = sum_b w_b (o_b - log t_b)^2 / sum_b w_b (targets
// t_b > 0 are factors, so the loss weighs halving and doubling alike).  Gradients flow
// straight through the BF16 rounding into the FP32 master weights, which Adam
// updates.  Every reduction runs in a fixed order, so training is reproducible.
//
// Kernels: k_round (BF16 copies of the weights), k_forward (one thread per row,
// weights in shared memory, activations kept for the backward pass), k_out_grad,
// k_hidden2_grad, k_hidden1_grad (activation gradients), k_atb (weight gradients
// A^T B tiled through shared memory), k_colsum (bias gradients), k_adam.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "internal.cuh"

namespace risq {

namespace {

constexpr int HM = 128;  // largest hidden width

struct Layout {
    int n_in, H;
    int64_t oW1, ob1, oW2, ob2, oW3, ob3, P;
    Layout(int n, int h) : n_in(n), H(h) {
        oW1 = 0;
        ob1 = oW1 + (int64_t)h * n;
        oW2 = ob1 + h;
        ob2 = oW2 + (int64_t)h * h;
        oW3 = ob2 + h;
        ob3 = oW3 + h;
        P = ob3 + 1;
    }
};

__device__ __forceinline__ float round_bf16(float f) {
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7f800000u) == 0x7f800000u) return __uint_as_float(u & 0xffff0000u);
    u += 0x7fffu + ((u >> 16) & 1u);
    return __uint_as_float(u & 0xffff0000u);
}

// rounded copy: weight matrices to BF16 precision, biases unchanged
__global__ void k_round(const float* __restrict__ p, float* __restrict__ r, int64_t oW1, int64_t ob1, int64_t oW2,
                        int64_t ob2, int64_t oW3, int64_t ob3, int64_t P) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P; i += (int64_t)gridDim.x * blockDim.x) {
        const bool w = (i >= oW1 && i < ob1) || (i >= oW2 && i < ob2) || (i >= oW3 && i < ob3);
        r[i] = w ? round_bf16(p[i]) : p[i];
    }
}

__global__ void __launch_bounds__(128) k_forward(const float* __restrict__ X, int64_t B, int n_in, int H,
                                                 const float* __restrict__ pr, int64_t oW1, int64_t ob1, int64_t oW2,
                                                 int64_t ob2, int64_t oW3, int64_t ob3, float* __restrict__ h1,
                                                 float* __restrict__ h2, float* __restrict__ out) {
    extern __shared__ float sm[];
    float* W1 = sm;
    float* W2 = W1 + H * n_in;
    float* B1 = W2 + H * H;
    float* B2 = B1 + H;
    float* W3 = B2 + H;
    for (int k = threadIdx.x; k < H * n_in; k += blockDim.x) W1[k] = pr[oW1 + k];
    for (int k = threadIdx.x; k < H * H; k += blockDim.x) W2[k] = pr[oW2 + k];
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        B1[k] = pr[ob1 + k];
        B2[k] = pr[ob2 + k];
        W3[k] = pr[oW3 + k];
    }
    __syncthreads();
    const float b3 = pr[ob3];
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x) {
        const float* x = X + b * n_in;
        float a1[HM];
#pragma unroll
        for (int j = 0; j < HM; j++) {
            if (j < H) {
                float s = B1[j];
                for (int i = 0; i < n_in; i++) s += W1[j * n_in + i] * x[i];
                a1[j] = fmaxf(s, 0.f);
                h1[b * H + j] = a1[j];
            } else {
                a1[j] = 0.f;
            }
        }
        float o = b3;
        for (int j2 = 0; j2 < H; j2++) {
            float s = B2[j2];
#pragma unroll
            for (int j = 0; j < HM; j++)
                if (j < H) s += W2[j2 * H + j] * a1[j];
            s = fmaxf(s, 0.f);
            h2[b * H + j2] = s;
            o += W3[j2] * s;
        }
        out[b] = o;
    }
}

// dL/do and the loss terms: do_b = 2 w_b (o_b - log t_b) / W
__global__ void k_out_grad(const float* __restrict__ o, const float* __restrict__ t, const float* __restrict__ w,
                           int64_t B, float inv_w, float* __restrict__ dout, float* __restrict__ lterm) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x) {
        const float d = o[b] - logf(t[b]);
        dout[b] = 2.f * w[b] * d * inv_w;
        lterm[b] = w[b] * d * d * inv_w;
    }
}

__global__ void k_hidden2_grad(const float* __restrict__ dout, const float* __restrict__ pr, int64_t oW3,
                               const float* __restrict__ h2, int64_t B, int H, float* __restrict__ dh2) {
    const int64_t n = B * H;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i / H;
        const int j = (int)(i % H);
        dh2[i] = h2[i] > 0.f ? dout[b] * pr[oW3 + j] : 0.f;
    }
}

__global__ void k_hidden1_grad(const float* __restrict__ dh2, const float* __restrict__ pr, int64_t oW2,
                               const float* __restrict__ h1, int64_t B, int H, float* __restrict__ dh1) {
    const int64_t n = B * H;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i / H;
        const int j1 = (int)(i % H);
        float s = 0.f;
        if (h1[i] > 0.f)
            for (int j2 = 0; j2 < H; j2++) s += dh2[b * H + j2] * pr[oW2 + (int64_t)j2 * H + j1];
        dh1[i] = s;
    }
}

// out[m][k] = sum_b A[b][m] * Bm[b][k]   (A: B x M, Bm: B x K, row-major), 16 x 16 tiles
__global__ void __launch_bounds__(256) k_atb(const float* __restrict__ A, const float* __restrict__ Bm, int64_t B, int M,
                                             int K, float* __restrict__ out) {
    __shared__ float As[32][16];
    __shared__ float Bs[32][16];
    const int tm = threadIdx.x / 16, tk = threadIdx.x % 16;
    const int m = blockIdx.x * 16 + tm, k = blockIdx.y * 16 + tk;
    float acc = 0.f;
    for (int64_t b0 = 0; b0 < B; b0 += 32) {
        for (int l = threadIdx.x; l < 32 * 16; l += 256) {
            const int r = l / 16, c = l % 16;
            const int64_t b = b0 + r;
            const int mm = blockIdx.x * 16 + c, kk = blockIdx.y * 16 + c;
            As[r][c] = (b < B && mm < M) ? A[b * M + mm] : 0.f;
            Bs[r][c] = (b < B && kk < K) ? Bm[b * K + kk] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 32; r++) acc += As[r][tm] * Bs[r][tk];
        __syncthreads();
    }
    if (m < M && k < K) out[(int64_t)m * K + k] = acc;
}

// out[m] = sum_b A[b][m]
__global__ void k_colsum(const float* __restrict__ A, int64_t B, int M, float* __restrict__ out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    float s = 0.f;
    for (int64_t b = 0; b < B; b++) s += A[b * M + m];
    out[m] = s;
}

// sum of a vector in a fixed order (one block)
__global__ void k_sum1(const float* __restrict__ a, int64_t n, float* __restrict__ out) {
    __shared__ float sh[256];
    float s = 0.f;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += a[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t P, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void k_gather_rows(const float* __restrict__ X, const float* __restrict__ t, const float* __restrict__ w,
                              const int64_t* __restrict__ idx, int64_t nb, int n_in, float* __restrict__ Xb,
                              float* __restrict__ tb, float* __restrict__ wb) {
    const int64_t n = nb * n_in;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / n_in;
        const int c = (int)(i % n_in);
        const int64_t src = idx[r];
        Xb[i] = X[src * n_in + c];
        if (c == 0) { tb[r] = t[src]; wb[r] = w[src]; }
    }
}

struct Trainer {
    Layout L;
    int64_t Bmax;
    cudaStream_t st = nullptr;
    float *pr = nullptr, *h1 = nullptr, *h2 = nullptr, *o = nullptr, *dout = nullptr, *lterm = nullptr;
    float *dh1 = nullptr, *dh2 = nullptr, *grad = nullptr, *ones = nullptr, *wsum = nullptr, *lsum = nullptr;
    std::string err;

    Trainer(int n_in, int H, int64_t bmax) : L(n_in, H), Bmax(bmax) {}
    template <typename T>
    int alloc(T*& p, size_t n) {
        if (cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            err = "cudaMalloc failed in MLP training";
            return RISQGPU_ERR_OOM;
        }
        return RISQGPU_OK;
    }
    int init() {
        RQ_TRY(alloc(pr, L.P));
        RQ_TRY(alloc(h1, Bmax * L.H));
        RQ_TRY(alloc(h2, Bmax * L.H));
        RQ_TRY(alloc(o, Bmax));
        RQ_TRY(alloc(dout, Bmax));
        RQ_TRY(alloc(lterm, Bmax));
        RQ_TRY(alloc(dh1, Bmax * L.H));
        RQ_TRY(alloc(dh2, Bmax * L.H));
        RQ_TRY(alloc(grad, L.P));
        RQ_TRY(alloc(ones, Bmax));
        RQ_TRY(alloc(wsum, 1));
        RQ_TRY(alloc(lsum, 1));
        std::vector<float> one(Bmax, 1.f);
        cudaMemcpy(ones, one.data(), sizeof(float) * Bmax, cudaMemcpyHostToDevice);
        return cudaGetLastError() == cudaSuccess ? RISQGPU_OK : RISQGPU_ERR_CUDA;
    }
    ~Trainer() {
        for (float* p : {pr, h1, h2, o, dout, lterm, dh1, dh2, grad, ones, wsum, lsum})
            if (p) cudaFree(p);
    }
    // loss and gradient of one batch on device rows (X, t, w), parameters p (device)
    int batch(const float* p, const float* X, const float* t, const float* w, int64_t B, float* loss_host) {
        const int n = L.n_in, H = L.H;
        const int g = (int)std::max<int64_t>(1, std::min<int64_t>((B * H + 255) / 256, 4096));
        k_round<<<64, 256, 0, st>>>(p, pr, L.oW1, L.ob1, L.oW2, L.ob2, L.oW3, L.ob3, L.P);
        const size_t smem = sizeof(float) * ((size_t)H * n + (size_t)H * H + 3 * H);
        cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_forward<<<(int)std::max<int64_t>(1, std::min<int64_t>((B + 127) / 128, 1184)), 128, smem, st>>>(
            X, B, n, H, pr, L.oW1, L.ob1, L.oW2, L.ob2, L.oW3, L.ob3, h1, h2, o);
        k_sum1<<<1, 256, 0, st>>>(w, B, wsum);
        float W = 0.f;
        cudaMemcpyAsync(&W, wsum, sizeof(float), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        if (!(W > 0.f)) { err = "sample weights must have a positive sum"; return RISQGPU_ERR_INVALID; }
        k_out_grad<<<g, 256, 0, st>>>(o, t, w, B, 1.f / W, dout, lterm);
        k_hidden2_grad<<<g, 256, 0, st>>>(dout, pr, L.oW3, h2, B, H, dh2);
        k_hidden1_grad<<<g, 256, 0, st>>>(dh2, pr, L.oW2, h1, B, H, dh1);
        // weight gradients
        k_atb<<<dim3((H + 15) / 16, (n + 15) / 16), 256, 0, st>>>(dh1, X, B, H, n, grad + L.oW1);
        k_colsum<<<(H + 127) / 128, 128, 0, st>>>(dh1, B, H, grad + L.ob1);
        k_atb<<<dim3((H + 15) / 16, (H + 15) / 16), 256, 0, st>>>(dh2, h1, B, H, H, grad + L.oW2);
        k_colsum<<<(H + 127) / 128, 128, 0, st>>>(dh2, B, H, grad + L.ob2);
        k_atb<<<dim3(1, (H + 15) / 16), 256, 0, st>>>(dout, h2, B, 1, H, grad + L.oW3);
        k_colsum<<<1, 128, 0, st>>>(dout, B, 1, grad + L.ob3);
        if (loss_host) {
            k_sum1<<<1, 256, 0, st>>>(lterm, B, lsum);
            cudaMemcpyAsync(loss_host, lsum, sizeof(float), cudaMemcpyDeviceToHost, st);
        }
        cudaError_t e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) { err = cudaGetErrorString(e); return RISQGPU_ERR_CUDA; }
        return RISQGPU_OK;
    }
};

int check_dims(int n_in, int hidden) {
    if (n_in < 1 || n_in > 258 || hidden < 1 || hidden > HM) return RISQGPU_ERR_INVALID;
    return RISQGPU_OK;
}

struct DevScope {
    int prev = -1;
    explicit DevScope(int d) {
        cudaGetDevice(&prev);
        if (prev != d) cudaSetDevice(d);
    }
    ~DevScope() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// targets are factors: the log-space loss needs every one finite and positive
bool targets_ok(const float* t, int64_t B) {
    for (int64_t b = 0; b < B; b++)
        if (!(t[b] > 0.f) || !std::isfinite(t[b])) return false;
    return true;
}

}  // namespace

}  // namespace risq

using namespace risq;

extern "C" int risqgpu_mlp_grad(int device, int n_in, int hidden, const float* params, const float* feats,
                                const float* target, const float* weight, int64_t B, float* loss, float* grad) {
    if (!params || !feats || !target || !weight || !loss || !grad || B < 1) return RISQGPU_ERR_INVALID;
    if (!targets_ok(target, B)) return RISQGPU_ERR_INVALID;
    RQ_TRY(check_dims(n_in, hidden));
    DevScope ds(device);
    Trainer T(n_in, hidden, B);
    RQ_TRY(T.init());
    float *p = nullptr, *X = nullptr, *t = nullptr, *w = nullptr;
    RQ_TRY(T.alloc(p, T.L.P));
    RQ_TRY(T.alloc(X, B * n_in));
    RQ_TRY(T.alloc(t, B));
    RQ_TRY(T.alloc(w, B));
    cudaMemcpy(p, params, sizeof(float) * T.L.P, cudaMemcpyHostToDevice);
    cudaMemcpy(X, feats, sizeof(float) * B * n_in, cudaMemcpyHostToDevice);
    cudaMemcpy(t, target, sizeof(float) * B, cudaMemcpyHostToDevice);
    cudaMemcpy(w, weight, sizeof(float) * B, cudaMemcpyHostToDevice);
    int rc = T.batch(p, X, t, w, B, loss);
    if (rc == RISQGPU_OK && cudaMemcpy(grad, T.grad, sizeof(float) * T.L.P, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = RISQGPU_ERR_CUDA;
    cudaFree(p); cudaFree(X); cudaFree(t); cudaFree(w);
    return rc;
}

extern "C" int risqgpu_mlp_train(int device, int n_in, int hidden, float* params, const float* feats,
                                 const float* target, const float* weight, int64_t B, int epochs, int batch,
                                 float lr, uint64_t seed, float* loss_hist) {
    if (!params || !feats || !target || !weight || B < 1 || epochs < 1 || batch < 1) return RISQGPU_ERR_INVALID;
    if (!targets_ok(target, B)) return RISQGPU_ERR_INVALID;
    RQ_TRY(check_dims(n_in, hidden));
    DevScope ds(device);
    const int64_t bs = std::min<int64_t>(batch, B);
    Trainer T(n_in, hidden, bs);
    RQ_TRY(T.init());
    const int64_t P = T.L.P;
    float *p = nullptr, *m = nullptr, *v = nullptr, *X = nullptr, *t = nullptr, *w = nullptr;
    float *Xb = nullptr, *tb = nullptr, *wb = nullptr;
    int64_t* idx = nullptr;
    RQ_TRY(T.alloc(p, P));
    RQ_TRY(T.alloc(m, P));
    RQ_TRY(T.alloc(v, P));
    RQ_TRY(T.alloc(X, B * n_in));
    RQ_TRY(T.alloc(t, B));
    RQ_TRY(T.alloc(w, B));
    RQ_TRY(T.alloc(Xb, bs * n_in));
    RQ_TRY(T.alloc(tb, bs));
    RQ_TRY(T.alloc(wb, bs));
    RQ_TRY(T.alloc(idx, B));
    cudaMemcpy(p, params, sizeof(float) * P, cudaMemcpyHostToDevice);
    cudaMemset(m, 0, sizeof(float) * P);
    cudaMemset(v, 0, sizeof(float) * P);
    cudaMemcpy(X, feats, sizeof(float) * B * n_in, cudaMemcpyHostToDevice);
    cudaMemcpy(t, target, sizeof(float) * B, cudaMemcpyHostToDevice);
    cudaMemcpy(w, weight, sizeof(float) * B, cudaMemcpyHostToDevice);
    std::vector<int64_t> order(B);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 rng(seed);
    int rc = RISQGPU_OK;
    int64_t step = 0;
    const float b1 = 0.9f, b2 = 0.999f;
    for (int ep = 0; ep < epochs && rc == RISQGPU_OK; ep++) {
        std::shuffle(order.begin(), order.end(), rng);
        cudaMemcpy(idx, order.data(), sizeof(int64_t) * B, cudaMemcpyHostToDevice);
        double lsum = 0.0;
        int nb = 0;
        for (int64_t b0 = 0; b0 < B && rc == RISQGPU_OK; b0 += bs) {
            const int64_t nbr = std::min(bs, B - b0);
            k_gather_rows<<<256, 256, 0, T.st>>>(X, t, w, idx + b0, nbr, n_in, Xb, tb, wb);
            float l = 0.f;
            rc = T.batch(p, Xb, tb, wb, nbr, &l);
            if (rc) break;
            step++;
            const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
            k_adam<<<64, 256, 0, T.st>>>(p, T.grad, m, v, P, lr, b1, b2, 1e-8f, c1, c2);
            lsum += l;
            nb++;
        }
        if (loss_hist) loss_hist[ep] = (float)(lsum / std::max(nb, 1));
    }
    if (rc == RISQGPU_OK && cudaMemcpy(params, p, sizeof(float) * P, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = RISQGPU_ERR_CUDA;
    for (float* q : {p, m, v, X, t, w, Xb, tb, wb}) cudaFree(q);
    cudaFree(idx);
    return rc;
}
