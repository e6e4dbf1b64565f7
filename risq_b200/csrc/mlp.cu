// Learned diagonal-preconditioner correction: per-determinant inference.
//
// The network maps determinant features to a multiplicative correction of the
// DPR step r_i / (lambda - H_ii): f_i = clamp(exp((MLP(x_i) + MLP(x~_i)) / 2), 0.25, 4),
// x~_i being the features with the alpha and beta occupations exchanged.
// Features x_i (2n + 2 values, n = orbitals): occupation of each alpha orbital
// then each beta orbital as +1 / -1, (H_ii - E - mu_e) * s_e, and
// (sum of h_pp over the occupied spin-orbitals - mu_h) * s_h, where (mu_e, s_e,
// mu_h, s_h) are the network's feature normalisation.  Layers
// (2n+2) -> hidden -> hidden -> 1 with ReLU; weights are rounded to BF16 (round
// to nearest even) on the device, every product accumulates in FP32, and the
// first layer's activations are rounded to BF16 (they are the A operand of the
// second layer's BF16 GEMM on the tensor-core path, mlp_tc.cu).
// There is no counterpart in the reference (which only has DPR,
// algorithms/davidson.rs:391-408); the reference's DPR is the fallback.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "internal.cuh"

namespace risq {

namespace {

__device__ __forceinline__ float bf16_to_f(uint16_t u) { return __uint_as_float(((uint32_t)u) << 16); }

__device__ __forceinline__ uint16_t f_to_bf16_dev(float f) {  // round to nearest even (finite values)
    uint32_t u = __float_as_uint(f);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

uint16_t f_to_bf16(float f) {  // round to nearest even
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);  // inf / nan
    uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
}

constexpr int HMAX = 128;

// Network output o for one spin order: occupations of `a` fill inputs 0..n-1 and
// those of `b` inputs n..2n-1.  W1, W2, W3, B1, B2 in shared memory (FP32 copies of
// the BF16 weights).
template <int W>
__device__ __forceinline__ float mlp_out(const uint64_t (&a)[W], const uint64_t (&b)[W], int norb, int n_in,
                                         int hidden, float dE, float sum_h, const float* W1, const float* B1,
                                         const float* W2, const float* B2, const float* W3, float bias3) {
    float hid[HMAX];
#pragma unroll
    for (int j = 0; j < HMAX; j++) {
        if (j < hidden) {
            const float* wr = W1 + j * n_in;
            float s = B1[j];
            for (int o = 0; o < norb; o++) {
                s += wr[o] * (((a[o >> 6] >> (o & 63)) & 1ull) ? 1.f : -1.f);
                s += wr[norb + o] * (((b[o >> 6] >> (o & 63)) & 1ull) ? 1.f : -1.f);
            }
            s += wr[2 * norb] * dE + wr[2 * norb + 1] * sum_h;
            hid[j] = bf16_to_f(f_to_bf16_dev(fmaxf(s, 0.f)));  // BF16 activations, as the tensor-core path
        } else {
            hid[j] = 0.f;
        }
    }
    float o3 = bias3;
    for (int j2 = 0; j2 < hidden; j2++) {
        const float* wr = W2 + j2 * hidden;
        float s = B2[j2];
#pragma unroll
        for (int j = 0; j < HMAX; j++) s += wr[j < hidden ? j : 0] * (j < hidden ? hid[j] : 0.f);
        o3 += W3[j2] * fmaxf(s, 0.f);
    }
    return o3;
}

// One thread per determinant; all weights staged in shared memory as FP32.  The
// factor is symmetric under the alpha <-> beta exchange, as the Hamiltonian is:
// f = clamp(exp((o(alpha, beta) + o(beta, alpha)) / 2), 0.25, 4), so a determinant
// and its spin-flipped partner get the same factor and the correction vector keeps
// the spin-flip symmetry of the start vectors.
template <int W>
__global__ void __launch_bounds__(128) k_mlp_scale(const uint64_t* __restrict__ up, const uint64_t* __restrict__ dn,
                                                   const double* __restrict__ diag, int64_t N, int norb,
                                                   const double* __restrict__ h1, double energy, int n_in, int hidden,
                                                   const uint16_t* __restrict__ w1, const float* __restrict__ b1,
                                                   const uint16_t* __restrict__ w2, const float* __restrict__ b2,
                                                   const uint16_t* __restrict__ w3, const float* __restrict__ b3,
                                                   float4 fnorm, float* __restrict__ out) {
    extern __shared__ float sm[];
    float* W1 = sm;                      // hidden x n_in
    float* W2 = W1 + hidden * n_in;      // hidden x hidden
    float* B1 = W2 + hidden * hidden;    // hidden
    float* B2 = B1 + hidden;             // hidden
    float* W3 = B2 + hidden;             // hidden
    float* HPP = W3 + hidden;            // norb
    for (int k = threadIdx.x; k < hidden * n_in; k += blockDim.x) W1[k] = bf16_to_f(w1[k]);
    for (int k = threadIdx.x; k < hidden * hidden; k += blockDim.x) W2[k] = bf16_to_f(w2[k]);
    for (int k = threadIdx.x; k < hidden; k += blockDim.x) {
        B1[k] = b1[k];
        B2[k] = b2[k];
        W3[k] = bf16_to_f(w3[k]);
    }
    for (int k = threadIdx.x; k < norb; k += blockDim.x) {
        uint32_t i = k + 1;
        HPP[k] = (float)h1[(i * (i - 1)) / 2 + i];
    }
    __syncthreads();
    const float bias3 = b3[0];
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        uint64_t a[W], b[W];
        for (int k = 0; k < W; k++) { a[k] = up[k * N + p]; b[k] = dn[k * N + p]; }
        float sum_h = 0.f;
        for (int o = 0; o < norb; o++) {
            if ((a[o >> 6] >> (o & 63)) & 1ull) sum_h += HPP[o];
            if ((b[o >> 6] >> (o & 63)) & 1ull) sum_h += HPP[o];
        }
        const float dE = ((float)(diag[p] - energy) - fnorm.x) * fnorm.y;
        sum_h = (sum_h - fnorm.z) * fnorm.w;
        const float o_ab = mlp_out<W>(a, b, norb, n_in, hidden, dE, sum_h, W1, B1, W2, B2, W3, bias3);
        const float o_ba = mlp_out<W>(b, a, norb, n_in, hidden, dE, sum_h, W1, B1, W2, B2, W3, bias3);
        float f = __expf(0.5f * (o_ab + o_ba));
        out[p] = fminf(fmaxf(f, 0.25f), 4.0f);
    }
}

}  // namespace

void free_mlp(risqgpu* h) {
    dfree(h->mlp.w1); dfree(h->mlp.w2); dfree(h->mlp.w3);
    dfree(h->mlp.b1); dfree(h->mlp.b2); dfree(h->mlp.b3);
    h->mlp.loaded = false;
}

int set_mlp_impl(risqgpu* h, int n_in, int hidden, const float* w1, const float* b1, const float* w2, const float* b2,
                 const float* w3, const float* b3, const float* feat_norm) {
    if (n_in != 2 * h->norb + 2) { h->err = "MLP input size must be 2*norb + 2"; return RISQGPU_ERR_INVALID; }
    if (hidden < 1 || hidden > HMAX) { h->err = "MLP hidden size must be in [1, 128]"; return RISQGPU_ERR_INVALID; }
    if (!w1 || !b1 || !w2 || !b2 || !w3 || !b3) { h->err = "null MLP weights"; return RISQGPU_ERR_INVALID; }
    free_mlp(h);
    auto up16 = [&](const float* src, size_t n, uint16_t*& dst) -> int {
        std::vector<uint16_t> t(n);
        for (size_t i = 0; i < n; i++) t[i] = f_to_bf16(src[i]);
        RQ_TRY(dalloc(h, dst, n));
        RQ_CUDA(h, cudaMemcpy(dst, t.data(), n * sizeof(uint16_t), cudaMemcpyHostToDevice));
        return RISQGPU_OK;
    };
    auto up32 = [&](const float* src, size_t n, float*& dst) -> int {
        RQ_TRY(dalloc(h, dst, n));
        RQ_CUDA(h, cudaMemcpy(dst, src, n * sizeof(float), cudaMemcpyHostToDevice));
        return RISQGPU_OK;
    };
    RQ_TRY(up16(w1, (size_t)hidden * n_in, h->mlp.w1));
    RQ_TRY(up16(w2, (size_t)hidden * hidden, h->mlp.w2));
    RQ_TRY(up16(w3, (size_t)hidden, h->mlp.w3));
    RQ_TRY(up32(b1, hidden, h->mlp.b1));
    RQ_TRY(up32(b2, hidden, h->mlp.b2));
    RQ_TRY(up32(b3, 1, h->mlp.b3));
    h->mlp.n_in = n_in;
    h->mlp.hidden = hidden;
    h->mlp.fnorm = feat_norm ? make_float4(feat_norm[0], feat_norm[1], feat_norm[2], feat_norm[3])
                             : make_float4(0.f, 1.f, 0.f, 1.f);
    h->mlp.loaded = true;
    return RISQGPU_OK;
}

int mlp_scale_tc(risqgpu* h, double energy, float* out);

int mlp_scale_impl(risqgpu* h, double energy, float* out) {
    if (!h->mlp.loaded) { h->err = "no MLP loaded"; return RISQGPU_ERR_INVALID; }
    // hidden width 128 with 2n <= 128 runs on the tensor cores; other shapes on the CUDA cores
    if (h->mlp.hidden == 128 && 2 * h->norb <= 128) return mlp_scale_tc(h, energy, out);
    const int hid = h->mlp.hidden, nin = h->mlp.n_in;
    size_t smem = sizeof(float) * ((size_t)hid * nin + (size_t)hid * hid + 3 * hid + h->norb);
    const int64_t N = (int64_t)h->N;
    int grid = std::max(1, std::min<int>((int)((N + 127) / 128), num_sms(h) * 2));
    if (h->W == 1) {
        RQ_CUDA(h, cudaFuncSetAttribute(k_mlp_scale<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_mlp_scale<1><<<grid, 128, smem, h->stream>>>(h->d_up, h->d_dn, h->d_diag, N, h->norb, h->d_h1, energy, nin,
                                                       hid, h->mlp.w1, h->mlp.b1, h->mlp.w2, h->mlp.b2, h->mlp.w3,
                                                       h->mlp.b3, h->mlp.fnorm, out);
    } else {
        RQ_CUDA(h, cudaFuncSetAttribute(k_mlp_scale<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_mlp_scale<2><<<grid, 128, smem, h->stream>>>(h->d_up, h->d_dn, h->d_diag, N, h->norb, h->d_h1, energy, nin,
                                                       hid, h->mlp.w1, h->mlp.b1, h->mlp.w2, h->mlp.b2, h->mlp.w3,
                                                       h->mlp.b3, h->mlp.fnorm, out);
    }
    return check_launch(h, "mlp scale");
}

__global__ void k_factors_to_caller(const float* __restrict__ fi, const int32_t* __restrict__ orig, int64_t n,
                                    float* __restrict__ fc) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        fc[orig[p]] = fi[p];
}

int precond_factors_impl(risqgpu* h, double energy, float* out) {
    if (h->N == 0) { h->err = "no determinants set"; return RISQGPU_ERR_INVALID; }
    const int64_t n = (int64_t)h->N;
    float *fi = nullptr, *fc = nullptr;
    ScopedFree<2> release(fi, fc);
    RQ_TRY(dalloc(h, fi, n));
    RQ_TRY(dalloc(h, fc, n));
    RQ_TRY(mlp_scale_impl(h, energy, fi));
    k_factors_to_caller<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, h->stream>>>(fi, h->d_orig, n, fc);
    RQ_TRY(check_launch(h, "factors"));
    RQ_CUDA(h, cudaMemcpyAsync(out, fc, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "factors"));
    dfree(fi);
    dfree(fc);
    return RISQGPU_OK;
}

}  // namespace risq
