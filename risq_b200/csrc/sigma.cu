// sigma = H x over full-row storage (both triangles, diagonal kept apart), and the
// dispatch to the tiled upper-triangle kernels (tiles.cu).
//
// Replaces SparseMatUpperTri::matrix_vector_prod (src/var/sparse.rs:64-78).  With
// both triangles stored every output is a private warp reduction: one warp per row,
// the column/value streams read once with evict-first loads so that the gathered
// vector x stays resident in L2.  Upper-triangle storage (the reference's own layout,
// half the bytes) goes through the tiled kernels.
#include <algorithm>
#include <type_traits>

#include "bits.cuh"
#include "internal.cuh"

namespace risq {

namespace {

constexpr unsigned FULL = 0xffffffffu;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// VK 0: FP64 values, FP64 vectors.  VK 1: FP32 values, FP32 vectors (FP32 sums).
// VK 2: FP32 value + FP32 remainder, FP64 vectors.  VK 3: FP32 values, FP64 vectors.
template <int VK, typename X>
__global__ void __launch_bounds__(256) k_spmv(int64_t N, const int64_t* __restrict__ row_start,
                                              const int32_t* __restrict__ row_len, const int32_t* __restrict__ cols,
                                              const double* __restrict__ v64, const float* __restrict__ v32,
                                              const float* __restrict__ vlo, const double* __restrict__ diag,
                                              const X* __restrict__ x, X* __restrict__ y) {
    using A = typename std::conditional<VK == 1, float, double>::type;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t p = warp; p < N; p += nwarps) {
        const int64_t s = row_start[p];
        const int len = row_len[p];
        A acc = 0;
        int k = lane;
        // four independent loads in flight per lane
        for (; k + 96 < len; k += 128) {
            int c0 = __ldcs(cols + s + k), c1 = __ldcs(cols + s + k + 32);
            int c2 = __ldcs(cols + s + k + 64), c3 = __ldcs(cols + s + k + 96);
            A a0, a1, a2, a3;
            if constexpr (VK == 0) {
                a0 = __ldcs(v64 + s + k); a1 = __ldcs(v64 + s + k + 32);
                a2 = __ldcs(v64 + s + k + 64); a3 = __ldcs(v64 + s + k + 96);
            } else if constexpr (VK == 2) {
                a0 = (double)__ldcs(v32 + s + k) + (double)__ldcs(vlo + s + k);
                a1 = (double)__ldcs(v32 + s + k + 32) + (double)__ldcs(vlo + s + k + 32);
                a2 = (double)__ldcs(v32 + s + k + 64) + (double)__ldcs(vlo + s + k + 64);
                a3 = (double)__ldcs(v32 + s + k + 96) + (double)__ldcs(vlo + s + k + 96);
            } else {
                a0 = (A)__ldcs(v32 + s + k); a1 = (A)__ldcs(v32 + s + k + 32);
                a2 = (A)__ldcs(v32 + s + k + 64); a3 = (A)__ldcs(v32 + s + k + 96);
            }
            acc += a0 * (A)__ldg(x + c0);
            acc += a1 * (A)__ldg(x + c1);
            acc += a2 * (A)__ldg(x + c2);
            acc += a3 * (A)__ldg(x + c3);
        }
        for (; k < len; k += 32) {
            int c = __ldcs(cols + s + k);
            A a;
            if constexpr (VK == 0) a = __ldcs(v64 + s + k);
            else if constexpr (VK == 2) a = (double)__ldcs(v32 + s + k) + (double)__ldcs(vlo + s + k);
            else a = (A)__ldcs(v32 + s + k);
            acc += a * (A)__ldg(x + c);
        }
        acc = warp_sum(acc);
        if (lane == 0) y[p] = (X)(diag[p] * (double)x[p] + (double)acc);
    }
}

// FP64 sigma that recomputes every stored element from the two determinants and
// the integrals (Slater-Condon in FP64, bitwise the values a FP64 build stores),
// reading only the int32 column stream from HBM.  SMEM: the packed integral tables
// are staged in shared memory (n <= 20 fits in 227 KB).
template <int W, bool SMEM>
__global__ void __launch_bounds__(1024, 1) k_spmv_otf(int64_t N, const uint64_t* __restrict__ up,
                                                      const uint64_t* __restrict__ dn,
                                                      const int64_t* __restrict__ row_start,
                                                      const int32_t* __restrict__ row_len,
                                                      const int32_t* __restrict__ cols,
                                                      const double* __restrict__ diag, Ints Ig, uint32_t n1,
                                                      uint32_t n2, const double* __restrict__ x,
                                                      double* __restrict__ y) {
    extern __shared__ double sm[];
    if constexpr (SMEM) {
        for (uint32_t k = threadIdx.x; k < n1; k += blockDim.x) sm[k] = Ig.h1[k];
        for (uint32_t k = threadIdx.x; k < n2; k += blockDim.x) sm[n1 + k] = Ig.h2[k];
        __syncthreads();
    }
    const IntsShared Is{sm, sm + n1, Ig.nuc};
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t p = warp; p < N; p += nwarps) {
        Bits<W> a, b;
#pragma unroll
        for (int k = 0; k < W; k++) { a.w[k] = __ldg(up + k * N + p); b.w[k] = __ldg(dn + k * N + p); }
        const int64_t s = row_start[p];
        const int len = row_len[p];
        double acc = 0.0;
        for (int k = lane; k < len; k += 32) {
            const int q = __ldcs(cols + s + k);
            Bits<W> aq, bq;
#pragma unroll
            for (int w = 0; w < W; w++) { aq.w[w] = __ldg(up + w * N + q); bq.w[w] = __ldg(dn + w * N + q); }
            double v;
            if constexpr (SMEM) v = sc_pair<W, IntsShared>(Is, a, b, aq, bq);
            else v = sc_pair<W, Ints>(Ig, a, b, aq, bq);
            acc += v * __ldg(x + q);
        }
        acc = warp_sum(acc);
        if (lane == 0) y[p] = diag[p] * x[p] + acc;
    }
}

template <int W>
int launch_otf(risqgpu* h, const double* x, double* y) {
    const int64_t n = (int64_t)h->N;
    Ints I{h->d_h1, h->d_h2, h->nuc};
    const size_t smem = sizeof(double) * (h->n1 + h->n2);
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    if (smem <= (size_t)max_smem) {
        RQ_CUDA(h, cudaFuncSetAttribute(k_spmv_otf<W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_spmv_otf<W, true><<<num_sms(h), 1024, smem, h->stream>>>(n, h->d_up, h->d_dn, h->d_row_start, h->d_row_len,
                                                                   h->d_cols, h->d_diag, I, (uint32_t)h->n1,
                                                                   (uint32_t)h->n2, x, y);
    } else {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_spmv_otf<W, false>, 1024, 0);
        k_spmv_otf<W, false><<<num_sms(h) * std::max(occ, 1), 1024, 0, h->stream>>>(
            n, h->d_up, h->d_dn, h->d_row_start, h->d_row_len, h->d_cols, h->d_diag, I, (uint32_t)h->n1,
            (uint32_t)h->n2, x, y);
    }
    return check_launch(h, "sigma otf");
}

__global__ void k_permute_in(const double* __restrict__ x, const int32_t* __restrict__ orig, int64_t n,
                             double* __restrict__ xi) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        xi[p] = x[orig[p]];
}
__global__ void k_permute_out(const double* __restrict__ yi, const int32_t* __restrict__ orig, int64_t n,
                              double* __restrict__ y) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        y[orig[p]] = yi[p];
}

// Second-order self-energy of every determinant over the stored matrix:
// S_i = -sum_{j != i} H_ij^2 / max(H_jj - E, gmin).  VK as in k_spmv (0 FP64 values,
// 1 FP32, 2 FP32 + remainder).  Full rows: one warp per row, private sum.  Upper
// triangle: each stored pair adds to both rows (atomics; `out` zeroed first).
template <int VK>
__global__ void __launch_bounds__(256) k_self_energy(int64_t N, const int64_t* __restrict__ row_start,
                                                     const int32_t* __restrict__ row_len,
                                                     const int32_t* __restrict__ cols, const double* __restrict__ v64,
                                                     const float* __restrict__ v32, const float* __restrict__ vlo,
                                                     const double* __restrict__ diag, double energy, double gmin,
                                                     int upper, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t p = warp; p < N; p += nwarps) {
        const int64_t s = row_start[p];
        const int len = row_len[p];
        const double gp = fmax(diag[p] - energy, gmin);
        double acc = 0.0;
        for (int k = lane; k < len; k += 32) {
            const int c = cols[s + k];
            double v;
            if constexpr (VK == 0) v = v64[s + k];
            else if constexpr (VK == 2) v = (double)v32[s + k] + (double)vlo[s + k];
            else v = (double)v32[s + k];
            const double v2 = v * v;
            acc += v2 / fmax(diag[c] - energy, gmin);
            if (upper) atomicAdd(out + c, -v2 / gp);
        }
        acc = warp_sum(acc);
        if (lane == 0) {
            if (upper) atomicAdd(out + p, -acc);
            else out[p] = -acc;
        }
    }
}

}  // namespace

int spmv_grid(risqgpu* h) {
    static int cached_dev = -1, cached = 0;
    if (cached_dev != h->device) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_spmv<0, double>, 256, 0);
        cached = num_sms(h) * std::max(occ, 1);
        cached_dev = h->device;
    }
    return cached;
}

int sigma_device(risqgpu* h, const void* x, void* y, int kind) {
    if (!h->built) { h->err = "sigma before build"; return RISQGPU_ERR_INVALID; }
    const int64_t n = (int64_t)h->N;
    const int grid = spmv_grid(h);
    if (h->upper) return sigma_tiles(h, x, y, kind);
    if (h->precision == RISQGPU_MATRIX_FREE) {
        if (kind != 0) {
            h->err = "a matrix-free build has only the FP64 sigma";
            return RISQGPU_ERR_INVALID;
        }
        return sigma_matrix_free(h, (const double*)x, (double*)y);
    }
    if (kind == 0) {
        const double* xd = (const double*)x;
        double* yd = (double*)y;
        if (h->precision == RISQGPU_FP64)
            k_spmv<0, double><<<grid, 256, 0, h->stream>>>(n, h->d_row_start, h->d_row_len, h->d_cols, h->d_val64,
                                                           nullptr, nullptr, h->d_diag, xd, yd);
        else if (h->precision == RISQGPU_MIXED)
            k_spmv<2, double><<<grid, 256, 0, h->stream>>>(n, h->d_row_start, h->d_row_len, h->d_cols, nullptr,
                                                           h->d_val32, h->d_val_lo, h->d_diag, xd, yd);
        else  // FP32 or columns-only storage: exact FP64 elements recomputed on the fly
            return h->W == 1 ? launch_otf<1>(h, xd, yd) : launch_otf<2>(h, xd, yd);
    } else {
        if (h->precision == RISQGPU_FP64 || h->precision == RISQGPU_COLS) {
            h->err = "FP32 sigma needs an FP32 or MIXED build";
            return RISQGPU_ERR_INVALID;
        }
        k_spmv<1, float><<<grid, 256, 0, h->stream>>>(n, h->d_row_start, h->d_row_len, h->d_cols, nullptr, h->d_val32,
                                                      nullptr, h->d_diag, (const float*)x, (float*)y);
    }
    return check_launch(h, "sigma");
}

int permute_in(risqgpu* h, const double* x, double* xi) {
    const int64_t n = (int64_t)h->N;
    const int g = std::max(1, (int)std::min<int64_t>((n + 255) / 256, 148 * 16));
    k_permute_in<<<g, 256, 0, h->stream>>>(x, h->d_orig, n, xi);
    return check_launch(h, "permute in");
}

int permute_out(risqgpu* h, const double* yi, double* y) {
    const int64_t n = (int64_t)h->N;
    const int g = std::max(1, (int)std::min<int64_t>((n + 255) / 256, 148 * 16));
    k_permute_out<<<g, 256, 0, h->stream>>>(yi, h->d_orig, n, y);
    return check_launch(h, "permute out");
}

int sigma_host(risqgpu* h, const double* x, double* y, int nvec) {
    if (!h->built) { h->err = "sigma before build"; return RISQGPU_ERR_INVALID; }
    if (nvec < 1) { h->err = "nvec < 1"; return RISQGPU_ERR_INVALID; }
    const int64_t n = (int64_t)h->N;
    double *dx = nullptr, *dxi = nullptr, *dyi = nullptr;
    ScopedFree<3> release(dx, dxi, dyi);
    RQ_TRY(dalloc(h, dx, n));
    RQ_TRY(dalloc(h, dxi, n));
    RQ_TRY(dalloc(h, dyi, n));
    for (int c = 0; c < nvec; c++) {
        RQ_CUDA(h, cudaMemcpyAsync(dx, x + (size_t)c * n, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
        RQ_TRY(permute_in(h, dx, dxi));
        RQ_TRY(sigma_device(h, dxi, dyi, 0));
        RQ_TRY(permute_out(h, dyi, dx));
        RQ_CUDA(h, cudaMemcpyAsync(y + (size_t)c * n, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    }
    return sync(h, "sigma_host");
}

int self_energy_impl(risqgpu* h, double energy, double gmin, double* out) {
    if (!h->built) { h->err = "self energy before build"; return RISQGPU_ERR_INVALID; }
    if (h->precision == RISQGPU_COLS || h->precision == RISQGPU_MATRIX_FREE) {
        h->err = "self energy needs stored values (not COLS or MATRIX_FREE)";
        return RISQGPU_ERR_INVALID;
    }
    if (!(gmin > 0.0)) { h->err = "gmin must be positive"; return RISQGPU_ERR_INVALID; }
    const int64_t n = (int64_t)h->N;
    double *si = nullptr, *sc = nullptr;
    ScopedFree<2> release(si, sc);
    RQ_TRY(dalloc(h, si, n));
    RQ_TRY(dalloc(h, sc, n));
    RQ_CUDA(h, cudaMemsetAsync(si, 0, sizeof(double) * n, h->stream));
    if (h->tiled) {
        RQ_TRY(tiles_self_energy(h, energy, gmin, si));
        RQ_TRY(permute_out(h, si, sc));
        RQ_CUDA(h, cudaMemcpyAsync(out, sc, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
        return sync(h, "self energy");
    }
    const int grid = spmv_grid(h);
    const int up = h->upper ? 1 : 0;
    if (h->precision == RISQGPU_FP64)
        k_self_energy<0><<<grid, 256, 0, h->stream>>>(n, h->d_row_start, h->d_row_len, h->d_cols, h->d_val64, nullptr,
                                                      nullptr, h->d_diag, energy, gmin, up, si);
    else if (h->precision == RISQGPU_MIXED)
        k_self_energy<2><<<grid, 256, 0, h->stream>>>(n, h->d_row_start, h->d_row_len, h->d_cols, nullptr, h->d_val32,
                                                      h->d_val_lo, h->d_diag, energy, gmin, up, si);
    else
        k_self_energy<1><<<grid, 256, 0, h->stream>>>(n, h->d_row_start, h->d_row_len, h->d_cols, nullptr, h->d_val32,
                                                      nullptr, h->d_diag, energy, gmin, up, si);
    RQ_TRY(check_launch(h, "self energy"));
    RQ_TRY(permute_out(h, si, sc));
    RQ_CUDA(h, cudaMemcpyAsync(out, sc, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    return sync(h, "self energy");
}

}  // namespace risq
