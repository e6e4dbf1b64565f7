// Block Davidson on the device.
//
// Follows Davidson::new (src/var/eigenvalues/algorithms/davidson.rs:106-277):
// lowest `nroots` pairs, search space nroots + 10 (Config::new, :53-79), DPR
// correction r / (lambda - H_ii) (:391-408), orthonormalisation of each new
// vector against the basis (MGS::orthonormalize, modified_gram_schmidt.rs:22-36),
// restart to the Ritz vectors when the space is full (:261-269), convergence when
// every residual norm < tol and every |lambda - lambda_prev| < etol (:179-193),
// early exits on a correction norm < 1e-9 (:210) and on a dependent new vector
// (:222).  The projected problem (at most 18 x 18) is solved on the host with
// the cyclic Jacobi method (Golub & Van Loan, Matrix Computations, 8.5); the
// reference uses nalgebra's SymmetricEigen (Householder + QR), which gives the
// same eigenpairs to rounding.
//
// Device work per iteration: one fused pass for Ritz vectors, residuals and the
// preconditioned correction; classical Gram-Schmidt applied twice (numerically
// equivalent to MGS for these sizes, two passes over the basis instead of one
// per column); one sigma; one pass for the new projected column.  All
// reductions are two-stage with a fixed grid, so results are reproducible.
// The restart takes H*ritz as the combination of the stored H*V columns rather
// than a fresh sigma (same vector, one sigma fewer).  The host waits twice per
// iteration: for the residual norms (convergence test) and for the new projected
// column, which arrives together with the squared norm of the new vector; the
// reference's dependent-vector exit is therefore taken after that vector's sigma,
// whose result is dropped.
//
// MIXED mode keeps V and H*V in FP32 and runs the FP32 sigma; dots, Gram-Schmidt
// coefficients, the projected matrix and the Ritz vectors stay FP64.  After it
// converges, FP64-sigma sweeps (FP32 value + FP32 remainder) restart from the
// FP64 Ritz vectors until the same criteria hold in FP64.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "internal.cuh"

namespace risq {

int sigma_device(risqgpu* h, const void* x, void* y, int kind);
int mlp_scale_impl(risqgpu* h, double energy, float* out);

namespace {

// sigma bracketed by CUDA events on the handle's stream; the events are read once the
// solve has finished (no synchronisation per sigma)
struct SigmaTimer {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    int run(risqgpu* h, const void* x, void* y, int kind) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, h->stream);
        int rc = sigma_device(h, x, y, kind);
        cudaEventRecord(b, h->stream);
        ev.emplace_back(a, b);
        return rc;
    }
    // after the stream has been synchronised
    void collect(risqgpu* h) {
        for (auto& e : ev) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, e.first, e.second) == cudaSuccess) h->sigma_ms_acc += ms;
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        ev.clear();
    }
    ~SigmaTimer() {
        for (auto& e : ev) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
    }
};

constexpr int KMAX = 64;   // basis columns (search space + the nroots new vectors)
constexpr int RMAX = 8;    // roots
constexpr int CCH = 16;    // basis columns per block of the dot-product kernels (blockIdx.y)
constexpr int DBLK = 256;  // threads per reduction block

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-reduce `m` per-thread values (acc[0..m)) into partial[blockIdx.x * stride + j].
template <int MMAX>
__device__ __forceinline__ void block_reduce_store(double (&acc)[MMAX], int m, double* __restrict__ partial, int stride) {
    __shared__ double sh[DBLK / 32][MMAX];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < MMAX; j++) {
        if (j < m) {
            double v = warp_sum_d(acc[j]);
            if (lane == 0) sh[w][j] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < m) {
        double s = 0.0;
        for (int k = 0; k < DBLK / 32; k++) s += sh[k][threadIdx.x];
        partial[blockIdx.x * stride + threadIdx.x] = s;
    }
}

// out[j] = sum over blocks of partial[b * stride + j], fixed order.
__global__ void k_reduce(const double* __restrict__ partial, int nblk, int m, int stride, double* __restrict__ out) {
    int j = blockIdx.x;
    if (j >= m) return;
    __shared__ double sh[DBLK];
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partial[b * stride + j];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = sh[0];
}

// Partial dot products <A_j, b> (A column-major, leading dimension N) for the columns
// j < m, and with `self` also <b, b> as column m; blockIdx.y takes CCH columns each.
// partial[blockIdx.x * (KMAX + 1) + j].
template <typename T>
__global__ void __launch_bounds__(DBLK) k_dots(const T* __restrict__ A, int m, const T* __restrict__ b, int self,
                                              int64_t N, double* __restrict__ partial) {
    const int j0 = blockIdx.y * CCH;
    const int mc = min(CCH, m + self - j0);
    double acc[CCH];
#pragma unroll
    for (int j = 0; j < CCH; j++) acc[j] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double bi = (double)b[i];
#pragma unroll
        for (int j = 0; j < CCH; j++)
            if (j < mc) acc[j] += (j0 + j < m ? (double)A[(int64_t)(j0 + j) * N + i] : bi) * bi;
    }
    block_reduce_store<CCH>(acc, mc, partial + j0, KMAX + 1);
}

// t -= sum_{j < m} coef[j] A_j, rounded to the basis type.
template <typename T>
__global__ void __launch_bounds__(DBLK) k_cgs_update(const T* __restrict__ A, int m, T* __restrict__ t, int64_t N,
                                                    const double* __restrict__ coef) {
    __shared__ double c[KMAX];
    if (threadIdx.x < KMAX) c[threadIdx.x] = threadIdx.x < m ? coef[threadIdx.x] : 0.0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        double ti = (double)t[i];
        for (int j = 0; j < m; j++) ti -= c[j] * (double)A[(int64_t)j * N + i];
        t[i] = (T)ti;
    }
}

// Thick restart: out_V[:, c] = sum_j V[:, j] Y[j, c], out_HV likewise, for the columns
// c of this block's chunk (blockIdx.y, CCH columns); Y: dim x keep, row-major.
template <typename T>
__global__ void __launch_bounds__(DBLK) k_combine(const T* __restrict__ V, const T* __restrict__ HV, int dim, int keep,
                                                 int64_t N, const double* __restrict__ Y, T* __restrict__ outV,
                                                 T* __restrict__ outHV) {
    __shared__ double ys[KMAX * CCH];
    const int c0 = blockIdx.y * CCH;
    const int kc = min(CCH, keep - c0);
    for (int k = threadIdx.x; k < dim * CCH; k += blockDim.x) {
        const int j = k / CCH, c = k % CCH;
        ys[k] = c < kc ? Y[j * keep + c0 + c] : 0.0;
    }
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        double a[CCH], b[CCH];
#pragma unroll
        for (int c = 0; c < CCH; c++) { a[c] = 0.0; b[c] = 0.0; }
        for (int j = 0; j < dim; j++) {
            const double v = (double)V[(int64_t)j * N + i], hv = (double)HV[(int64_t)j * N + i];
#pragma unroll
            for (int c = 0; c < CCH; c++) {
                a[c] += v * ys[j * CCH + c];
                b[c] += hv * ys[j * CCH + c];
            }
        }
#pragma unroll
        for (int c = 0; c < CCH; c++)
            if (c < kc) {
                outV[(int64_t)(c0 + c) * N + i] = (T)a[c];
                outHV[(int64_t)(c0 + c) * N + i] = (T)b[c];
            }
    }
}

template <typename T>
__global__ void k_scale(T* __restrict__ t, int64_t N, const double* __restrict__ nrm2) {
    double s = 1.0 / sqrt(*nrm2);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        t[i] = (T)((double)t[i] * s);
}

// Ritz vectors, H*ritz, residuals and the preconditioned correction for each root.
// sm: Y (dim x nr, row-major Y[j*nr + c]) followed by lambda[nr].  Writes
// ritz/hr (FP64, N x nr), the correction into V[:, dim + c] when `room`, and
// partial sums: |r_c|^2 (slot c), sum_c |t_c|^2 (slot nr).
template <typename T>
__global__ void __launch_bounds__(DBLK) k_ritz(const T* __restrict__ V, const T* __restrict__ HV, int dim, int nr,
                                              int64_t N, const double* __restrict__ small, const double* __restrict__ diag,
                                              const float* __restrict__ fscale, int room, double* __restrict__ ritz,
                                              double* __restrict__ hr, T* __restrict__ Vnew, double* __restrict__ partial) {
    __shared__ double Y[KMAX * RMAX];
    __shared__ double lam[RMAX];
    for (int k = threadIdx.x; k < dim * nr; k += blockDim.x) Y[k] = small[k];
    if (threadIdx.x < nr) lam[threadIdx.x] = small[dim * nr + threadIdx.x];
    __syncthreads();
    double acc[RMAX + 1];
#pragma unroll
    for (int c = 0; c <= RMAX; c++) acc[c] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        double rz[RMAX], hz[RMAX];
#pragma unroll
        for (int c = 0; c < RMAX; c++) { rz[c] = 0.0; hz[c] = 0.0; }
        for (int j = 0; j < dim; j++) {
            double v = (double)V[j * N + i], hv = (double)HV[j * N + i];
#pragma unroll
            for (int c = 0; c < RMAX; c++)
                if (c < nr) { rz[c] += v * Y[j * nr + c]; hz[c] += hv * Y[j * nr + c]; }
        }
        double d = diag[i];
        double f = fscale ? (double)fscale[i] : 1.0;
#pragma unroll
        for (int c = 0; c < RMAX; c++) {
            if (c < nr) {
                double r = hz[c] - rz[c] * lam[c];
                ritz[c * N + i] = rz[c];
                hr[c * N + i] = hz[c];
                acc[c] += r * r;
                if (room) {
                    double tc = r / (lam[c] - d) * f;
                    T tt = (T)tc;
                    Vnew[c * N + i] = tt;
                    acc[RMAX] += (double)tt * (double)tt;
                }
            }
        }
    }
    double out[RMAX + 1];
#pragma unroll
    for (int c = 0; c <= RMAX; c++) out[c] = c < nr ? acc[c] : (c == nr ? acc[RMAX] : 0.0);
    block_reduce_store<RMAX + 1>(out, nr + 1, partial, KMAX + 1);
}

template <typename T>
__global__ void k_set_cols(T* __restrict__ V, T* __restrict__ HV, const double* __restrict__ ritz,
                           const double* __restrict__ hr, int nr, int64_t N) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        for (int c = 0; c < nr; c++) {
            V[c * N + i] = (T)ritz[c * N + i];
            if (HV) HV[c * N + i] = (T)hr[c * N + i];
        }
}

template <typename T>
__global__ void k_fill_init(T* __restrict__ V, int ncol, int64_t N, const double* __restrict__ src /* internal order or null */,
                            const int32_t* __restrict__ inv, int e0, int e1) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        for (int c = 0; c < ncol; c++) {
            double v;
            if (src) v = src[c * N + i];
            else v = (i == inv[c == 0 ? e0 : e1]) ? 1.0 : 0.0;
            V[c * N + i] = (T)v;
        }
    }
}

__global__ void k_to_internal(const double* __restrict__ x, const int32_t* __restrict__ orig, int64_t N, int ncol,
                              double* __restrict__ xi) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
        for (int c = 0; c < ncol; c++) xi[c * N + p] = x[c * N + orig[p]];
}
__global__ void k_to_caller(const double* __restrict__ xi, const int32_t* __restrict__ orig, int64_t N, int ncol,
                            double* __restrict__ x) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
        for (int c = 0; c < ncol; c++) x[c * N + orig[p]] = xi[c * N + p];
}

// Cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (row-major),
// eigenvalues ascending, Y[r*n + c] = component r of eigenvector c.
void jacobi_sorted(int n, const double* A, double* w, double* Y) {
    std::vector<double> a(A, A + n * n), v(n * n, 0.0);
    for (int i = 0; i < n; i++) v[i * n + i] = 1.0;
    for (int sweep = 0; sweep < 64; sweep++) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) (i == j ? diag : off) += a[i * n + j] * a[i * n + j];
        if (off == 0.0 || off < 1e-32 * diag) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = a[p * n + q];
                // threshold Jacobi (Rutishauser): an element at rounding level of its
                // diagonal pair is set to zero instead of rotated away
                if (std::fabs(apq) <= 1e-17 * std::max(std::fabs(a[p * n + p]), std::fabs(a[q * n + q]))) {
                    a[p * n + q] = a[q * n + p] = 0.0;
                    continue;
                }
                double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++) {
                    double x = a[k * n + p], y = a[k * n + q];
                    a[k * n + p] = c * x - s * y;
                    a[k * n + q] = s * x + c * y;
                }
                for (int k = 0; k < n; k++) {
                    double x = a[p * n + k], y = a[q * n + k];
                    a[p * n + k] = c * x - s * y;
                    a[q * n + k] = s * x + c * y;
                }
                for (int k = 0; k < n; k++) {
                    double x = v[k * n + p], y = v[k * n + q];
                    v[k * n + p] = c * x - s * y;
                    v[k * n + q] = s * x + c * y;
                }
            }
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return a[x * n + x] < a[y * n + y]; });
    for (int c = 0; c < n; c++) {
        w[c] = a[idx[c] * n + idx[c]];
        for (int r = 0; r < n; r++) Y[r * n + c] = v[r * n + idx[c]];
    }
}

struct Work {
    risqgpu* h;
    int64_t N;
    int grid;
    double* partial = nullptr;  // grid x (KMAX+1)
    double* red = nullptr;      // KMAX+1
    double* small = nullptr;    // Y + lambda
    double* coef = nullptr;     // KMAX+1
    double* cols = nullptr;     // (RMAX + KMAX) x (KMAX+1): reduced projected columns, then saved norms
    SigmaTimer timer;
    // partial dots of the columns j < m of A with b (and <b, b> as column m when self)
    template <typename T>
    int dots(const T* A, int m, const T* b, bool self) {
        const int cols = m + (self ? 1 : 0);
        if (cols <= 0) return RISQGPU_OK;
        dim3 g2(grid, (cols + CCH - 1) / CCH);
        k_dots<T><<<g2, DBLK, 0, h->stream>>>(A, m, b, self ? 1 : 0, N, partial);
        return check_launch(h, "dots");
    }
    int reduce_to(int m, double* dev_out) {
        k_reduce<<<m, DBLK, 0, h->stream>>>(partial, grid, m, KMAX + 1, dev_out);
        return check_launch(h, "reduce");
    }
    int reduce(int m, double* host_out) {
        k_reduce<<<m, DBLK, 0, h->stream>>>(partial, grid, m, KMAX + 1, red);
        RQ_TRY(check_launch(h, "reduce"));
        if (host_out) {
            RQ_CUDA(h, cudaMemcpyAsync(host_out, red, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream));
            RQ_TRY(sync(h, "reduce"));
        }
        return RISQGPU_OK;
    }
};

struct LoopOut {
    int iters = 0, n_sigma = 0, reason = -1, fallbacks = 0;
    bool converged = false;
    double evals[RMAX] = {0};
    double res[RMAX] = {0};
};

// One Davidson run with basis type T.  init_int: internal-order FP64 columns (ninit)
// or null for identity columns.  On return ritz (N x nr, FP64, internal order) holds
// the last Ritz vectors.  space: largest basis before a restart (the reference's
// nroots + 10); keep: vectors kept at a restart (the reference keeps the nroots Ritz
// vectors; more gives a thick restart with the lowest `keep` Ritz vectors).
template <typename T>
int davidson_loop(Work& wk, int nr, const double* init_int, int ninit, bool normalize_init, const double* last_init,
                  double tol, double etol, int max_iter, int sigma_kind, float* fscale, double* ritz, double* hr,
                  int space, int keep, LoopOut& out) {
    risqgpu* h = wk.h;
    const int64_t N = wk.N;
    const int mss = (int64_t)space < N ? space : (int)N;
    keep = std::max(nr, std::min(keep, mss - nr));
    const bool thick = keep > nr;
    T *V = nullptr, *HV = nullptr;
    double* ybuf = nullptr;
    ScopedFree<3> release(V, HV, ybuf);
    // columns: the basis (mss), the new vectors (nr), and for a thick restart room for
    // the kept combinations before they move to the front
    const size_t ncols = (size_t)(mss + nr) + (thick ? (size_t)keep : 0);
    RQ_TRY(dalloc(h, V, ncols * N));
    RQ_TRY(dalloc(h, HV, ncols * N));
    if (thick) RQ_TRY(dalloc(h, ybuf, (size_t)KMAX * KMAX));
    const int g = wk.grid;
    // initial subspace (generate_subspace, davidson.rs:318-338)
    int dim = init_int ? ninit : std::min(2, mss);
    if (dim > mss) dim = mss;
    {
        int32_t e1 = N > 1 ? 1 : 0;
        k_fill_init<T><<<g, DBLK, 0, h->stream>>>(V, dim, N, init_int, h->d_inv, 0, e1);
        RQ_TRY(check_launch(h, "init"));
    }
    // Gram-Schmidt of column `col` of V against the columns before it, twice (classical
    // Gram-Schmidt applied twice matches MGS to rounding); leaves |t|^2 in wk.red[col]
    auto orthogonalise = [&](int col) -> int {
        T* t = V + (size_t)col * N;
        if (col > 0) {
            RQ_TRY(wk.dots(V, col, t, false));
            RQ_TRY(wk.reduce(col, nullptr));
            for (int pass = 0; pass < 2; pass++) {
                RQ_CUDA(h, cudaMemcpyAsync(wk.coef, wk.red, sizeof(double) * col, cudaMemcpyDeviceToDevice, h->stream));
                k_cgs_update<T><<<g, DBLK, 0, h->stream>>>(V, col, t, N, wk.coef);
                RQ_TRY(check_launch(h, "gram-schmidt"));
                RQ_TRY(wk.dots(V, col, t, true));
                RQ_TRY(wk.reduce(col + 1, nullptr));
            }
        } else {
            RQ_TRY(wk.dots(V, 0, t, true));
            RQ_TRY(wk.reduce(1, nullptr));
        }
        return RISQGPU_OK;
    };
    // orthonormalise multi-column initial guesses; a single caller guess is used as given, as
    // in the reference, but a guess carried over from the FP32 stage is renormalised in FP64
    // (an FP32-rounded norm error of 1e-7 would shift the Rayleigh quotient by 1e-7 |E|)
    if (init_int && (dim > 1 || normalize_init)) {
        for (int c = 0; c < dim; c++) {
            RQ_TRY(orthogonalise(c));
            k_scale<T><<<g, DBLK, 0, h->stream>>>(V + (size_t)c * N, N, wk.red + c);
        }
    }
    for (int c = 0; c < dim; c++) RQ_TRY(wk.timer.run(h, V + (size_t)c * N, HV + (size_t)c * N, sigma_kind));
    out.n_sigma += dim;
    std::vector<double> P((size_t)KMAX * KMAX, 0.0);
    // P[i][c] for i < m, c in [c0, c1): every column reduced on the device, then one copy
    // to the host, which also brings the saved squared norm of the last new vector
    // (slot `extra` of the buffer, when extra >= 0)
    double saved_norm2 = 0.0;
    auto proj_cols = [&](int c0, int c1, int m, int extra) -> int {
        const int nc = c1 - c0;
        for (int c = c0; c < c1; c++) {
            RQ_TRY(wk.dots(V, m, HV + (size_t)c * N, false));
            RQ_TRY(wk.reduce_to(m, wk.cols + (size_t)(c - c0) * (KMAX + 1)));
        }
        const int nread = extra >= 0 ? extra + 1 : nc * (KMAX + 1);
        std::vector<double> buf((size_t)nread);
        RQ_CUDA(h, cudaMemcpyAsync(buf.data(), wk.cols, sizeof(double) * nread, cudaMemcpyDeviceToHost, h->stream));
        RQ_TRY(sync(h, "projected columns"));
        for (int c = c0; c < c1; c++)
            for (int i = 0; i < m; i++) {
                const double v = buf[(size_t)(c - c0) * (KMAX + 1) + i];
                P[i * KMAX + c] = v;
                P[c * KMAX + i] = v;
            }
        if (extra >= 0) saved_norm2 = buf[extra];
        return RISQGPU_OK;
    };
    RQ_TRY(proj_cols(0, dim, dim, -1));
    std::vector<double> last(nr, 0.0);
    if (last_init) for (int c = 0; c < nr; c++) last[c] = last_init[c];
    std::vector<double> w(KMAX), Y(KMAX * KMAX), Pd(KMAX * KMAX), hostsmall(KMAX * RMAX + RMAX), ykeep(KMAX * KMAX);
    std::vector<double> red(KMAX + 1);
    double e_feat = NAN;
    std::vector<double> res_hist;
    int it;
    out.converged = false;
    for (it = 0; it < max_iter; it++) {
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < dim; j++) Pd[i * dim + j] = P[i * KMAX + j];
        jacobi_sorted(dim, Pd.data(), w.data(), Y.data());
        const bool room = dim + nr <= mss;
        for (int j = 0; j < dim; j++)
            for (int c = 0; c < nr; c++) hostsmall[j * nr + c] = Y[j * dim + c];
        for (int c = 0; c < nr; c++) hostsmall[dim * nr + c] = w[c];
        RQ_CUDA(h, cudaMemcpyAsync(wk.small, hostsmall.data(), sizeof(double) * (dim * nr + nr), cudaMemcpyHostToDevice,
                                   h->stream));
        // learned scaling: refresh the per-determinant factors when the energy used in
        // their features moved by more than 0.1 Ha (the network is trained on features
        // at the Ritz values of whole trajectories, so coarse refreshes suffice); fall
        // back to plain DPR for an iteration whenever the residual stalled (no new
        // minimum in the last 3 iterations)
        const float* fs = nullptr;
        if (fscale) {
            if (std::isnan(e_feat) || std::fabs(w[0] - e_feat) > 0.1) {
                e_feat = w[0];
                RQ_TRY(mlp_scale_impl(h, e_feat, fscale));
            }
            const size_t k = res_hist.size();
            bool stalled = false;
            if (k >= 4) {
                double best_before = res_hist[0];
                for (size_t j = 1; j + 3 < k; j++) best_before = std::min(best_before, res_hist[j]);
                double best_recent = std::min(res_hist[k - 1], std::min(res_hist[k - 2], res_hist[k - 3]));
                stalled = !(best_recent < best_before);
            }
            if (stalled) out.fallbacks++;
            else fs = fscale;
        }
        k_ritz<T><<<g, DBLK, 0, h->stream>>>(V, HV, dim, nr, N, wk.small, h->d_diag, fs, room ? 1 : 0, ritz, hr,
                                             V + (size_t)dim * N, wk.partial);
        RQ_TRY(check_launch(h, "ritz"));
        RQ_TRY(wk.reduce(nr + 1, red.data()));
        bool all_small = true, all_e = true;
        res_hist.push_back(std::sqrt(red[0]));
        for (int c = 0; c < nr; c++) {
            out.res[c] = std::sqrt(red[c]);
            out.evals[c] = w[c];
            if (!(out.res[c] < tol)) all_small = false;
            if (!(std::fabs(w[c] - last[c]) < etol)) all_e = false;
        }
        if (N <= 2 || (all_small && all_e)) {
            out.converged = true;
            out.reason = N <= 2 ? 3 : 0;
            break;
        }
        for (int c = 0; c < nr; c++) last[c] = w[c];
        if (room) {
            if (std::sqrt(red[nr]) < 1e-9) { out.converged = true; out.reason = 1; break; }
            // slot of the last new vector's squared norm: after the nr projected columns
            const int norm_slot = nr * (KMAX + 1);
            for (int c = 0; c < nr; c++) {
                const int col = dim + c;
                RQ_TRY(orthogonalise(col));
                if (c == nr - 1)
                    RQ_CUDA(h, cudaMemcpyAsync(wk.cols + norm_slot, wk.red + col, sizeof(double),
                                               cudaMemcpyDeviceToDevice, h->stream));
                k_scale<T><<<g, DBLK, 0, h->stream>>>(V + (size_t)col * N, N, wk.red + col);
            }
            for (int c = 0; c < nr; c++)
                RQ_TRY(wk.timer.run(h, V + (size_t)(dim + c) * N, HV + (size_t)(dim + c) * N, sigma_kind));
            RQ_TRY(proj_cols(dim, dim + nr, dim + nr, norm_slot));
            // a dependent last vector (MGS norm < 1e-9, modified_gram_schmidt.rs:22-36) ends the
            // solve; its sigma and projected column, computed before the norm reached the host,
            // are dropped, so the result is the one of stopping before them
            if (std::sqrt(saved_norm2) < 1e-9) { out.converged = true; out.reason = 2; break; }
            out.n_sigma += nr;
            dim += nr;
        } else if (!thick) {
            // restart to the Ritz vectors (davidson.rs:261-269)
            k_set_cols<T><<<g, DBLK, 0, h->stream>>>(V, HV, ritz, hr, nr, N);
            RQ_TRY(check_launch(h, "restart"));
            dim = nr;
            std::fill(P.begin(), P.end(), 0.0);
            RQ_TRY(proj_cols(0, dim, dim, -1));
        } else {
            // thick restart: the lowest `keep` Ritz vectors and their H products, formed
            // from the basis in the spare columns, then moved to the front
            for (int j = 0; j < dim; j++)
                for (int c = 0; c < keep; c++) ykeep[j * keep + c] = Y[j * dim + c];
            RQ_CUDA(h, cudaMemcpyAsync(ybuf, ykeep.data(), sizeof(double) * dim * keep, cudaMemcpyHostToDevice,
                                       h->stream));
            T* sv = V + (size_t)(mss + nr) * N;
            T* shv = HV + (size_t)(mss + nr) * N;
            dim3 g2(g, (keep + CCH - 1) / CCH);
            k_combine<T><<<g2, DBLK, 0, h->stream>>>(V, HV, dim, keep, N, ybuf, sv, shv);
            RQ_TRY(check_launch(h, "thick restart"));
            RQ_CUDA(h, cudaMemcpyAsync(V, sv, sizeof(T) * keep * N, cudaMemcpyDeviceToDevice, h->stream));
            RQ_CUDA(h, cudaMemcpyAsync(HV, shv, sizeof(T) * keep * N, cudaMemcpyDeviceToDevice, h->stream));
            dim = keep;
            std::fill(P.begin(), P.end(), 0.0);
            RQ_TRY(proj_cols(0, dim, dim, -1));
        }
    }
    out.iters += it + (it < max_iter ? 1 : 0);
    return sync(h, "davidson");
}

}  // namespace

int davidson_impl(risqgpu* h, int nroots, const double* init, int ninit, double tol, double etol, int max_iter,
                  int mode, int precond, double* evals, double* evecs, risqgpu_dstats* st) {
    auto t0 = std::chrono::steady_clock::now();
    h->sigma_ms_acc = 0.0;
    if (!h->built) { h->err = "davidson before build"; return RISQGPU_ERR_INVALID; }
    if (nroots < 1 || nroots > RMAX) { h->err = "nroots must be in [1, 8]"; return RISQGPU_ERR_INVALID; }
    if ((size_t)nroots > h->N) { h->err = "nroots > N"; return RISQGPU_ERR_INVALID; }
    // search space and restart size: the reference's (nroots + 10, nroots) unless the
    // handle was given others (risqgpu_set_subspace)
    const int space = h->dav_space > 0 ? h->dav_space : nroots + 10;
    const int keep = h->dav_keep > 0 ? h->dav_keep : nroots;
    if (space + nroots > KMAX || space < 2 * nroots) {
        h->err = "search space must lie in [2 nroots, " + std::to_string(KMAX) + " - nroots]";
        return RISQGPU_ERR_INVALID;
    }
    if (init && (ninit < 1 || ninit > space)) { h->err = "bad ninit"; return RISQGPU_ERR_INVALID; }
    if (init && nroots > 1 && ninit < nroots) { h->err = "ninit must be >= nroots for several roots"; return RISQGPU_ERR_INVALID; }
    if (mode != RISQGPU_MODE_FP64 &&
        (h->precision == RISQGPU_FP64 || h->precision == RISQGPU_COLS || h->precision == RISQGPU_MATRIX_FREE)) {
        h->err = "the FP32 sigma of MIXED / FP32 mode needs an FP32 or MIXED build";
        return RISQGPU_ERR_INVALID;
    }
    if (h->upper && h->precision == RISQGPU_FP32 && mode != RISQGPU_MODE_FP32) {
        h->err = "an FP32 upper-triangle build has no FP64 sigma; use MIXED_UPPER or FP32 mode";
        return RISQGPU_ERR_INVALID;
    }
    if (precond == RISQGPU_PRECOND_LEARNED && !h->mlp.loaded) {
        h->err = "learned preconditioner requested but no MLP loaded";
        return RISQGPU_ERR_INVALID;
    }
    const int64_t N = (int64_t)h->N;
    if (init) {
        const size_t n_in = (size_t)ninit * h->N;
        for (size_t i = 0; i < n_in; i++)
            if (!std::isfinite(init[i])) {
                h->err = "initial guess holds a non-finite value at index " + std::to_string(i);
                return RISQGPU_ERR_INVALID;
            }
    }
    Work wk;
    wk.h = h;
    wk.N = N;
    double *ritz = nullptr, *hr = nullptr, *init_int = nullptr, *tmp = nullptr, *seed = nullptr, *outv = nullptr;
    float* fscale = nullptr;
    ScopedFree<5> release_work(wk.partial, wk.red, wk.small, wk.coef, wk.cols);
    ScopedFree<7> release_vecs(ritz, hr, init_int, tmp, seed, outv, fscale);
    wk.grid = std::max(1, std::min<int>((int)((N + DBLK - 1) / DBLK), num_sms(h) * 4));
    RQ_TRY(dalloc(h, wk.partial, (size_t)wk.grid * (KMAX + 1)));
    RQ_TRY(dalloc(h, wk.red, KMAX + 1));
    RQ_TRY(dalloc(h, wk.small, KMAX * RMAX + RMAX));
    RQ_TRY(dalloc(h, wk.coef, KMAX + 1));
    RQ_TRY(dalloc(h, wk.cols, (size_t)(KMAX + 2) * (KMAX + 1)));
    RQ_TRY(dalloc(h, ritz, (size_t)nroots * N));
    RQ_TRY(dalloc(h, hr, (size_t)nroots * N));
    int use_init = init ? std::min(ninit, space) : 0;
    if (init) {
        RQ_TRY(dalloc(h, tmp, (size_t)use_init * N));
        RQ_TRY(dalloc(h, init_int, (size_t)use_init * N));
        RQ_CUDA(h, cudaMemcpyAsync(tmp, init, sizeof(double) * use_init * N, cudaMemcpyHostToDevice, h->stream));
        k_to_internal<<<wk.grid, DBLK, 0, h->stream>>>(tmp, h->d_orig, N, use_init, init_int);
        RQ_TRY(check_launch(h, "init"));
    }
    LoopOut lo;
    int n64 = 0;
    if (mode == RISQGPU_MODE_FP64) {
        if (precond == RISQGPU_PRECOND_LEARNED) RQ_TRY(dalloc(h, fscale, N));
        RQ_TRY(davidson_loop<double>(wk, nroots, init_int, use_init, false, nullptr, tol, etol, max_iter, 0, fscale, ritz, hr,
                                     space, keep, lo));
        n64 = lo.n_sigma;
    } else {
        if (precond == RISQGPU_PRECOND_LEARNED) RQ_TRY(dalloc(h, fscale, N));
        RQ_TRY(davidson_loop<float>(wk, nroots, init_int, use_init, false, nullptr, tol, etol, max_iter, 1, fscale, ritz, hr,
                                    space, keep, lo));
        const int n32 = lo.n_sigma;
        // closing FP64-sigma sweeps (stored FP32 + remainder, or elements recomputed in FP64);
        // FP32 mode stops after the FP32 stage
        if (lo.converged && mode == RISQGPU_MODE_MIXED) {
            // closing FP64-sigma sweeps from the FP64 Ritz vectors
            LoopOut lr;
            RQ_TRY(dalloc(h, seed, (size_t)nroots * N));
            RQ_CUDA(h, cudaMemcpyAsync(seed, ritz, sizeof(double) * nroots * N, cudaMemcpyDeviceToDevice, h->stream));
            RQ_TRY(davidson_loop<double>(wk, nroots, seed, nroots, true, lo.evals, tol, etol, max_iter, 0, nullptr, ritz, hr,
                                         space, keep, lr));
            dfree(seed);
            lr.iters += lo.iters;
            lr.fallbacks = lo.fallbacks;
            n64 = lr.n_sigma;
            lr.n_sigma += n32;
            lo = lr;
        }
    }
    for (int c = 0; c < nroots; c++) evals[c] = lo.evals[c];
    if (evecs) {
        RQ_TRY(dalloc(h, outv, (size_t)nroots * N));
        k_to_caller<<<wk.grid, DBLK, 0, h->stream>>>(ritz, h->d_orig, N, nroots, outv);
        RQ_CUDA(h, cudaMemcpyAsync(evecs, outv, sizeof(double) * nroots * N, cudaMemcpyDeviceToHost, h->stream));
        RQ_TRY(sync(h, "evecs"));
    }
    RQ_TRY(sync(h, "davidson end"));
    wk.timer.collect(h);
    if (st) {
        st->iters = lo.iters;
        st->n_sigma = lo.n_sigma;
        st->n_sigma_fp64 = n64;
        st->converged = lo.converged ? 1 : 0;
        st->reason = lo.reason;
        st->learned_fallbacks = lo.fallbacks;
        for (int c = 0; c < nroots && c < 8; c++) st->residual[c] = lo.res[c];
        st->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        st->ms_sigma = h->sigma_ms_acc;
    }
    return lo.converged ? RISQGPU_OK : RISQGPU_ERR_NOT_CONVERGED;
}

}  // namespace risq
