// Internal state of a risqgpu handle and shared host helpers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/risqgpu.h"

namespace risq {

// A failed CUDA call inside a handle method: record and return.
#define RQ_CUDA(h, call)                                                                         \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            (h)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                       \
            return e_ == cudaErrorMemoryAllocation ? RISQGPU_ERR_OOM : RISQGPU_ERR_CUDA;         \
        }                                                                                        \
    } while (0)

#define RQ_TRY(call)                 \
    do {                             \
        int s_ = (call);             \
        if (s_ != RISQGPU_OK) return s_; \
    } while (0)

struct MlpWeights {
    int n_in = 0, hidden = 0;
    // device copies: bf16 weights as raw u16 + fp32 biases
    uint16_t *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
    float *b1 = nullptr, *b2 = nullptr, *b3 = nullptr;
    float4 fnorm = {0.f, 1.f, 0.f, 1.f};  // (mu_e, 1/sd_e, mu_h, 1/sd_h)
    bool loaded = false;
};

}  // namespace risq

struct risqgpu {
    int device = 0;
    cudaStream_t stream = nullptr;        // stream all work is issued on
    cudaStream_t own_stream = nullptr;    // the handle's own stream
    double sigma_ms_acc = 0.0;            // event time of sigma launches inside Davidson
    bool time_sigma = false;
    std::string err;

    // integrals (reference packed layout)
    int norb = 0;
    double nuc = 0.0;
    size_t n1 = 0, n2 = 0;
    double* d_h1 = nullptr;
    double* d_h2 = nullptr;
    std::vector<double> h_h1, h_h2;  // host copies (excitation tables, diagonal of HF)

    // determinant set, internal order = sorted by (up, dn)
    int W = 1;        // 64-bit words per spin string
    size_t N = 0;     // determinants
    size_t nsh = 0;   // n_stored_h of the pending build
    int n_up = 0, n_dn = 0;
    uint64_t* d_up = nullptr;    // SoA [W][N]
    uint64_t* d_dn = nullptr;    // SoA [W][N]
    uint64_t* d_up_b = nullptr;  // alpha strings in beta-group order, SoA [W][N]
    int32_t* d_orig = nullptr;   // internal -> caller index
    int32_t* d_inv = nullptr;    // caller -> internal index
    double* d_diag = nullptr;    // H_ii, internal order

    // alpha groups over the internal order
    int32_t G_a = 0;
    int32_t* d_ga = nullptr;        // group of each det
    int32_t* d_ga_start = nullptr;  // G_a + 1
    // beta groups: order_b lists internal indices sorted by (dn, up)
    int32_t G_b = 0;
    int32_t* d_gb = nullptr;        // group of each det (internal index)
    int32_t* d_gb_start = nullptr;  // G_b + 1 (positions in order_b)
    int32_t* d_order_b = nullptr;
    int32_t* d_pos_b = nullptr;     // position of each det in order_b
    // single-excitation partners between alpha groups
    int32_t* d_pa_start = nullptr;  // G_a + 1
    int32_t* d_pa_list = nullptr;
    size_t n_pa = 0;
    // open-addressing table (alpha group, beta string) -> internal index, one-word
    // strings only (norb <= 64); 2^ht_bits slots {beta lo, beta hi, group, index},
    // index -1 = empty
    int4* d_ht = nullptr;
    int ht_bits = 0;

    // sparse H: both triangles, rows in internal order, diagonal separate
    int precision = -1;   // value storage: FP64, FP32, MIXED or COLS
    bool upper = false;   // only pairs with q > p (internal order) are stored
    bool built = false;
    int64_t* d_row_start = nullptr;  // N + 1 (segment starts; capacity per row)
    int32_t* d_row_len = nullptr;    // stored elements per row
    int32_t* d_cols = nullptr;
    double* d_val64 = nullptr;
    float* d_val32 = nullptr;
    float* d_val_lo = nullptr;  // FP64 - FP32 remainder (MIXED)
    size_t cap = 0;             // allocated element slots
    uint64_t nnz_full = 0;
    uint64_t nnz_upper = 0;

    // previous build kept for an incremental extension
    size_t prev_N = 0;
    int32_t* d_prev_orig = nullptr;
    int64_t* d_prev_row_start = nullptr;
    int32_t* d_prev_row_len = nullptr;
    int32_t* d_prev_cols = nullptr;
    double* d_prev_val64 = nullptr;
    float* d_prev_val32 = nullptr;
    float* d_prev_val_lo = nullptr;
    int prev_precision = -1;

    // host copy of the caller-order determinants (incremental prefix check)
    std::vector<uint64_t> h_dets;

    risq::MlpWeights mlp;

    // variational wavefunction of the last risqgpu_variational run (caller order)
    std::vector<uint64_t> wf_dets;
    std::vector<double> wf_coeffs, wf_diag;
    double wf_energy = 0.0;
    std::vector<risqgpu_var_iter> var_log;
    // result of the last risqgpu_find_new_dets
    std::vector<uint64_t> pend_dets;
    std::vector<double> pend_diag;
};

namespace risq {

// Free a device pointer (ignores null) and reset it.
template <typename T>
inline void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

template <typename T>
inline int dalloc(risqgpu* h, T*& p, size_t count) {
    dfree(p);
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        h->err = "cudaMalloc(" + std::to_string(count * sizeof(T)) + " bytes): " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? RISQGPU_ERR_OOM : RISQGPU_ERR_CUDA;
    }
    return RISQGPU_OK;
}

inline int check_launch(risqgpu* h, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        h->err = std::string(what) + ": " + cudaGetErrorString(e);
        return RISQGPU_ERR_CUDA;
    }
    return RISQGPU_OK;
}

inline int sync(risqgpu* h, const char* what) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        h->err = std::string(what) + ": " + cudaGetErrorString(e);
        return RISQGPU_ERR_CUDA;
    }
    return RISQGPU_OK;
}

inline int num_sms(risqgpu* h) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, h->device);
    return v;
}

// builder pieces (build_h.cu)
int set_dets_impl(risqgpu* h, const uint64_t* dets, size_t n, size_t nsh, const double* diag);
int build_h_impl(risqgpu* h, int precision, int builder, risqgpu_hstats* st);
int export_upper_impl(risqgpu* h, int64_t* rowptr, int64_t* cols, double* vals, size_t cap, double* diag);
int ham_elements_impl(risqgpu* h, const uint64_t* d1, const uint64_t* d2, size_t n, double* out, bool diag_only);
void free_csr(risqgpu* h);
void free_dets(risqgpu* h);

// sigma (sigma.cu).  kind: 0 = FP64 values (or FP32 hi + lo in MIXED storage) on
// FP64 vectors, 1 = FP32 values on FP32 vectors.
int sigma_device(risqgpu* h, const void* x, void* y, int kind);
int sigma_host(risqgpu* h, const double* x, double* y, int nvec);

// davidson (davidson.cu)
int davidson_impl(risqgpu* h, int nroots, const double* init, int ninit, double tol, double etol, int max_iter,
                  int mode, int precond, double* evals, double* evecs, risqgpu_dstats* st);
int set_mlp_impl(risqgpu* h, int n_in, int hidden, const float* w1, const float* b1, const float* w2,
                 const float* b2, const float* w3, const float* b3, const float* feat_norm);
void free_mlp(risqgpu* h);
int precond_factors_impl(risqgpu* h, double energy, float* out);
int self_energy_impl(risqgpu* h, double energy, double gmin, double* out);

}  // namespace risq
