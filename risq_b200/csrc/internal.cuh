// Internal state of a risqgpu handle and shared host helpers.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>
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
    // device memory held by this handle through dalloc, and the caller's bound on it
    // (0 = none; risqgpu_set_memory_limit)
    size_t mem_used = 0;
    size_t mem_limit = 0;

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
    int precision = -1;   // value storage: FP64, FP32, MIXED, COLS or MATRIX_FREE
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
    // matrix-free storage: the sigma's row counter and the builder's singles threshold
    int* d_mf_counter = nullptr;
    double mf_thr = 0.0;

    // Tiled upper-triangle storage (upper builds).  Rows are cut into panels of
    // 2^tile_rb consecutive rows and columns into windows of 2^tile_cb.  Each panel
    // holds its dense (panel, window) tiles, elements coded (row in panel << tile_cb |
    // column in window), followed by its leftover elements (pairs in tiles too sparse
    // to stage), coded by their column, in row order.  Values share d_val64 / d_val32
    // / d_val_lo with the element index.
    bool tiled = false;
    int tile_rb = 0, tile_cb = 0;
    int64_t n_panels = 0;
    int64_t n_tiles = 0;
    uint64_t n_dense_el = 0;          // stored pairs in dense tiles
    int64_t* d_panel_tile = nullptr;  // n_panels + 1: first tile of each panel
    // sigma work units: runs of one panel's tiles of about equal pair counts, largest
    // first; 3 int64 each: first tile, end tile, panel * 2 + (1 if the unit also takes
    // the panel's leftover pairs)
    int64_t n_units = 0;
    int64_t* d_units = nullptr;
    int32_t* d_tile_win = nullptr;    // window of each tile
    float* d_tile_bound = nullptr;    // FP32 values: largest row or column sum of |H| in each tile
    int32_t* d_tile_len = nullptr;    // elements of each tile
    int64_t* d_tile_off = nullptr;    // first element of each tile
    int64_t* d_left_off = nullptr;    // N: first leftover element of each row
    int32_t* d_left_len = nullptr;    // N: leftover elements of each row
    uint32_t* d_el_idx = nullptr;     // element index (coded as above)
    double h_row_abs_max = 0.0;       // max over rows of sum_q |H_pq| (both triangles), for the fixed-point scale
    // sigma work space, allocated with the matrix: int64 fixed-point accumulators
    // (N) and two scalars (max |x|, scale)
    long long* d_acc = nullptr;
    double* d_sig_scalars = nullptr;

    // Row-block partition for several GPUs (risqgpu_set_partition): this handle builds
    // and applies the row panels [part_p_lo, part_p_hi) of the tiled layout; partial
    // sums are added across the ranks by the caller's all-reduce.
    bool reproducible = false;  // FP32 sigma in fixed point too (risqgpu_set_reproducible)
    int part_rank = 0, part_n = 1;
    risqgpu_allreduce_fn part_reduce = nullptr;
    void* part_user = nullptr;
    int64_t part_p_lo = 0, part_p_hi = 0;

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
    // Davidson search space and restart size (0 = the reference's nroots + 10 and nroots)
    int dav_space = 0;
    int dav_keep = 0;

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

// Allocation ledger: every allocation made through dalloc is recorded with its handle
// and size, so that dfree can return the bytes to that handle's count (mem_used).
void mem_record(risqgpu* h, void* p, size_t bytes);
void mem_forget(void* p);

// Free a device pointer (ignores null) and reset it.
template <typename T>
inline void dfree(T*& p) {
    if (p) {
        mem_forget((void*)p);
        cudaFree(p);
    }
    p = nullptr;
}

template <typename T>
inline int dalloc(risqgpu* h, T*& p, size_t count) {
    dfree(p);
    if (count == 0) count = 1;
    const size_t bytes = count * sizeof(T);
    if (h->mem_limit && h->mem_used + bytes > h->mem_limit) {
        h->err = "allocation of " + std::to_string(bytes) + " bytes exceeds the handle's device memory limit (" +
                 std::to_string(h->mem_used) + " of " + std::to_string(h->mem_limit) + " bytes in use)";
        return RISQGPU_ERR_OOM;
    }
    cudaError_t e = cudaMalloc((void**)&p, bytes);
    if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        h->err = "cudaMalloc(" + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? RISQGPU_ERR_OOM : RISQGPU_ERR_CUDA;
    }
    mem_record(h, (void*)p, bytes);
    return RISQGPU_OK;
}

// Device bytes a new allocation may take: free device memory, bounded by the handle's limit.
inline size_t mem_available(risqgpu* h) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        fr = 0;
    }
    if (h->mem_limit) fr = std::min(fr, h->mem_limit > h->mem_used ? h->mem_limit - h->mem_used : (size_t)0);
    return fr;
}

// Frees the device pointers it was given when it goes out of scope, so that every
// early return of a function releases its work buffers.
template <int K>
struct ScopedFree {
    void** slots[K];
    template <typename... T>
    explicit ScopedFree(T*&... p) : slots{reinterpret_cast<void**>(&p)...} {
        static_assert(sizeof...(T) == K, "ScopedFree<K> takes K pointers");
    }
    ~ScopedFree() {
        for (void** s : slots) dfree(*s);
    }
    ScopedFree(const ScopedFree&) = delete;
    ScopedFree& operator=(const ScopedFree&) = delete;
};

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
// One FP64 vector between the caller's determinant order and the internal (sorted)
// order, on the handle's stream: xi[p] = x[orig[p]] / y[orig[p]] = yi[p].
int permute_in(risqgpu* h, const double* x, double* xi);
int permute_out(risqgpu* h, const double* yi, double* y);

// tiled upper-triangle storage (tiles.cu)
int tile_shape(int64_t N, int& rb, int& cb);
int sigma_tiles(risqgpu* h, const void* x, void* y, int kind);
// FP64 sigma of a matrix-free build (build_h.cu), internal order
int sigma_matrix_free(risqgpu* h, const double* x, double* y);
// Sum `count` int64 values in place across the partition's ranks (the caller's all-reduce,
// on the handle's stream).
int part_allreduce(risqgpu* h, void* buf_dev, size_t count);
int tiles_coo(risqgpu* h, int32_t* p, int32_t* q, double* v);
int tiles_self_energy(risqgpu* h, double energy, double gmin, double* out);
int tiles_rows(risqgpu* h, const uint32_t* mark, int64_t* out_r, int64_t* out_c, double* out_v,
               unsigned long long* count, unsigned long long cap);
int export_rows_impl(risqgpu* h, const int64_t* rows, size_t k, int64_t* out_r, int64_t* out_c, double* out_v,
                     size_t cap, size_t* count);
void free_tiles(risqgpu* h);
// Converts the CSR rows of a build, chunk by chunk of whole panels, into the tiled
// arrays (d_el_idx and the value arrays must already hold room for every element).
struct TileBuilder {
    risqgpu* h = nullptr;
    unsigned long long* row_abs = nullptr;  // N: sum_q |H_pq| over both triangles, units of 2^-32
    unsigned long long* absmax = nullptr;
    size_t tile_cap = 0;
    int64_t el_cap = 0;
    int64_t el_next = 0, tile_next = 0;
    std::vector<int64_t> panel_el;  // host: first element of each panel, and the end
    int begin(risqgpu* h, int64_t n_panels, int64_t element_capacity);
    template <typename VIN>
    int chunk(int64_t p_lo, int64_t p_hi, const int64_t* row_start, int64_t base, const int32_t* row_len,
              const int32_t* cols, const VIN* vin, const float* vlo_in, VIN* vout, float* vlo_out);
    int finish();
    int make_units();
    ~TileBuilder();
};

// davidson (davidson.cu)
int davidson_impl(risqgpu* h, int nroots, const double* init, int ninit, double tol, double etol, int max_iter,
                  int mode, int precond, double* evals, double* evecs, risqgpu_dstats* st);
int set_mlp_impl(risqgpu* h, int n_in, int hidden, const float* w1, const float* b1, const float* w2,
                 const float* b2, const float* w3, const float* b3, const float* feat_norm);
void free_mlp(risqgpu* h);
int precond_factors_impl(risqgpu* h, double energy, float* out);
int self_energy_impl(risqgpu* h, double energy, double gmin, double* out);

}  // namespace risq
