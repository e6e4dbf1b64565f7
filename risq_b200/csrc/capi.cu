// extern "C" entry points of librisqgpu.so (declared in include/risqgpu.h).
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <unordered_map>

#include "internal.cuh"

namespace risq {

namespace {
std::mutex g_ledger_mu;
std::unordered_map<void*, std::pair<risqgpu*, size_t>> g_ledger;
}  // namespace

void mem_record(risqgpu* h, void* p, size_t bytes) {
    std::lock_guard<std::mutex> lk(g_ledger_mu);
    g_ledger[p] = {h, bytes};
    h->mem_used += bytes;
}

void mem_forget(void* p) {
    std::lock_guard<std::mutex> lk(g_ledger_mu);
    auto it = g_ledger.find(p);
    if (it == g_ledger.end()) return;
    it->second.first->mem_used -= it->second.second;
    g_ledger.erase(it);
}

}  // namespace risq

using namespace risq;

namespace {

// Make the handle's device current for the duration of a call.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

size_t combine_2_host(long p, long q) {
    long i = p < 0 ? -p : p, j = q < 0 ? -q : q;
    return i > j ? (size_t)((i * (i - 1)) / 2 + j) : (size_t)((j * (j - 1)) / 2 + i);
}

}  // namespace

extern "C" {

const char* risqgpu_version(void) { return "risq_b200 0.1 (sm_100a)"; }

int risqgpu_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int risqgpu_create(int norb, const double* one_body, size_t n1, const double* two_body, size_t n2, double e_nuc,
                   int device, risqgpu_t** out) {
    if (!out) return RISQGPU_ERR_INVALID;
    *out = nullptr;
    if (norb < 1 || norb > 128 || !one_body || !two_body) return RISQGPU_ERR_INVALID;
    size_t e1 = combine_2_host(norb + 1, norb + 1);
    size_t c2n = combine_2_host(norb + 1, norb + 1);
    size_t e2 = combine_2_host((long)c2n, (long)c2n);
    if (n1 != e1 || n2 != e2) return RISQGPU_ERR_INVALID;
    int ndev = risqgpu_device_count();
    if (ndev == 0) return RISQGPU_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return RISQGPU_ERR_INVALID;
    risqgpu* h = new (std::nothrow) risqgpu();
    if (!h) return RISQGPU_ERR_OOM;
    h->device = device;
    DeviceGuard g(device);
    h->norb = norb;
    h->W = norb > 64 ? 2 : 1;
    h->nuc = e_nuc;
    h->n1 = n1;
    h->n2 = n2;
    int rc = RISQGPU_OK;
    if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) rc = RISQGPU_ERR_CUDA;
    h->stream = h->own_stream;
    if (!rc) rc = dalloc(h, h->d_h1, n1);
    if (!rc) rc = dalloc(h, h->d_h2, n2);
    if (!rc && cudaMemcpy(h->d_h1, one_body, n1 * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) rc = RISQGPU_ERR_CUDA;
    if (!rc && cudaMemcpy(h->d_h2, two_body, n2 * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) rc = RISQGPU_ERR_CUDA;
    if (!rc) {
        h->h_h1.assign(one_body, one_body + n1);
        h->h_h2.assign(two_body, two_body + n2);
    }
    if (rc) {
        risqgpu_destroy(h);
        return rc;
    }
    *out = h;
    return RISQGPU_OK;
}

void risqgpu_destroy(risqgpu_t* h) {
    if (!h) return;
    DeviceGuard g(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_dets(h);
    free_mlp(h);
    dfree(h->d_h1);
    dfree(h->d_h2);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
}

const char* risqgpu_last_error(const risqgpu_t* h) { return h ? h->err.c_str() : "null handle"; }

int risqgpu_set_dets(risqgpu_t* h, const uint64_t* dets, size_t n, size_t n_stored_h, const double* diag) {
    if (!h) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    h->err.clear();
    return set_dets_impl(h, dets, n, n_stored_h, diag);
}

int risqgpu_build_h(risqgpu_t* h, int precision, int builder, risqgpu_hstats* stats) {
    if (!h) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    return build_h_impl(h, precision, builder, stats);
}

int risqgpu_nnz(const risqgpu_t* h, uint64_t* nnz_upper, uint64_t* nnz_full) {
    if (!h) return RISQGPU_ERR_INVALID;
    if (nnz_upper) *nnz_upper = h->nnz_upper;
    if (nnz_full) *nnz_full = h->nnz_full;
    return h->built ? RISQGPU_OK : RISQGPU_ERR_INVALID;
}

int risqgpu_export_upper(risqgpu_t* h, int64_t* rowptr, int64_t* cols, double* vals, size_t cap, double* diag) {
    if (!h || !rowptr || (!cols && cap) || (!vals && cap)) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    return export_upper_impl(h, rowptr, cols, vals, cap, diag);
}

int risqgpu_export_rows(risqgpu_t* h, const int64_t* rows, size_t k, int64_t* out_row, int64_t* out_col,
                        double* out_val, size_t cap, size_t* count) {
    if (!h || !count || (k && !rows) || (cap && (!out_row || !out_col || !out_val))) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    *count = 0;
    return export_rows_impl(h, rows, k, out_row, out_col, out_val, cap, count);
}

int risqgpu_sigma(risqgpu_t* h, const double* x, double* y, int nvec) {
    if (!h || !x || !y) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    if (nvec >= 1 && h->built) {
        const size_t n = h->N * (size_t)nvec;
        for (size_t i = 0; i < n; i++)
            if (!std::isfinite(x[i])) {
                h->err = "x holds a non-finite value at index " + std::to_string(i);
                return RISQGPU_ERR_INVALID;
            }
    }
    return sigma_host(h, x, y, nvec);
}

int risqgpu_sigma_device(risqgpu_t* h, const void* x_dev, void* y_dev, int dtype) {
    if (!h || !x_dev || !y_dev || (dtype != 0 && dtype != 1)) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    int rc = sigma_device(h, x_dev, y_dev, dtype);
    if (rc) return rc;
    return sync(h, "sigma_device");
}

int risqgpu_davidson(risqgpu_t* h, int nroots, const double* init, int ninit, double tol, double etol, int max_iter,
                     int mode, int precond, double* evals, double* evecs, risqgpu_dstats* stats) {
    if (!h || !evals || max_iter < 1 || mode < 0 || mode > 2 || (precond != 0 && precond != 1))
        return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    return davidson_impl(h, nroots, init, ninit, tol, etol, max_iter, mode, precond, evals, evecs, stats);
}

int risqgpu_sparse_optimize(risqgpu_t* h, const double* init_coeffs, double coeff_eps, double energy_eps,
                            int max_iter, int precision, int mode, int precond, double* energy, double* coeffs,
                            risqgpu_hstats* hstats, risqgpu_dstats* dstats) {
    if (!h || !energy || !coeffs || max_iter < 1) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    if (hstats) std::memset(hstats, 0, sizeof(*hstats));
    if (dstats) std::memset(dstats, 0, sizeof(*dstats));
    int rc = build_h_impl(h, precision, RISQGPU_BUILDER_AUTO, hstats);
    if (rc) return rc;
    double e = 0.0;
    std::vector<double> v(h->N);
    rc = davidson_impl(h, 1, init_coeffs, init_coeffs ? 1 : 0, coeff_eps, energy_eps, max_iter, mode, precond, &e,
                       v.data(), dstats);
    if (rc == RISQGPU_ERR_NOT_CONVERGED) {
        h->err = "Davidson Algorithm did not converge!";
        return rc;  // energy and coefficients are left unchanged (var/davidson.rs:109-111)
    }
    if (rc) return rc;
    *energy = e;
    std::memcpy(coeffs, v.data(), sizeof(double) * h->N);
    return RISQGPU_OK;
}

int risqgpu_set_subspace(risqgpu_t* h, int max_space, int keep) {
    if (!h || max_space < 0 || keep < 0 || max_space > 56 || (max_space > 0 && keep > max_space / 2)) {
        if (h) h->err = "max_space must lie in [0, 56] and keep in [0, max_space / 2]";
        return RISQGPU_ERR_INVALID;
    }
    h->dav_space = max_space;
    h->dav_keep = keep;
    return RISQGPU_OK;
}

int risqgpu_set_partition(risqgpu_t* h, int rank, int nranks, risqgpu_allreduce_fn reduce, void* user) {
    if (!h) return RISQGPU_ERR_INVALID;
    if (nranks < 1 || rank < 0 || rank >= nranks || (nranks > 1 && !reduce)) {
        h->err = "partition needs 0 <= rank < nranks and, for nranks > 1, a reduce function";
        return RISQGPU_ERR_INVALID;
    }
    h->part_rank = rank;
    h->part_n = nranks;
    h->part_reduce = nranks > 1 ? reduce : nullptr;
    h->part_user = user;
    return RISQGPU_OK;
}

int risqgpu_set_reproducible(risqgpu_t* h, int on) {
    if (!h) return RISQGPU_ERR_INVALID;
    h->reproducible = on != 0;
    return RISQGPU_OK;
}

int risqgpu_set_memory_limit(risqgpu_t* h, size_t bytes) {
    if (!h) return RISQGPU_ERR_INVALID;
    h->mem_limit = bytes;
    return RISQGPU_OK;
}

int risqgpu_memory_used(const risqgpu_t* h, size_t* used, size_t* limit) {
    if (!h) return RISQGPU_ERR_INVALID;
    if (used) *used = h->mem_used;
    if (limit) *limit = h->mem_limit;
    return RISQGPU_OK;
}

int risqgpu_set_stream(risqgpu_t* h, void* stream) {
    if (!h) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return RISQGPU_ERR_CUDA;
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return RISQGPU_OK;
}

int risqgpu_ham_diag(risqgpu_t* h, const uint64_t* dets, size_t n, double* out) {
    if (!h || (n && (!dets || !out))) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    return ham_elements_impl(h, dets, nullptr, n, out, true);
}

int risqgpu_ham_off_diag(risqgpu_t* h, const uint64_t* d1, const uint64_t* d2, size_t n, double* out) {
    if (!h || (n && (!d1 || !d2 || !out))) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    return ham_elements_impl(h, d1, d2, n, out, false);
}

int risqgpu_set_precond_mlp(risqgpu_t* h, int n_in, int hidden, const float* w1, const float* b1, const float* w2,
                            const float* b2, const float* w3, const float* b3, const float* feat_norm) {
    if (!h) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    return set_mlp_impl(h, n_in, hidden, w1, b1, w2, b2, w3, b3, feat_norm);
}

int risqgpu_precond_factors(risqgpu_t* h, double energy, float* out) {
    if (!h || !out) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    return precond_factors_impl(h, energy, out);
}

int risqgpu_self_energy(risqgpu_t* h, double energy, double gmin, double* out) {
    if (!h || !out) return RISQGPU_ERR_INVALID;
    DeviceGuard g(h->device);
    return self_energy_impl(h, energy, gmin, out);
}

}  // extern "C"
