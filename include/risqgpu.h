/*
 * risqgpu.h -- C ABI of the B200 HCI variational hot path.
 *
 * One handle holds, on one GPU: the integrals, the determinant set, the sparse
 * Hamiltonian over it and the Davidson workspace.  The entry points map onto
 * the reference crate (aaholmes/risq) as follows:
 *
 *   risqgpu_create        Ham + Ints after read_ints      src/ham/read_ints.rs:73-190, src/ham/mod.rs:34-40
 *   risqgpu_set_dets      VarWf.wf.dets / n_stored_h      src/wf/mod.rs:44-80, :1635-1683
 *   risqgpu_build_h       gen_sparse_ham_fast_lookup /    src/var/fast_ham.rs:527-575
 *                         gen_sparse_ham_fast             src/var/ham_gen.rs:60-292
 *                         + sort_remove_duplicates        src/var/sparse.rs:44-56
 *   risqgpu_sigma         MatrixOperations::matrix_vector_prod / matrix_matrix_prod
 *                                                         src/var/sparse.rs:64-88, matrix_operations.rs:14-27
 *   risqgpu_davidson      Davidson::new (DPR, Lowest)     src/var/eigenvalues/algorithms/davidson.rs:106-277
 *   risqgpu_sparse_optimize  sparse_optimize              src/var/davidson.rs:43-113
 *   risqgpu_ham_diag / risqgpu_ham_off_diag
 *                         Ham::ham_diag / ham_off_diag_no_excite   src/ham/mod.rs:92-124, :256-303
 *
 * Conventions
 *  - Determinants: uint64_t[N][4] rows {up_lo, up_hi, dn_lo, dn_hi}: the
 *    reference's Config{up: u128, dn: u128} (src/wf/det.rs:16-19) split into
 *    little-endian halves, bit i = spatial orbital i (0-based).
 *  - Integrals: the reference's packed 1-based layout; one_body has
 *    combine_2(norb+1, norb+1) entries and two_body combine_4(norb+1, ...)
 *    entries (src/utils/ints.rs:38-68, src/ham/read_ints.rs:79-80).
 *  - Vectors: host pointers in the caller's determinant order unless a name ends
 *    in _device.  Block vectors are column-major: nvec columns of N doubles.
 *  - Every function returns RISQGPU_OK (0) or an error code; nothing aborts.
 *    risqgpu_last_error() returns a message for the last failure on a handle.
 *  - One handle = one CUDA stream; calls are synchronous at return; a handle is
 *    not re-entrant (the reference is single-threaded).
 */
#ifndef RISQGPU_H
#define RISQGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define RISQGPU_API __attribute__((visibility("default")))
#else
#define RISQGPU_API
#endif

typedef struct risqgpu risqgpu_t;

enum risqgpu_status {
    RISQGPU_OK = 0,
    RISQGPU_ERR_INVALID = 1,        /* bad argument, or call order violated */
    RISQGPU_ERR_OOM = 2,            /* device allocation failed */
    RISQGPU_ERR_CUDA = 3,           /* CUDA runtime error */
    RISQGPU_ERR_NOT_CONVERGED = 4,  /* Davidson hit max_iter (DavidsonError, davidson.rs:81-90) */
    RISQGPU_ERR_NO_DEVICE = 5,
    RISQGPU_ERR_CAPACITY = 6        /* output buffer too small */
};

/* Storage precision of the sparse Hamiltonian values. */
enum risqgpu_precision {
    RISQGPU_FP64 = 0,   /* FP64 values, int32 columns */
    RISQGPU_FP32 = 1,   /* FP32 values (rounded from FP64 Slater-Condon), int32 columns */
    RISQGPU_MIXED = 2,  /* FP32 values plus an FP32 remainder, so both FP32 and ~FP64 sigma run */
    RISQGPU_COLS = 3,   /* int32 columns only: the FP64 sigma recomputes every element on the fly
                           (bitwise the stored FP64 values) for sets whose values do not fit */
    /* Upper triangle only (each pair once, as the reference's SparseMatUpperTri): half the
     * storage.  The pairs are regrouped into row-panel x column-window tiles whose x and
     * y windows sigma stages in shared memory.  The FP64 sigma sums in 64-bit fixed
     * point, so it and the solves built on it are bitwise reproducible; the FP32 sigma
     * sums in FP32 (order-dependent in the last bits) unless risqgpu_set_reproducible
     * asks for fixed point too.  Built from scratch every time (no n_stored_h reuse). */
    RISQGPU_FP64_UPPER = 4,
    RISQGPU_FP32_UPPER = 5,
    RISQGPU_MIXED_UPPER = 6,
    /* Nothing stored: the FP64 sigma runs the build's connection search and evaluates
     * every element of every row itself (both triangles, the elements a FP64 build with
     * the same builder rule stores, bitwise), one warp per row with a private sum, so it
     * is bitwise reproducible.  For sets whose columns do not fit; about 20x the time of
     * a stored sigma.  No FP32 sigma, export, self energy or row-block partition. */
    RISQGPU_MATRIX_FREE = 7
};

/* Which reference builder's rule decides the stored set (src/var/davidson.rs:55-61). */
enum risqgpu_builder {
    RISQGPU_BUILDER_AUTO = 0,   /* the reference's switch: N > 100 -> FAST, else LEGACY */
    RISQGPU_BUILDER_FAST = 1,   /* fast_ham.rs: singles kept iff |H| > 1e-12, doubles iff H != 0 */
    RISQGPU_BUILDER_LEGACY = 2  /* ham_gen.rs: every element kept iff H != 0 (spin-flip-closed sets) */
};

/* Davidson arithmetic. */
enum risqgpu_mode {
    RISQGPU_MODE_FP64 = 0,   /* FP64 sigma, FP64 vectors */
    RISQGPU_MODE_MIXED = 1,  /* FP32 sigma and FP32 basis; FP64 dots, Gram-Schmidt and Rayleigh-Ritz;
                                closing FP64-sigma sweeps */
    RISQGPU_MODE_FP32 = 2    /* the FP32 stage of MIXED alone, without the closing FP64 sweeps */
};

/* Davidson preconditioner. */
enum risqgpu_precond {
    RISQGPU_PRECOND_DPR = 0,      /* r / (lambda - H_ii)  (davidson.rs:391-408) */
    RISQGPU_PRECOND_LEARNED = 1   /* DPR scaled per determinant by the loaded MLP, DPR when stalled */
};

typedef struct {
    uint64_t n_dets;
    uint64_t nnz_upper;       /* stored upper-triangle off-diagonal elements (the reference's count) */
    uint64_t nnz_full;        /* both triangles as held on the device */
    uint64_t candidates;      /* structural candidate pairs visited by the fill pass (both triangles) */
    double ms_setup;          /* sort, grouping, partner tables */
    double ms_count;          /* candidate count pass */
    double ms_fill;           /* Slater-Condon + CSR fill pass */
    double ms_total;
    uint64_t bytes_csr;       /* bytes written for columns + values */
    double gpu_ms_count;      /* CUDA-event durations on the handle's stream */
    double gpu_ms_fill;       /* fill (and, for upper-triangle storage, the regrouping into tiles) */
    uint64_t n_tiles;         /* upper-triangle storage: dense (row panel, column window) tiles */
    uint64_t nnz_dense;       /* upper-triangle storage: stored pairs that lie in dense tiles */
} risqgpu_hstats;

typedef struct {
    int iters;                /* outer Davidson iterations */
    int n_sigma;              /* sigma products (columns) */
    int n_sigma_fp64;         /* of which FP64 */
    int converged;
    int reason;               /* 0 residual+energy, 1 tiny correction, 2 redundant vector, 3 n<=2, -1 not converged */
    int learned_fallbacks;    /* iterations where the learned preconditioner fell back to DPR */
    double ms_total;
    double ms_sigma;          /* CUDA-event time of the sigma launches */
    double residual[8];       /* final residual norms per root */
} risqgpu_dstats;

/* One iteration of risqgpu_variational (the loop body of variational, src/var/mod.rs:70-123). */
typedef struct {
    double eps;               /* selection threshold used */
    uint64_t n_dets;          /* determinants after the iteration */
    uint64_t n_new;           /* determinants added (with spin flips) */
    uint64_t candidates;      /* excitations above eps not yet in the space */
    uint64_t nnz_upper;
    double energy;
    int dav_iters;
    int dav_converged;        /* 1 converged, 0 not (max iterations), -1 the matrix did not fit any storage:
                                 the stage stopped after this iteration's selection (energy NaN) */
    double ms_select, ms_build, ms_davidson;
    int storage;              /* the iteration's H storage (RISQGPU_FP64 ... RISQGPU_MATRIX_FREE), -1 none */
} risqgpu_var_iter;

/* Library version string. */
RISQGPU_API const char* risqgpu_version(void);

/* Number of visible CUDA devices (0 if none or the runtime is unavailable). */
RISQGPU_API int risqgpu_device_count(void);

/* Create a handle on `device`, copying the integrals (reference packed layout). */
RISQGPU_API int risqgpu_create(int norb, const double* one_body, size_t n1, const double* two_body, size_t n2,
                   double e_nuc, int device, risqgpu_t** out);

RISQGPU_API void risqgpu_destroy(risqgpu_t* h);

RISQGPU_API const char* risqgpu_last_error(const risqgpu_t* h);

/* Set the determinant set.  dets: N rows of 4 u64.  diag: the stored H_ii (the
 * reference keeps the incrementally updated value from selection,
 * src/wf/mod.rs:1525,1569,1618); NULL computes ham_diag on the device.
 * n_stored_h: determinants 0..n_stored_h-1 must equal the previous call's first
 * n_stored_h determinants; their stored elements are kept and only pairs with at
 * least one index >= n_stored_h are built next (expand_sparse_ham_rows,
 * src/wf/mod.rs:1664-1683).  Pass 0 for a fresh build. */
RISQGPU_API int risqgpu_set_dets(risqgpu_t* h, const uint64_t* dets, size_t n, size_t n_stored_h, const double* diag);

/* Build (or extend) the sparse Hamiltonian over the current set. */
RISQGPU_API int risqgpu_build_h(risqgpu_t* h, int precision, int builder, risqgpu_hstats* stats);

/* Stored elements after the last build. */
RISQGPU_API int risqgpu_nnz(const risqgpu_t* h, uint64_t* nnz_upper, uint64_t* nnz_full);

/* Export the stored upper triangle in the caller's determinant indices, each row
 * sorted by column: rowptr[N+1], cols[nnz_upper], vals[nnz_upper] (FP64; the
 * FP32 modes export their stored values widened), diag[N] (nullable). */
RISQGPU_API int risqgpu_export_upper(risqgpu_t* h, int64_t* rowptr, int64_t* cols, double* vals, size_t cap, double* diag);

/* Export the stored elements of the given rows (caller indices, distinct) in both
 * triangles: (out_row[i], out_col[i], out_val[i]) for every stored H_rc with r one of
 * the rows, FP64 values (the FP32 modes widened, FP32 + remainder summed), in no
 * particular order; *count receives the number of entries, and RISQGPU_ERR_CAPACITY
 * is returned when it exceeds cap.  A row of the reference's SparseMatUpperTri
 * (src/var/sparse.rs:24-36) together with the column of the same index: used to
 * check sampled rows of sets too large to export whole.  Needs stored values. */
RISQGPU_API int risqgpu_export_rows(risqgpu_t* h, const int64_t* rows, size_t k, int64_t* out_row, int64_t* out_col,
                                    double* out_val, size_t cap, size_t* count);

/* y = H x for nvec column vectors (FP64 host buffers, caller order). */
RISQGPU_API int risqgpu_sigma(risqgpu_t* h, const double* x, double* y, int nvec);

/* Same on device buffers in the library's internal (sorted) order; dtype 0 =
 * FP64 vectors and FP64 elements (stored FP64, stored FP32 + remainder, or
 * recomputed from the columns for FP32 / COLS storage), 1 = FP32 vectors with the
 * stored FP32 values.  Used for timing without host transfers. */
RISQGPU_API int risqgpu_sigma_device(risqgpu_t* h, const void* x_dev, void* y_dev, int dtype);

/* Lowest nroots eigenpairs.  init: N x ninit column-major (caller order) or NULL
 * (identity columns 0 and 1, davidson.rs:318-326).  evals[nroots],
 * evecs[N x nroots] column-major (nullable).  Returns RISQGPU_ERR_NOT_CONVERGED
 * if max_iter passes without convergence (evals/evecs then hold the last Ritz
 * pairs). */
RISQGPU_API int risqgpu_davidson(risqgpu_t* h, int nroots, const double* init, int ninit, double tol, double etol,
                     int max_iter, int mode, int precond, double* evals, double* evecs, risqgpu_dstats* stats);

/* sparse_optimize (src/var/davidson.rs:43-113): build/extend H for the set, run
 * Davidson for one root with tolerances (coeff_eps, energy_eps), write energy and
 * coefficients.  init_coeffs NULL = no initial guess.  max_iter: Davidson iterations
 * (the reference fixes 50, algorithms/davidson.rs:73). */
RISQGPU_API int risqgpu_sparse_optimize(risqgpu_t* h, const double* init_coeffs, double coeff_eps, double energy_eps,
                            int max_iter, int precision, int mode, int precond, double* energy, double* coeffs,
                            risqgpu_hstats* hstats, risqgpu_dstats* dstats);

/* Davidson search space of this handle's solves (risqgpu_davidson, sparse_optimize,
 * variational).  max_space: basis vectors before a restart; keep: Ritz vectors kept
 * at a restart.  0, 0 (the default) is the reference's Config::new, nroots + 10 and a
 * restart to the nroots Ritz vectors (src/var/eigenvalues/algorithms/davidson.rs:53-79,
 * :261-269).  A larger space with keep > nroots is a thick restart: the lowest `keep`
 * Ritz vectors carry over, which keeps more of the Krylov information between
 * restarts.  No counterpart in the reference beyond its fixed choice.  max_space <= 56,
 * keep <= max_space / 2. */
RISQGPU_API int risqgpu_set_subspace(risqgpu_t* h, int max_space, int keep);

/* Reproducible sums for the FP32 sigma of upper-triangle storage.  By default it sums
 * in FP32 with atomic adds, whose order (and so the last bits of the result) varies
 * from run to run; on = 1 makes it sum in 64-bit fixed point like the FP64 sigma,
 * bitwise reproducible, about 10 % slower.  FP64 sigma and partitioned handles always
 * sum in fixed point.  The reference's serial sums are reproducible by construction
 * (tests/integration_test_suite.rs:413-440). */
RISQGPU_API int risqgpu_set_reproducible(risqgpu_t* h, int on);

/* All-reduce supplied by a multi-GPU caller: sum `count` int64 values at device
 * address buf_dev in place across the ranks, ordered after the work already issued on
 * `stream` (a cudaStream_t) and before the work issued there after the call returns;
 * return 0 on success.  Every rank calls it at the same points with the same count. */
typedef int (*risqgpu_allreduce_fn)(void* buf_dev, size_t count, void* stream, void* user);

/* Row-block partition of the upper-triangle storage for nranks GPUs (one handle and one
 * process per GPU, every rank holding the same determinant set).  The next upper-triangle
 * build of this handle (FP64_UPPER, FP32_UPPER or MIXED_UPPER) stores only rank `rank`'s
 * share of the row panels (contiguous panels cut so that the shares hold equal numbers of
 * pairs), and every sigma sums this share into 64-bit fixed-point partial sums that
 * `reduce` adds across the ranks; integer sums are exact, so every rank gets the sigma of
 * the whole matrix, bitwise equal to a single-GPU build's, and the replicated Davidson
 * solves on the ranks stay identical.  The reference is single-threaded and has no
 * counterpart (its matrix_vector_prod, src/var/sparse.rs:64-78, splits naturally by rows).
 * nranks = 1 (reduce may be NULL) restores the undivided build.  Statistics and
 * risqgpu_nnz then count this rank's pairs. */
RISQGPU_API int risqgpu_set_partition(risqgpu_t* h, int rank, int nranks, risqgpu_allreduce_fn reduce, void* user);

/* Bound the device memory this handle may hold (bytes; 0 = no bound beyond the
 * device).  An allocation past the bound fails with RISQGPU_ERR_OOM, as a failed
 * cudaMalloc would, and leaves the handle usable.  No counterpart in the reference:
 * it lets a caller share one GPU between the library and its own work, and lets
 * tests drive the out-of-memory paths without exhausting a shared device. */
RISQGPU_API int risqgpu_set_memory_limit(risqgpu_t* h, size_t bytes);
/* Device memory the handle holds now (used) and its bound (limit, 0 = none). */
RISQGPU_API int risqgpu_memory_used(const risqgpu_t* h, size_t* used, size_t* limit);

/* Run the handle's work on `stream` (a cudaStream_t on the handle's device; NULL
 * restores the handle's own stream), so that a caller can order and time it with
 * its own events. */
RISQGPU_API int risqgpu_set_stream(risqgpu_t* h, void* stream);

/* HCI selection step (find_new_dets / iterate_excites, src/wf/mod.rs:1418-1631) over the
 * current determinant set (the last risqgpu_set_dets): heat-bath expansion of every
 * determinant with threshold eps / |coeffs[i]| (coeffs in caller order), singles only
 * when `singles` is non-zero (the reference enables them at the target eps), new
 * determinants in the reference's push order with spin-flipped partners
 * (push_and_spin_flipped, src/wf/mod.rs:99-116) and their diagonal updated from the
 * parent.  ncore: orbitals frozen by lowest h_ii (src/ham/read_ints.rs:161-184).
 * The result stays in the handle; read it with risqgpu_get_new_dets. */
RISQGPU_API int risqgpu_find_new_dets(risqgpu_t* h, const double* coeffs, double eps, int singles, int ncore,
                                      size_t* n_new);
RISQGPU_API int risqgpu_get_new_dets(risqgpu_t* h, uint64_t* dets, double* diag, size_t cap);

/* The whole variational stage (init_var_wf + variational, src/wf/mod.rs:1687-1740,
 * src/var/mod.rs:59-134) on the device: HF start, eps schedule, selection,
 * incremental H build and Davidson each iteration.  z_sym must be 1.  max_iter: HCI
 * iterations (the reference uses 20); dav_max_iter: Davidson iterations per solve (the
 * reference uses 50).  precision -1 stores FP64 both triangles while they fit, then
 * falls back, as the set grows, to FP64_UPPER, COLS and MATRIX_FREE (each OOM moves
 * one step down); otherwise the given storage every iteration.  The final
 * wavefunction stays in the handle (risqgpu_get_wf). */
RISQGPU_API int risqgpu_variational(risqgpu_t* h, int nup, int ndn, int ncore, int z_sym, double eps_var,
                                    int max_iter, int dav_max_iter, int precision, int mode, int precond,
                                    double* energy, uint64_t* n_dets);
RISQGPU_API int risqgpu_get_wf(risqgpu_t* h, uint64_t* dets, double* coeffs, double* diag, size_t cap);
RISQGPU_API int risqgpu_var_log(risqgpu_t* h, risqgpu_var_iter* out, int cap, int* n);

/* y = H x like risqgpu_sigma, but the call allocates no device memory.  This entry
 * point has no counterpart in the reference.  It is for callers that cannot let a
 * library allocate device memory during a solve: a host code whose pool allocator
 * owns the device memory budget, or a Davidson loop that overlaps work on several
 * streams, where the cudaMalloc/cudaFree pair inside risqgpu_sigma would add a
 * device-wide synchronisation to every iteration.  x_dev and y_dev are device
 * pointers to N doubles in the caller's determinant order (allocated by the
 * caller; x_dev may equal y_dev); the two internal-order copies live in one static
 * device array of 2 x 2^20 doubles (16 MiB), held by every GPU that loads the
 * library until the process exits, so sets of more than 1,048,576 determinants
 * are rejected with RISQGPU_ERR_CAPACITY.
 * Ordering: the call runs on the handle's stream, which by default does not wait
 * for other streams.  x_dev must therefore be complete before the call, or the
 * caller routes the handle onto the stream that produces x_dev with
 * risqgpu_set_stream.  The call synchronises the handle's stream before it returns,
 * so it cannot be recorded into a CUDA graph by stream capture.  The first call on
 * each device also looks up the array's device address (cudaGetSymbolAddress, with
 * the handle's device current).  All calls share the array, so
 * calls that overlap on the GPU (other handles or threads, other streams) race;
 * the contents left by a previous call are never read. */
RISQGPU_API int risqgpu_sigma_noalloc(risqgpu_t* h, const double* x_dev, double* y_dev);

/* Element-level entry points (parity tests): H_ii and H_ij of dets[k] / (d1[k], d2[k]). */
RISQGPU_API int risqgpu_ham_diag(risqgpu_t* h, const uint64_t* dets, size_t n, double* out);
RISQGPU_API int risqgpu_ham_off_diag(risqgpu_t* h, const uint64_t* d1, const uint64_t* d2, size_t n, double* out);

/* Learned preconditioner (no counterpart in the reference, which has DPR only):
 * an MLP (2n+2) -> hidden -> hidden -> 1 (ReLU) gives each determinant a factor
 * f = clamp(exp((out(x) + out(x~)) / 2), 0.25, 4), x~ being the features with the
 * alpha and beta occupations exchanged (the factor is spin-flip symmetric, like
 * H_ii), applied to its DPR step r_i / (lambda - H_ii).
 * Features: 2n occupations as +1/-1 (alpha orbitals, then beta), then
 * (H_ii - E - mu_e) * s_e and (sum of occupied h_pp - mu_h) * s_h with
 * feat_norm = {mu_e, s_e, mu_h, s_h} (NULL = {0, 1, 0, 1}).  Weights are row-major
 * FP32 (W1: hidden x n_in, W2: hidden x hidden, W3: 1 x hidden); the device rounds
 * them to BF16 and accumulates in FP32. */
RISQGPU_API int risqgpu_set_precond_mlp(risqgpu_t* h, int n_in, int hidden, const float* w1, const float* b1,
                            const float* w2, const float* b2, const float* w3, const float* b3,
                            const float* feat_norm);

/* Per-determinant preconditioner factors of the loaded MLP for energy E, caller
 * order (N floats).  For checking the network against a CPU evaluation. */
RISQGPU_API int risqgpu_precond_factors(risqgpu_t* h, double energy, float* out);

/* Second-order (Epstein-Nesbet) self-energy of every determinant at energy E over
 * the stored matrix, caller order: out[i] = -sum_{j != i} H_ij^2 / max(H_jj - E, gmin)
 * (N doubles; gmin > 0 keeps the sum finite when E reaches a diagonal).  No
 * counterpart in the reference: it gives the learned preconditioner its training
 * target f_i = sqrt((H_ii - E) / (H_ii - E + out[i])) at the converged FP64
 * Davidson energy.  Needs stored values (not RISQGPU_COLS). */
RISQGPU_API int risqgpu_self_energy(risqgpu_t* h, double energy, double gmin, double* out);

/* MLP training on the device (forward and backward kernels of this library, Adam).
 * params: packed FP32 [W1 (H x n_in), b1 (H), W2 (H x H), b2 (H), W3 (H), b3 (1)];
 * feats: B x n_in features (already normalised), target: B factors, weight: B
 * sample weights.  Loss in log space, L = sum_b w_b (o_b - log t_b)^2 / sum_b w_b,
 * with o the network output computed from BF16-rounded weights (one spin order;
 * targets must be finite and positive, else RISQGPU_ERR_INVALID).
 * risqgpu_mlp_grad: L and dL/dparams (FP32, straight through the rounding) for
 * one batch.  risqgpu_mlp_train: `epochs` passes of Adam (lr, betas 0.9/0.999)
 * over shuffled minibatches of `batch` rows; params updated in place; loss_hist
 * (epochs entries, nullable) receives the mean loss of each epoch. */
RISQGPU_API int risqgpu_mlp_grad(int device, int n_in, int hidden, const float* params, const float* feats,
                                 const float* target, const float* weight, int64_t B, float* loss, float* grad);
RISQGPU_API int risqgpu_mlp_train(int device, int n_in, int hidden, float* params, const float* feats,
                                  const float* target, const float* weight, int64_t B, int epochs, int batch,
                                  float lr, uint64_t seed, float* loss_hist);

#ifdef __cplusplus
}
#endif

#endif /* RISQGPU_H */
