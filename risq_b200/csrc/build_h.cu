// Sparse Hamiltonian construction on the device.
//
// Replaces gen_sparse_ham_fast_lookup (src/var/fast_ham.rs:527-575) and
// gen_sparse_ham_fast (src/var/ham_gen.rs:60-292) + sort_remove_duplicates
// (src/var/sparse.rs:44-56).  Both reference builders store the same set: every
// pair (i, j) at excitation degree 1 or 2 with at least one index >= n_stored_h
// whose element passes the rule (doubles: H != 0; singles: |H| > 1e-12 in the
// fast builder, H != 0 in the legacy one, off_diag.rs:33, fast_ham.rs:505).
//
// Layout.  Determinants are re-ordered by (up, dn) so that every alpha group is
// a contiguous index range; a second order by (dn, up) lists each beta group.
// Alpha strings that differ by one electron are linked through a sorted table of
// "string minus one electron" keys (the reference's alpha_singles,
// fast_ham.rs:105-134).  A row's neighbours are then three index ranges:
//   (1) its alpha group            -> beta singles and beta-beta doubles
//   (2) its beta group             -> alpha singles and alpha-alpha doubles
//   (3) its alpha-partner groups   -> opposite-spin doubles (beta differs by one)
// The matrix is held either with both triangles (each element computed once per
// side; ham_sing/ham_doub are bitwise symmetric, see bits.cuh), so that every sigma
// output is a private row sum, or as the upper triangle only (each pair once, the
// reference's SparseMatUpperTri), regrouped into row-panel x column-window tiles
// for sigma (tiles.cu).  One warp builds one row: a count pass sizes the rows, a
// fill pass evaluates FP64 Slater-Condon and compacts the non-zeros with warp
// ballots.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>

#include "bits.cuh"
#include "internal.cuh"

namespace risq {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__global__ void k_iota(int32_t* p, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = (int32_t)i;
}

// key[i] = src[perm[i] * stride + off]
__global__ void k_gather_key(const uint64_t* __restrict__ src, int64_t stride, int off, const int32_t* __restrict__ perm,
                             int64_t n, uint64_t* __restrict__ key) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        key[i] = src[(int64_t)perm[i] * stride + off];
}

// AoS caller rows -> SoA strings in sorted order, plus the two index maps.
__global__ void k_scatter_soa(const uint64_t* __restrict__ aos, const int32_t* __restrict__ perm, int64_t n, int W,
                              uint64_t* __restrict__ up, uint64_t* __restrict__ dn, int32_t* __restrict__ orig,
                              int32_t* __restrict__ inv) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        int64_t c = perm[p];
        for (int k = 0; k < W; k++) {
            up[k * n + p] = aos[c * 4 + k];
            dn[k * n + p] = aos[c * 4 + 2 + k];
        }
        orig[p] = (int32_t)c;
        inv[c] = (int32_t)p;
    }
}

__global__ void k_gather_f64(const double* __restrict__ src, const int32_t* __restrict__ perm, int64_t n,
                             double* __restrict__ dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[perm[i]];
}

// Electron counts and duplicate / group-boundary flags over the sorted order.
template <int W>
__global__ void k_flags_alpha(const uint64_t* __restrict__ up, const uint64_t* __restrict__ dn, int64_t n, int nup,
                              int ndn, int32_t* __restrict__ head, int* __restrict__ bad) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        int cu = 0, cd = 0;
        bool same_up = p > 0, same_dn = p > 0;
        for (int k = 0; k < W; k++) {
            uint64_t u = up[k * n + p], d = dn[k * n + p];
            cu += __popcll(u);
            cd += __popcll(d);
            if (p > 0) {
                same_up = same_up && (u == up[k * n + p - 1]);
                same_dn = same_dn && (d == dn[k * n + p - 1]);
            }
        }
        if (cu != nup || cd != ndn) atomicOr(bad, 1);
        if (same_up && same_dn) atomicOr(bad, 2);
        head[p] = (p == 0 || !same_up) ? 1 : 0;
    }
}

// head flags for a sorted W-word key array (SoA [W][n])
template <int W>
__global__ void k_flags_keys(const uint64_t* __restrict__ key, int64_t n, int32_t* __restrict__ head) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        bool same = p > 0;
        if (p > 0)
            for (int k = 0; k < W; k++) same = same && key[k * n + p] == key[k * n + p - 1];
        head[p] = same ? 0 : 1;
    }
}

// ids = inclusive_sum(head) - 1 ; start[id] = p at each head ; start[G] = n
__global__ void k_segment_starts(const int32_t* __restrict__ incl, int64_t n, int32_t* __restrict__ ids,
                                 int32_t* __restrict__ start) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        int id = incl[p] - 1;
        ids[p] = id;
        if (p == 0 || incl[p - 1] != incl[p]) start[id] = (int32_t)p;
        if (p == n - 1) start[id + 1] = (int32_t)n;
    }
}

// beta-ordered copies: gb[order_b[t]] = group, up_b[t] = up[order_b[t]]
template <int W>
__global__ void k_beta_views(const int32_t* __restrict__ order_b, const int32_t* __restrict__ gid_t,
                             const uint64_t* __restrict__ up, int64_t n, int32_t* __restrict__ gb,
                             int32_t* __restrict__ pos_b, uint64_t* __restrict__ up_b) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t p = order_b[t];
        gb[p] = gid_t[t];
        pos_b[p] = (int32_t)t;
        for (int k = 0; k < W; k++) up_b[k * n + t] = up[k * n + p];
    }
}

// "alpha minus one electron" keys: entry e = g * nup + j removes the j-th
// occupied orbital of unique alpha string g.
template <int W>
__global__ void k_remove1_keys(const uint64_t* __restrict__ up, int64_t n, const int32_t* __restrict__ ga_start,
                               int64_t G, int nup, uint64_t* __restrict__ key) {
    int64_t E = G * nup;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t g = e / nup;
        int j = (int)(e % nup);
        int64_t p = ga_start[g];
        Bits<W> s;
        for (int k = 0; k < W; k++) s.w[k] = up[k * n + p];
        for (int c = 0; c < j; c++) s.pop_lowest();
        Bits<W> full;
        for (int k = 0; k < W; k++) full.w[k] = up[k * n + p];
        full.clear(s.ctz());
        for (int k = 0; k < W; k++) key[k * E + e] = full.w[k];
    }
}

// per sorted entry: partner count (run length - 1) stored at the entry's original index
__global__ void k_run_counts(const int32_t* __restrict__ run_id, const int32_t* __restrict__ run_start,
                             const int32_t* __restrict__ ent, int64_t E, int32_t* __restrict__ cnt_e) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < E; s += (int64_t)gridDim.x * blockDim.x) {
        int r = run_id[s];
        cnt_e[ent[s]] = run_start[r + 1] - run_start[r] - 1;
    }
}

__global__ void k_run_fill(const int32_t* __restrict__ run_id, const int32_t* __restrict__ run_start,
                           const int32_t* __restrict__ ent, int64_t E, const int64_t* __restrict__ off_e, int nup,
                           int32_t* __restrict__ pa_list) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < E; s += (int64_t)gridDim.x * blockDim.x) {
        int r = run_id[s];
        int64_t o = off_e[ent[s]];
        for (int64_t y = run_start[r]; y < run_start[r + 1]; y++) {
            if (y == s) continue;
            pa_list[o++] = ent[y] / nup;
        }
    }
}

__global__ void k_pa_start(const int64_t* __restrict__ off_e, int64_t G, int nup, int64_t total,
                           int32_t* __restrict__ pa_start) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g <= G; g += (int64_t)gridDim.x * blockDim.x)
        pa_start[g] = (int32_t)(g < G ? off_e[g * nup] : total);
}

// Hash of (alpha group, beta string) for the determinant table (splitmix64 finaliser).
__device__ __forceinline__ uint64_t det_hash(uint32_t g, uint64_t beta) {
    uint64_t h = beta * 0x9E3779B97F4A7C15ull ^ ((uint64_t)(g + 1) * 0xC2B2AE3D27D4EB4Full);
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    return h;
}

// Insert every determinant (one-word strings) into the open-addressing table.  A slot
// is {beta low, beta high, alpha group, internal index} (16 bytes, one vector load per
// probe); index -1 marks an empty slot.
__global__ void k_ht_insert(int64_t n, const int32_t* __restrict__ ga, const uint64_t* __restrict__ dn, int bits,
                            int4* __restrict__ ht) {
    const uint32_t mask = (1u << bits) - 1u;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t beta = dn[q];
        const int g = ga[q];
        uint32_t slot = (uint32_t)(det_hash((uint32_t)g, beta) >> (64 - bits));
        // the table has at least 2n slots, so an empty one is always found
        for (uint32_t t = 0; t <= mask; t++) {
            if (atomicCAS(&ht[slot].w, -1, (int32_t)q) == -1) {
                ht[slot].x = (int)(uint32_t)beta;
                ht[slot].y = (int)(uint32_t)(beta >> 32);
                ht[slot].z = g;
                break;
            }
            slot = (slot + 1) & mask;
        }
    }
}

template <int W>
struct SetView {
    const uint64_t* __restrict__ up;
    const uint64_t* __restrict__ dn;
    const uint64_t* __restrict__ up_b;
    int64_t N;
    const int32_t* __restrict__ ga;
    const int32_t* __restrict__ ga_start;
    const int32_t* __restrict__ gb;
    const int32_t* __restrict__ gb_start;
    const int32_t* __restrict__ order_b;
    const int32_t* __restrict__ pos_b;
    const int32_t* __restrict__ pa_start;
    const int32_t* __restrict__ pa_list;
    const int32_t* __restrict__ orig;
    int64_t nsh;
    int norb;
    // (alpha group, beta string) -> internal index, or null (two-word strings)
    const int4* __restrict__ ht;
    int ht_bits;
    // previous build (incremental extension)
    const int32_t* __restrict__ prev_inv_of_caller;  // caller -> previous internal (or null)
    const int64_t* __restrict__ prev_row_start;
    const int32_t* __restrict__ prev_row_len;
    const int32_t* __restrict__ prev_cols;
    const int32_t* __restrict__ prev_orig;
    const int32_t* __restrict__ inv;
    const double* __restrict__ prev_v64;
    const float* __restrict__ prev_v32;
    const float* __restrict__ prev_vlo;

    __device__ __forceinline__ Bits<W> up_at(int64_t p) const {
        Bits<W> b;
#pragma unroll
        for (int k = 0; k < W; k++) b.w[k] = __ldg(up + k * N + p);
        return b;
    }
    __device__ __forceinline__ Bits<W> dn_at(int64_t p) const {
        Bits<W> b;
#pragma unroll
        for (int k = 0; k < W; k++) b.w[k] = __ldg(dn + k * N + p);
        return b;
    }
    __device__ __forceinline__ Bits<W> upb_at(int64_t t) const {
        Bits<W> b;
#pragma unroll
        for (int k = 0; k < W; k++) b.w[k] = __ldg(up_b + k * N + t);
        return b;
    }
    // internal index of the determinant (alpha group g, beta string beta), or -1
    __device__ __forceinline__ int find(int g, uint64_t beta) const {
        const uint32_t mask = (1u << ht_bits) - 1u;
        uint32_t slot = (uint32_t)(det_hash((uint32_t)g, beta) >> (64 - ht_bits));
        const int lo = (int)(uint32_t)beta, hi = (int)(uint32_t)(beta >> 32);
        for (uint32_t t = 0; t <= mask; t++) {
            const int4 e = __ldg(ht + slot);
            if (e.w < 0) return -1;
            if (e.x == lo && e.y == hi && e.z == g) return e.w;
            slot = (slot + 1) & mask;
        }
        return -1;
    }
};

// n-th (0-based) set bit of x; 64 if there is none
__device__ __forceinline__ int nth_set_bit(uint64_t x, int n) {
    for (int k = 0; k < n && x; k++) x &= x - 1;
    return x ? __ffsll((long long)x) - 1 : 64;
}

// Alpha partner groups with more determinants than this are searched through the
// determinant table rather than scanned.
constexpr int LOOKUP_MIN_GROUP = 256;

// Kinds of structural hits, evaluated in batches.
enum HitKind : int { K_SING_B = 0, K_SING_A = 1, K_DOUB_B = 2, K_DOUB_A = 3, K_OPP = 4 };

// Vectors of the matrix-free sigma (MODE 5), internal order.
struct SigmaIO {
    const double* __restrict__ x;
    double* __restrict__ y;
    const double* __restrict__ diag;
};

// MODE 0: count structural candidates per row.  MODE 1/2/3: evaluate and store
// FP64 / FP32 / FP32 + FP32 remainder.  MODE 4: evaluate, store the columns only.
// MODE 5: matrix-free sigma, y_p = H_pp x_p + sum_q H_pq x_q over the row's
// connections found and evaluated here (full rows, nothing stored); each lane sums its
// hits in queue order and the warp adds the lanes in a fixed order, so a row's sum
// does not depend on the schedule.
//
// One warp per row.  The scans visit candidates 32 at a time; only a minority are
// connected, so evaluating Slater-Condon in place would run with a few lanes
// active.  Connected candidates are appended instead to one of two per-warp queues
// in shared memory (singles, which sum over the occupied orbitals, and doubles,
// which read one or two integrals), and each queue is evaluated whenever it holds
// 32 entries, with every lane busy.  Stored elements are written in queue order.
template <int W, int MODE>
__global__ void __launch_bounds__(256) k_build_rows(SetView<W> v, Ints I, double thr_single, int upper,
                                                    int* __restrict__ row_counter,
                                                    int64_t* __restrict__ cnt, const int64_t* __restrict__ row_start,
                                                    int32_t* __restrict__ row_len, int32_t* __restrict__ cols,
                                                    double* __restrict__ v64, float* __restrict__ v32,
                                                    float* __restrict__ vlo, int64_t row_lo, int64_t row_hi,
                                                    int64_t base_off, SigmaIO io) {
    constexpr int WARPS = 256 / 32;
    constexpr int QCAP = 64;  // < 32 pending + 32 new
    __shared__ int s_q[WARPS][2][QCAP];
    __shared__ unsigned char s_k[WARPS][2][QCAP];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    int* const qs = s_q[wib][0];
    int* const qd = s_q[wib][1];
    unsigned char* const ks = s_k[wib][0];
    unsigned char* const kd = s_k[wib][1];
    for (;;) {
        int p = 0;
        if (lane == 0) p = (int)row_lo + atomicAdd(row_counter, 1);
        p = __shfl_sync(FULL, p, 0);
        if (p >= row_hi) break;
        const Bits<W> a = v.up_at(p), b = v.dn_at(p);
        const bool p_new = v.nsh == 0 || v.orig[p] >= v.nsh;
        int64_t base = (MODE >= 1 && MODE <= 4) ? row_start[p] - base_off : 0;
        int count = 0;
        double acc = 0.0;  // MODE 5
        int ns = 0, nd = 0;  // queue fill, warp-uniform

        auto store = [&](int64_t pos, int q, double val) {
            cols[pos] = q;
            if (MODE == 1) v64[pos] = val;
            if (MODE == 2) v32[pos] = (float)val;
            if (MODE == 3) {
                float hi = (float)val;
                v32[pos] = hi;
                vlo[pos] = (float)(val - (double)hi);
            }
        };
        // evaluate queue entries [0, take) on lanes [0, take), store the non-zero ones
        auto flush = [&](int* qq, unsigned char* kk, int& nq, int take) {
            bool ok = false;
            double val = 0.0;
            int q = -1;
            if (lane < take) {
                q = qq[lane];
                const int kind = kk[lane];
                const Bits<W> aq = v.up_at(q), bq = v.dn_at(q);
                if (kind == K_SING_B) { val = sc_single<W>(I, b, bq, a); ok = fabs(val) > thr_single; }
                else if (kind == K_SING_A) { val = sc_single<W>(I, a, aq, b); ok = fabs(val) > thr_single; }
                else if (kind == K_DOUB_B) { val = sc_double_same<W>(I, b, bq); ok = val != 0.0; }
                else if (kind == K_DOUB_A) { val = sc_double_same<W>(I, a, aq); ok = val != 0.0; }
                else { val = sc_double_opp<W>(I, a, b, aq, bq); ok = val != 0.0; }
            }
            if constexpr (MODE == 5) {
                if (ok) acc += val * __ldg(io.x + q);
            } else {
                const unsigned m = __ballot_sync(FULL, ok);
                if (ok) store(base + count + __popc(m & lt), q, val);
                count += __popc(m);
            }
            const int rem = nq - take;
            int tq = 0;
            unsigned char tk = 0;
            if (lane < rem) { tq = qq[take + lane]; tk = kk[take + lane]; }
            __syncwarp();
            if (lane < rem) { qq[lane] = tq; kk[lane] = tk; }
            __syncwarp();
            nq = rem;
        };
        auto push = [&](bool hit, bool single, int q, int kind) {
            hit = hit && (!upper || q > p);
            if (MODE == 0) {
                count += __popc(__ballot_sync(FULL, hit));
                return;
            }
            const unsigned ms = __ballot_sync(FULL, hit && single);
            const unsigned md = __ballot_sync(FULL, hit && !single);
            if (hit && single) { const int pos = ns + __popc(ms & lt); qs[pos] = q; ks[pos] = (unsigned char)kind; }
            if (hit && !single) { const int pos = nd + __popc(md & lt); qd[pos] = q; kd[pos] = (unsigned char)kind; }
            ns += __popc(ms);
            nd += __popc(md);
            __syncwarp();
            if (ns >= 32) flush(qs, ks, ns, 32);
            if (nd >= 32) flush(qd, kd, nd, 32);
        };

        // (0) elements kept from the previous build (pairs of old determinants)
        if (MODE != 5 && !p_new && v.prev_inv_of_caller) {
            int op = v.prev_inv_of_caller[v.orig[p]];
            int64_t ps = v.prev_row_start[op];
            int pl = v.prev_row_len[op];
            if (MODE) {
                for (int t = lane; t < pl; t += 32) {
                    int oq = v.prev_cols[ps + t];
                    int q = v.inv[v.prev_orig[oq]];
                    int64_t pos = base + t;
                    cols[pos] = q;
                    if (MODE == 1) v64[pos] = v.prev_v64[ps + t];
                    if (MODE == 2) v32[pos] = v.prev_v32[ps + t];
                    if (MODE == 3) { v32[pos] = v.prev_v32[ps + t]; vlo[pos] = v.prev_vlo[ps + t]; }
                    // MODE 4 keeps columns only
                }
            }
            count += pl;
        }

        // (1) same alpha string: beta singles and beta-beta doubles
        // (upper storage only needs q > p: the group is contiguous, start after p)
        {
            const int g = v.ga[p];
            const int s = upper ? p + 1 : v.ga_start[g], e = v.ga_start[g + 1];
            for (int t0 = s; t0 < e; t0 += 32) {
                const int q = t0 + lane;
                bool hit = false;
                int d = 0;
                if (q < e && q != p) {
                    d = (b ^ v.dn_at(q)).popc();
                    hit = d <= 4 && (p_new || v.orig[q] >= v.nsh);
                }
                push(hit, d == 2, q, d == 2 ? K_SING_B : K_DOUB_B);
            }
        }
        // (2) same beta string: alpha singles and alpha-alpha doubles
        // (a beta group lists its dets in increasing internal index: start after p's slot)
        {
            const int g = v.gb[p];
            const int s = upper ? v.pos_b[p] + 1 : v.gb_start[g], e = v.gb_start[g + 1];
            for (int t0 = s; t0 < e; t0 += 32) {
                const int t = t0 + lane;
                bool hit = false;
                int d = 0, q = -1;
                if (t < e) {
                    d = (a ^ v.upb_at(t)).popc();
                    if (d != 0 && d <= 4) {
                        q = v.order_b[t];
                        hit = p_new || v.orig[q] >= v.nsh;
                    }
                }
                push(hit, d == 2, q, d == 2 ? K_SING_A : K_DOUB_A);
            }
        }
        // (3) alpha single-partner groups: opposite-spin doubles.  A small partner group
        // is scanned for beta strings one single excitation away; a large one (one-word
        // strings) is probed in the determinant table with the single excitations of
        // beta_p instead (n_beta x (norb - n_beta) lookups in place of |group| tests).
        {
            const int g = v.ga[p];
            const int ps = v.pa_start[g], pe = v.pa_start[g + 1];
            // this row's occupied / virtual beta orbitals, k-th of each in lane k % 32, word k / 32
            int occ0 = 64, occ1 = 64, vir0 = 64, vir1 = 64, n_occ = 0, n_vir = 0;
            if constexpr (W == 1) {
                if (v.ht) {
                    const uint64_t all = v.norb >= 64 ? ~0ull : ((1ull << v.norb) - 1ull);
                    const uint64_t bo = b.w[0], bv = ~b.w[0] & all;
                    n_occ = __popcll(bo);
                    n_vir = __popcll(bv);
                    occ0 = nth_set_bit(bo, lane);
                    occ1 = nth_set_bit(bo, lane + 32);
                    vir0 = nth_set_bit(bv, lane);
                    vir1 = nth_set_bit(bv, lane + 32);
                }
            }
            for (int c0 = ps; c0 < pe; c0 += 32) {
                const int nvalid = min(32, pe - c0);
                int gs = 0, gl = 0, g2 = -1;
                bool probe = false;
                if (lane < nvalid) {
                    g2 = v.pa_list[c0 + lane];
                    gs = v.ga_start[g2];
                    // groups are ordered by index: a lower group holds only q < p
                    gl = (upper && g2 < g) ? 0 : v.ga_start[g2 + 1] - gs;
                    if (W == 1 && v.ht && gl > LOOKUP_MIN_GROUP) {
                        probe = true;
                        gl = 0;
                    }
                }
                // large groups: probe the table with the single excitations of beta_p
                if constexpr (W == 1) {
                    unsigned big = __ballot_sync(FULL, probe);
                    while (big) {
                        const int src = __ffs(big) - 1;
                        big &= big - 1;
                        const int gg = __shfl_sync(FULL, g2, src);
                        const int total = n_occ * n_vir;
                        for (int t0 = 0; t0 < total; t0 += 32) {
                            const int idx = t0 + lane;
                            bool hit = false;
                            int q = -1;
                            const int io = idx / max(n_vir, 1), iv = idx - io * max(n_vir, 1);
                            // the requesting lane picks the word: shuffle both, select after
                            const int o0 = __shfl_sync(FULL, occ0, io & 31), o1 = __shfl_sync(FULL, occ1, io & 31);
                            const int v0 = __shfl_sync(FULL, vir0, iv & 31), v1 = __shfl_sync(FULL, vir1, iv & 31);
                            const int oi = io < 32 ? o0 : o1, vi = iv < 32 ? v0 : v1;
                            if (idx < total) {
                                const uint64_t beta = b.w[0] ^ (1ull << oi) ^ (1ull << vi);
                                q = v.find(gg, beta);
                                hit = q >= 0 && (p_new || v.orig[q] >= v.nsh);
                            }
                            push(hit, false, q, K_OPP);
                        }
                    }
                }
                int incl = gl;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += y;
                }
                const int total = __shfl_sync(FULL, incl, 31);
                const int excl = incl - gl;
                for (int t0 = 0; t0 < total; t0 += 32) {
                    const int my = t0 + lane;
                    // j = number of partner groups whose inclusive end is <= my
                    int j = 0;
#pragma unroll
                    for (int step = 16; step >= 1; step >>= 1) {
                        const int vv = __shfl_sync(FULL, incl, j + step - 1);
                        if (vv <= my) j += step;
                    }
                    const int gsj = __shfl_sync(FULL, gs, j);
                    const int exj = __shfl_sync(FULL, excl, j);
                    bool hit = false;
                    int q = -1;
                    if (my < total) {
                        q = gsj + (my - exj);
                        hit = (b ^ v.dn_at(q)).popc() == 2 && (p_new || v.orig[q] >= v.nsh);
                    }
                    push(hit, false, q, K_OPP);
                }
            }
        }
        if (MODE) {
            if (ns > 0) flush(qs, ks, ns, ns);
            if (nd > 0) flush(qd, kd, nd, nd);
        }
        if constexpr (MODE == 5) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
            if (lane == 0) io.y[p] = io.diag[p] * io.x[p] + acc;
        } else if (lane == 0) {
            // row capacities are rounded up to 4 elements so that every row starts on a
            // 16-byte (columns) / 32-byte (FP64 values) boundary for vector loads
            if (MODE == 0) cnt[p] = (count + 3) & ~3;
            else row_len[p] = count;
        }
    }
}

// FP64 values of the stored elements (export of a columns-only build).
template <int W>
__global__ void k_stored_values(const uint64_t* __restrict__ up, const uint64_t* __restrict__ dn, int64_t n,
                                const int64_t* __restrict__ row_start, const int32_t* __restrict__ row_len,
                                const int32_t* __restrict__ cols, Ints I, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t p = warp; p < n; p += nwarps) {
        Bits<W> a, b;
        for (int k = 0; k < W; k++) { a.w[k] = up[k * n + p]; b.w[k] = dn[k * n + p]; }
        for (int k = lane; k < row_len[p]; k += 32) {
            const int64_t e = row_start[p] + k;
            const int q = cols[e];
            Bits<W> aq, bq;
            for (int w = 0; w < W; w++) { aq.w[w] = up[w * n + q]; bq.w[w] = dn[w * n + q]; }
            out[e] = sc_pair<W>(I, a, b, aq, bq);
        }
    }
}

template <int W>
__global__ void k_ham_diag(const uint64_t* __restrict__ up, const uint64_t* __restrict__ dn, int64_t n, Ints I,
                           double* __restrict__ out) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        Bits<W> a, b;
        for (int k = 0; k < W; k++) { a.w[k] = up[k * n + p]; b.w[k] = dn[k * n + p]; }
        out[p] = sc_diag<W>(I, a, b);
    }
}

// ham_off_diag_no_excite (src/ham/mod.rs:256-303) on AoS pairs, or ham_diag.
template <int W>
__global__ void k_ham_pairs(const uint64_t* __restrict__ d1, const uint64_t* __restrict__ d2, int64_t n, Ints I,
                            int diag_only, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        Bits<W> a1, b1, a2, b2;
        for (int k = 0; k < W; k++) {
            a1.w[k] = d1[i * 4 + k];
            b1.w[k] = d1[i * 4 + 2 + k];
        }
        if (diag_only) { out[i] = sc_diag<W>(I, a1, b1); continue; }
        for (int k = 0; k < W; k++) {
            a2.w[k] = d2[i * 4 + k];
            b2.w[k] = d2[i * 4 + 2 + k];
        }
        bool su = a1 == a2, sd = b1 == b2;
        double r = 0.0;
        if (su && sd) r = 0.0;
        else if (!su && !sd) {
            if (a1.andnot(a2).popc() > 1 || b1.andnot(b2).popc() > 1) r = 0.0;
            else r = sc_double_opp<W>(I, a1, b1, a2, b2);
        } else if (su) {
            int m = b1.andnot(b2).popc();
            r = m > 2 ? 0.0 : (m == 1 ? sc_single<W>(I, b1, b2, a1) : sc_double_same<W>(I, b1, b2));
        } else {
            int m = a1.andnot(a2).popc();
            r = m > 2 ? 0.0 : (m == 1 ? sc_single<W>(I, a1, a2, b1) : sc_double_same<W>(I, a1, a2));
        }
        out[i] = r;
    }
}

inline int grid_for(risqgpu* h, int64_t n, int block = 256) {
    int64_t g = (n + block - 1) / block;
    int64_t cap = (int64_t)num_sms(h) * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// Stable LSD radix sort of `perm` (values) by a multi-word key.  words: list of
// (source array, stride, offset) from least to most significant; the key of
// element i in pass k is src[perm[i]*stride + off].
struct KeyWord {
    const uint64_t* src;
    int64_t stride;
    int off;
    int bits;
};

int lsd_sort(risqgpu* h, int32_t*& perm, int64_t n, const std::vector<KeyWord>& words) {
    if (n <= 1) return RISQGPU_OK;
    uint64_t *k0 = nullptr, *k1 = nullptr;
    int32_t* v1 = nullptr;
    RQ_TRY(dalloc(h, k0, n));
    RQ_TRY(dalloc(h, k1, n));
    RQ_TRY(dalloc(h, v1, n));
    size_t tmp_bytes = 0;
    char* tmp = nullptr;
    {
        cub::DoubleBuffer<uint64_t> dk(k0, k1);
        cub::DoubleBuffer<int32_t> dv(perm, v1);
        cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, dk, dv, (int)n, 0, 64, h->stream);
    }
    int rc = dalloc(h, tmp, tmp_bytes);
    if (rc) { dfree(k0); dfree(k1); dfree(v1); return rc; }
    int32_t* cur = perm;
    int32_t* alt = v1;
    for (const KeyWord& w : words) {
        if (w.bits <= 0) continue;
        k_gather_key<<<grid_for(h, n), 256, 0, h->stream>>>(w.src, w.stride, w.off, cur, n, k0);
        cub::DoubleBuffer<uint64_t> dk(k0, k1);
        cub::DoubleBuffer<int32_t> dv(cur, alt);
        cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, dk, dv, (int)n, 0, std::min(64, w.bits), h->stream);
        if (dv.Current() != cur) std::swap(cur, alt);
    }
    int lrc = check_launch(h, "lsd_sort");
    if (cur != perm) cudaMemcpyAsync(perm, cur, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, h->stream);
    RQ_TRY(sync(h, "lsd_sort"));
    dfree(k0); dfree(k1); dfree(v1);
    dfree(tmp);
    return lrc;
}

// head flags -> segment ids and starts; returns the number of segments
int segments(risqgpu* h, const int32_t* head, int64_t n, int32_t* ids, int32_t*& starts, int32_t& G) {
    int32_t* incl = nullptr;
    RQ_TRY(dalloc(h, incl, n));
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, head, incl, (int)n, h->stream);
    char* tmp = nullptr;
    RQ_TRY(dalloc(h, tmp, tb));
    cub::DeviceScan::InclusiveSum(tmp, tb, head, incl, (int)n, h->stream);
    int32_t last = 0;
    RQ_CUDA(h, cudaMemcpyAsync(&last, incl + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "segments"));
    G = last;
    RQ_TRY(dalloc(h, starts, (size_t)G + 1));
    k_segment_starts<<<grid_for(h, n), 256, 0, h->stream>>>(incl, n, ids, starts);
    RQ_TRY(check_launch(h, "segments"));
    RQ_TRY(sync(h, "segments"));
    dfree(incl);
    dfree(tmp);
    return RISQGPU_OK;
}

template <int W>
int build_groups(risqgpu* h, const uint64_t* d_aos, const double* d_diag_in) {
    const int64_t n = (int64_t)h->N;
    const int norb = h->norb;
    // (up, dn) order
    int32_t* perm = nullptr;
    RQ_TRY(dalloc(h, perm, n));
    k_iota<<<grid_for(h, n), 256, 0, h->stream>>>(perm, n);
    std::vector<KeyWord> kw;
    for (int k = 0; k < W; k++) kw.push_back({d_aos, 4, 2 + k, norb - 64 * k});
    for (int k = 0; k < W; k++) kw.push_back({d_aos, 4, k, norb - 64 * k});
    RQ_TRY(lsd_sort(h, perm, n, kw));
    RQ_TRY(dalloc(h, h->d_up, (size_t)W * n));
    RQ_TRY(dalloc(h, h->d_dn, (size_t)W * n));
    RQ_TRY(dalloc(h, h->d_orig, n));
    RQ_TRY(dalloc(h, h->d_inv, n));
    RQ_TRY(dalloc(h, h->d_diag, n));
    k_scatter_soa<<<grid_for(h, n), 256, 0, h->stream>>>(d_aos, perm, n, W, h->d_up, h->d_dn, h->d_orig, h->d_inv);
    Ints I{h->d_h1, h->d_h2, h->nuc};
    if (d_diag_in) k_gather_f64<<<grid_for(h, n), 256, 0, h->stream>>>(d_diag_in, perm, n, h->d_diag);
    else k_ham_diag<W><<<grid_for(h, n), 256, 0, h->stream>>>(h->d_up, h->d_dn, n, I, h->d_diag);
    RQ_TRY(check_launch(h, "scatter"));
    // alpha groups, electron-count and duplicate checks
    int32_t* head = nullptr;
    int* bad = nullptr;
    RQ_TRY(dalloc(h, head, n));
    RQ_TRY(dalloc(h, bad, 1));
    RQ_CUDA(h, cudaMemsetAsync(bad, 0, sizeof(int), h->stream));
    k_flags_alpha<W><<<grid_for(h, n), 256, 0, h->stream>>>(h->d_up, h->d_dn, n, h->n_up, h->n_dn, head, bad);
    int hbad = 0;
    RQ_CUDA(h, cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "flags"));
    if (hbad & 1) { h->err = "determinants must all hold the same numbers of up and down electrons"; return RISQGPU_ERR_INVALID; }
    if (hbad & 2) { h->err = "duplicate determinant in the set"; return RISQGPU_ERR_INVALID; }
    RQ_TRY(dalloc(h, h->d_ga, n));
    RQ_TRY(segments(h, head, n, h->d_ga, h->d_ga_start, h->G_a));
    // beta order over internal indices, by (dn, up)
    RQ_TRY(dalloc(h, h->d_order_b, n));
    k_iota<<<grid_for(h, n), 256, 0, h->stream>>>(h->d_order_b, n);
    std::vector<KeyWord> kb;
    for (int k = 0; k < W; k++) kb.push_back({h->d_up + k * n, 1, 0, norb - 64 * k});
    for (int k = 0; k < W; k++) kb.push_back({h->d_dn + k * n, 1, 0, norb - 64 * k});
    RQ_TRY(lsd_sort(h, h->d_order_b, n, kb));
    // beta group heads over the beta order
    uint64_t* dnb = nullptr;
    RQ_TRY(dalloc(h, dnb, (size_t)W * n));
    for (int k = 0; k < W; k++)
        k_gather_key<<<grid_for(h, n), 256, 0, h->stream>>>(h->d_dn + k * n, 1, 0, h->d_order_b, n, dnb + k * n);
    k_flags_keys<W><<<grid_for(h, n), 256, 0, h->stream>>>(dnb, n, head);
    RQ_TRY(check_launch(h, "beta flags"));
    int32_t* gid_t = nullptr;
    RQ_TRY(dalloc(h, gid_t, n));
    RQ_TRY(segments(h, head, n, gid_t, h->d_gb_start, h->G_b));
    RQ_TRY(dalloc(h, h->d_gb, n));
    RQ_TRY(dalloc(h, h->d_pos_b, n));
    RQ_TRY(dalloc(h, h->d_up_b, (size_t)W * n));
    k_beta_views<W><<<grid_for(h, n), 256, 0, h->stream>>>(h->d_order_b, gid_t, h->d_up, n, h->d_gb, h->d_pos_b,
                                                           h->d_up_b);
    RQ_TRY(check_launch(h, "beta views"));
    dfree(dnb);
    dfree(gid_t);
    dfree(head);
    dfree(bad);
    dfree(perm);

    // alpha single partners through "minus one electron" keys
    const int64_t G = h->G_a;
    const int nup = h->n_up;
    const int64_t E = G * nup;
    if (E == 0) {
        RQ_TRY(dalloc(h, h->d_pa_start, G + 1));
        RQ_CUDA(h, cudaMemsetAsync(h->d_pa_start, 0, sizeof(int32_t) * (G + 1), h->stream));
        RQ_TRY(dalloc(h, h->d_pa_list, 1));
        h->n_pa = 0;
        return sync(h, "partners");
    }
    uint64_t* keys = nullptr;
    RQ_TRY(dalloc(h, keys, (size_t)W * E));
    k_remove1_keys<W><<<grid_for(h, E), 256, 0, h->stream>>>(h->d_up, n, h->d_ga_start, G, nup, keys);
    int32_t* ent = nullptr;
    RQ_TRY(dalloc(h, ent, E));
    k_iota<<<grid_for(h, E), 256, 0, h->stream>>>(ent, E);
    std::vector<KeyWord> kr;
    for (int k = 0; k < W; k++) kr.push_back({keys + k * E, 1, 0, norb - 64 * k});
    RQ_TRY(lsd_sort(h, ent, E, kr));
    uint64_t* skeys = nullptr;
    RQ_TRY(dalloc(h, skeys, (size_t)W * E));
    for (int k = 0; k < W; k++)
        k_gather_key<<<grid_for(h, E), 256, 0, h->stream>>>(keys + k * E, 1, 0, ent, E, skeys + k * E);
    int32_t* ehead = nullptr;
    RQ_TRY(dalloc(h, ehead, E));
    k_flags_keys<W><<<grid_for(h, E), 256, 0, h->stream>>>(skeys, E, ehead);
    int32_t *run_id = nullptr, *run_start = nullptr;
    int32_t R = 0;
    RQ_TRY(dalloc(h, run_id, E));
    RQ_TRY(segments(h, ehead, E, run_id, run_start, R));
    int32_t* cnt_e = nullptr;
    int64_t* off_e = nullptr;
    RQ_TRY(dalloc(h, cnt_e, E));
    RQ_TRY(dalloc(h, off_e, E + 1));
    k_run_counts<<<grid_for(h, E), 256, 0, h->stream>>>(run_id, run_start, ent, E, cnt_e);
    {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt_e, off_e, (int)E, h->stream);
        char* tmp = nullptr;
        RQ_TRY(dalloc(h, tmp, tb));
        cub::DeviceScan::ExclusiveSum(tmp, tb, cnt_e, off_e, (int)E, h->stream);
        RQ_TRY(sync(h, "partner scan"));
        dfree(tmp);
    }
    int64_t last_off = 0;
    int32_t last_cnt = 0;
    RQ_CUDA(h, cudaMemcpyAsync(&last_off, off_e + E - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(&last_cnt, cnt_e + E - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "partner total"));
    const int64_t total = last_off + last_cnt;
    if (total >= (int64_t)INT32_MAX) { h->err = "alpha partner table exceeds int32 range"; return RISQGPU_ERR_INVALID; }
    h->n_pa = (size_t)total;
    RQ_TRY(dalloc(h, h->d_pa_list, total));
    RQ_TRY(dalloc(h, h->d_pa_start, G + 1));
    k_run_fill<<<grid_for(h, E), 256, 0, h->stream>>>(run_id, run_start, ent, E, off_e, nup, h->d_pa_list);
    k_pa_start<<<grid_for(h, G + 1), 256, 0, h->stream>>>(off_e, G, nup, total, h->d_pa_start);
    RQ_TRY(check_launch(h, "partners"));
    RQ_TRY(sync(h, "partners"));
    dfree(keys); dfree(ent); dfree(skeys); dfree(ehead); dfree(run_id); dfree(run_start); dfree(cnt_e); dfree(off_e);
    return RISQGPU_OK;
}

template <int W>
SetView<W> make_view(risqgpu* h, bool with_prev, const int32_t* prev_inv_caller) {
    SetView<W> v;
    v.up = h->d_up; v.dn = h->d_dn; v.up_b = h->d_up_b; v.N = (int64_t)h->N;
    v.ga = h->d_ga; v.ga_start = h->d_ga_start; v.gb = h->d_gb; v.gb_start = h->d_gb_start;
    v.order_b = h->d_order_b; v.pos_b = h->d_pos_b; v.pa_start = h->d_pa_start; v.pa_list = h->d_pa_list;
    v.orig = h->d_orig; v.nsh = (int64_t)h->nsh; v.inv = h->d_inv;
    v.norb = h->norb;
    v.ht = h->d_ht;
    v.ht_bits = h->ht_bits;
    v.prev_inv_of_caller = with_prev ? prev_inv_caller : nullptr;
    v.prev_row_start = h->d_prev_row_start; v.prev_row_len = h->d_prev_row_len; v.prev_cols = h->d_prev_cols;
    v.prev_orig = h->d_prev_orig; v.prev_v64 = h->d_prev_val64; v.prev_v32 = h->d_prev_val32;
    v.prev_vlo = h->d_prev_val_lo;
    return v;
}

__global__ void k_invert(const int32_t* __restrict__ orig, int64_t n, int32_t* __restrict__ inv) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        inv[orig[p]] = (int32_t)p;
}

template <int W>
int launch_fill(risqgpu* h, const SetView<W>& v, const Ints& I, double thr, int upper, int precision, int* counter,
                int blocks, int threads, int32_t* cols, double* v64, float* v32, float* vlo, int64_t row_lo,
                int64_t row_hi, int64_t base) {
    if (precision == RISQGPU_FP64)
        k_build_rows<W, 1><<<blocks, threads, 0, h->stream>>>(v, I, thr, upper, counter, nullptr, h->d_row_start,
                                                              h->d_row_len, cols, v64, nullptr, nullptr, row_lo,
                                                              row_hi, base, SigmaIO{});
    else if (precision == RISQGPU_FP32)
        k_build_rows<W, 2><<<blocks, threads, 0, h->stream>>>(v, I, thr, upper, counter, nullptr, h->d_row_start,
                                                              h->d_row_len, cols, nullptr, v32, nullptr, row_lo,
                                                              row_hi, base, SigmaIO{});
    else if (precision == RISQGPU_MIXED)
        k_build_rows<W, 3><<<blocks, threads, 0, h->stream>>>(v, I, thr, upper, counter, nullptr, h->d_row_start,
                                                              h->d_row_len, cols, nullptr, v32, vlo, row_lo, row_hi,
                                                              base, SigmaIO{});
    else
        k_build_rows<W, 4><<<blocks, threads, 0, h->stream>>>(v, I, thr, upper, counter, nullptr, h->d_row_start,
                                                              h->d_row_len, cols, nullptr, nullptr, nullptr, row_lo,
                                                              row_hi, base, SigmaIO{});
    return check_launch(h, "fill rows");
}

__global__ void k_panel_starts(const int64_t* __restrict__ row_start, int64_t n, int rb, int64_t np,
                               int64_t* __restrict__ out) {
    for (int64_t P = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; P <= np; P += (int64_t)gridDim.x * blockDim.x)
        out[P] = row_start[min(n, P << rb)];
}

// Upper-triangle fill through the tiled layout: the rows are filled chunk by chunk of
// whole panels into a CSR buffer that holds one chunk, and every chunk is regrouped
// into tiles before the next is filled, so that the device holds the tiled arrays
// plus one chunk rather than two copies of the matrix.
template <int W>
int fill_tiled(risqgpu* h, const SetView<W>& v, const Ints& I, double thr, int precision, int* counter, int64_t cap,
               int blocks, int threads) {
    const int64_t n = (int64_t)h->N;
    int rb = 0, cb = 0;
    if (tile_shape(n, rb, cb) != RISQGPU_OK) {
        h->err = "determinant set too large for the tiled upper-triangle layout";
        return RISQGPU_ERR_INVALID;
    }
    h->tile_rb = rb;
    h->tile_cb = cb;
    const int64_t np = (n + ((int64_t)1 << rb) - 1) >> rb;
    std::vector<int64_t> ps((size_t)np + 1);
    {
        int64_t* dps = nullptr;
        ScopedFree<1> release(dps);
        RQ_TRY(dalloc(h, dps, (size_t)np + 1));
        k_panel_starts<<<grid_for(h, np + 1), 256, 0, h->stream>>>(h->d_row_start, n, rb, np, dps);
        RQ_CUDA(h, cudaMemcpyAsync(ps.data(), dps, sizeof(int64_t) * (np + 1), cudaMemcpyDeviceToHost, h->stream));
        RQ_TRY(sync(h, "panel starts"));
    }
    // this handle's panels: all of them, or with a row-block partition the rank's share,
    // contiguous panels cut where the counted pairs reach rank / nranks of the total
    int64_t own_lo = 0, own_hi = np;
    if (h->part_n > 1) {
        auto cut = [&](int r) -> int64_t {
            const int64_t goal = (int64_t)((double)ps[np] * r / h->part_n);
            return (int64_t)(std::lower_bound(ps.begin(), ps.end() - 1, goal) - ps.begin());
        };
        own_lo = h->part_rank == 0 ? 0 : cut(h->part_rank);
        own_hi = h->part_rank == h->part_n - 1 ? np : cut(h->part_rank + 1);
        own_hi = std::max(own_hi, own_lo);
        // rows of other ranks' panels hold no stored pairs here
        RQ_CUDA(h, cudaMemsetAsync(h->d_row_len, 0, sizeof(int32_t) * n, h->stream));
    }
    h->part_p_lo = own_lo;
    h->part_p_hi = own_hi;
    const int64_t own_cap = ps[own_hi] - ps[own_lo];
    const size_t vb = precision == RISQGPU_FP64 ? 8 : (precision == RISQGPU_MIXED ? 8 : 4);
    const size_t per_el = 4 + vb;
    // bytes held besides the element arrays: per-row tile data and accumulators, plus a
    // margin for the conversion's work buffers that grows with the set (at most 256 MiB)
    const size_t base_need = (size_t)own_cap * per_el + (size_t)n * 32;
    const size_t fixed = base_need + std::max((size_t)8 << 20, std::min((size_t)256 << 20, base_need / 32));
    const size_t avail = mem_available(h);
    // chunks: the fewest whose largest chunk fits beside the tiled arrays; chunk k ends at
    // the panel boundary nearest to k/K of the pairs, so the chunks hold about equal shares
    std::vector<int64_t> cuts;
    int64_t max_chunk = 0;
    const int64_t own_np = own_hi - own_lo;
    for (int64_t K = 1;; K = K < 8 ? K + 1 : K * 2) {
        cuts.assign(1, own_lo);
        for (int64_t k = 1; k < K; k++) {
            const int64_t goal = ps[own_lo] + (int64_t)((double)own_cap * k / K);
            int64_t P = std::lower_bound(ps.begin() + cuts.back() + 1, ps.begin() + own_hi, goal) - ps.begin();
            if (P > cuts.back() + 1 && goal - ps[P - 1] < ps[P] - goal) P--;
            if (P < own_hi) cuts.push_back(P);
        }
        if (cuts.back() != own_hi) cuts.push_back(own_hi);
        max_chunk = 0;
        for (size_t c = 0; c + 1 < cuts.size(); c++) max_chunk = std::max(max_chunk, ps[cuts[c + 1]] - ps[cuts[c]]);
        if (fixed + (size_t)max_chunk * per_el <= avail) break;
        if (K >= own_np) {
            h->err = "tiled upper-triangle H needs " + std::to_string((fixed + (size_t)max_chunk * per_el) >> 20) +
                     " MiB, " + std::to_string(avail >> 20) + " MiB available";
            return RISQGPU_ERR_OOM;
        }
    }
    int32_t* ccols = nullptr;
    double* c64 = nullptr;
    float *c32 = nullptr, *clo = nullptr;
    ScopedFree<4> release(ccols, c64, c32, clo);
    RQ_TRY(dalloc(h, h->d_el_idx, (size_t)own_cap));
    if (precision == RISQGPU_FP64) RQ_TRY(dalloc(h, h->d_val64, (size_t)own_cap));
    else RQ_TRY(dalloc(h, h->d_val32, (size_t)own_cap));
    if (precision == RISQGPU_MIXED) RQ_TRY(dalloc(h, h->d_val_lo, (size_t)own_cap));
    RQ_TRY(dalloc(h, ccols, (size_t)max_chunk));
    if (precision == RISQGPU_FP64) RQ_TRY(dalloc(h, c64, (size_t)max_chunk));
    else RQ_TRY(dalloc(h, c32, (size_t)max_chunk));
    if (precision == RISQGPU_MIXED) RQ_TRY(dalloc(h, clo, (size_t)max_chunk));
    TileBuilder tb;
    RQ_TRY(tb.begin(h, np, own_cap));
    const bool verbose = std::getenv("RISQGPU_VERBOSE") != nullptr;
    if (verbose)
        std::fprintf(stderr, "[risqgpu] tiled build: %zu chunks, largest %lld pairs, %zu MiB available\n",
                     cuts.size() - 1, (long long)max_chunk, avail >> 20);
    for (size_t c = 0; c + 1 < cuts.size(); c++) {
        const auto tc0 = std::chrono::steady_clock::now();
        const int64_t p_lo = cuts[c], p_hi = cuts[c + 1];
        const int64_t r_lo = p_lo << rb, r_hi = std::min(n, p_hi << rb);
        const int64_t base = ps[p_lo];
        RQ_CUDA(h, cudaMemsetAsync(counter, 0, sizeof(int), h->stream));
        RQ_TRY(launch_fill<W>(h, v, I, thr, 1, precision, counter, blocks, threads, ccols, c64, c32, clo, r_lo, r_hi,
                              base));
        if (verbose) RQ_TRY(sync(h, "fill"));
        const auto tc1 = std::chrono::steady_clock::now();
        if (precision == RISQGPU_FP64)
            RQ_TRY(tb.chunk<double>(p_lo, p_hi, h->d_row_start, base, h->d_row_len, ccols, c64, nullptr, h->d_val64,
                                    nullptr));
        else
            RQ_TRY(tb.chunk<float>(p_lo, p_hi, h->d_row_start, base, h->d_row_len, ccols, c32, clo, h->d_val32,
                                   h->d_val_lo));
        if (verbose)
            std::fprintf(stderr, "[risqgpu]   chunk %zu: panels %lld..%lld fill %.1f ms, regroup %.1f ms\n", c,
                         (long long)p_lo, (long long)p_hi,
                         std::chrono::duration<double, std::milli>(tc1 - tc0).count(),
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc1).count());
    }
    RQ_TRY(tb.finish());
    // every stored element went into the tiles exactly once
    int64_t* sum = nullptr;
    char* tmp = nullptr;
    ScopedFree<2> release_sum(sum, tmp);
    RQ_TRY(dalloc(h, sum, 1));
    size_t tbytes = 0;
    cub::DeviceReduce::Sum(nullptr, tbytes, h->d_row_len, sum, (int)n, h->stream);
    RQ_TRY(dalloc(h, tmp, tbytes));
    cub::DeviceReduce::Sum(tmp, tbytes, h->d_row_len, sum, (int)n, h->stream);
    int64_t stored = 0;
    RQ_CUDA(h, cudaMemcpyAsync(&stored, sum, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "tiled count check"));
    if (stored != tb.el_next) {
        h->err = "tiled layout holds " + std::to_string(tb.el_next) + " elements for " + std::to_string(stored) +
                 " stored";
        return RISQGPU_ERR_INVALID;
    }
    return RISQGPU_OK;
}

// stored count, statistics and handle state after a fill
int finish_build(risqgpu* h, int precision, int upper, int64_t cap, std::chrono::steady_clock::time_point t0,
                 std::chrono::steady_clock::time_point t1, std::chrono::steady_clock::time_point t2, cudaEvent_t* ev,
                 risqgpu_hstats* st) {
    using clk = std::chrono::steady_clock;
    const int64_t n = (int64_t)h->N;
    int64_t* sum = nullptr;
    char* tmp = nullptr;
    ScopedFree<2> release(sum, tmp);
    RQ_TRY(dalloc(h, sum, 1));
    size_t tb = 0;
    cub::DeviceReduce::Sum(nullptr, tb, h->d_row_len, sum, (int)n, h->stream);
    RQ_TRY(dalloc(h, tmp, tb));
    cub::DeviceReduce::Sum(tmp, tb, h->d_row_len, sum, (int)n, h->stream);
    RQ_TRY(sync(h, "fill rows"));
    auto t3 = clk::now();
    int64_t nnz = 0;
    RQ_CUDA(h, cudaMemcpyAsync(&nnz, sum, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "nnz"));
    h->cap = (size_t)cap;
    h->nnz_full = upper ? 2 * (uint64_t)nnz : (uint64_t)nnz;
    h->nnz_upper = upper ? (uint64_t)nnz : (uint64_t)nnz / 2;
    h->precision = precision;
    h->upper = upper != 0;
    float ms_c = 0.f, ms_f = 0.f;
    cudaEventElapsedTime(&ms_c, ev[0], ev[1]);
    cudaEventElapsedTime(&ms_f, ev[2], ev[3]);
    if (st) {
        st->gpu_ms_count = ms_c;
        st->gpu_ms_fill = ms_f;
        st->candidates = (uint64_t)cap;
        st->ms_count = std::chrono::duration<double, std::milli>(t1 - t0).count();
        st->ms_fill = std::chrono::duration<double, std::milli>(t3 - t2).count();
        size_t vb = precision == RISQGPU_FP64 ? 8 : (precision == RISQGPU_FP32 ? 4 : (precision == RISQGPU_COLS ? 0 : 8));
        st->bytes_csr = (uint64_t)nnz * (4 + vb);
        st->n_tiles = (uint64_t)h->n_tiles;
        st->nnz_dense = h->n_dense_el;
    }
    return RISQGPU_OK;
}

// Destroys the build's timing events on every exit.
struct BuildEvents {
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    ~BuildEvents() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
};

template <int W>
int build_rows(risqgpu* h, int precision, int upper, double thr, risqgpu_hstats* st) {
    using clk = std::chrono::steady_clock;
    const int64_t n = (int64_t)h->N;
    const bool incremental = h->nsh > 0 && h->d_prev_row_start != nullptr;
    int32_t* prev_inv = nullptr;
    int* counter = nullptr;
    int64_t* cnt = nullptr;
    ScopedFree<3> release(prev_inv, counter, cnt);
    if (incremental) {
        RQ_TRY(dalloc(h, prev_inv, h->prev_N));
        k_invert<<<grid_for(h, h->prev_N), 256, 0, h->stream>>>(h->d_prev_orig, (int64_t)h->prev_N, prev_inv);
    }
    SetView<W> v = make_view<W>(h, incremental, prev_inv);
    Ints I{h->d_h1, h->d_h2, h->nuc};
    RQ_TRY(dalloc(h, counter, 1));
    RQ_TRY(dalloc(h, cnt, n + 1));
    RQ_TRY(dalloc(h, h->d_row_start, n + 1));
    RQ_TRY(dalloc(h, h->d_row_len, n));
    const int threads = 256;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_build_rows<W, 1>, threads, 0);
    const int blocks = num_sms(h) * std::max(occ, 1);

    RQ_TRY(sync(h, "pre-count"));
    BuildEvents be;
    cudaEvent_t* ev = be.ev;
    for (int k = 0; k < 4; k++) RQ_CUDA(h, cudaEventCreate(&ev[k]));
    auto t0 = clk::now();
    RQ_CUDA(h, cudaMemsetAsync(counter, 0, sizeof(int), h->stream));
    RQ_CUDA(h, cudaEventRecord(ev[0], h->stream));
    k_build_rows<W, 0><<<blocks, threads, 0, h->stream>>>(v, I, thr, upper, counter, cnt, nullptr, nullptr, nullptr,
                                                          nullptr, nullptr, nullptr, 0, n, 0, SigmaIO{});
    RQ_CUDA(h, cudaEventRecord(ev[1], h->stream));
    RQ_TRY(check_launch(h, "count rows"));
    {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, h->d_row_start, (int)(n + 1), h->stream);
        char* tmp = nullptr;
        ScopedFree<1> release_tmp(tmp);
        RQ_TRY(dalloc(h, tmp, tb));
        RQ_CUDA(h, cudaMemsetAsync(cnt + n, 0, sizeof(int64_t), h->stream));
        cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, h->d_row_start, (int)(n + 1), h->stream);
        RQ_TRY(sync(h, "row scan"));
    }
    int64_t cap = 0;
    RQ_CUDA(h, cudaMemcpyAsync(&cap, h->d_row_start + n, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "count rows"));
    dfree(cnt);
    auto t1 = clk::now();
    if (upper) {
        // upper-triangle storage: filled chunk by chunk and regrouped into tiles
        auto t2 = clk::now();
        RQ_CUDA(h, cudaEventRecord(ev[2], h->stream));
        RQ_TRY(fill_tiled<W>(h, v, I, thr, precision, counter, cap, blocks, threads));
        RQ_CUDA(h, cudaEventRecord(ev[3], h->stream));
        return finish_build(h, precision, upper, cap, t0, t1, t2, ev, st);
    }
    {
        // refuse up front when the rows cannot be stored, leaving the handle unchanged
        size_t vb = precision == RISQGPU_FP64 ? 8 : (precision == RISQGPU_FP32 ? 4 : (precision == RISQGPU_COLS ? 0 : 8));
        const size_t arrays = (size_t)cap * (4 + vb);
        size_t need = arrays + std::max((size_t)8 << 20, std::min((size_t)64 << 20, arrays / 16));
        const size_t fr = mem_available(h);
        if (need > fr) {
            h->err = "sparse H needs " + std::to_string(need >> 20) + " MiB, " + std::to_string(fr >> 20) +
                     " MiB available";
            return RISQGPU_ERR_OOM;
        }
    }
    RQ_TRY(dalloc(h, h->d_cols, cap));
    if (precision == RISQGPU_FP64) RQ_TRY(dalloc(h, h->d_val64, cap));
    else if (precision != RISQGPU_COLS) RQ_TRY(dalloc(h, h->d_val32, cap));
    if (precision == RISQGPU_MIXED) RQ_TRY(dalloc(h, h->d_val_lo, cap));
    RQ_TRY(sync(h, "alloc"));
    auto t2 = clk::now();
    RQ_CUDA(h, cudaMemsetAsync(counter, 0, sizeof(int), h->stream));
    RQ_CUDA(h, cudaEventRecord(ev[2], h->stream));
    RQ_TRY(launch_fill<W>(h, v, I, thr, upper, precision, counter, blocks, threads, h->d_cols, h->d_val64, h->d_val32,
                          h->d_val_lo, 0, n, 0));
    RQ_CUDA(h, cudaEventRecord(ev[3], h->stream));
    return finish_build(h, precision, upper, cap, t0, t1, t2, ev, st);
}

// Matrix-free FP64 sigma: the build's connection search and Slater-Condon evaluation
// run inside sigma, one warp per row over both triangles, so nothing but the
// determinant tables is held (the replacement for stored columns when even those do
// not fit).  The elements are those a full FP64 build with the same builder rule
// stores, bit for bit.
template <int W>
int sigma_mf(risqgpu* h, const double* x, double* y) {
    SetView<W> v = make_view<W>(h, false, nullptr);
    v.nsh = 0;  // every pair, old and new determinants alike
    Ints I{h->d_h1, h->d_h2, h->nuc};
    static int cached_dev[2] = {-1, -1}, cached_blocks[2] = {0, 0};
    if (cached_dev[W - 1] != h->device) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_build_rows<W, 5>, 256, 0);
        cached_blocks[W - 1] = num_sms(h) * std::max(occ, 1);
        cached_dev[W - 1] = h->device;
    }
    RQ_CUDA(h, cudaMemsetAsync(h->d_mf_counter, 0, sizeof(int), h->stream));
    k_build_rows<W, 5><<<cached_blocks[W - 1], 256, 0, h->stream>>>(v, I, h->mf_thr, 0, h->d_mf_counter, nullptr,
                                                                    nullptr, nullptr, nullptr, nullptr, nullptr,
                                                                    nullptr, 0, (int64_t)h->N, 0,
                                                                    SigmaIO{x, y, h->d_diag});
    return check_launch(h, "matrix-free sigma");
}

}  // namespace

int sigma_matrix_free(risqgpu* h, const double* x, double* y) {
    return h->W == 1 ? sigma_mf<1>(h, x, y) : sigma_mf<2>(h, x, y);
}

void free_csr(risqgpu* h) {
    dfree(h->d_mf_counter);
    dfree(h->d_row_start); dfree(h->d_row_len); dfree(h->d_cols);
    dfree(h->d_val64); dfree(h->d_val32); dfree(h->d_val_lo);
    free_tiles(h);
    h->built = false;
    h->cap = 0;
    h->nnz_full = h->nnz_upper = 0;
}

static void free_prev(risqgpu* h) {
    dfree(h->d_prev_orig); dfree(h->d_prev_row_start); dfree(h->d_prev_row_len); dfree(h->d_prev_cols);
    dfree(h->d_prev_val64); dfree(h->d_prev_val32); dfree(h->d_prev_val_lo);
    h->prev_N = 0;
    h->prev_precision = -1;
}

void free_dets(risqgpu* h) {
    dfree(h->d_up); dfree(h->d_dn); dfree(h->d_up_b); dfree(h->d_orig); dfree(h->d_inv); dfree(h->d_diag);
    dfree(h->d_ga); dfree(h->d_ga_start); dfree(h->d_gb); dfree(h->d_gb_start); dfree(h->d_order_b);
    dfree(h->d_pos_b); dfree(h->d_pa_start); dfree(h->d_pa_list); dfree(h->d_ht);
    h->ht_bits = 0;
    free_csr(h);
    free_prev(h);
    h->N = 0;
}

static bool within_norb(const risqgpu* h, const uint64_t* d) {
    if (h->norb >= 128) return true;
    uint64_t m0 = h->norb >= 64 ? 0ull : (~0ull << h->norb);
    uint64_t m1 = h->norb <= 64 ? ~0ull : (~0ull << (h->norb - 64));
    return !((d[0] & m0) || (d[1] & m1) || (d[2] & m0) || (d[3] & m1));
}

int set_dets_impl(risqgpu* h, const uint64_t* dets, size_t n, size_t nsh, const double* diag) {
    if (!dets && n) { h->err = "dets is null"; return RISQGPU_ERR_INVALID; }
    if (n >= (size_t)INT32_MAX) { h->err = "more than 2^31-1 determinants"; return RISQGPU_ERR_INVALID; }
    if (nsh > n) { h->err = "n_stored_h > n"; return RISQGPU_ERR_INVALID; }
    if (nsh > 0) {
        if (h->upper) {
            h->err = "an upper-triangle build cannot be extended; rebuild with n_stored_h = 0";
            return RISQGPU_ERR_INVALID;
        }
        if (!h->built || h->N != nsh) {
            h->err = "n_stored_h must equal the size of the previously built set";
            return RISQGPU_ERR_INVALID;
        }
        if (std::memcmp(h->h_dets.data(), dets, sizeof(uint64_t) * 4 * nsh) != 0) {
            h->err = "the first n_stored_h determinants differ from the previous set";
            return RISQGPU_ERR_INVALID;
        }
    }
    // electron counts from the first determinant; all must agree (checked on device)
    int nu = 0, nd = 0;
    if (n) {
        nu = __builtin_popcountll(dets[0]) + __builtin_popcountll(dets[1]);
        nd = __builtin_popcountll(dets[2]) + __builtin_popcountll(dets[3]);
    }
    for (size_t i = 0; i < n; i++) {
        // every orbital index must address the integral tables
        if (!within_norb(h, dets + 4 * i)) {
            h->err = "determinant " + std::to_string(i) + " occupies an orbital >= norb";
            return RISQGPU_ERR_INVALID;
        }
    }
    // keep the previous matrix for an incremental extension
    if (nsh > 0) {
        free_prev(h);
        h->prev_N = h->N;
        h->prev_precision = h->precision;
        h->d_prev_orig = h->d_orig; h->d_orig = nullptr;
        h->d_prev_row_start = h->d_row_start; h->d_row_start = nullptr;
        h->d_prev_row_len = h->d_row_len; h->d_row_len = nullptr;
        h->d_prev_cols = h->d_cols; h->d_cols = nullptr;
        h->d_prev_val64 = h->d_val64; h->d_val64 = nullptr;
        h->d_prev_val32 = h->d_val32; h->d_val32 = nullptr;
        h->d_prev_val_lo = h->d_val_lo; h->d_val_lo = nullptr;
        free_csr(h);
        dfree(h->d_up); dfree(h->d_dn); dfree(h->d_up_b); dfree(h->d_inv); dfree(h->d_diag);
        dfree(h->d_ga); dfree(h->d_ga_start); dfree(h->d_gb); dfree(h->d_gb_start); dfree(h->d_order_b);
        dfree(h->d_pos_b); dfree(h->d_pa_start); dfree(h->d_pa_list); dfree(h->d_ht);
        h->ht_bits = 0;
        h->N = 0;
    } else {
        free_dets(h);
    }
    h->N = n;
    h->nsh = nsh;
    h->n_up = nu;
    h->n_dn = nd;
    h->h_dets.assign(dets, dets + 4 * n);
    if (n == 0) return RISQGPU_OK;
    uint64_t* d_aos = nullptr;
    double* d_dg = nullptr;
    RQ_TRY(dalloc(h, d_aos, 4 * n));
    RQ_CUDA(h, cudaMemcpyAsync(d_aos, dets, sizeof(uint64_t) * 4 * n, cudaMemcpyHostToDevice, h->stream));
    if (diag) {
        RQ_TRY(dalloc(h, d_dg, n));
        RQ_CUDA(h, cudaMemcpyAsync(d_dg, diag, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    }
    int rc = h->W == 1 ? build_groups<1>(h, d_aos, d_dg) : build_groups<2>(h, d_aos, d_dg);
    if (rc == RISQGPU_OK && h->W == 1) {
        // determinant table for the opposite-spin search: at least 2n slots
        int bits = 10;
        while (((int64_t)1 << bits) < 2 * (int64_t)n) bits++;
        if (bits > 31) {
            h->err = "determinant table exceeds 2^31 slots";
            rc = RISQGPU_ERR_INVALID;
        } else {
            h->ht_bits = bits;
            RQ_TRY(dalloc(h, h->d_ht, (size_t)1 << bits));
            RQ_CUDA(h, cudaMemsetAsync(h->d_ht, 0xff, sizeof(int4) << bits, h->stream));
            k_ht_insert<<<grid_for(h, (int64_t)n), 256, 0, h->stream>>>((int64_t)n, h->d_ga, h->d_dn, bits, h->d_ht);
            RQ_TRY(check_launch(h, "determinant table"));
        }
    }
    RQ_TRY(sync(h, "set_dets"));
    dfree(d_aos);
    dfree(d_dg);
    return rc;
}

int build_h_impl(risqgpu* h, int precision, int builder, risqgpu_hstats* st) {
    if (precision < 0 || precision > RISQGPU_MATRIX_FREE) { h->err = "bad precision"; return RISQGPU_ERR_INVALID; }
    if (builder < 0 || builder > 2) { h->err = "bad builder"; return RISQGPU_ERR_INVALID; }
    if (h->N == 0) { h->err = "no determinants set"; return RISQGPU_ERR_INVALID; }
    if (h->nsh > 0 && (h->prev_precision != precision || precision >= RISQGPU_FP64_UPPER)) {
        h->err = "an incremental build must keep the previous build's full-row precision";
        return RISQGPU_ERR_INVALID;
    }
    bool fast = builder == RISQGPU_BUILDER_FAST || (builder == RISQGPU_BUILDER_AUTO && h->N > 100);
    double thr = fast ? 1e-12 : 0.0;
    auto t0 = std::chrono::steady_clock::now();
    free_csr(h);
    if (precision == RISQGPU_MATRIX_FREE) {
        // nothing to store: sigma finds and evaluates every row's elements itself
        if (h->part_n > 1) {
            h->err = "matrix-free storage has no row-block partition";
            return RISQGPU_ERR_INVALID;
        }
        RQ_TRY(dalloc(h, h->d_mf_counter, 1));
        h->precision = RISQGPU_MATRIX_FREE;
        h->upper = false;
        h->mf_thr = thr;
        h->built = true;
        h->nsh = 0;
        if (st) {
            std::memset(st, 0, sizeof(*st));
            st->n_dets = h->N;
            st->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        return RISQGPU_OK;
    }
    // upper-triangle storage modes map onto the value types with the upper flag set
    int upper = precision >= RISQGPU_FP64_UPPER ? 1 : 0;
    int vprec = precision == RISQGPU_FP64_UPPER ? RISQGPU_FP64
              : precision == RISQGPU_FP32_UPPER ? RISQGPU_FP32
              : precision == RISQGPU_MIXED_UPPER ? RISQGPU_MIXED : precision;
    int rc = h->W == 1 ? build_rows<1>(h, vprec, upper, thr, st) : build_rows<2>(h, vprec, upper, thr, st);
    if (rc) return rc;
    h->built = true;
    if (h->nsh > 0) free_prev(h);
    h->nsh = 0;
    if (st) {
        st->n_dets = h->N;
        st->nnz_upper = h->nnz_upper;
        st->nnz_full = h->nnz_full;
        st->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return RISQGPU_OK;
}

int export_upper_impl(risqgpu* h, int64_t* rowptr, int64_t* cols, double* vals, size_t cap, double* diag) {
    if (!h->built) { h->err = "no built matrix"; return RISQGPU_ERR_INVALID; }
    if (h->precision == RISQGPU_MATRIX_FREE) { h->err = "a matrix-free build stores nothing to export"; return RISQGPU_ERR_INVALID; }
    const size_t n = h->N;
    if (cap < h->nnz_upper) { h->err = "export capacity too small"; return RISQGPU_ERR_CAPACITY; }
    std::vector<int64_t> rs(n + 1);
    std::vector<int32_t> rl(n), ci(h->cap), orig(n);
    std::vector<double> v(h->cap);
    if (h->tiled) {
        // tiled storage: decode every pair to (p, q, value), then present it as rows of
        // consecutive elements (row_start / row_len over the decoded order, sorted by p)
        const size_t nz = h->nnz_upper;
        int32_t *dp = nullptr, *dq = nullptr;
        double* dv = nullptr;
        ScopedFree<3> release(dp, dq, dv);
        RQ_TRY(dalloc(h, dp, nz));
        RQ_TRY(dalloc(h, dq, nz));
        RQ_TRY(dalloc(h, dv, nz));
        RQ_TRY(tiles_coo(h, dp, dq, dv));
        RQ_TRY(sync(h, "tiled pairs"));
        std::vector<int32_t> hp(nz);
        ci.resize(nz);
        v.resize(nz);
        RQ_CUDA(h, cudaMemcpy(hp.data(), dp, sizeof(int32_t) * nz, cudaMemcpyDeviceToHost));
        RQ_CUDA(h, cudaMemcpy(ci.data(), dq, sizeof(int32_t) * nz, cudaMemcpyDeviceToHost));
        RQ_CUDA(h, cudaMemcpy(v.data(), dv, sizeof(double) * nz, cudaMemcpyDeviceToHost));
        std::vector<int64_t> cnt(n + 1, 0);
        for (size_t k = 0; k < nz; k++) cnt[hp[k] + 1]++;
        for (size_t p = 0; p < n; p++) cnt[p + 1] += cnt[p];
        std::vector<int32_t> c2(nz);
        std::vector<double> v2(nz);
        std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
        for (size_t k = 0; k < nz; k++) {
            const int64_t at = fill[hp[k]]++;
            c2[at] = ci[k];
            v2[at] = v[k];
        }
        ci.swap(c2);
        v.swap(v2);
        for (size_t p = 0; p < n; p++) {
            rs[p] = cnt[p];
            rl[p] = (int32_t)(cnt[p + 1] - cnt[p]);
        }
        rs[n] = cnt[n];
        RQ_CUDA(h, cudaMemcpy(orig.data(), h->d_orig, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    } else {
    RQ_CUDA(h, cudaMemcpy(rs.data(), h->d_row_start, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost));
    RQ_CUDA(h, cudaMemcpy(rl.data(), h->d_row_len, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    RQ_CUDA(h, cudaMemcpy(ci.data(), h->d_cols, sizeof(int32_t) * h->cap, cudaMemcpyDeviceToHost));
    RQ_CUDA(h, cudaMemcpy(orig.data(), h->d_orig, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    if (h->precision == RISQGPU_FP64) {
        RQ_CUDA(h, cudaMemcpy(v.data(), h->d_val64, sizeof(double) * h->cap, cudaMemcpyDeviceToHost));
    } else if (h->precision == RISQGPU_COLS) {
        double* dv = nullptr;
        RQ_TRY(dalloc(h, dv, h->cap));
        Ints I{h->d_h1, h->d_h2, h->nuc};
        if (h->W == 1)
            k_stored_values<1><<<grid_for(h, (int64_t)n * 32), 256, 0, h->stream>>>(h->d_up, h->d_dn, (int64_t)n,
                h->d_row_start, h->d_row_len, h->d_cols, I, dv);
        else
            k_stored_values<2><<<grid_for(h, (int64_t)n * 32), 256, 0, h->stream>>>(h->d_up, h->d_dn, (int64_t)n,
                h->d_row_start, h->d_row_len, h->d_cols, I, dv);
        RQ_TRY(check_launch(h, "stored values"));
        RQ_TRY(sync(h, "stored values"));
        RQ_CUDA(h, cudaMemcpy(v.data(), dv, sizeof(double) * h->cap, cudaMemcpyDeviceToHost));
        dfree(dv);
    } else {
        std::vector<float> hi(h->cap), lo;
        RQ_CUDA(h, cudaMemcpy(hi.data(), h->d_val32, sizeof(float) * h->cap, cudaMemcpyDeviceToHost));
        if (h->precision == RISQGPU_MIXED) {
            lo.resize(h->cap);
            RQ_CUDA(h, cudaMemcpy(lo.data(), h->d_val_lo, sizeof(float) * h->cap, cudaMemcpyDeviceToHost));
        }
        for (size_t k = 0; k < h->cap; k++) v[k] = (double)hi[k] + (lo.empty() ? 0.0 : (double)lo[k]);
    }
    }
    // count per caller row
    // full rows hold each pair twice (keep the caller-order upper one); upper storage
    // holds it once in internal order, which maps to (min, max) in caller order
    std::vector<int64_t> cnt(n + 1, 0);
    for (size_t p = 0; p < n; p++) {
        int64_t r = orig[p];
        for (int64_t k = rs[p]; k < rs[p] + rl[p]; k++) {
            int64_t c = orig[ci[k]];
            if (h->upper) cnt[std::min(r, c)]++;
            else if (c > r) cnt[r]++;
        }
    }
    rowptr[0] = 0;
    for (size_t r = 0; r < n; r++) rowptr[r + 1] = rowptr[r] + cnt[r];
    std::vector<int64_t> fill(rowptr, rowptr + n);
    for (size_t p = 0; p < n; p++) {
        int64_t r = orig[p];
        for (int64_t k = rs[p]; k < rs[p] + rl[p]; k++) {
            int64_t c = orig[ci[k]];
            if (!h->upper && c <= r) continue;
            const int64_t lo = std::min(r, c), hi = std::max(r, c);
            cols[fill[lo]] = hi;
            vals[fill[lo]] = v[k];
            fill[lo]++;
        }
    }
    std::vector<std::pair<int64_t, double>> tmp;
    for (size_t r = 0; r < n; r++) {
        tmp.clear();
        for (int64_t k = rowptr[r]; k < rowptr[r + 1]; k++) tmp.emplace_back(cols[k], vals[k]);
        std::sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t k = 0; k < tmp.size(); k++) { cols[rowptr[r] + k] = tmp[k].first; vals[rowptr[r] + k] = tmp[k].second; }
    }
    if (diag) {
        std::vector<double> dg(n);
        RQ_CUDA(h, cudaMemcpy(dg.data(), h->d_diag, sizeof(double) * n, cudaMemcpyDeviceToHost));
        for (size_t p = 0; p < n; p++) diag[orig[p]] = dg[p];
    }
    return RISQGPU_OK;
}

namespace {

__global__ void k_mark_rows(const int64_t* __restrict__ rows, int64_t k, const int32_t* __restrict__ inv,
                            uint32_t* __restrict__ mark) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = inv[rows[i]];
        atomicOr(mark + (p >> 5), 1u << (p & 31));
    }
}

// full-row storage: the marked rows hold every element of themselves
template <typename V, bool VLO>
__global__ void k_rows_full(const int64_t* __restrict__ rows, int64_t k, const int32_t* __restrict__ inv,
                            const int32_t* __restrict__ orig, const int64_t* __restrict__ row_start,
                            const int32_t* __restrict__ row_len, const int32_t* __restrict__ cols,
                            const V* __restrict__ vals, const float* __restrict__ vlo, int64_t* __restrict__ out_r,
                            int64_t* __restrict__ out_c, double* __restrict__ out_v,
                            unsigned long long* __restrict__ count, unsigned long long cap) {
    for (int64_t i = blockIdx.x; i < k; i += gridDim.x) {
        const int32_t p = inv[rows[i]];
        const int64_t s = row_start[p];
        for (int t = threadIdx.x; t < row_len[p]; t += blockDim.x) {
            double v = (double)vals[s + t];
            if constexpr (VLO) v += (double)vlo[s + t];
            const unsigned long long at = atomicAdd(count, 1ull);
            if (at < cap) {
                out_r[at] = rows[i];
                out_c[at] = orig[cols[s + t]];
                out_v[at] = v;
            }
        }
    }
}

}  // namespace

int export_rows_impl(risqgpu* h, const int64_t* rows, size_t k, int64_t* out_r, int64_t* out_c, double* out_v,
                     size_t cap, size_t* count) {
    if (!h->built) { h->err = "no built matrix"; return RISQGPU_ERR_INVALID; }
    if (h->precision == RISQGPU_COLS || h->precision == RISQGPU_MATRIX_FREE) {
        h->err = "row export needs stored values (not COLS or MATRIX_FREE)";
        return RISQGPU_ERR_INVALID;
    }
    for (size_t i = 0; i < k; i++)
        if (rows[i] < 0 || (size_t)rows[i] >= h->N) { h->err = "row index out of range"; return RISQGPU_ERR_INVALID; }
    // rows must be distinct (each is exported once per stored element)
    {
        std::vector<int64_t> sr(rows, rows + k);
        std::sort(sr.begin(), sr.end());
        if (std::adjacent_find(sr.begin(), sr.end()) != sr.end()) { h->err = "repeated row index"; return RISQGPU_ERR_INVALID; }
    }
    const int64_t n = (int64_t)h->N;
    int64_t *drows = nullptr, *dr = nullptr, *dc = nullptr;
    double* dv = nullptr;
    uint32_t* mark = nullptr;
    unsigned long long* cnt = nullptr;
    ScopedFree<6> release(drows, dr, dc, dv, mark, cnt);
    RQ_TRY(dalloc(h, drows, k));
    RQ_TRY(dalloc(h, dr, cap));
    RQ_TRY(dalloc(h, dc, cap));
    RQ_TRY(dalloc(h, dv, cap));
    RQ_TRY(dalloc(h, mark, (size_t)(n + 31) / 32));
    RQ_TRY(dalloc(h, cnt, 1));
    RQ_CUDA(h, cudaMemcpyAsync(drows, rows, sizeof(int64_t) * k, cudaMemcpyHostToDevice, h->stream));
    RQ_CUDA(h, cudaMemsetAsync(mark, 0, sizeof(uint32_t) * ((n + 31) / 32), h->stream));
    RQ_CUDA(h, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), h->stream));
    if (h->tiled) {
        k_mark_rows<<<grid_for(h, (int64_t)k), 256, 0, h->stream>>>(drows, (int64_t)k, h->d_inv, mark);
        RQ_TRY(tiles_rows(h, mark, dr, dc, dv, cnt, cap));
    } else {
        const int g = (int)std::max<size_t>(1, std::min<size_t>(k, 4096));
        if (h->precision == RISQGPU_FP64)
            k_rows_full<double, false><<<g, 256, 0, h->stream>>>(drows, (int64_t)k, h->d_inv, h->d_orig, h->d_row_start,
                h->d_row_len, h->d_cols, h->d_val64, nullptr, dr, dc, dv, cnt, cap);
        else if (h->precision == RISQGPU_MIXED)
            k_rows_full<float, true><<<g, 256, 0, h->stream>>>(drows, (int64_t)k, h->d_inv, h->d_orig, h->d_row_start,
                h->d_row_len, h->d_cols, h->d_val32, h->d_val_lo, dr, dc, dv, cnt, cap);
        else
            k_rows_full<float, false><<<g, 256, 0, h->stream>>>(drows, (int64_t)k, h->d_inv, h->d_orig, h->d_row_start,
                h->d_row_len, h->d_cols, h->d_val32, nullptr, dr, dc, dv, cnt, cap);
        RQ_TRY(check_launch(h, "row export"));
    }
    unsigned long long c = 0;
    RQ_CUDA(h, cudaMemcpyAsync(&c, cnt, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "row export"));
    *count = (size_t)c;
    if (c > cap) { h->err = "row export capacity too small: " + std::to_string(c) + " entries"; return RISQGPU_ERR_CAPACITY; }
    RQ_CUDA(h, cudaMemcpy(out_r, dr, sizeof(int64_t) * c, cudaMemcpyDeviceToHost));
    RQ_CUDA(h, cudaMemcpy(out_c, dc, sizeof(int64_t) * c, cudaMemcpyDeviceToHost));
    RQ_CUDA(h, cudaMemcpy(out_v, dv, sizeof(double) * c, cudaMemcpyDeviceToHost));
    return RISQGPU_OK;
}

int ham_elements_impl(risqgpu* h, const uint64_t* d1, const uint64_t* d2, size_t n, double* out, bool diag_only) {
    if (n == 0) return RISQGPU_OK;
    for (size_t i = 0; i < n; i++) {
        // every orbital index must address the integral tables
        if (!within_norb(h, d1 + 4 * i) || (!diag_only && !within_norb(h, d2 + 4 * i))) {
            h->err = "determinant pair " + std::to_string(i) + " occupies an orbital >= norb";
            return RISQGPU_ERR_INVALID;
        }
    }
    uint64_t *a = nullptr, *b = nullptr;
    double* o = nullptr;
    RQ_TRY(dalloc(h, a, 4 * n));
    RQ_TRY(dalloc(h, o, n));
    RQ_CUDA(h, cudaMemcpyAsync(a, d1, sizeof(uint64_t) * 4 * n, cudaMemcpyHostToDevice, h->stream));
    if (!diag_only) {
        RQ_TRY(dalloc(h, b, 4 * n));
        RQ_CUDA(h, cudaMemcpyAsync(b, d2, sizeof(uint64_t) * 4 * n, cudaMemcpyHostToDevice, h->stream));
    }
    Ints I{h->d_h1, h->d_h2, h->nuc};
    int grid = grid_for(h, (int64_t)n);
    if (h->W == 1) k_ham_pairs<1><<<grid, 256, 0, h->stream>>>(a, b, (int64_t)n, I, diag_only ? 1 : 0, o);
    else k_ham_pairs<2><<<grid, 256, 0, h->stream>>>(a, b, (int64_t)n, I, diag_only ? 1 : 0, o);
    RQ_TRY(check_launch(h, "ham pairs"));
    RQ_CUDA(h, cudaMemcpyAsync(out, o, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "ham pairs"));
    dfree(a); dfree(b); dfree(o);
    return RISQGPU_OK;
}

}  // namespace risq
