// HCI selection on the device: find_new_dets / iterate_excites (src/wf/mod.rs:1418-1631).
//
// The reference walks the determinants in order and, for each, the heat-bath
// sorted excitation lists (src/excite/init.rs:81-280) until |H| < eps / |c|,
// pushing every excited determinant that is not yet in the variational space
// or in the output (first occurrence wins, with the diagonal updated from that
// parent, src/wf/det.rs:271-420), and finally push_and_spin_flipped's each new
// determinant (src/wf/mod.rs:99-116).  Here one warp expands one determinant;
// the candidates of each determinant are written at a prefix-sum offset in the
// same order the reference visits them, so a candidate's index in the buffer is
// its position in the reference's sequence.  "First occurrence wins" then
// becomes a stable sort by configuration keeping the first of each run, and the
// spin-flip pushes become a second stable unique over [flip(d), d] pairs.
// Membership in the current space is a binary search over the (up, dn)-sorted
// determinant set the handle already holds.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bits.cuh"
#include "internal.cuh"
#include "select.cuh"

namespace risq {

namespace {

constexpr unsigned FULL = 0xffffffffu;

inline int grid_of(risqgpu* h, int64_t n, int block = 256) {
    int64_t g = (n + block - 1) / block;
    int64_t cap = (int64_t)num_sms(h) * 16;
    return (int)std::max<int64_t>(1, std::min(g, cap));
}

template <int W>
struct SortedSet {  // the handle's determinant set, sorted by (up, dn)
    const uint64_t* __restrict__ up;
    const uint64_t* __restrict__ dn;
    int64_t N;
    // lexicographic compare of (up, dn) with the most significant word of up first
    __device__ __forceinline__ int cmp(int64_t p, const Bits<W>& a, const Bits<W>& b) const {
#pragma unroll
        for (int k = W - 1; k >= 0; k--) {
            uint64_t x = __ldg(up + k * N + p);
            if (x != a.w[k]) return x < a.w[k] ? -1 : 1;
        }
#pragma unroll
        for (int k = W - 1; k >= 0; k--) {
            uint64_t x = __ldg(dn + k * N + p);
            if (x != b.w[k]) return x < b.w[k] ? -1 : 1;
        }
        return 0;
    }
    __device__ __forceinline__ bool contains(const Bits<W>& a, const Bits<W>& b) const {
        int64_t lo = 0, hi = N;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            int c = cmp(mid, a, b);
            if (c == 0) return true;
            if (c < 0) lo = mid + 1;
            else hi = mid;
        }
        return false;
    }
};

struct Tables {  // heat-bath lists on the device (see select.cuh)
    const int32_t* __restrict__ opp_off;   // n*n + 1
    const int32_t* __restrict__ same_off;  // n*n + 1
    const int32_t* __restrict__ sing_off;  // n + 1
    const uint8_t* __restrict__ r;
    const uint8_t* __restrict__ s;
    const double* __restrict__ habs;
    int norb;
    double max_opp, max_same, max_sing;
};

// Excitation codes: kind (0 opp, 1 same-up, 2 same-dn, 3 single-up, 4 single-dn) in
// bits 28..30 and four 7-bit orbitals i, j, r, s.
__device__ __forceinline__ uint32_t ecode(int kind, int i, int j, int r, int s) {
    return ((uint32_t)kind << 28) | ((uint32_t)i << 21) | ((uint32_t)j << 14) | ((uint32_t)r << 7) | (uint32_t)s;
}

// One warp per determinant (caller order).  FILL = false: count the candidates
// of each determinant; FILL = true: write them at off[d].
template <int W, bool FILL>
__global__ void __launch_bounds__(256) k_expand(const uint64_t* __restrict__ aos, const double* __restrict__ coeff,
                                                int64_t N, double eps, int singles_on, Tables T, Bits<W> valence,
                                                Ints I, SortedSet<W> set, int* __restrict__ row_counter,
                                                int64_t* __restrict__ cnt, const int64_t* __restrict__ off,
                                                uint64_t* __restrict__ out_cfg, int32_t* __restrict__ out_parent,
                                                uint32_t* __restrict__ out_code, int64_t M) {
    const int lane = threadIdx.x & 31;
    const int n = T.norb;
    for (;;) {
        int d = 0;
        if (lane == 0) d = atomicAdd(row_counter, 1);
        d = __shfl_sync(FULL, d, 0);
        if (d >= N) break;
        Bits<W> up, dn;
#pragma unroll
        for (int k = 0; k < W; k++) { up.w[k] = aos[(int64_t)d * 4 + k]; dn.w[k] = aos[(int64_t)d * 4 + 2 + k]; }
        const double local_eps = eps / fabs(coeff[d]);
        int64_t base = FILL ? off[d] : 0;
        int64_t count = 0;

        auto emit_chunk = [&](int my_n, auto&& gen) {
            // lanes hold my_n candidates each; place them in lane order
            int incl = my_n;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += y;
            }
            int total = __shfl_sync(FULL, incl, 31);
            if (FILL && my_n > 0) gen(base + count + (incl - my_n));
            count += total;
        };

        // (1) opposite-spin doubles (mod.rs:1487-1534)
        if (T.max_opp >= local_eps) {
            Bits<W> vu = up & valence, vd = dn & valence;
            const int nu = vu.popc(), nd = vd.popc();
            const int npair = nu * nd;
            for (int c0 = 0; c0 < npair; c0 += 32) {
                const int pidx = c0 + lane;
                int i = -1, j = -1;
                int my_n = 0;
                if (pidx < npair) {
                    Bits<W> t = vu;
                    for (int k = 0; k < pidx / nd; k++) t.pop_lowest();
                    i = t.ctz();
                    Bits<W> u = vd;
                    for (int k = 0; k < pidx % nd; k++) u.pop_lowest();
                    j = u.ctz();
                    const int lo = T.opp_off[i * n + j], hi = T.opp_off[i * n + j + 1];
                    for (int k = lo; k < hi; k++) {
                        if (T.habs[k] < local_eps) break;
                        const int r = T.r[k], s = T.s[k];
                        if (up.test(r) || dn.test(s)) continue;
                        Bits<W> nu2 = up, nd2 = dn;
                        nu2.clear(i); nu2.set(r);
                        nd2.clear(j); nd2.set(s);
                        if (!set.contains(nu2, nd2)) my_n++;
                    }
                }
                emit_chunk(my_n, [&](int64_t pos) {
                    const int lo = T.opp_off[i * n + j], hi = T.opp_off[i * n + j + 1];
                    for (int k = lo; k < hi; k++) {
                        if (T.habs[k] < local_eps) break;
                        const int r = T.r[k], s = T.s[k];
                        if (up.test(r) || dn.test(s)) continue;
                        Bits<W> nu2 = up, nd2 = dn;
                        nu2.clear(i); nu2.set(r);
                        nd2.clear(j); nd2.set(s);
                        if (set.contains(nu2, nd2)) continue;
                        for (int q = 0; q < W; q++) { out_cfg[q * M + pos] = nu2.w[q]; out_cfg[(W + q) * M + pos] = nd2.w[q]; }
                        out_parent[pos] = d;
                        out_code[pos] = ecode(0, i, j, r, s);
                        pos++;
                    }
                });
            }
        }
        // (2) same-spin doubles (mod.rs:1536-1580)
        if (T.max_same >= local_eps) {
            for (int sp = 0; sp < 2; sp++) {
                const Bits<W> x = sp == 0 ? up : dn;
                const Bits<W> vx = x & valence;
                const int nv = vx.popc();
                const int npair = nv * (nv - 1) / 2;
                for (int c0 = 0; c0 < npair; c0 += 32) {
                    const int pidx = c0 + lane;
                    int i = -1, j = -1;
                    int my_n = 0;
                    if (pidx < npair) {
                        // bit_pairs order: (a, b) with a < b, a-major
                        int a = 0, rem = pidx;
                        while (rem >= nv - 1 - a) { rem -= nv - 1 - a; a++; }
                        int b = a + 1 + rem;
                        Bits<W> t = vx;
                        for (int k = 0; k < a; k++) t.pop_lowest();
                        i = t.ctz();
                        for (int k = a; k < b; k++) t.pop_lowest();
                        j = t.ctz();
                        const int lo = T.same_off[i * n + j], hi = T.same_off[i * n + j + 1];
                        for (int k = lo; k < hi; k++) {
                            if (T.habs[k] < local_eps) break;
                            const int r = T.r[k], s = T.s[k];
                            if (x.test(r) || x.test(s)) continue;
                            Bits<W> nx = x;
                            nx.clear(i); nx.clear(j); nx.set(r); nx.set(s);
                            if (!(sp == 0 ? set.contains(nx, dn) : set.contains(up, nx))) my_n++;
                        }
                    }
                    emit_chunk(my_n, [&](int64_t pos) {
                        const int lo = T.same_off[i * n + j], hi = T.same_off[i * n + j + 1];
                        for (int k = lo; k < hi; k++) {
                            if (T.habs[k] < local_eps) break;
                            const int r = T.r[k], s = T.s[k];
                            if (x.test(r) || x.test(s)) continue;
                            Bits<W> nx = x;
                            nx.clear(i); nx.clear(j); nx.set(r); nx.set(s);
                            const Bits<W> a2 = sp == 0 ? nx : up, b2 = sp == 0 ? dn : nx;
                            if (set.contains(a2, b2)) continue;
                            for (int q = 0; q < W; q++) { out_cfg[q * M + pos] = a2.w[q]; out_cfg[(W + q) * M + pos] = b2.w[q]; }
                            out_parent[pos] = d;
                            out_code[pos] = ecode(1 + sp, i, j, r, s);
                            pos++;
                        }
                    });
                }
            }
        }
        // (3) singles, only at the target eps (mod.rs:1582-1628)
        if (singles_on && T.max_sing >= local_eps) {
            for (int sp = 0; sp < 2; sp++) {
                const Bits<W> x = sp == 0 ? up : dn;
                const Bits<W> other = sp == 0 ? dn : up;
                const Bits<W> vx = x & valence;
                const int nv = vx.popc();
                for (int c0 = 0; c0 < nv; c0 += 32) {
                    const int pidx = c0 + lane;
                    int i = -1;
                    int my_n = 0;
                    if (pidx < nv) {
                        Bits<W> t = vx;
                        for (int k = 0; k < pidx; k++) t.pop_lowest();
                        i = t.ctz();
                        const int lo = T.sing_off[i], hi = T.sing_off[i + 1];
                        for (int k = lo; k < hi; k++) {
                            if (T.habs[k] < local_eps) break;
                            const int r = T.r[k];
                            if (x.test(r)) continue;
                            Bits<W> nx = x;
                            nx.clear(i); nx.set(r);
                            const Bits<W> a2 = sp == 0 ? nx : up, b2 = sp == 0 ? dn : nx;
                            if (set.contains(a2, b2)) continue;
                            if (fabs(sc_single<W>(I, x, nx, other)) > local_eps) my_n++;
                        }
                    }
                    emit_chunk(my_n, [&](int64_t pos) {
                        const int lo = T.sing_off[i], hi = T.sing_off[i + 1];
                        for (int k = lo; k < hi; k++) {
                            if (T.habs[k] < local_eps) break;
                            const int r = T.r[k];
                            if (x.test(r)) continue;
                            Bits<W> nx = x;
                            nx.clear(i); nx.set(r);
                            const Bits<W> a2 = sp == 0 ? nx : up, b2 = sp == 0 ? dn : nx;
                            if (set.contains(a2, b2)) continue;
                            if (!(fabs(sc_single<W>(I, x, nx, other)) > local_eps)) continue;
                            for (int q = 0; q < W; q++) { out_cfg[q * M + pos] = a2.w[q]; out_cfg[(W + q) * M + pos] = b2.w[q]; }
                            out_parent[pos] = d;
                            out_code[pos] = ecode(3 + sp, i, 0, r, 0);
                            pos++;
                        }
                    });
                }
            }
        }
        if (!FILL && lane == 0) cnt[d] = count;
    }
}

// Diagonal of a new determinant from its parent's (Det::new_diag_*, src/wf/det.rs:271-420).
template <int W>
__device__ double new_diag(const Ints& I, const Bits<W>& up, const Bits<W>& dn, double pdiag, uint32_t code) {
    const int kind = (code >> 28) & 7;
    const int p = (code >> 21) & 127, q = (code >> 14) & 127, r = (code >> 7) & 127, s = code & 127;
    if (kind == 0) {  // new_diag_opp
        double nd = pdiag + one_body(I, r, r) + one_body(I, s, s) - one_body(I, p, p) - one_body(I, q, q);
        nd += direct(I, r, s, r, s) - direct(I, p, q, p, q);
        Bits<W> t = up;
        while (!t.is_zero()) {
            int i = t.ctz();
            t.pop_lowest();
            if (i == p) continue;
            nd += dpe(I, i, r, i, r) - dpe(I, i, p, i, p);
            nd += direct(I, i, s, i, s) - direct(I, i, q, i, q);
        }
        t = dn;
        while (!t.is_zero()) {
            int i = t.ctz();
            t.pop_lowest();
            if (i == q) continue;
            nd += dpe(I, i, s, i, s) - dpe(I, i, q, i, q);
            nd += direct(I, i, r, i, r) - direct(I, i, p, i, p);
        }
        return nd;
    }
    if (kind == 1 || kind == 2) {  // new_diag_same
        const bool alpha = kind == 1;
        double nd = pdiag + one_body(I, r, r) + one_body(I, s, s) - one_body(I, p, p) - one_body(I, q, q);
        nd += dpe(I, r, s, r, s) - dpe(I, p, q, p, q);
        Bits<W> t = alpha ? up : dn;
        while (!t.is_zero()) {
            int i = t.ctz();
            t.pop_lowest();
            if (i == p || i == q) continue;
            nd += dpe(I, i, r, i, r) + dpe(I, i, s, i, s) - dpe(I, i, p, i, p) - dpe(I, i, q, i, q);
        }
        t = alpha ? dn : up;
        while (!t.is_zero()) {
            int i = t.ctz();
            t.pop_lowest();
            nd += direct(I, i, r, i, r) + direct(I, i, s, i, s) - direct(I, i, p, i, p) - direct(I, i, q, i, q);
        }
        return nd;
    }
    // new_diag_sing
    const bool alpha = kind == 3;
    double nd = pdiag + one_body(I, r, r) - one_body(I, p, p);
    Bits<W> t = alpha ? up : dn;
    while (!t.is_zero()) {
        int i = t.ctz();
        t.pop_lowest();
        if (i == p) continue;
        nd += dpe(I, i, r, i, r) - dpe(I, i, p, i, p);
    }
    t = alpha ? dn : up;
    while (!t.is_zero()) {
        int i = t.ctz();
        t.pop_lowest();
        nd += direct(I, i, r, i, r) - direct(I, i, p, i, p);
    }
    return nd;
}

// Kept candidate k (generation order): its diagonal, and the [flip(d), d] pair
// entries at 2k and 2k+1 (a flip equal to d is the same configuration twice).
template <int W>
__global__ void k_finish(const int64_t* __restrict__ kept, int64_t K, const uint64_t* __restrict__ cfg, int64_t M,
                         const int32_t* __restrict__ parent, const uint32_t* __restrict__ code,
                         const uint64_t* __restrict__ aos, const double* __restrict__ pdiag_caller, Ints I,
                         uint64_t* __restrict__ pair_cfg, double* __restrict__ pair_diag) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = kept[k];
        const int32_t par = parent[c];
        Bits<W> pu, pd, u, dd;
#pragma unroll
        for (int q = 0; q < W; q++) {
            pu.w[q] = aos[(int64_t)par * 4 + q];
            pd.w[q] = aos[(int64_t)par * 4 + 2 + q];
            u.w[q] = cfg[q * M + c];
            dd.w[q] = cfg[(W + q) * M + c];
        }
        const double dg = new_diag<W>(I, pu, pd, pdiag_caller[par], code[c]);
        const int64_t e0 = 2 * k, e1 = 2 * k + 1, L = 2 * K;
#pragma unroll
        for (int q = 0; q < W; q++) {
            pair_cfg[q * L + e0] = dd.w[q];        // flip: up <- dn
            pair_cfg[(W + q) * L + e0] = u.w[q];
            pair_cfg[q * L + e1] = u.w[q];
            pair_cfg[(W + q) * L + e1] = dd.w[q];
        }
        pair_diag[e0] = dg;
        pair_diag[e1] = dg;
    }
}

// head[t] = 1 where the sorted (by configuration) entry t starts a run
template <int W>
__global__ void k_heads(const uint64_t* __restrict__ cfg, int64_t M, const int64_t* __restrict__ perm, int64_t n,
                        int32_t* __restrict__ head) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        bool same = t > 0;
        if (t > 0) {
            const int64_t a = perm[t], b = perm[t - 1];
            for (int q = 0; q < 2 * W; q++) same = same && cfg[q * M + a] == cfg[q * M + b];
        }
        head[t] = same ? 0 : 1;
    }
}

template <int W>
__global__ void k_not_in_set(const uint64_t* __restrict__ cfg, int64_t M, SortedSet<W> set,
                             int32_t* __restrict__ keep) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < M; t += (int64_t)gridDim.x * blockDim.x) {
        Bits<W> a, b;
        for (int q = 0; q < W; q++) { a.w[q] = cfg[q * M + t]; b.w[q] = cfg[(W + q) * M + t]; }
        keep[t] = set.contains(a, b) ? 0 : 1;
    }
}

__global__ void k_iota64(int64_t* p, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = i;
}

__global__ void k_gather_word(const uint64_t* __restrict__ src, const int64_t* __restrict__ perm, int64_t n,
                              uint64_t* __restrict__ key) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        key[i] = src[perm[i]];
}

// Stable LSD sort of an int64 permutation by a (2W)-word configuration
// (dn words first, then up words: up is the most significant).
template <int W>
int sort_by_cfg(risqgpu* h, const uint64_t* cfg, int64_t M, int64_t* perm, int64_t n) {
    if (n <= 1) return RISQGPU_OK;
    uint64_t *k0 = nullptr, *k1 = nullptr;
    int64_t* v1 = nullptr;
    RQ_TRY(dalloc(h, k0, n));
    RQ_TRY(dalloc(h, k1, n));
    RQ_TRY(dalloc(h, v1, n));
    size_t tb = 0;
    {
        cub::DoubleBuffer<uint64_t> dk(k0, k1);
        cub::DoubleBuffer<int64_t> dv(perm, v1);
        cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, (int)n, 0, 64, h->stream);
    }
    char* tmp = nullptr;
    RQ_TRY(dalloc(h, tmp, tb));
    int64_t* cur = perm;
    int64_t* alt = v1;
    // (row of cfg, significant bits) from least to most significant: dn words, then up words
    std::vector<std::pair<int, int>> words;
    for (int k = 0; k < W; k++) words.push_back({W + k, std::min(64, h->norb - 64 * k)});
    for (int k = 0; k < W; k++) words.push_back({k, std::min(64, h->norb - 64 * k)});
    for (const auto& wb : words) {
        if (wb.second <= 0) continue;
        k_gather_word<<<grid_of(h, n), 256, 0, h->stream>>>(cfg + (int64_t)wb.first * M, cur, n, k0);
        cub::DoubleBuffer<uint64_t> dk(k0, k1);
        cub::DoubleBuffer<int64_t> dv(cur, alt);
        cub::DeviceRadixSort::SortPairs(tmp, tb, dk, dv, (int)n, 0, wb.second, h->stream);
        if (dv.Current() != cur) std::swap(cur, alt);
    }
    if (cur != perm) RQ_CUDA(h, cudaMemcpyAsync(perm, cur, sizeof(int64_t) * n, cudaMemcpyDeviceToDevice, h->stream));
    RQ_TRY(check_launch(h, "sort_by_cfg"));
    RQ_TRY(sync(h, "sort_by_cfg"));
    dfree(k0); dfree(k1); dfree(v1); dfree(tmp);
    return RISQGPU_OK;
}

// Select flagged elements of `in` (keeping order) into `out`; returns the count.
int compact_i64(risqgpu* h, const int64_t* in, const int32_t* flags, int64_t n, int64_t* out, int64_t& nout) {
    int64_t* dn = nullptr;
    RQ_TRY(dalloc(h, dn, 1));
    size_t tb = 0;
    cub::DeviceSelect::Flagged(nullptr, tb, in, flags, out, dn, (int)n, h->stream);
    char* tmp = nullptr;
    RQ_TRY(dalloc(h, tmp, tb));
    cub::DeviceSelect::Flagged(tmp, tb, in, flags, out, dn, (int)n, h->stream);
    RQ_CUDA(h, cudaMemcpyAsync(&nout, dn, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "compact"));
    dfree(tmp);
    dfree(dn);
    return RISQGPU_OK;
}

int sort_i64(risqgpu* h, int64_t* keys, int64_t n) {
    if (n <= 1) return RISQGPU_OK;
    int64_t* alt = nullptr;
    RQ_TRY(dalloc(h, alt, n));
    size_t tb = 0;
    cub::DoubleBuffer<int64_t> dk(keys, alt);
    cub::DeviceRadixSort::SortKeys(nullptr, tb, dk, (int)n, 0, 64, h->stream);
    char* tmp = nullptr;
    RQ_TRY(dalloc(h, tmp, tb));
    cub::DeviceRadixSort::SortKeys(tmp, tb, dk, (int)n, 0, 64, h->stream);
    if (dk.Current() != keys) RQ_CUDA(h, cudaMemcpyAsync(keys, dk.Current(), sizeof(int64_t) * n, cudaMemcpyDeviceToDevice, h->stream));
    RQ_TRY(sync(h, "sort_i64"));
    dfree(alt);
    dfree(tmp);
    return RISQGPU_OK;
}

// Unique by configuration keeping the smallest index: `idx` (n entries, values
// index cfg columns) in increasing order on entry; on return the kept indices in
// increasing order and their count.
template <int W>
int unique_first(risqgpu* h, const uint64_t* cfg, int64_t M, int64_t* idx, int64_t n, int64_t& nk) {
    RQ_TRY(sort_by_cfg<W>(h, cfg, M, idx, n));
    int32_t* head = nullptr;
    int64_t* out = nullptr;
    RQ_TRY(dalloc(h, head, n));
    RQ_TRY(dalloc(h, out, n));
    k_heads<W><<<grid_of(h, n), 256, 0, h->stream>>>(cfg, M, idx, n, head);
    RQ_TRY(check_launch(h, "heads"));
    RQ_TRY(compact_i64(h, idx, head, n, out, nk));
    RQ_TRY(sort_i64(h, out, nk));
    RQ_CUDA(h, cudaMemcpyAsync(idx, out, sizeof(int64_t) * nk, cudaMemcpyDeviceToDevice, h->stream));
    RQ_TRY(sync(h, "unique"));
    dfree(head);
    dfree(out);
    return RISQGPU_OK;
}

__global__ void k_gather_out(const int64_t* __restrict__ idx, int64_t K, const uint64_t* __restrict__ cfg, int64_t L,
                             const double* __restrict__ dg, int W, uint64_t* __restrict__ aos,
                             double* __restrict__ dout) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = idx[k];
        for (int q = 0; q < 2; q++) {
            aos[k * 4 + q] = q < W ? cfg[q * L + e] : 0ull;
            aos[k * 4 + 2 + q] = q < W ? cfg[(W + q) * L + e] : 0ull;
        }
        dout[k] = dg[e];
    }
}

template <int W>
int find_new_impl(risqgpu* h, const double* coeffs, double eps, bool singles, const SelectTables& tab,
                  std::vector<uint64_t>& new_dets, std::vector<double>& new_diag, SelectStats* st) {
    const int64_t N = (int64_t)h->N;
    new_dets.clear();
    new_diag.clear();
    // caller-order determinants, coefficients and diagonals on the device
    uint64_t* aos = nullptr;
    double *cf = nullptr, *dgc = nullptr;
    RQ_TRY(dalloc(h, aos, 4 * N));
    RQ_TRY(dalloc(h, cf, N));
    RQ_TRY(dalloc(h, dgc, N));
    RQ_CUDA(h, cudaMemcpyAsync(aos, h->h_dets.data(), sizeof(uint64_t) * 4 * N, cudaMemcpyHostToDevice, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(cf, coeffs, sizeof(double) * N, cudaMemcpyHostToDevice, h->stream));
    {
        std::vector<double> dg_int(N), dg_c(N);
        std::vector<int32_t> orig(N);
        RQ_CUDA(h, cudaMemcpyAsync(dg_int.data(), h->d_diag, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
        RQ_CUDA(h, cudaMemcpyAsync(orig.data(), h->d_orig, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, h->stream));
        RQ_TRY(sync(h, "select prep"));
        for (int64_t p = 0; p < N; p++) dg_c[orig[p]] = dg_int[p];
        RQ_CUDA(h, cudaMemcpy(dgc, dg_c.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
    }
    // tables
    int32_t *oo = nullptr, *so = nullptr, *go = nullptr;
    uint8_t *tr = nullptr, *ts = nullptr;
    double* th = nullptr;
    RQ_TRY(dalloc(h, oo, tab.opp_off.size()));
    RQ_TRY(dalloc(h, so, tab.same_off.size()));
    RQ_TRY(dalloc(h, go, tab.sing_off.size()));
    RQ_TRY(dalloc(h, tr, tab.r.size()));
    RQ_TRY(dalloc(h, ts, tab.s.size()));
    RQ_TRY(dalloc(h, th, tab.habs.size()));
    RQ_CUDA(h, cudaMemcpyAsync(oo, tab.opp_off.data(), 4 * tab.opp_off.size(), cudaMemcpyHostToDevice, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(so, tab.same_off.data(), 4 * tab.same_off.size(), cudaMemcpyHostToDevice, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(go, tab.sing_off.data(), 4 * tab.sing_off.size(), cudaMemcpyHostToDevice, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(tr, tab.r.data(), tab.r.size(), cudaMemcpyHostToDevice, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(ts, tab.s.data(), tab.s.size(), cudaMemcpyHostToDevice, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(th, tab.habs.data(), 8 * tab.habs.size(), cudaMemcpyHostToDevice, h->stream));
    Tables T{oo, so, go, tr, ts, th, h->norb, tab.max_opp, tab.max_same, tab.max_sing};
    Bits<W> val;
    for (int q = 0; q < W; q++) val.w[q] = tab.valence[q];
    Ints I{h->d_h1, h->d_h2, h->nuc};
    SortedSet<W> set{h->d_up, h->d_dn, N};
    int* counter = nullptr;
    int64_t *cnt = nullptr, *off = nullptr;
    RQ_TRY(dalloc(h, counter, 1));
    RQ_TRY(dalloc(h, cnt, N + 1));
    RQ_TRY(dalloc(h, off, N + 1));
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_expand<W, true>, 256, 0);
    const int blocks = num_sms(h) * std::max(occ, 1);
    RQ_CUDA(h, cudaMemsetAsync(counter, 0, sizeof(int), h->stream));
    RQ_CUDA(h, cudaMemsetAsync(cnt + N, 0, sizeof(int64_t), h->stream));
    k_expand<W, false><<<blocks, 256, 0, h->stream>>>(aos, cf, N, eps, singles ? 1 : 0, T, val, I, set, counter, cnt,
                                                      nullptr, nullptr, nullptr, nullptr, 0);
    RQ_TRY(check_launch(h, "expand count"));
    {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, (int)(N + 1), h->stream);
        char* tmp = nullptr;
        RQ_TRY(dalloc(h, tmp, tb));
        cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, (int)(N + 1), h->stream);
        RQ_TRY(sync(h, "expand scan"));
        dfree(tmp);
    }
    int64_t M = 0;
    RQ_CUDA(h, cudaMemcpy(&M, off + N, sizeof(int64_t), cudaMemcpyDeviceToHost));
    if (st) st->candidates = (uint64_t)M;
    if (M > 0) {
        uint64_t* cfg = nullptr;
        int32_t* parent = nullptr;
        uint32_t* code = nullptr;
        RQ_TRY(dalloc(h, cfg, (size_t)2 * W * M));
        RQ_TRY(dalloc(h, parent, M));
        RQ_TRY(dalloc(h, code, M));
        RQ_CUDA(h, cudaMemsetAsync(counter, 0, sizeof(int), h->stream));
        k_expand<W, true><<<blocks, 256, 0, h->stream>>>(aos, cf, N, eps, singles ? 1 : 0, T, val, I, set, counter,
                                                         nullptr, off, cfg, parent, code, M);
        RQ_TRY(check_launch(h, "expand fill"));
        // first occurrence of each configuration
        int64_t* idx = nullptr;
        RQ_TRY(dalloc(h, idx, M));
        k_iota64<<<grid_of(h, M), 256, 0, h->stream>>>(idx, M);
        int64_t K = 0;
        RQ_TRY(unique_first<W>(h, cfg, M, idx, M, K));
        // diagonals and [flip(d), d] pairs
        const int64_t L = 2 * K;
        uint64_t* pcfg = nullptr;
        double* pdg = nullptr;
        RQ_TRY(dalloc(h, pcfg, (size_t)2 * W * L));
        RQ_TRY(dalloc(h, pdg, L));
        k_finish<W><<<grid_of(h, K), 256, 0, h->stream>>>(idx, K, cfg, M, parent, code, aos, dgc, I, pcfg, pdg);
        RQ_TRY(check_launch(h, "finish"));
        dfree(cfg); dfree(parent); dfree(code); dfree(idx);
        // drop flips already in the space, then first occurrence again
        int32_t* keep = nullptr;
        int64_t *lidx = nullptr, *lkeep = nullptr;
        RQ_TRY(dalloc(h, keep, L));
        RQ_TRY(dalloc(h, lidx, L));
        RQ_TRY(dalloc(h, lkeep, L));
        k_not_in_set<W><<<grid_of(h, L), 256, 0, h->stream>>>(pcfg, L, set, keep);
        k_iota64<<<grid_of(h, L), 256, 0, h->stream>>>(lidx, L);
        int64_t L2 = 0;
        RQ_TRY(compact_i64(h, lidx, keep, L, lkeep, L2));
        int64_t F = 0;
        RQ_TRY(unique_first<W>(h, pcfg, L, lkeep, L2, F));
        uint64_t* outd = nullptr;
        double* outg = nullptr;
        RQ_TRY(dalloc(h, outd, 4 * std::max<int64_t>(F, 1)));
        RQ_TRY(dalloc(h, outg, std::max<int64_t>(F, 1)));
        k_gather_out<<<grid_of(h, std::max<int64_t>(F, 1)), 256, 0, h->stream>>>(lkeep, F, pcfg, L, pdg, W, outd, outg);
        RQ_TRY(check_launch(h, "gather out"));
        new_dets.resize(4 * F);
        new_diag.resize(F);
        RQ_CUDA(h, cudaMemcpyAsync(new_dets.data(), outd, sizeof(uint64_t) * 4 * F, cudaMemcpyDeviceToHost, h->stream));
        RQ_CUDA(h, cudaMemcpyAsync(new_diag.data(), outg, sizeof(double) * F, cudaMemcpyDeviceToHost, h->stream));
        RQ_TRY(sync(h, "select out"));
        if (st) { st->unique = (uint64_t)K; st->added = (uint64_t)F; }
        dfree(pcfg); dfree(pdg); dfree(keep); dfree(lidx); dfree(lkeep); dfree(outd); dfree(outg);
    } else if (st) {
        st->unique = st->added = 0;
    }
    dfree(aos); dfree(cf); dfree(dgc); dfree(oo); dfree(so); dfree(go); dfree(tr); dfree(ts); dfree(th);
    dfree(counter); dfree(cnt); dfree(off);
    return RISQGPU_OK;
}

}  // namespace

int find_new_dets_impl(risqgpu* h, const double* coeffs, double eps, bool singles, const SelectTables& tab,
                       std::vector<uint64_t>& new_dets, std::vector<double>& new_diag, SelectStats* st) {
    if (h->N == 0) { h->err = "no determinants set"; return RISQGPU_ERR_INVALID; }
    return h->W == 1 ? find_new_impl<1>(h, coeffs, eps, singles, tab, new_dets, new_diag, st)
                     : find_new_impl<2>(h, coeffs, eps, singles, tab, new_dets, new_diag, st);
}

}  // namespace risq
