// The variational HCI loop around the hot path, driven from the host.
//
//   build_select_tables   init_excite_generator      src/excite/init.rs:81-280
//   init_eps / Eps::next  starting threshold, x0.1    src/wf/eps.rs:41-172
//   variational_impl      init_var_wf + variational  src/wf/mod.rs:1687-1740, src/var/mod.rs:59-134
// Selection, the sparse H build and Davidson run on the device; this file only
// keeps the determinant list, coefficients and diagonals in caller order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "select.cuh"

namespace risq {

namespace {

struct HostInts {
    const risqgpu* h;
    static size_t c2(long i, long j) { return i > j ? (size_t)((i * (i - 1)) / 2 + j) : (size_t)((j * (j - 1)) / 2 + i); }
    double one_body(int p, int q) const { return h->h_h1[c2(p + 1, q + 1)]; }
    double get(int p, int q, int r, int s) const { return h->h_h2[c2((long)c2(p, q), (long)c2(r, s))]; }
    double direct(int p, int q, int r, int s) const { return get(p + 1, r + 1, q + 1, s + 1); }
    double dpe(int p, int q, int r, int s) const { return get(p + 1, r + 1, q + 1, s + 1) - get(p + 1, s + 1, q + 1, r + 1); }
};

struct Entry {
    int r, s;
    double h;
};

void stable_desc(std::vector<Entry>& v) {
    std::stable_sort(v.begin(), v.end(), [](const Entry& a, const Entry& b) { return a.h > b.h; });
}

inline bool bit(const uint64_t* w, int b) { return (w[b >> 6] >> (b & 63)) & 1ull; }

struct Eps {
    double next_one, target;
    double next() {  // Eps::next (src/wf/eps.rs:41-53)
        double curr = next_one;
        double prop = next_one * 0.1;
        next_one = prop > target ? prop : target;
        return curr;
    }
};

// init_eps for the HF start with z_sym == 1 (src/wf/eps.rs:82-172).
Eps init_eps(const SelectTables& t, int n, const uint64_t* hf, double eps_var) {
    double max_sym = eps_var, max_asym = eps_var;
    const uint64_t up[2] = {hf[0], hf[1]}, dn[2] = {hf[2], hf[3]};
    const uint64_t vu[2] = {up[0] & t.valence[0], up[1] & t.valence[1]};
    const uint64_t vd[2] = {dn[0] & t.valence[0], dn[1] & t.valence[1]};
    for (int i = 0; i < n; i++) {
        if (!bit(vu, i)) continue;
        for (int j = 0; j < n; j++) {
            if (!bit(vd, j)) continue;
            bool fs = false, fa = false;
            for (int k = t.opp_off[i * n + j]; k < t.opp_off[i * n + j + 1]; k++) {
                const int r = t.r[k], s = t.s[k];
                if (!bit(up, r) && !bit(dn, s)) {
                    const double th = t.habs[k];
                    if (i == j && r == s) {
                        fs = true;
                        if (th > max_sym) max_sym = th;
                    } else {
                        fa = true;
                        if (th > max_asym) max_asym = th;
                    }
                    if (fs && fa) break;
                }
            }
        }
    }
    for (int sp = 0; sp < 2; sp++) {
        const uint64_t* x = sp == 0 ? up : dn;
        const uint64_t vx[2] = {x[0] & t.valence[0], x[1] & t.valence[1]};
        for (int i = 0; i < n; i++) {
            if (!bit(vx, i)) continue;
            for (int j = i + 1; j < n; j++) {
                if (!bit(vx, j)) continue;
                for (int k = t.same_off[i * n + j]; k < t.same_off[i * n + j + 1]; k++) {
                    if (!bit(x, t.r[k]) && !bit(x, t.s[k])) {
                        if (t.habs[k] > max_asym) max_asym = t.habs[k];
                        break;
                    }
                }
            }
        }
    }
    const double max_doub = max_sym > max_asym ? max_sym : max_asym;
    return Eps{max_doub - 1e-9, eps_var};
}

}  // namespace

int build_select_tables(risqgpu* h, int ncore, int n_up, int n_dn, SelectTables& t) {
    const int n = h->norb;
    if (ncore < 0 || ncore >= n) { h->err = "ncore must be in [0, norb)"; return RISQGPU_ERR_INVALID; }
    HostInts I{h};
    // core / valence by ascending h_ii, stable (src/ham/read_ints.rs:161-184)
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return I.one_body(a, a) < I.one_body(b, b); });
    t.core_orbs.assign(order.begin(), order.begin() + ncore);
    t.valence_orbs.assign(order.begin() + ncore, order.end());
    t.valence[0] = t.valence[1] = 0;
    for (int v : t.valence_orbs) t.valence[v >> 6] |= 1ull << (v & 63);
    const std::vector<int>& vo = t.valence_orbs;
    t.opp_off.assign((size_t)n * n + 1, 0);
    t.same_off.assign((size_t)n * n + 1, 0);
    t.sing_off.assign((size_t)n + 1, 0);
    t.r.clear(); t.s.clear(); t.habs.clear();
    t.max_opp = t.max_same = t.max_sing = 0.0;
    std::vector<std::vector<Entry>> opp((size_t)n * n), same((size_t)n * n), sing(n);
    std::vector<Entry> v;
    for (int p : vo)
        for (int q : vo) {
            v.clear();
            for (int r : vo) {
                if (p == r) continue;
                for (int s : vo) {
                    if (q == s) continue;
                    double hv = std::fabs(I.direct(p, q, r, s));
                    if (hv > t.max_opp) t.max_opp = hv;
                    v.push_back({r, s, hv});
                }
            }
            stable_desc(v);
            opp[(size_t)p * n + q] = v;
        }
    for (int p : vo)
        for (int q : vo) {
            if (p >= q) continue;
            v.clear();
            for (int r : vo) {
                if (p == r || q == r) continue;
                for (int s : vo) {
                    if (r >= s) continue;
                    if (p == s || q == s) continue;
                    double hv = std::fabs(I.dpe(p, q, r, s));
                    if (hv > t.max_same) t.max_same = hv;
                    v.push_back({r, s, hv});
                }
            }
            stable_desc(v);
            same[(size_t)p * n + q] = v;
        }
    std::vector<double> vs, vp;
    for (int p : vo) {
        v.clear();
        for (int r : vo) {
            if (p == r) continue;
            vs.clear();
            vp.clear();
            for (int q = 0; q < n; q++) {
                if (p == q || q == r) continue;
                vs.push_back(I.dpe(p, q, r, q));
                vp.push_back(I.direct(p, q, r, q));
            }
            std::stable_sort(vs.begin(), vs.end());
            std::stable_sort(vp.begin(), vp.end());
            const int L = (int)vs.size();
            if (n_up - 1 > L || n_dn > L) { h->err = "too many electrons for the orbital space"; return RISQGPU_ERR_INVALID; }
            double s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
            for (int k = 0; k < n_up - 1; k++) s1 += vs[k];
            for (int k = 0; k < n_dn; k++) s2 += vp[k];
            for (int k = L - (n_up - 1); k < L; k++) s3 += vs[k];
            for (int k = L - n_dn; k < L; k++) s4 += vp[k];
            const double max1 = I.one_body(p, r) + s1 + s2;
            const double max2 = I.one_body(p, r) + s3 + s4;
            v.push_back({r, 0, std::fabs(max1) > std::fabs(max2) ? std::fabs(max1) : std::fabs(max2)});
        }
        stable_desc(v);
        sing[p] = v;
    }
    for (int p : vo) {
        double x = sing[p].empty() ? 0.0 : sing[p][0].h;
        t.max_sing = std::fmax(t.max_sing, x);
    }
    auto flatten = [&](std::vector<std::vector<Entry>>& lists, std::vector<int32_t>& off) {
        for (size_t k = 0; k < lists.size(); k++) {
            off[k] = (int32_t)t.habs.size();
            for (const Entry& e : lists[k]) {
                t.r.push_back((uint8_t)e.r);
                t.s.push_back((uint8_t)e.s);
                t.habs.push_back(e.h);
            }
        }
        off[lists.size()] = (int32_t)t.habs.size();
    };
    flatten(opp, t.opp_off);
    flatten(same, t.same_off);
    flatten(sing, t.sing_off);
    return RISQGPU_OK;
}

int variational_impl(risqgpu* h, int nup, int ndn, int ncore, double eps_var, int max_iter, int dav_max_iter,
                     int precision, int mode, int precond, double* energy, uint64_t* n_dets) {
    using clk = std::chrono::steady_clock;
    if (nup < 0 || ndn < 0 || nup > h->norb || ndn > h->norb) { h->err = "bad electron counts"; return RISQGPU_ERR_INVALID; }
    if (!(eps_var > 0)) { h->err = "eps_var must be positive"; return RISQGPU_ERR_INVALID; }
    SelectTables tab;
    RQ_TRY(build_select_tables(h, ncore, nup, ndn, tab));
    // HF determinant: lowest nup / ndn orbitals (src/wf/mod.rs:1697-1698)
    uint64_t hf[4] = {0, 0, 0, 0};
    for (int i = 0; i < nup; i++) hf[i >> 6] |= 1ull << (i & 63);
    for (int i = 0; i < ndn; i++) hf[2 + (i >> 6)] |= 1ull << (i & 63);
    double hf_diag = 0.0;
    RQ_TRY(ham_elements_impl(h, hf, nullptr, 1, &hf_diag, true));
    h->wf_dets.assign(hf, hf + 4);
    h->wf_coeffs.assign(1, 1.0);
    h->wf_diag.assign(1, hf_diag);
    h->wf_energy = hf_diag;
    h->var_log.clear();
    Eps eps_iter = init_eps(tab, h->norb, hf, eps_var);
    free_dets(h);
    RQ_TRY(set_dets_impl(h, h->wf_dets.data(), 1, 0, h->wf_diag.data()));
    size_t n_stored = 0;
    const bool verbose = std::getenv("RISQGPU_VERBOSE") != nullptr;
    // precision -1: FP64 values while they fit in device memory, then columns only with
    // the FP64 elements recomputed in sigma (FP64 arithmetic throughout)
    const bool auto_prec = precision < 0;
    int cur_prec = auto_prec ? RISQGPU_FP64 : precision;
    int cur_mode = auto_prec ? RISQGPU_MODE_FP64 : mode;
    for (int iter = 1; iter <= max_iter; iter++) {
        risqgpu_var_iter rec;
        std::memset(&rec, 0, sizeof(rec));
        auto t0 = clk::now();
        const double eps = eps_iter.next();  // find_new_dets (src/wf/mod.rs:1418-1425)
        std::vector<uint64_t> nd;
        std::vector<double> ng;
        SelectStats ss;
        RQ_TRY(find_new_dets_impl(h, h->wf_coeffs.data(), eps, eps == eps_var, tab, nd, ng, &ss));
        const size_t added = ng.size();
        h->wf_dets.insert(h->wf_dets.end(), nd.begin(), nd.end());
        h->wf_diag.insert(h->wf_diag.end(), ng.begin(), ng.end());
        h->wf_coeffs.resize(h->wf_diag.size(), 0.0);
        auto t1 = clk::now();
        rec.eps = eps;
        rec.n_new = added;
        rec.candidates = ss.candidates;
        rec.ms_select = std::chrono::duration<double, std::milli>(t1 - t0).count();
        if (eps == eps_var && ss.unique == 0) break;  // converged (src/var/mod.rs:83-87)
        // sparse_optimize (src/var/davidson.rs:43-113)
        const size_t N = h->wf_diag.size();
        if (!(h->built && added == 0)) {
            // upper-triangle storage is rebuilt from scratch every time
            const size_t nsh = cur_prec >= RISQGPU_FP64_UPPER ? 0 : n_stored;
            RQ_TRY(set_dets_impl(h, h->wf_dets.data(), N, nsh, h->wf_diag.data()));
            int rc = build_h_impl(h, cur_prec, RISQGPU_BUILDER_AUTO, nullptr);
            if (rc == RISQGPU_ERR_OOM && n_stored > 0) {
                // no room for the kept previous matrix next to the new one: rebuild every pair
                // (the stored set then differs from the reference's history only by singles of
                // magnitude <= 1e-12 that a legacy-rule build (N <= 100) had kept)
                if (verbose) std::fprintf(stderr, "[risqgpu] iter %d: incremental build does not fit, rebuilding\n", iter);
                RQ_TRY(set_dets_impl(h, h->wf_dets.data(), N, 0, h->wf_diag.data()));
                rc = build_h_impl(h, cur_prec, RISQGPU_BUILDER_AUTO, nullptr);
            }
            if (rc == RISQGPU_ERR_OOM && auto_prec && cur_prec == RISQGPU_FP64) {
                // both triangles do not fit: store each pair once (the reference's own layout)
                if (verbose) std::fprintf(stderr, "[risqgpu] iter %d: full FP64 rows do not fit, upper triangle from here\n", iter);
                cur_prec = RISQGPU_FP64_UPPER;
                RQ_TRY(set_dets_impl(h, h->wf_dets.data(), N, 0, h->wf_diag.data()));
                rc = build_h_impl(h, cur_prec, RISQGPU_BUILDER_AUTO, nullptr);
            }
            if (rc == RISQGPU_ERR_OOM && auto_prec && cur_prec == RISQGPU_FP64_UPPER) {
                // FP64 values do not fit at all: keep the columns only and recompute the FP64
                // elements inside sigma (the same values, a third of the storage)
                if (verbose) std::fprintf(stderr, "[risqgpu] iter %d: FP64 values do not fit, columns only from here\n", iter);
                cur_prec = RISQGPU_COLS;
                RQ_TRY(set_dets_impl(h, h->wf_dets.data(), N, 0, h->wf_diag.data()));
                rc = build_h_impl(h, cur_prec, RISQGPU_BUILDER_AUTO, nullptr);
            }
            if (rc == RISQGPU_ERR_OOM && auto_prec && cur_prec == RISQGPU_COLS) {
                // not even the columns fit: find and evaluate the elements inside sigma
                if (verbose) std::fprintf(stderr, "[risqgpu] iter %d: columns do not fit, matrix-free from here\n", iter);
                cur_prec = RISQGPU_MATRIX_FREE;
                RQ_TRY(set_dets_impl(h, h->wf_dets.data(), N, 0, h->wf_diag.data()));
                rc = build_h_impl(h, cur_prec, RISQGPU_BUILDER_AUTO, nullptr);
            }
            if (rc != RISQGPU_OK) {
                // the space outgrew every storage mode: log the selection that got that far
                rec.n_dets = N;
                rec.energy = NAN;
                rec.dav_converged = -1;
                rec.storage = -1;
                h->var_log.push_back(rec);
                return rc;
            }
            n_stored = N;
        }
        auto t2 = clk::now();
        double e = 0.0;
        std::vector<double> vec(N);
        risqgpu_dstats ds;
        std::memset(&ds, 0, sizeof(ds));
        int rc = davidson_impl(h, 1, iter > 1 ? h->wf_coeffs.data() : nullptr, iter > 1 ? 1 : 0, 1e-4, 1e-8,
                               dav_max_iter, cur_mode, precond, &e, vec.data(), &ds);
        if (rc == RISQGPU_OK) {
            h->wf_energy = e;
            h->wf_coeffs = vec;
        } else if (rc != RISQGPU_ERR_NOT_CONVERGED) {
            return rc;
        }  // on non-convergence energy and coefficients stay (src/var/davidson.rs:109-111)
        auto t3 = clk::now();
        rec.n_dets = N;
        rec.storage = cur_prec;
        rec.nnz_upper = h->nnz_upper;
        rec.energy = h->wf_energy;
        rec.dav_iters = ds.iters;
        rec.dav_converged = rc == RISQGPU_OK ? 1 : 0;
        rec.ms_build = std::chrono::duration<double, std::milli>(t2 - t1).count();
        rec.ms_davidson = std::chrono::duration<double, std::milli>(t3 - t2).count();
        h->var_log.push_back(rec);
        if (verbose)
            std::fprintf(stderr,
                         "[risqgpu] iter %d eps %.3g N %llu new %llu nnz_upper %llu E %.10f dav %d%s "
                         "sel %.1f ms build %.1f ms dav %.1f ms\n",
                         iter, eps, (unsigned long long)N, (unsigned long long)added,
                         (unsigned long long)h->nnz_upper, h->wf_energy, ds.iters, rc == RISQGPU_OK ? "" : " (not converged)",
                         rec.ms_select, rec.ms_build, rec.ms_davidson);
        eps_iter.next();  // src/var/mod.rs:123
    }
    if (energy) *energy = h->wf_energy;
    if (n_dets) *n_dets = h->wf_diag.size();
    return RISQGPU_OK;
}

}  // namespace risq

using namespace risq;

extern "C" {

int risqgpu_find_new_dets(risqgpu_t* h, const double* coeffs, double eps, int singles, int ncore, size_t* n_new) {
    if (!h || !coeffs || !n_new) return RISQGPU_ERR_INVALID;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != h->device) cudaSetDevice(h->device);
    SelectTables tab;
    int rc = build_select_tables(h, ncore, h->n_up, h->n_dn, tab);
    if (rc == RISQGPU_OK) {
        SelectStats ss;
        rc = find_new_dets_impl(h, coeffs, eps, singles != 0, tab, h->pend_dets, h->pend_diag, &ss);
        *n_new = h->pend_diag.size();
    }
    if (prev >= 0 && prev != h->device) cudaSetDevice(prev);
    return rc;
}

int risqgpu_get_new_dets(risqgpu_t* h, uint64_t* dets, double* diag, size_t cap) {
    if (!h) return RISQGPU_ERR_INVALID;
    const size_t n = h->pend_diag.size();
    if (cap < n) return RISQGPU_ERR_CAPACITY;
    if (n && (!dets || !diag)) return RISQGPU_ERR_INVALID;
    std::memcpy(dets, h->pend_dets.data(), sizeof(uint64_t) * 4 * n);
    std::memcpy(diag, h->pend_diag.data(), sizeof(double) * n);
    return RISQGPU_OK;
}

int risqgpu_variational(risqgpu_t* h, int nup, int ndn, int ncore, int z_sym, double eps_var, int max_iter,
                        int dav_max_iter, int precision, int mode, int precond, double* energy, uint64_t* n_dets) {
    if (!h || z_sym != 1 || max_iter < 1 || dav_max_iter < 1) {
        if (h) h->err = "z_sym must be 1 and the iteration limits positive";
        return RISQGPU_ERR_INVALID;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != h->device) cudaSetDevice(h->device);
    int rc = variational_impl(h, nup, ndn, ncore, eps_var, max_iter, dav_max_iter, precision, mode, precond, energy,
                              n_dets);
    if (prev >= 0 && prev != h->device) cudaSetDevice(prev);
    return rc;
}

int risqgpu_get_wf(risqgpu_t* h, uint64_t* dets, double* coeffs, double* diag, size_t cap) {
    if (!h) return RISQGPU_ERR_INVALID;
    const size_t n = h->wf_diag.size();
    if (cap < n) return RISQGPU_ERR_CAPACITY;
    if (dets) std::memcpy(dets, h->wf_dets.data(), sizeof(uint64_t) * 4 * n);
    if (coeffs) std::memcpy(coeffs, h->wf_coeffs.data(), sizeof(double) * n);
    if (diag) std::memcpy(diag, h->wf_diag.data(), sizeof(double) * n);
    return RISQGPU_OK;
}

int risqgpu_var_log(risqgpu_t* h, risqgpu_var_iter* out, int cap, int* n) {
    if (!h || !n) return RISQGPU_ERR_INVALID;
    *n = (int)h->var_log.size();
    for (int i = 0; i < *n && i < cap; i++) out[i] = h->var_log[i];
    return RISQGPU_OK;
}

}  // extern "C"
