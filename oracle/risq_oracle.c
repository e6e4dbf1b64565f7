/*
 * risq_oracle.c -- CPU restatement of RISQ's HCI variational path.
 *
 * TEST INFRASTRUCTURE. This library is the checker for the CUDA path: only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark load it.
 * Nothing in the shipped library links, imports or calls it.
 *
 * Every function restates one piece of the reference Rust crate (aaholmes/risq);
 * the file:line it follows is given beside it.  Orbital indices are 0-based in
 * determinants and 1-based in the packed integral tables, exactly as in the
 * reference.  u128 determinant strings are held as `unsigned __int128`; across
 * the C ABI they travel as two little-endian u64 halves {lo, hi}.
 *
 * Parity pins (see tests/): the golden variational energies of the reference's
 * integration tests (tests/integration_test_suite.rs:34,44,64,74), the parity
 * known-answer cases (src/utils/bits.rs:197-211), the fast_ham lookup-table unit
 * tests (src/var/fast_ham.rs:638-786) and MGS orthonormality
 * (src/var/eigenvalues/modified_gram_schmidt.rs:45-67).
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <errno.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

#define OR_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------- */
/* utils/bits.rs                                                              */
/* ------------------------------------------------------------------------- */

static inline int popc128(u128 x) {
    return __builtin_popcountll((uint64_t)x) + __builtin_popcountll((uint64_t)(x >> 64));
}

static inline int ctz128(u128 x) {
    uint64_t lo = (uint64_t)x;
    if (lo) return __builtin_ctzll(lo);
    return 64 + __builtin_ctzll((uint64_t)(x >> 64));
}

static inline u128 bit128(int b) { return ((u128)1) << b; }

/* parity(n): xor-fold, +1 for an even number of set bits (src/utils/bits.rs:171-180). */
static inline int parity128(u128 n) {
    n ^= n >> 64;
    n ^= n >> 32;
    n ^= n >> 16;
    n ^= n >> 8;
    n ^= n >> 4;
    n ^= n >> 2;
    n ^= n >> 1;
    return 1 - 2 * (int)(n & 1);
}

/* bits(n) iterates set bits from the lowest (src/utils/bits.rs:14-25); callers
 * below write that loop inline as: for (t = n; t; t &= t - 1) k = ctz128(t). */

/* ------------------------------------------------------------------------- */
/* utils/ints.rs                                                              */
/* ------------------------------------------------------------------------- */

/* combine_2 (src/utils/ints.rs:38-46): 1-based triangular index, sign ignored. */
static inline size_t combine_2(int p, int q) {
    long i = labs((long)p), j = labs((long)q);
    if (i > j) return (size_t)((i * (i - 1)) / 2 + j);
    return (size_t)((j * (j - 1)) / 2 + i);
}

/* combine_2_usize (src/utils/ints.rs:49-55). */
static inline size_t combine_2u(size_t i, size_t j) {
    if (i > j) return (i * (i - 1)) / 2 + j;
    return (j * (j - 1)) / 2 + i;
}

/* combine_4 (src/utils/ints.rs:66-68). */
static inline size_t combine_4(int p, int q, int r, int s) {
    return combine_2u(combine_2(p, q), combine_2(r, s));
}

/* permute (src/utils/ints.rs:76-82): parity of the occupied bits strictly
 * between the two differing orbitals. */
static inline int permute1(u128 d1, u128 d2) {
    if (d1 > d2) return parity128(d1 & (d1 - d2));
    return parity128(d2 & (d2 - d1));
}

/* permute_2 (src/utils/ints.rs:92-97). */
static inline int permute2(u128 d1, u128 d2, const int v[4]) {
    u128 m = (bit128(v[0]) - 1) ^ (bit128(v[1]) - 1) ^ (bit128(v[2]) - 1) ^ (bit128(v[3]) - 1);
    return parity128(d1 & d2 & m);
}

/* ------------------------------------------------------------------------- */
/* ham/read_ints.rs + ham/mod.rs                                              */
/* ------------------------------------------------------------------------- */

typedef struct {
    int norb;
    double nuc;
    size_t n1, n2;
    double *one_body; /* combine_2(p,q), 1-based   (src/ham/read_ints.rs:79) */
    double *two_body; /* combine_4(p,q,r,s), 1-based (src/ham/read_ints.rs:80) */
    int ncore, nval;
    int *core_orbs;
    int *valence_orbs;
} Ham;

static inline double get_int(const Ham *h, int p, int q, int r, int s) { /* ham/mod.rs:49-55 */
    return h->two_body[combine_4(p, q, r, s)];
}
static inline double one_body(const Ham *h, int p, int q) { /* ham/mod.rs:65-67 */
    return h->one_body[combine_2(p + 1, q + 1)];
}
static inline double direct(const Ham *h, int p, int q, int r, int s) { /* ham/mod.rs:72-74 */
    return get_int(h, p + 1, r + 1, q + 1, s + 1);
}
static inline double dpe(const Ham *h, int p, int q, int r, int s) { /* ham/mod.rs:80-82 */
    return get_int(h, p + 1, r + 1, q + 1, s + 1) - get_int(h, p + 1, s + 1, q + 1, r + 1);
}

/* Core/valence split by ascending h_ii with a stable sort (src/ham/read_ints.rs:161-184). */
static void ham_split_core(Ham *h, int ncore) {
    int n = h->norb;
    int *idx = malloc(sizeof(int) * n);
    double *f = malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++) { idx[i] = i; f[i] = one_body(h, i, i); }
    /* stable insertion sort by f */
    for (int i = 1; i < n; i++) {
        int ki = idx[i];
        double kf = f[i];
        int j = i - 1;
        while (j >= 0 && f[j] > kf) { f[j + 1] = f[j]; idx[j + 1] = idx[j]; j--; }
        f[j + 1] = kf; idx[j + 1] = ki;
    }
    h->ncore = 0; h->nval = 0;
    h->core_orbs = malloc(sizeof(int) * (n > 0 ? n : 1));
    h->valence_orbs = malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int i = 0; i < n; i++) {
        if (i < ncore) h->core_orbs[h->ncore++] = idx[i];
        else h->valence_orbs[h->nval++] = idx[i];
    }
    free(idx); free(f);
}

static Ham *ham_alloc(int norb) {
    Ham *h = calloc(1, sizeof(Ham));
    h->norb = norb;
    h->n1 = combine_2(norb + 1, norb + 1);
    h->n2 = combine_4(norb + 1, norb + 1, norb + 1, norb + 1);
    h->one_body = calloc(h->n1, sizeof(double));
    h->two_body = calloc(h->n2, sizeof(double));
    return h;
}

OR_EXPORT void or_ham_free(Ham *h) {
    if (!h) return;
    free(h->one_body); free(h->two_body); free(h->core_orbs); free(h->valence_orbs); free(h);
}

/* A token is a float only if the whole token parses (lexical::parse semantics
 * as used at src/ham/read_ints.rs:102-105). */
static int parse_full_double(const char *tok, double *out) {
    char *end;
    errno = 0;
    double v = strtod(tok, &end);
    if (end == tok || *end != '\0') return 0;
    /* lexical rejects hexadecimal floats and "inf"/"nan" spelled words that strtod accepts */
    for (const char *c = tok; *c; c++)
        if (*c == 'x' || *c == 'X' || *c == 'n' || *c == 'N' || *c == 'i' || *c == 'I') return 0;
    *out = v;
    return 1;
}

static int parse_full_int(const char *tok, int *out) {
    char *end;
    errno = 0;
    long v = strtol(tok, &end, 10);
    if (end == tok || *end != '\0' || errno) return 0;
    *out = (int)v;
    return 1;
}

/* read_ints (src/ham/read_ints.rs:73-190).  Returns NULL and fills err on failure. */
OR_EXPORT Ham *or_ham_read_fcidump(const char *path, int norb, int ncore, char *err, int errlen) {
    FILE *fp = fopen(path, "r");
    if (!fp) { snprintf(err, errlen, "cannot open %s", path); return NULL; }
    Ham *h = ham_alloc(norb);
    char *line = NULL;
    size_t cap = 0;
    long lineno = 0;
    while (getline(&line, &cap, fp) >= 0) {
        lineno++;
        char *save = NULL;
        char *tok = strtok_r(line, " \t\r\n", &save);
        if (!tok) { snprintf(err, errlen, "line %ld: Missing integral value", lineno); goto fail; }
        double val;
        if (!parse_full_double(tok, &val)) continue; /* header line */
        int idx[4];
        const char *names[4] = {"p", "q", "r", "s"};
        for (int k = 0; k < 4; k++) {
            char *t = strtok_r(NULL, " \t\r\n", &save);
            if (!t) { snprintf(err, errlen, "line %ld: Missing %s index", lineno, names[k]); goto fail; }
            if (!parse_full_int(t, &idx[k])) { snprintf(err, errlen, "line %ld: Invalid %s index: '%s'", lineno, names[k], t); goto fail; }
            if (idx[k] < 0 || idx[k] > norb) { snprintf(err, errlen, "line %ld: Index %s out of range [0, %d]: %d", lineno, names[k], norb, idx[k]); goto fail; }
        }
        int p = idx[0], q = idx[1], r = idx[2], s = idx[3];
        if (p == 0 && q == 0 && r == 0 && s == 0) h->nuc = val;
        else if (r == 0 && s == 0) {
            size_t id = combine_2(p, q);
            if (id >= h->n1) { snprintf(err, errlen, "line %ld: one_body index %zu >= %zu", lineno, id, h->n1); goto fail; }
            h->one_body[id] = val;
        } else {
            size_t id = combine_4(p, q, r, s);
            if (id >= h->n2) { snprintf(err, errlen, "line %ld: two_body index %zu >= %zu", lineno, id, h->n2); goto fail; }
            h->two_body[id] = val;
        }
    }
    free(line);
    fclose(fp);
    ham_split_core(h, ncore);
    return h;
fail:
    free(line);
    fclose(fp);
    or_ham_free(h);
    return NULL;
}

/* Build a Ham from arrays already in the reference's packed layout. */
OR_EXPORT Ham *or_ham_from_arrays(int norb, int ncore, double nuc, const double *ob, const double *tb) {
    Ham *h = ham_alloc(norb);
    h->nuc = nuc;
    memcpy(h->one_body, ob, sizeof(double) * h->n1);
    memcpy(h->two_body, tb, sizeof(double) * h->n2);
    ham_split_core(h, ncore);
    return h;
}

OR_EXPORT void or_ham_sizes(const Ham *h, size_t *n1, size_t *n2) { *n1 = h->n1; *n2 = h->n2; }
OR_EXPORT void or_ham_copy(const Ham *h, double *nuc, double *ob, double *tb) {
    *nuc = h->nuc;
    memcpy(ob, h->one_body, sizeof(double) * h->n1);
    memcpy(tb, h->two_body, sizeof(double) * h->n2);
}
OR_EXPORT int or_ham_orbs(const Ham *h, int *core, int *val) {
    memcpy(core, h->core_orbs, sizeof(int) * h->ncore);
    memcpy(val, h->valence_orbs, sizeof(int) * h->nval);
    return h->ncore;
}

typedef struct { u128 up, dn; } Config;

static inline Config cfg_from(const uint64_t *w) {
    Config c;
    c.up = ((u128)w[1] << 64) | w[0];
    c.dn = ((u128)w[3] << 64) | w[2];
    return c;
}
static inline void cfg_to(Config c, uint64_t *w) {
    w[0] = (uint64_t)c.up; w[1] = (uint64_t)(c.up >> 64);
    w[2] = (uint64_t)c.dn; w[3] = (uint64_t)(c.dn >> 64);
}

/* ham_diag (src/ham/mod.rs:92-124). */
static double ham_diag(const Ham *h, Config det) {
    double diag = h->nuc;
    for (u128 t = det.up; t; t &= t - 1) { int i = ctz128(t); diag += one_body(h, i, i); }
    for (u128 t = det.dn; t; t &= t - 1) { int i = ctz128(t); diag += one_body(h, i, i); }
    for (u128 t = det.up; t; t &= t - 1) {
        int i = ctz128(t);
        for (u128 u = det.dn; u; u &= u - 1) { int j = ctz128(u); diag += direct(h, i, j, i, j); }
    }
    /* bit_pairs (src/utils/bits.rs:31-52): (i, j) with i < j, i-major order */
    for (int s = 0; s < 2; s++) {
        u128 x = s == 0 ? det.up : det.dn;
        for (u128 t = x; t; t &= t - 1) {
            int i = ctz128(t);
            for (u128 u = t & (t - 1); u; u &= u - 1) { int j = ctz128(u); diag += dpe(h, i, j, i, j); }
        }
    }
    return diag;
}

/* ham_sing (src/ham/mod.rs:135-168). */
static double ham_sing(const Ham *h, Config d1, Config d2) {
    double out;
    u128 same1, opp1, a1, a2;
    if (d1.dn == d2.dn) { same1 = d1.up; opp1 = d1.dn; a1 = d1.up; a2 = d2.up; }
    else { same1 = d1.dn; opp1 = d1.up; a1 = d1.dn; a2 = d2.dn; }
    int i = ctz128(a1 & ~a2);
    int j = ctz128(a2 & ~a1);
    out = one_body(h, i, j);
    for (u128 t = same1; t; t &= t - 1) { int k = ctz128(t); out += dpe(h, i, k, j, k); }
    for (u128 t = opp1; t; t &= t - 1) { int k = ctz128(t); out += direct(h, i, k, j, k); }
    out *= (double)permute1(a1, a2);
    return out;
}

/* ham_doub (src/ham/mod.rs:179-233). */
static double ham_doub(const Ham *h, Config d1, Config d2) {
    if (d1.dn == d2.dn || d1.up == d2.up) {
        u128 x1 = d1.dn == d2.dn ? d1.up : d1.dn;
        u128 x2 = d1.dn == d2.dn ? d2.up : d2.dn;
        int ind[4] = {0, 0, 0, 0};
        int n = 0;
        for (u128 t = x1 & ~x2; t && n < 4; t &= t - 1) ind[n++] = ctz128(t);
        for (u128 t = x2 & ~x1; t && n < 4; t &= t - 1) ind[n++] = ctz128(t);
        return (double)permute2(x1, x2, ind) * dpe(h, ind[0], ind[1], ind[2], ind[3]);
    }
    int i1[2], i2[2];
    i1[0] = ctz128(d1.up & ~d2.up); i1[1] = ctz128(d2.up & ~d1.up);
    i2[0] = ctz128(d1.dn & ~d2.dn); i2[1] = ctz128(d2.dn & ~d1.dn);
    return (double)(permute1(d1.up, d2.up) * permute1(d1.dn, d2.dn)) * direct(h, i1[0], i2[0], i1[1], i2[1]);
}

/* ham_off_diag_no_excite (src/ham/mod.rs:256-303). */
static double ham_off_diag_no_excite(const Ham *h, Config d1, Config d2) {
    int same_up = d1.up == d2.up, same_dn = d1.dn == d2.dn;
    if (same_up && same_dn) return 0.0;
    if (!same_up && !same_dn) {
        if (popc128(d1.up & ~d2.up) > 1 || popc128(d1.dn & ~d2.dn) > 1) return 0.0;
        return ham_doub(h, d1, d2);
    }
    u128 x = same_up ? (d1.dn & ~d2.dn) : (d1.up & ~d2.up);
    int n = popc128(x);
    if (n > 2) return 0.0;
    return n == 1 ? ham_sing(h, d1, d2) : ham_doub(h, d1, d2);
}

OR_EXPORT void or_ham_diag_batch(const Ham *h, const uint64_t *dets, size_t n, double *out) {
    for (size_t i = 0; i < n; i++) out[i] = ham_diag(h, cfg_from(dets + 4 * i));
}
OR_EXPORT void or_ham_off_diag_batch(const Ham *h, const uint64_t *d1, const uint64_t *d2, size_t n, double *out) {
    for (size_t i = 0; i < n; i++) out[i] = ham_off_diag_no_excite(h, cfg_from(d1 + 4 * i), cfg_from(d2 + 4 * i));
}
OR_EXPORT int or_parity(uint64_t lo, uint64_t hi) { return parity128(((u128)hi << 64) | lo); }
OR_EXPORT int or_permute(uint64_t lo1, uint64_t hi1, uint64_t lo2, uint64_t hi2) {
    return permute1(((u128)hi1 << 64) | lo1, ((u128)hi2 << 64) | lo2);
}
OR_EXPORT size_t or_combine_4(int p, int q, int r, int s) { return combine_4(p, q, r, s); }

/* ------------------------------------------------------------------------- */
/* Hash map Config -> index (the reference's HashMap<Config, usize>).          */
/* ------------------------------------------------------------------------- */

typedef struct {
    size_t cap, n;
    Config *keys;
    int64_t *vals; /* -1 = empty */
} CfgMap;

static inline uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}
static inline uint64_t cfg_hash(Config c) {
    uint64_t h = mix64((uint64_t)c.up ^ 0x9e3779b97f4a7c15ULL);
    h = mix64(h ^ (uint64_t)(c.up >> 64));
    h = mix64(h ^ (uint64_t)c.dn);
    return mix64(h ^ (uint64_t)(c.dn >> 64));
}
static void map_init(CfgMap *m, size_t cap) {
    size_t c = 16;
    while (c < cap * 2) c <<= 1;
    m->cap = c; m->n = 0;
    m->keys = malloc(sizeof(Config) * c);
    m->vals = malloc(sizeof(int64_t) * c);
    for (size_t i = 0; i < c; i++) m->vals[i] = -1;
}
static void map_free(CfgMap *m) { free(m->keys); free(m->vals); m->keys = NULL; m->vals = NULL; m->cap = m->n = 0; }
static int64_t map_get(const CfgMap *m, Config k) {
    size_t mask = m->cap - 1, i = cfg_hash(k) & mask;
    while (m->vals[i] >= 0) {
        if (m->keys[i].up == k.up && m->keys[i].dn == k.dn) return m->vals[i];
        i = (i + 1) & mask;
    }
    return -1;
}
static void map_put(CfgMap *m, Config k, int64_t v);
static void map_grow(CfgMap *m) {
    CfgMap n2;
    map_init(&n2, m->cap);
    for (size_t i = 0; i < m->cap; i++) if (m->vals[i] >= 0) map_put(&n2, m->keys[i], m->vals[i]);
    map_free(m);
    *m = n2;
}
static void map_put(CfgMap *m, Config k, int64_t v) {
    if ((m->n + 1) * 2 > m->cap) map_grow(m);
    size_t mask = m->cap - 1, i = cfg_hash(k) & mask;
    while (m->vals[i] >= 0) {
        if (m->keys[i].up == k.up && m->keys[i].dn == k.dn) { m->vals[i] = v; return; }
        i = (i + 1) & mask;
    }
    m->keys[i] = k; m->vals[i] = v; m->n++;
}

/* ------------------------------------------------------------------------- */
/* wf/det.rs (Det + incremental diagonal) and wf/mod.rs (Wf)                   */
/* ------------------------------------------------------------------------- */

typedef struct {
    Config config;
    double coeff;
    double diag;
    int has_diag;
} Det;

typedef struct {
    size_t n, cap;
    Det *dets;
    CfgMap inds;
    double energy;
} Wf;

static void wf_init(Wf *w, size_t cap) {
    w->n = 0; w->cap = cap > 4 ? cap : 4;
    w->dets = malloc(sizeof(Det) * w->cap);
    map_init(&w->inds, w->cap);
    w->energy = 0.0;
}
static void wf_free(Wf *w) { free(w->dets); map_free(&w->inds); w->dets = NULL; w->n = w->cap = 0; }
static void wf_append(Wf *w, Det d) {
    if (w->n == w->cap) { w->cap *= 2; w->dets = realloc(w->dets, sizeof(Det) * w->cap); }
    map_put(&w->inds, d.config, (int64_t)w->n);
    w->dets[w->n++] = d;
}
/* Wf::push (src/wf/mod.rs:87-93). */
static void wf_push(Wf *w, Det d) { if (map_get(&w->inds, d.config) < 0) wf_append(w, d); }
/* Wf::push_and_spin_flipped (src/wf/mod.rs:99-116): the flipped det goes first. */
static void wf_push_and_spin_flipped(Wf *w, Det d) {
    if (d.config.up == d.config.dn) { wf_push(w, d); return; }
    Config f = {d.config.dn, d.config.up};
    if (map_get(&w->inds, f) < 0) {
        Det df = d;
        df.config = f;
        wf_append(w, df);
        wf_push(w, d);
    } else {
        wf_push(w, d);
    }
}

/* new_diag_opp (src/wf/det.rs:271-299); one_body helper (:303-307). */
static double new_diag_opp(const Ham *h, const Det *d, int p, int q, int r, int s) {
    double nd = d->diag + one_body(h, r, r) + one_body(h, s, s) - one_body(h, p, p) - one_body(h, q, q);
    nd += direct(h, r, s, r, s) - direct(h, p, q, p, q);
    for (u128 t = d->config.up; t; t &= t - 1) {
        int i = ctz128(t);
        if (i == p) continue;
        nd += dpe(h, i, r, i, r) - dpe(h, i, p, i, p);
        nd += direct(h, i, s, i, s) - direct(h, i, q, i, q);
    }
    for (u128 t = d->config.dn; t; t &= t - 1) {
        int i = ctz128(t);
        if (i == q) continue;
        nd += dpe(h, i, s, i, s) - dpe(h, i, q, i, q);
        nd += direct(h, i, r, i, r) - direct(h, i, p, i, p);
    }
    return nd;
}

/* new_diag_same (src/wf/det.rs:316-356) with helpers :360-378. */
static double new_diag_same(const Ham *h, const Det *d, int p, int q, int r, int s, int is_alpha) {
    double nd = d->diag + one_body(h, r, r) + one_body(h, s, s) - one_body(h, p, p) - one_body(h, q, q);
    nd += dpe(h, r, s, r, s) - dpe(h, p, q, p, q);
    u128 same = is_alpha ? d->config.up : d->config.dn;
    u128 opp = is_alpha ? d->config.dn : d->config.up;
    for (u128 t = same; t; t &= t - 1) {
        int i = ctz128(t);
        if (i == p || i == q) continue;
        nd += dpe(h, i, r, i, r) + dpe(h, i, s, i, s) - dpe(h, i, p, i, p) - dpe(h, i, q, i, q);
    }
    for (u128 t = opp; t; t &= t - 1) {
        int i = ctz128(t);
        nd += direct(h, i, r, i, r) + direct(h, i, s, i, s) - direct(h, i, p, i, p) - direct(h, i, q, i, q);
    }
    return nd;
}

/* new_diag_sing (src/wf/det.rs:387-420). */
static double new_diag_sing(const Ham *h, const Det *d, int p, int r, int is_alpha) {
    double nd = d->diag + one_body(h, r, r) - one_body(h, p, p);
    u128 same = is_alpha ? d->config.up : d->config.dn;
    u128 opp = is_alpha ? d->config.dn : d->config.up;
    for (u128 t = same; t; t &= t - 1) {
        int i = ctz128(t);
        if (i == p) continue;
        nd += dpe(h, i, r, i, r) - dpe(h, i, p, i, p);
    }
    for (u128 t = opp; t; t &= t - 1) {
        int i = ctz128(t);
        nd += direct(h, i, r, i, r) - direct(h, i, p, i, p);
    }
    return nd;
}

/* ------------------------------------------------------------------------- */
/* excite/init.rs: ExciteGenerator                                            */
/* ------------------------------------------------------------------------- */

typedef struct { int r, s; double abs_h; } Stored;
typedef struct { Stored *v; int n; } StoredList;

typedef struct {
    int norb;
    double max_opp_doub, max_same_doub, max_sing;
    StoredList *opp;  /* [p*norb+q] */
    StoredList *same; /* [p*norb+q], p<q */
    StoredList *sing; /* [p] */
    u128 valence;
} ExciteGen;

/* Stable sort by abs_h descending (Rust's sort_by is stable; init.rs:126,170,253). */
static void stable_sort_desc(Stored *v, int n) {
    if (n < 2) return;
    Stored *tmp = malloc(sizeof(Stored) * n);
    for (int w = 1; w < n; w *= 2) {
        for (int lo = 0; lo < n; lo += 2 * w) {
            int mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            int a = lo, b = mid, k = lo;
            while (a < mid && b < hi) {
                /* take from right only if strictly greater: keeps the stable order */
                if (v[b].abs_h > v[a].abs_h) tmp[k++] = v[b++];
                else tmp[k++] = v[a++];
            }
            while (a < mid) tmp[k++] = v[a++];
            while (b < hi) tmp[k++] = v[b++];
        }
        memcpy(v, tmp, sizeof(Stored) * n);
    }
    free(tmp);
}

static void sort_doubles_asc(double *v, int n) { /* v_same/v_opp sort (init.rs:214-215) */
    for (int i = 1; i < n; i++) {
        double k = v[i];
        int j = i - 1;
        while (j >= 0 && v[j] > k) { v[j + 1] = v[j]; j--; }
        v[j + 1] = k;
    }
}

/* init_excite_generator (src/excite/init.rs:81-280). */
static ExciteGen *excite_gen_new(const Ham *h, int n_up, int n_dn) {
    int n = h->norb;
    ExciteGen *eg = calloc(1, sizeof(ExciteGen));
    eg->norb = n;
    eg->opp = calloc((size_t)n * n, sizeof(StoredList));
    eg->same = calloc((size_t)n * n, sizeof(StoredList));
    eg->sing = calloc((size_t)n, sizeof(StoredList));
    for (int a = 0; a < h->nval; a++) eg->valence |= bit128(h->valence_orbs[a]);
    const int *vo = h->valence_orbs;
    int nv = h->nval;
    for (int a = 0; a < nv; a++) for (int b = 0; b < nv; b++) {
        int p = vo[a], q = vo[b];
        Stored *v = malloc(sizeof(Stored) * (size_t)(nv * nv + 1));
        int m = 0;
        for (int c = 0; c < nv; c++) {
            int r = vo[c];
            if (p == r) continue;
            for (int d = 0; d < nv; d++) {
                int s = vo[d];
                if (q == s) continue;
                double hv = fabs(direct(h, p, q, r, s));
                if (hv > eg->max_opp_doub) eg->max_opp_doub = hv;
                v[m].r = r; v[m].s = s; v[m].abs_h = hv; m++;
            }
        }
        stable_sort_desc(v, m);
        eg->opp[p * n + q].v = v; eg->opp[p * n + q].n = m;
    }
    for (int a = 0; a < nv; a++) for (int b = 0; b < nv; b++) {
        int p = vo[a], q = vo[b];
        if (p >= q) continue;
        Stored *v = malloc(sizeof(Stored) * (size_t)(nv * nv + 1));
        int m = 0;
        for (int c = 0; c < nv; c++) {
            int r = vo[c];
            if (p == r || q == r) continue;
            for (int d = 0; d < nv; d++) {
                int s = vo[d];
                if (r >= s) continue;
                if (p == s || q == s) continue;
                double hv = fabs(dpe(h, p, q, r, s));
                if (hv > eg->max_same_doub) eg->max_same_doub = hv;
                v[m].r = r; v[m].s = s; v[m].abs_h = hv; m++;
            }
        }
        stable_sort_desc(v, m);
        eg->same[p * n + q].v = v; eg->same[p * n + q].n = m;
    }
    double *vs = malloc(sizeof(double) * (n + 1)), *vp = malloc(sizeof(double) * (n + 1));
    for (int a = 0; a < nv; a++) {
        int p = vo[a];
        Stored *v = malloc(sizeof(Stored) * (size_t)(nv + 1));
        int m = 0;
        for (int c = 0; c < nv; c++) {
            int r = vo[c];
            if (p == r) continue;
            int L = 0;
            for (int q = 0; q < n; q++) {
                if (p == q || q == r) continue;
                vs[L] = dpe(h, p, q, r, q);
                vp[L] = direct(h, p, q, r, q);
                L++;
            }
            sort_doubles_asc(vs, L);
            sort_doubles_asc(vp, L);
            /* Iterator::sum over f64 folds left from zero (init.rs:216-225) */
            double s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
            for (int k = 0; k < n_up - 1; k++) s1 += vs[k];
            for (int k = 0; k < n_dn; k++) s2 += vp[k];
            for (int k = L - (n_up - 1); k < L; k++) s3 += vs[k];
            for (int k = L - n_dn; k < L; k++) s4 += vp[k];
            double max1 = one_body(h, p, r) + s1 + s2;
            double max2 = one_body(h, p, r) + s3 + s4;
            v[m].r = r; v[m].s = -1;
            v[m].abs_h = fabs(max1) > fabs(max2) ? fabs(max1) : fabs(max2);
            m++;
        }
        stable_sort_desc(v, m);
        eg->sing[p].v = v; eg->sing[p].n = m;
    }
    free(vs); free(vp);
    double mx = 0.0;
    for (int a = 0; a < nv; a++) {
        int p = vo[a];
        double x = eg->sing[p].n ? eg->sing[p].v[0].abs_h : 0.0;
        mx = fmax(mx, x); /* fold(0., f64::max) (init.rs:268) */
    }
    eg->max_sing = mx;
    return eg;
}

static void excite_gen_free(ExciteGen *eg) {
    if (!eg) return;
    int n = eg->norb;
    for (int i = 0; i < n * n; i++) { free(eg->opp[i].v); free(eg->same[i].v); }
    for (int i = 0; i < n; i++) free(eg->sing[i].v);
    free(eg->opp); free(eg->same); free(eg->sing); free(eg);
}

/* ------------------------------------------------------------------------- */
/* var/sparse.rs: SparseMatUpperTri                                           */
/* ------------------------------------------------------------------------- */

typedef struct { int64_t col; double val; } Entry;
typedef struct { Entry *e; size_t n, cap; } Row;

typedef struct {
    size_t n;
    double *diag;
    size_t *nnz; /* per-row count after the last dedup (sparse.rs:31-33) */
    Row *rows;
    int err;     /* set where the reference would panic (missing spin-flipped det) */
} Sparse;

static void row_push(Row *r, int64_t col, double val) {
    if (r->n == r->cap) { r->cap = r->cap ? 2 * r->cap : 8; r->e = realloc(r->e, sizeof(Entry) * r->cap); }
    r->e[r->n].col = col; r->e[r->n].val = val; r->n++;
}

OR_EXPORT Sparse *or_sparse_new(void) { return calloc(1, sizeof(Sparse)); }
OR_EXPORT void or_sparse_free(Sparse *s) {
    if (!s) return;
    for (size_t i = 0; i < s->n; i++) free(s->rows[i].e);
    free(s->rows); free(s->diag); free(s->nnz); free(s);
}

/* new_sparse_ham / expand_sparse_ham_rows (src/wf/mod.rs:1646-1683). */
static void sparse_expand(Sparse *s, size_t n, const double *diag) {
    if (n < s->n) n = s->n;
    s->diag = realloc(s->diag, sizeof(double) * (n ? n : 1));
    s->nnz = realloc(s->nnz, sizeof(size_t) * (n ? n : 1));
    s->rows = realloc(s->rows, sizeof(Row) * (n ? n : 1));
    for (size_t i = s->n; i < n; i++) {
        s->diag[i] = diag[i];
        s->nnz[i] = 0;
        s->rows[i].e = NULL; s->rows[i].n = s->rows[i].cap = 0;
    }
    s->n = n;
}

/* add_off_diag_elem (src/var/off_diag.rs:45-53). */
static void add_off_diag_elem(Sparse *s, size_t i, size_t j, double elem) {
    if (i < j) row_push(&s->rows[i], (int64_t)j, elem);
    else row_push(&s->rows[j], (int64_t)i, elem);
}

/* add_el with elem == None (src/var/off_diag.rs:26-39). */
static void add_el(Sparse *s, const Ham *h, const Config *cf, size_t i, size_t j) {
    if (i == j) return;
    double e = ham_off_diag_no_excite(h, cf[i], cf[j]);
    if (e != 0.0) add_off_diag_elem(s, i, j, e);
}

/* Stable sort of a row slice by column (Rust slice::sort_by_key is stable). */
static void stable_sort_cols(Entry *v, size_t n) {
    if (n < 2) return;
    Entry *tmp = malloc(sizeof(Entry) * n);
    for (size_t w = 1; w < n; w *= 2) {
        for (size_t lo = 0; lo < n; lo += 2 * w) {
            size_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            size_t a = lo, b = mid, k = lo;
            while (a < mid && b < hi) {
                if (v[b].col < v[a].col) tmp[k++] = v[b++];
                else tmp[k++] = v[a++];
            }
            while (a < mid) tmp[k++] = v[a++];
            while (b < hi) tmp[k++] = v[b++];
        }
        memcpy(v, tmp, sizeof(Entry) * n);
    }
    free(tmp);
}

/* sort_remove_duplicates (src/var/sparse.rs:44-56): sort the rows' new tails by
 * column, then drop consecutive duplicates keeping the first. */
static size_t sparse_sort_remove_duplicates(Sparse *s) {
    size_t total = 0;
    for (size_t i = 0; i < s->n; i++) {
        Row *r = &s->rows[i];
        size_t start = s->nnz[i] < r->n ? s->nnz[i] : r->n;
        stable_sort_cols(r->e + start, r->n - start);
        size_t w = 0;
        for (size_t k = 0; k < r->n; k++) {
            if (w > 0 && r->e[w - 1].col == r->e[k].col) continue;
            r->e[w++] = r->e[k];
        }
        r->n = w;
        s->nnz[i] = w;
        total += w;
    }
    return total;
}

OR_EXPORT size_t or_sparse_nnz(const Sparse *s) {
    size_t t = 0;
    for (size_t i = 0; i < s->n; i++) t += s->rows[i].n;
    return t;
}
OR_EXPORT size_t or_sparse_n(const Sparse *s) { return s->n; }

/* Export the upper triangle as CSR with each row sorted by column (the
 * reference keeps each insertion batch sorted; the set is what parity checks). */
OR_EXPORT void or_sparse_export(const Sparse *s, int64_t *rowptr, int64_t *cols, double *vals, double *diag) {
    size_t k = 0;
    rowptr[0] = 0;
    for (size_t i = 0; i < s->n; i++) {
        Row *r = &s->rows[i];
        Entry *tmp = malloc(sizeof(Entry) * (r->n ? r->n : 1));
        memcpy(tmp, r->e, sizeof(Entry) * r->n);
        stable_sort_cols(tmp, r->n);
        for (size_t j = 0; j < r->n; j++) { cols[k] = tmp[j].col; vals[k] = tmp[j].val; k++; }
        free(tmp);
        rowptr[i + 1] = (int64_t)k;
        if (diag) diag[i] = s->diag[i];
    }
}

/* matrix_vector_prod (src/var/sparse.rs:64-78): symmetric scatter. */
static void sparse_mv(const Sparse *s, const double *x, double *y) {
    for (size_t i = 0; i < s->n; i++) y[i] = 0.0;
    for (size_t i = 0; i < s->n; i++) {
        y[i] += s->diag[i] * x[i];
        const Row *r = &s->rows[i];
        for (size_t k = 0; k < r->n; k++) {
            y[i] += r->e[k].val * x[r->e[k].col];
            y[r->e[k].col] += r->e[k].val * x[i];
        }
    }
}
OR_EXPORT void or_sparse_mv(const Sparse *s, const double *x, double *y) { sparse_mv(s, x, y); }

/* ------------------------------------------------------------------------- */
/* var/fast_ham.rs: lookup-based H construction (n > 100)                     */
/* ------------------------------------------------------------------------- */

typedef struct { u128 key; int64_t a; } KeyIdx;

static int cmp_keyidx(const void *x, const void *y) {
    const KeyIdx *a = x, *b = y;
    if (a->key < b->key) return -1;
    if (a->key > b->key) return 1;
    if (a->a < b->a) return -1;
    return a->a > b->a;
}

/* Groups of equal 128-bit strings: `order` lists det indices sorted by
 * (string, det index); `start[g]..start[g+1]` is group g; `gid[det]` its group. */
typedef struct {
    size_t ng;
    u128 *str;      /* unique strings, ascending */
    size_t *start;  /* ng+1 */
    int64_t *order; /* N */
    size_t *gid;    /* N */
} Groups;

static void groups_build(Groups *g, const Config *cf, size_t N, int use_dn) {
    KeyIdx *ki = malloc(sizeof(KeyIdx) * (N ? N : 1));
    for (size_t i = 0; i < N; i++) { ki[i].key = use_dn ? cf[i].dn : cf[i].up; ki[i].a = (int64_t)i; }
    qsort(ki, N, sizeof(KeyIdx), cmp_keyidx);
    g->order = malloc(sizeof(int64_t) * (N ? N : 1));
    g->gid = malloc(sizeof(size_t) * (N ? N : 1));
    g->str = malloc(sizeof(u128) * (N ? N : 1));
    g->start = malloc(sizeof(size_t) * (N + 1));
    g->ng = 0;
    for (size_t i = 0; i < N; i++) {
        if (i == 0 || ki[i].key != ki[i - 1].key) { g->str[g->ng] = ki[i].key; g->start[g->ng] = i; g->ng++; }
        g->order[i] = ki[i].a;
        g->gid[ki[i].a] = g->ng - 1;
    }
    g->start[g->ng] = N;
    free(ki);
}
static void groups_free(Groups *g) { free(g->order); free(g->gid); free(g->str); free(g->start); }

static size_t groups_find(const Groups *g, u128 s) { /* binary search; ng if absent */
    size_t lo = 0, hi = g->ng;
    while (lo < hi) {
        size_t mid = (lo + hi) / 2;
        if (g->str[mid] < s) lo = mid + 1; else hi = mid;
    }
    return (lo < g->ng && g->str[lo] == s) ? lo : g->ng;
}

/* Single-excitation partners among unique strings through "remove one
 * electron" keys (build_alpha_singles / build_beta_singles, fast_ham.rs:105-173). */
typedef struct { size_t *start; size_t *part; } Partners;

static void partners_build(Partners *P, const Groups *g) {
    size_t ne = 0;
    for (size_t i = 0; i < g->ng; i++) ne += popc128(g->str[i]);
    KeyIdx *ki = malloc(sizeof(KeyIdx) * (ne ? ne : 1));
    size_t k = 0;
    for (size_t i = 0; i < g->ng; i++)
        for (u128 t = g->str[i]; t; t &= t - 1) { ki[k].key = g->str[i] & ~bit128(ctz128(t)); ki[k].a = (int64_t)i; k++; }
    qsort(ki, ne, sizeof(KeyIdx), cmp_keyidx);
    size_t *cnt = calloc(g->ng + 1, sizeof(size_t));
    for (size_t a = 0; a < ne;) {
        size_t b = a;
        while (b < ne && ki[b].key == ki[a].key) b++;
        for (size_t x = a; x < b; x++) cnt[ki[x].a] += (b - a - 1);
        a = b;
    }
    P->start = malloc(sizeof(size_t) * (g->ng + 1));
    P->start[0] = 0;
    for (size_t i = 0; i < g->ng; i++) P->start[i + 1] = P->start[i] + cnt[i];
    P->part = malloc(sizeof(size_t) * (P->start[g->ng] ? P->start[g->ng] : 1));
    size_t *fill = calloc(g->ng + 1, sizeof(size_t));
    for (size_t a = 0; a < ne;) {
        size_t b = a;
        while (b < ne && ki[b].key == ki[a].key) b++;
        for (size_t x = a; x < b; x++)
            for (size_t y = a; y < b; y++)
                if (x != y) P->part[P->start[ki[x].a] + fill[ki[x].a]++] = (size_t)ki[y].a;
        a = b;
    }
    free(cnt); free(fill); free(ki);
}
static void partners_free(Partners *P) { free(P->start); free(P->part); }

/* are_strings_double_connected (fast_ham.rs:321-336). */
static inline int double_connected(u128 a, u128 b) {
    return popc128(a ^ b) == 4 && popc128(a) == popc128(b);
}

/* find_single_excitations (fast_ham.rs:473-517).  `grouped` replaces the
 * O(N_new * N) scan with scans of the same-alpha and same-beta groups; both
 * visit the same (i, j) pairs and apply the same |elem| > 1e-12 rule. */
static void fast_singles(Sparse *s, const Ham *h, const Config *cf, size_t N, size_t nsh,
                         const Groups *ga, const Groups *gb, int grouped) {
    for (size_t src = nsh; src < N; src++) {
        Config sc = cf[src];
        if (!grouped) {
            for (size_t tgt = 0; tgt < N; tgt++) {
                if (tgt == src) continue;
                Config tc = cf[tgt];
                int ud = popc128(sc.up ^ tc.up), dd = popc128(sc.dn ^ tc.dn);
                if (!((ud == 2 && dd == 0) || (ud == 0 && dd == 2))) continue;
                if (src < tgt) {
                    double e = ham_off_diag_no_excite(h, sc, tc);
                    if (fabs(e) > 1e-12) row_push(&s->rows[src], (int64_t)tgt, e);
                } else {
                    double e = ham_off_diag_no_excite(h, tc, sc);
                    if (fabs(e) > 1e-12) row_push(&s->rows[tgt], (int64_t)src, e);
                }
            }
        } else {
            for (int pass = 0; pass < 2; pass++) {
                const Groups *g = pass == 0 ? ga : gb;
                size_t gi = g->gid[src];
                for (size_t k = g->start[gi]; k < g->start[gi + 1]; k++) {
                    size_t tgt = (size_t)g->order[k];
                    if (tgt == src) continue;
                    Config tc = cf[tgt];
                    int ud = popc128(sc.up ^ tc.up), dd = popc128(sc.dn ^ tc.dn);
                    if (!((ud == 2 && dd == 0) || (ud == 0 && dd == 2))) continue;
                    if (src < tgt) {
                        double e = ham_off_diag_no_excite(h, sc, tc);
                        if (fabs(e) > 1e-12) row_push(&s->rows[src], (int64_t)tgt, e);
                    } else {
                        double e = ham_off_diag_no_excite(h, tc, sc);
                        if (fabs(e) > 1e-12) row_push(&s->rows[tgt], (int64_t)src, e);
                    }
                }
            }
        }
    }
}

/* gen_sparse_ham_fast_lookup (fast_ham.rs:527-575) with
 * find_all_connections_original_pattern (:341-366). */
static void gen_sparse_ham_fast_lookup(Sparse *s, const Ham *h, const Config *cf, size_t N, size_t nsh, int grouped_singles) {
    Groups ga, gb;
    groups_build(&ga, cf, N, 0);
    groups_build(&gb, cf, N, 1);
    Partners pa, pb;
    partners_build(&pa, &ga);
    partners_build(&pb, &gb);
    /* singles */
    fast_singles(s, h, cf, N, nsh, &ga, &gb, grouped_singles);
    /* new alpha strings */
    char *is_new = calloc(ga.ng + 1, 1);
    for (size_t d = nsh; d < N; d++) is_new[ga.gid[d]] = 1;
    /* opposite spin (find_opposite_spin_for_alpha_string, :369-407) */
    for (size_t a = 0; a < ga.ng; a++) {
        if (!is_new[a]) continue;
        for (size_t pk = pa.start[a]; pk < pa.start[a + 1]; pk++) {
            size_t a2 = pa.part[pk];
            for (size_t x = ga.start[a]; x < ga.start[a + 1]; x++) {
                size_t sd = (size_t)ga.order[x];
                u128 sb = cf[sd].dn;
                for (size_t y = ga.start[a2]; y < ga.start[a2 + 1]; y++) {
                    size_t cd = (size_t)ga.order[y];
                    u128 cb = cf[cd].dn;
                    /* are_beta_strings_single_connected (:310-316) */
                    if (sb == cb || popc128(sb ^ cb) != 2) continue;
                    if (sd >= nsh || cd >= nsh) add_el(s, h, cf, sd, cd);
                }
            }
        }
    }
    /* same spin (find_same_spin_for_alpha_string, :410-470) */
    for (size_t a = 0; a < ga.ng; a++) {
        int has_new = 0;
        for (size_t x = ga.start[a]; x < ga.start[a + 1]; x++) if ((size_t)ga.order[x] >= nsh) { has_new = 1; break; }
        if (!has_new) continue;
        for (size_t x = ga.start[a]; x < ga.start[a + 1]; x++) {
            size_t d1 = (size_t)ga.order[x];
            for (size_t y = x + 1; y < ga.start[a + 1]; y++) {
                size_t d2 = (size_t)ga.order[y];
                if (d1 >= nsh || d2 >= nsh)
                    if (double_connected(cf[d1].dn, cf[d2].dn)) add_el(s, h, cf, d1, d2);
            }
        }
        /* alpha doubles: other alpha strings double-connected, same beta (:444-467);
         * the beta-grouped scan visits exactly the dets with that beta string. */
        for (size_t x = ga.start[a]; x < ga.start[a + 1]; x++) {
            size_t nd = (size_t)ga.order[x];
            if (nd < nsh) continue;
            size_t gbi = gb.gid[nd];
            for (size_t y = gb.start[gbi]; y < gb.start[gbi + 1]; y++) {
                size_t od = (size_t)gb.order[y];
                if (cf[od].up != cf[nd].up && double_connected(cf[nd].up, cf[od].up)) add_el(s, h, cf, nd, od);
            }
        }
    }
    free(is_new);
    partners_free(&pa); partners_free(&pb);
    groups_free(&ga); groups_free(&gb);
}

/* ------------------------------------------------------------------------- */
/* var/ham_gen.rs: legacy construction (n <= 100), opp_algo = 1, same_algo = 1 */
/* ------------------------------------------------------------------------- */

/* add_el_and_spin_flipped (src/var/off_diag.rs:73-102). */
static void add_el_and_spin_flipped(Sparse *s, const Ham *h, const Config *cf, const CfgMap *inds, size_t i, size_t j) {
    if (i == j) return;
    double e = ham_off_diag_no_excite(h, cf[i], cf[j]);
    if (e == 0.0) return;
    add_off_diag_elem(s, i, j, e);
    Config fi = {cf[i].dn, cf[i].up}, fj = {cf[j].dn, cf[j].up};
    int64_t ii = map_get(inds, fi), jj = map_get(inds, fj);
    if (ii < 0 || jj < 0) { s->err = 1; return; } /* the reference panics here (off_diag.rs:88-99) */
    add_off_diag_elem(s, (size_t)ii, (size_t)jj, e);
}

/* gen_sparse_ham_fast with opp_algo 1 and same_algo 1 (src/var/ham_gen.rs:60-292,
 * :406-447, :621-637).  The hash-map iteration orders there only change the
 * order of insertion into rows, which the final sort and dedup remove. */
static void gen_sparse_ham_legacy(Sparse *s, const Ham *h, const Config *cf, size_t N, size_t nsh) {
    CfgMap inds;
    map_init(&inds, N);
    for (size_t i = 0; i < N; i++) map_put(&inds, cf[i], (int64_t)i);
    Groups ga;
    groups_build(&ga, cf, N, 0);
    Partners pa;
    partners_build(&pa, &ga);
    /* new unique up strings */
    char *is_new = calloc(ga.ng + 1, 1);
    for (size_t d = nsh; d < N; d++) is_new[ga.gid[d]] = 1;
    /* opposite spin, opp_algo 1 (:406-447).  up_singles[u] = unique ups single-connected
     * to a new unique up u; dn_candidates maps a dn string to the new dets (with up u)
     * whose dn is single-connected to it, looked up through up_singles keyed by dn. */
    for (size_t a = 0; a < ga.ng; a++) {
        if (!is_new[a]) continue;
        if (pa.start[a + 1] == pa.start[a]) continue; /* up_singles.get(&u) == None */
        for (size_t pk = pa.start[a]; pk < pa.start[a + 1]; pk++) {
            size_t a2 = pa.part[pk];
            for (size_t y = ga.start[a2]; y < ga.start[a2 + 1]; y++) {
                size_t ind1 = (size_t)ga.order[y];
                u128 dn_all = cf[ind1].dn;
                for (size_t x = ga.start[a]; x < ga.start[a + 1]; x++) {
                    size_t nd = (size_t)ga.order[x];
                    if (nd < nsh) continue; /* only new dets of this up string */
                    u128 dn_new = cf[nd].dn;
                    /* dn_candidates[dn_all] contains nd iff dn_all is in up_singles[dn_new]:
                     * dn_new must be a new unique up string and dn_all a unique up string
                     * single-connected to it. */
                    size_t gd = groups_find(&ga, dn_new);
                    if (gd == ga.ng || !is_new[gd]) continue;
                    if (groups_find(&ga, dn_all) == ga.ng) continue;
                    if (dn_all == dn_new || popc128(dn_all ^ dn_new) != 2) continue;
                    add_el(s, h, cf, ind1, nd);
                }
            }
        }
    }
    /* same spin, same_algo 1 (:621-637) */
    for (size_t a = 0; a < ga.ng; a++) {
        for (size_t x = ga.start[a]; x < ga.start[a + 1]; x++) {
            size_t i1 = (size_t)ga.order[x];
            for (size_t y = ga.start[a]; y < ga.start[a + 1]; y++) {
                size_t i2 = (size_t)ga.order[y];
                if (i2 < nsh) continue;
                if (i2 > i1) add_el_and_spin_flipped(s, h, cf, &inds, i1, i2);
            }
        }
    }
    free(is_new);
    partners_free(&pa);
    groups_free(&ga);
    map_free(&inds);
}

/* Build or extend the stored upper triangle for dets[0..N) given that rows for
 * dets[0..nsh) were built before.  builder: 0 = the reference's switch at n > 100
 * (src/var/davidson.rs:55-61), 1 = fast lookup, 2 = legacy. */
static void sparse_build(Sparse *s, const Ham *h, const Config *cf, size_t N, size_t nsh, const double *diag,
                         int builder, int grouped_singles) {
    sparse_expand(s, N, diag);
    int use_fast = builder == 1 || (builder == 0 && N > 100);
    if (use_fast) gen_sparse_ham_fast_lookup(s, h, cf, N, nsh, grouped_singles);
    else gen_sparse_ham_legacy(s, h, cf, N, nsh);
    sparse_sort_remove_duplicates(s);
}

OR_EXPORT int or_sparse_build(Sparse *s, const Ham *h, const uint64_t *dets, size_t N, size_t nsh,
                              const double *diag, int builder, int grouped_singles) {
    if (nsh > N || (s->n && s->n != nsh)) return -1;
    Config *cf = malloc(sizeof(Config) * (N ? N : 1));
    for (size_t i = 0; i < N; i++) cf[i] = cfg_from(dets + 4 * i);
    sparse_build(s, h, cf, N, nsh, diag, builder, grouped_singles);
    free(cf);
    return s->err ? -2 : 0;
}

/* ------------------------------------------------------------------------- */
/* Dense symmetric eigensolver for the projected problem.                      */
/* The reference calls nalgebra 0.26.2 SymmetricEigen (Householder + implicit   */
/* QR).  Here: the cyclic Jacobi method (Rutishauser 1966; Golub & Van Loan,    */
/* "Matrix Computations", section 8.5) which gives the same eigenpairs to       */
/* rounding, then sort_eigenpairs (eigenvalues/utils.rs:48-79).                 */
/* ------------------------------------------------------------------------- */

static void jacobi_eig(int n, const double *A_in, double *w, double *V) {
    double *A = malloc(sizeof(double) * n * n);
    memcpy(A, A_in, sizeof(double) * n * n);
    for (int i = 0; i < n * n; i++) V[i] = 0.0;
    for (int i = 0; i < n; i++) V[i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) {
            tot += A[i * n + j] * A[i * n + j];
            if (i != j) off += A[i * n + j] * A[i * n + j];
        }
        if (off <= 1e-30 * (tot > 0 ? tot : 1.0) || off == 0.0) break;
        for (int p = 0; p < n - 1; p++) for (int q = p + 1; q < n; q++) {
            double apq = A[p * n + q];
            if (apq == 0.0) continue;
            double app = A[p * n + p], aqq = A[q * n + q];
            double theta = (aqq - app) / (2.0 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
            for (int k = 0; k < n; k++) {
                double akp = A[k * n + p], akq = A[k * n + q];
                A[k * n + p] = c * akp - sn * akq;
                A[k * n + q] = sn * akp + c * akq;
            }
            for (int k = 0; k < n; k++) {
                double apk = A[p * n + k], aqk = A[q * n + k];
                A[p * n + k] = c * apk - sn * aqk;
                A[q * n + k] = sn * apk + c * aqk;
            }
            for (int k = 0; k < n; k++) { /* V column-major by eigenvector: V[k*n + col] row k */
                double vkp = V[k * n + p], vkq = V[k * n + q];
                V[k * n + p] = c * vkp - sn * vkq;
                V[k * n + q] = sn * vkp + c * vkq;
            }
        }
    }
    for (int i = 0; i < n; i++) w[i] = A[i * n + i];
    free(A);
}

/* SymmetricEigen + sort_eigenpairs(ascending): returns eigenvalues ascending and
 * Y (row-major n x n: Y[r*n + c] = component r of eigenvector c). */
static void sym_eig_sorted(int n, const double *A, double *w, double *Y) {
    double *wt = malloc(sizeof(double) * n), *Vt = malloc(sizeof(double) * n * n);
    int *idx = malloc(sizeof(int) * n);
    jacobi_eig(n, A, wt, Vt);
    for (int i = 0; i < n; i++) idx[i] = i;
    for (int i = 1; i < n; i++) {
        int k = idx[i], j = i - 1;
        while (j >= 0 && wt[idx[j]] > wt[k]) { idx[j + 1] = idx[j]; j--; }
        idx[j + 1] = k;
    }
    for (int c = 0; c < n; c++) {
        w[c] = wt[idx[c]];
        for (int r = 0; r < n; r++) Y[r * n + c] = Vt[r * n + idx[c]];
    }
    free(wt); free(Vt); free(idx);
}

OR_EXPORT void or_sym_eig(int n, const double *A, double *w, double *Y) { sym_eig_sorted(n, A, w, Y); }

/* ------------------------------------------------------------------------- */
/* var/eigenvalues: MGS + Davidson                                             */
/* ------------------------------------------------------------------------- */

/* MGS::orthonormalize (modified_gram_schmidt.rs:22-36); B is column-major N x ncol. */
static int mgs_orthonormalize(double *B, size_t N, int start, int end) {
    for (int i = start; i < end; i++) {
        double *vi = B + (size_t)i * N;
        for (int j = 0; j < i; j++) {
            const double *vj = B + (size_t)j * N;
            double d12 = 0.0, d11 = 0.0;
            for (size_t k = 0; k < N; k++) { d12 += vj[k] * vi[k]; d11 += vj[k] * vj[k]; }
            double mag = d12 / d11;
            for (size_t k = 0; k < N; k++) vi[k] -= vj[k] * mag;
        }
        double nrm = 0.0;
        for (size_t k = 0; k < N; k++) nrm += vi[k] * vi[k];
        nrm = sqrt(nrm);
        if (i == end - 1 && nrm < 1e-9) return 0;
        for (size_t k = 0; k < N; k++) vi[k] /= nrm;
    }
    return 1;
}
OR_EXPORT int or_mgs(double *B, size_t N, int start, int end) { return mgs_orthonormalize(B, N, start, end); }

typedef struct {
    int iters;    /* outer iterations executed */
    int n_sigma;  /* matrix_vector_prod calls */
    int converged;
    int reason;   /* 0 residual+energy, 1 small correction, 2 redundant vector, 3 n<=2, -1 failed */
} DavStats;

/* A matrix operator: y = H x for each column. */
typedef void (*MatVec)(const void *ctx, const double *x, double *y);

/* Davidson::new (algorithms/davidson.rs:106-277) with DPR correction (:391-408),
 * nvalues roots, SpectrumTarget::Lowest.  init: N x ninit column-major or NULL.
 * Returns 0 on convergence, 1 when max_iters passed without it (DavidsonError). */
static int davidson(const void *ctx, MatVec mv, const double *dg, size_t N, int nvalues, const double *init,
                    double tol, double etol, int max_iters, double *evals, double *evecs, DavStats *st) {
    int init_dim = init ? 1 : 2;
    int mss = (size_t)(nvalues + 10) < N ? nvalues + 10 : (int)N; /* Config::new (:62-66) */
    int update_dim = nvalues, reset_dim = nvalues;
    double *basis = calloc((size_t)mss * N, sizeof(double));
    for (int c = 0; c < mss && (size_t)c < N; c++) basis[(size_t)c * N + c] = 1.0; /* identity */
    if (init) { /* generate_subspace (:318-338) */
        memcpy(basis + (size_t)(init_dim - 1) * N, init, sizeof(double) * N);
        if (init_dim > 1) mgs_orthonormalize(basis, N, init_dim - 1, init_dim);
    }
    int dim_sub = init_dim;
    if (dim_sub > mss) dim_sub = mss;
    double *HV = calloc((size_t)(mss + 1) * N, sizeof(double));
    for (int c = 0; c < dim_sub; c++) mv(ctx, basis + (size_t)c * N, HV + (size_t)c * N);
    st->n_sigma = dim_sub;
    int K = mss + nvalues;
    double *P = calloc((size_t)K * K, sizeof(double)); /* projected, row-major dim_sub x dim_sub */
    for (int i = 0; i < dim_sub; i++) for (int j = 0; j < dim_sub; j++) {
        double s = 0.0;
        const double *a = basis + (size_t)i * N, *b = HV + (size_t)j * N;
        for (size_t k = 0; k < N; k++) s += a[k] * b[k];
        P[i * dim_sub + j] = s;
    }
    double *last = calloc(nvalues, sizeof(double));
    double *w = malloc(sizeof(double) * K), *Y = malloc(sizeof(double) * K * K);
    double *ritz = malloc(sizeof(double) * (size_t)K * N), *res = malloc(sizeof(double) * (size_t)K * N);
    double *corr = malloc(sizeof(double) * (size_t)nvalues * N);
    int result = 1;
    st->converged = 0; st->reason = -1;
    int it;
    for (it = 0; it < max_iters; it++) {
        sym_eig_sorted(dim_sub, P, w, Y);
        /* ritz = V[:, :dim_sub] * Y ; residues = HV * Y - ritz * Lambda (:165-166, :301-315) */
        for (int c = 0; c < dim_sub; c++) {
            double *rz = ritz + (size_t)c * N, *rs = res + (size_t)c * N;
            for (size_t k = 0; k < N; k++) { rz[k] = 0.0; rs[k] = 0.0; }
            for (int j = 0; j < dim_sub; j++) {
                double y = Y[j * dim_sub + c];
                const double *vj = basis + (size_t)j * N, *hj = HV + (size_t)j * N;
                for (size_t k = 0; k < N; k++) { rz[k] += vj[k] * y; rs[k] += hj[k] * y; }
            }
            for (size_t k = 0; k < N; k++) rs[k] -= rz[k] * w[c];
        }
        int all_small = 1, all_e = 1;
        for (int c = 0; c < nvalues && c < dim_sub; c++) {
            double nr = 0.0;
            const double *rs = res + (size_t)c * N;
            for (size_t k = 0; k < N; k++) nr += rs[k] * rs[k];
            if (!(sqrt(nr) < tol)) all_small = 0;
            if (!(fabs(w[c] - last[c]) < etol)) all_e = 0;
        }
        int conv = N <= 2 || (all_small && all_e);
        if (conv) { result = 0; st->reason = N <= 2 ? 3 : 0; break; }
        for (int c = 0; c < nvalues; c++) last[c] = w[c];
        if (dim_sub + update_dim <= mss) {
            /* DPR (:391-408); correction.norm() is the Frobenius norm (:210) */
            double cn = 0.0;
            for (int c = 0; c < update_dim; c++) {
                double *t = corr + (size_t)c * N;
                const double *rs = res + (size_t)c * N;
                for (size_t k = 0; k < N; k++) { t[k] = rs[k] / (w[c] - dg[k]); cn += t[k] * t[k]; }
            }
            if (sqrt(cn) < 1e-9) { result = 0; st->reason = 1; break; }
            for (int c = 0; c < update_dim; c++) memcpy(basis + (size_t)(dim_sub + c) * N, corr + (size_t)c * N, sizeof(double) * N);
            if (!mgs_orthonormalize(basis, N, dim_sub, dim_sub + update_dim)) { result = 0; st->reason = 2; break; }
            for (int c = 0; c < update_dim; c++) mv(ctx, basis + (size_t)(dim_sub + c) * N, HV + (size_t)(dim_sub + c) * N);
            st->n_sigma += update_dim;
            int nd = dim_sub + update_dim;
            double *P2 = calloc((size_t)nd * nd, sizeof(double));
            for (int i = 0; i < dim_sub; i++) for (int j = 0; j < dim_sub; j++) P2[i * nd + j] = P[i * dim_sub + j];
            for (int i = 0; i < nd; i++) for (int c = dim_sub; c < nd; c++) {
                double s = 0.0;
                const double *a = basis + (size_t)i * N, *b = HV + (size_t)c * N;
                for (size_t k = 0; k < N; k++) s += a[k] * b[k];
                P2[i * nd + c] = s;
                P2[c * nd + i] = s;
            }
            memcpy(P, P2, sizeof(double) * nd * nd);
            free(P2);
            dim_sub = nd;
        } else {
            /* restart to the Ritz vectors (:261-269) */
            dim_sub = reset_dim;
            memset(basis, 0, sizeof(double) * (size_t)mss * N);
            memcpy(basis, ritz, sizeof(double) * (size_t)dim_sub * N);
            for (int c = 0; c < dim_sub; c++) mv(ctx, basis + (size_t)c * N, HV + (size_t)c * N);
            st->n_sigma += dim_sub;
            for (int i = 0; i < dim_sub; i++) for (int j = 0; j < dim_sub; j++) {
                double s = 0.0;
                const double *a = basis + (size_t)i * N, *b = HV + (size_t)j * N;
                for (size_t k = 0; k < N; k++) s += a[k] * b[k];
                P[i * dim_sub + j] = s;
            }
        }
    }
    st->iters = it + (it < max_iters ? 1 : 0);
    st->converged = result == 0;
    /* create_results (:280-298): the first nvalues Ritz pairs */
    for (int c = 0; c < nvalues && c < dim_sub; c++) {
        evals[c] = w[c];
        if (evecs) memcpy(evecs + (size_t)c * N, ritz + (size_t)c * N, sizeof(double) * N);
    }
    free(basis); free(HV); free(P); free(last); free(w); free(Y); free(ritz); free(res); free(corr);
    return result;
}

static void sparse_mv_cb(const void *ctx, const double *x, double *y) { sparse_mv((const Sparse *)ctx, x, y); }

OR_EXPORT int or_davidson(const Sparse *s, int nvalues, const double *init, double tol, double etol, int max_iters,
                          double *evals, double *evecs, int *stats4) {
    DavStats st = {0};
    int r = davidson(s, sparse_mv_cb, s->diag, s->n, nvalues, init, tol, etol, max_iters, evals, evecs, &st);
    if (stats4) { stats4[0] = st.iters; stats4[1] = st.n_sigma; stats4[2] = st.converged; stats4[3] = st.reason; }
    return r;
}

/* ------------------------------------------------------------------------- */
/* Multi-threaded (OpenMP) fast build and sigma, for the CPU baseline on every  */
/* host core.  The build produces the pairs and values of                       */
/* gen_sparse_ham_fast_lookup with n_stored_h = 0 (fast_ham.rs:527-575): every   */
/* pair i < j at excitation degree 1 or 2 is found once, by its row i, through   */
/* the same alpha group, the same beta group, or an alpha single-partner group,  */
/* and valued ham_off_diag_no_excite(det_i, det_j); singles are kept iff         */
/* |H| > 1e-12 (fast_ham.rs:505,510), doubles iff H != 0 (off_diag.rs:33).  The  */
/* serial builder computes the singles with the same argument order and the     */
/* doubles are symmetric in their arguments, so the stored values are the same.  */
/* sigma is matrix_vector_prod (sparse.rs:64-78) with the rows shared out        */
/* round-robin between the threads, each thread scattering into its own copy of  */
/* y; the copies are summed in thread order.                                     */
/* ------------------------------------------------------------------------- */

OR_EXPORT int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

OR_EXPORT int or_sparse_build_par(Sparse *s, const Ham *h, const uint64_t *dets, size_t N, const double *diag) {
    if (s->n) return -1;
    Config *cf = malloc(sizeof(Config) * (N ? N : 1));
    for (size_t i = 0; i < N; i++) cf[i] = cfg_from(dets + 4 * i);
    sparse_expand(s, N, diag);
    Groups ga, gb;
    groups_build(&ga, cf, N, 0);
    groups_build(&gb, cf, N, 1);
    Partners pa;
    partners_build(&pa, &ga);
#pragma omp parallel for schedule(dynamic, 64)
    for (size_t i = 0; i < N; i++) {
        Row *r = &s->rows[i];
        const Config ci = cf[i];
        /* same alpha string: beta singles and beta-beta doubles */
        size_t g = ga.gid[i];
        for (size_t k = ga.start[g]; k < ga.start[g + 1]; k++) {
            const size_t j = (size_t)ga.order[k];
            if (j <= i) continue;
            const int d = popc128(ci.dn ^ cf[j].dn);
            if (d != 2 && d != 4) continue;
            const double e = ham_off_diag_no_excite(h, ci, cf[j]);
            if (d == 2 ? fabs(e) > 1e-12 : e != 0.0) row_push(r, (int64_t)j, e);
        }
        /* same beta string: alpha singles and alpha-alpha doubles */
        g = gb.gid[i];
        for (size_t k = gb.start[g]; k < gb.start[g + 1]; k++) {
            const size_t j = (size_t)gb.order[k];
            if (j <= i) continue;
            const int d = popc128(ci.up ^ cf[j].up);
            if (d != 2 && d != 4) continue;
            const double e = ham_off_diag_no_excite(h, ci, cf[j]);
            if (d == 2 ? fabs(e) > 1e-12 : e != 0.0) row_push(r, (int64_t)j, e);
        }
        /* opposite-spin doubles: alpha single partners whose beta differs by one electron */
        const size_t a = ga.gid[i];
        for (size_t pk = pa.start[a]; pk < pa.start[a + 1]; pk++) {
            const size_t a2 = pa.part[pk];
            for (size_t k = ga.start[a2]; k < ga.start[a2 + 1]; k++) {
                const size_t j = (size_t)ga.order[k];
                if (j <= i || popc128(ci.dn ^ cf[j].dn) != 2) continue;
                const double e = ham_off_diag_no_excite(h, ci, cf[j]);
                if (e != 0.0) row_push(r, (int64_t)j, e);
            }
        }
        stable_sort_cols(r->e, r->n);
        s->nnz[i] = r->n;
    }
    partners_free(&pa);
    groups_free(&ga);
    groups_free(&gb);
    free(cf);
    return 0;
}

/* Full rows of the sampled determinants against the whole set, by brute force (no
 * lookup tables): for row r every j != r at excitation degree 1 or 2 whose element
 * passes the fast builder's rule, valued as the fast builder values the pair
 * (ham_off_diag_no_excite(det_min(r,j), det_max(r,j)), fast_ham.rs:473-517;
 * off_diag.rs:26-39).  Entries of row rows[i] fill out_* from off[i], with
 * off[k] = total; columns ascending within a row.  Returns 0, or -1 when the
 * total exceeds cap (off[] is filled either way). */
static int brute_row(const Ham *h, const Config *cf, size_t N, size_t r, int64_t *oc, double *ov) {
    int n = 0;
    const Config a = cf[r];
    for (size_t j = 0; j < N; j++) {
        if (j == r) continue;
        const int du = popc128(a.up ^ cf[j].up), dd = popc128(a.dn ^ cf[j].dn);
        const int d = du + dd;
        if (d != 2 && d != 4) continue;
        const double e = r < j ? ham_off_diag_no_excite(h, a, cf[j]) : ham_off_diag_no_excite(h, cf[j], a);
        const int keep = d == 2 ? fabs(e) > 1e-12 : e != 0.0;
        if (!keep) continue;
        if (oc) { oc[n] = (int64_t)j; ov[n] = e; }
        n++;
    }
    return n;
}

OR_EXPORT int or_rows_bruteforce(const Ham *h, const uint64_t *dets, size_t N, const int64_t *rows, size_t k,
                                 int64_t *off, int64_t *out_c, double *out_v, size_t cap) {
    Config *cf = malloc(sizeof(Config) * (N ? N : 1));
    for (size_t i = 0; i < N; i++) cf[i] = cfg_from(dets + 4 * i);
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t i = 0; i < k; i++) off[i + 1] = brute_row(h, cf, N, (size_t)rows[i], NULL, NULL);
    off[0] = 0;
    for (size_t i = 0; i < k; i++) off[i + 1] += off[i];
    int rc = (size_t)off[k] > cap ? -1 : 0;
    if (rc == 0) {
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t i = 0; i < k; i++) brute_row(h, cf, N, (size_t)rows[i], out_c + off[i], out_v + off[i]);
    }
    free(cf);
    return rc;
}

typedef struct { const Sparse *s; double *buf; int nt; } ParCtx;

static void sparse_mv_par(const void *ctx, const double *x, double *y) {
    const ParCtx *c = ctx;
    const Sparse *s = c->s;
    const size_t n = s->n;
#pragma omp parallel num_threads(c->nt)
    {
#ifdef _OPENMP
        const int t = omp_get_thread_num();
#else
        const int t = 0;
#endif
        double *yt = c->buf + (size_t)t * n;
        for (size_t i = 0; i < n; i++) yt[i] = 0.0;
#pragma omp barrier
#pragma omp for schedule(static, 64)
        for (size_t i = 0; i < n; i++) {
            const Row *r = &s->rows[i];
            const double xi = x[i];
            double acc = s->diag[i] * xi;
            for (size_t k = 0; k < r->n; k++) {
                acc += r->e[k].val * x[r->e[k].col];
                yt[r->e[k].col] += r->e[k].val * xi;
            }
            yt[i] += acc;
        }
#pragma omp for schedule(static)
        for (size_t i = 0; i < n; i++) {
            double v = 0.0;
            for (int u = 0; u < c->nt; u++) v += c->buf[(size_t)u * n + i];
            y[i] = v;
        }
    }
}

OR_EXPORT void or_sparse_mv_par(const Sparse *s, const double *x, double *y) {
    ParCtx c = {s, NULL, or_num_threads()};
    c.buf = malloc(sizeof(double) * (size_t)c.nt * (s->n ? s->n : 1));
    sparse_mv_par(&c, x, y);
    free(c.buf);
}

OR_EXPORT int or_davidson_par(const Sparse *s, int nvalues, const double *init, double tol, double etol,
                              int max_iters, double *evals, double *evecs, int *stats4) {
    ParCtx c = {s, NULL, or_num_threads()};
    c.buf = malloc(sizeof(double) * (size_t)c.nt * (s->n ? s->n : 1));
    DavStats st = {0};
    int r = davidson(&c, sparse_mv_par, s->diag, s->n, nvalues, init, tol, etol, max_iters, evals, evecs, &st);
    if (stats4) { stats4[0] = st.iters; stats4[1] = st.n_sigma; stats4[2] = st.converged; stats4[3] = st.reason; }
    free(c.buf);
    return r;
}

/* Davidson over a dense symmetric matrix (row-major), used to pin the solver. */
typedef struct { const double *A; size_t n; } DenseCtx;
static void dense_mv_cb(const void *ctx, const double *x, double *y) {
    const DenseCtx *d = ctx;
    for (size_t i = 0; i < d->n; i++) {
        double s = 0.0;
        for (size_t j = 0; j < d->n; j++) s += d->A[i * d->n + j] * x[j];
        y[i] = s;
    }
}
OR_EXPORT int or_davidson_dense(const double *A, size_t n, int nvalues, const double *init, double tol, double etol,
                                int max_iters, double *evals, double *evecs, int *stats4) {
    double *dg = malloc(sizeof(double) * n);
    for (size_t i = 0; i < n; i++) dg[i] = A[i * n + i];
    DenseCtx ctx = {A, n};
    DavStats st = {0};
    int r = davidson(&ctx, dense_mv_cb, dg, n, nvalues, init, tol, etol, max_iters, evals, evecs, &st);
    if (stats4) { stats4[0] = st.iters; stats4[1] = st.n_sigma; stats4[2] = st.converged; stats4[3] = st.reason; }
    free(dg);
    return r;
}

/* ------------------------------------------------------------------------- */
/* wf/eps.rs, wf/mod.rs selection, var/mod.rs HCI loop                         */
/* ------------------------------------------------------------------------- */

typedef struct { double next_one, target; } Eps;

/* Eps::next (src/wf/eps.rs:41-53). */
static double eps_next(Eps *e) {
    double curr = e->next_one;
    double prop = e->next_one * 0.1;
    e->next_one = prop > e->target ? prop : e->target;
    return curr;
}

static inline int btest(u128 n, int b) { return (n & bit128(b)) != 0; }

/* init_eps (src/wf/eps.rs:82-172). */
static Eps init_eps(const Wf *wf, double eps_var, int z_sym, const ExciteGen *eg) {
    double max_sym = eps_var, max_asym = eps_var, max_conn = eps_var;
    int n = eg->norb;
    for (size_t d = 0; d < wf->n; d++) {
        Config c = wf->dets[d].config;
        for (u128 t = eg->valence & c.up; t; t &= t - 1) {
            int i = ctz128(t);
            for (u128 u = eg->valence & c.dn; u; u &= u - 1) {
                int j = ctz128(u);
                int found_sym = 0, found_asym = 0;
                const StoredList *L = &eg->opp[i * n + j];
                for (int k = 0; k < L->n; k++) {
                    int r = L->v[k].r, s = L->v[k].s;
                    if (!btest(c.up, r) && !btest(c.dn, s)) {
                        double th = L->v[k].abs_h;
                        if (i == j && r == s) { found_sym = 1; if (th > max_sym) max_sym = th; }
                        else {
                            found_asym = 1;
                            if (th > max_asym) max_asym = th;
                            if (i == j || r == s) if (th > max_conn) max_conn = th;
                        }
                        if (found_sym && found_asym) break;
                    }
                }
            }
        }
        for (int sp = 0; sp < 2; sp++) {
            u128 x = sp == 0 ? c.up : c.dn;
            u128 vx = eg->valence & x;
            for (u128 t = vx; t; t &= t - 1) {
                int i = ctz128(t);
                for (u128 u = t & (t - 1); u; u &= u - 1) {
                    int j = ctz128(u);
                    const StoredList *L = &eg->same[i * n + j];
                    for (int k = 0; k < L->n; k++) {
                        if (!btest(x, L->v[k].r) && !btest(x, L->v[k].s)) {
                            if (L->v[k].abs_h > max_asym) max_asym = L->v[k].abs_h;
                            break;
                        }
                    }
                }
            }
        }
    }
    double max_doub = z_sym == 1 ? (max_sym > max_asym ? max_sym : max_asym) : max_conn;
    Eps e = {max_doub - 1e-9, eps_var};
    return e;
}

/* Opaque HCI state (VarWf + Global subset + ExciteGenerator). */
typedef struct {
    const Ham *ham;
    ExciteGen *eg;
    int nup, ndn, z_sym;
    double eps_var;
    Wf wf;
    Eps eps_iter;
    double eps;
    size_t n_stored_h;
    Sparse *sp;
    int converged;
    int builder, grouped_singles;
    int dav_max_iter, parallel;
    /* per-iteration log */
    int nlog;
    double log_eps[64], log_energy[64];
    size_t log_ndets[64], log_nnz[64];
    int log_dav[64][4];
} Hci;

/* iterate_excites with matmul == false (src/wf/mod.rs:1474-1631). */
static void iterate_excites(Hci *H, Wf *out) {
    const Ham *h = H->ham;
    const ExciteGen *eg = H->eg;
    int n = eg->norb;
    for (size_t di = 0; di < H->wf.n; di++) {
        const Det *det = &H->wf.dets[di];
        double local_eps = H->eps / fabs(det->coeff);
        Config c = det->config;
        if (eg->max_opp_doub >= local_eps) {
            for (u128 t = eg->valence & c.up; t; t &= t - 1) {
                int i = ctz128(t);
                for (u128 u = eg->valence & c.dn; u; u &= u - 1) {
                    int j = ctz128(u);
                    const StoredList *L = &eg->opp[i * n + j];
                    for (int k = 0; k < L->n; k++) {
                        if (L->v[k].abs_h < local_eps) break;
                        int r = L->v[k].r, s = L->v[k].s;
                        if (btest(c.up, r) || btest(c.dn, s)) continue; /* is_valid (det.rs:87-118) */
                        Config d = {(c.up & ~bit128(i)) | bit128(r), (c.dn & ~bit128(j)) | bit128(s)};
                        if (map_get(&H->wf.inds, d) < 0 && map_get(&out->inds, d) < 0) {
                            Det nd = {d, 0.0, new_diag_opp(h, det, i, j, r, s), 1};
                            wf_push(out, nd);
                        }
                    }
                }
            }
        }
        if (eg->max_same_doub >= local_eps) {
            for (int sp = 0; sp < 2; sp++) {
                u128 x = sp == 0 ? c.up : c.dn;
                int is_alpha = sp == 0;
                for (u128 t = eg->valence & x; t; t &= t - 1) {
                    int i = ctz128(t);
                    for (u128 u = t & (t - 1); u; u &= u - 1) {
                        int j = ctz128(u);
                        const StoredList *L = &eg->same[i * n + j];
                        for (int k = 0; k < L->n; k++) {
                            if (L->v[k].abs_h < local_eps) break;
                            int r = L->v[k].r, s = L->v[k].s;
                            if (btest(x, r) || btest(x, s)) continue;
                            u128 nx = (x & ~bit128(i) & ~bit128(j)) | bit128(r) | bit128(s);
                            Config d = is_alpha ? (Config){nx, c.dn} : (Config){c.up, nx};
                            if (map_get(&H->wf.inds, d) < 0 && map_get(&out->inds, d) < 0) {
                                Det nd = {d, 0.0, new_diag_same(h, det, i, j, r, s, is_alpha), 1};
                                wf_push(out, nd);
                            }
                        }
                    }
                }
            }
        }
        if (H->eps == H->eps_var && eg->max_sing >= local_eps) {
            for (int sp = 0; sp < 2; sp++) {
                u128 x = sp == 0 ? c.up : c.dn;
                int is_alpha = sp == 0;
                for (u128 t = eg->valence & x; t; t &= t - 1) {
                    int i = ctz128(t);
                    const StoredList *L = &eg->sing[i];
                    for (int k = 0; k < L->n; k++) {
                        if (L->v[k].abs_h < local_eps) break;
                        int r = L->v[k].r;
                        if (btest(x, r)) continue;
                        u128 nx = (x & ~bit128(i)) | bit128(r);
                        Config d = is_alpha ? (Config){nx, c.dn} : (Config){c.up, nx};
                        if (map_get(&H->wf.inds, d) < 0 && map_get(&out->inds, d) < 0) {
                            if (fabs(ham_sing(h, c, d)) > local_eps) {
                                Det nd = {d, 0.0, new_diag_sing(h, det, i, r, is_alpha), 1};
                                wf_push(out, nd);
                            }
                        }
                    }
                }
            }
        }
    }
}

/* find_new_dets (src/wf/mod.rs:1418-1467).  Returns 1 when no new dets. */
static int find_new_dets(Hci *H) {
    H->eps = eps_next(&H->eps_iter);
    Wf out;
    wf_init(&out, 64);
    iterate_excites(H, &out);
    for (size_t k = 0; k < out.n; k++) {
        if (H->z_sym == 1) wf_push_and_spin_flipped(&H->wf, out.dets[k]);
        else if (out.dets[k].config.up != out.dets[k].config.dn) wf_push_and_spin_flipped(&H->wf, out.dets[k]);
    }
    int none = out.n == 0;
    wf_free(&out);
    return none;
}

/* sparse_optimize (src/var/davidson.rs:43-113). */
static void sparse_optimize(Hci *H, double coeff_eps, double energy_eps, int init_last_iter, int *davstats) {
    size_t N = H->wf.n;
    Config *cf = malloc(sizeof(Config) * N);
    double *diag = malloc(sizeof(double) * N);
    for (size_t i = 0; i < N; i++) { cf[i] = H->wf.dets[i].config; diag[i] = H->wf.dets[i].diag; }
    if (H->parallel) {
        /* every pair rebuilt on all cores (the fast builder's rule for the whole set) */
        or_sparse_free(H->sp);
        H->sp = or_sparse_new();
        uint64_t *d4 = malloc(sizeof(uint64_t) * 4 * (N ? N : 1));
        for (size_t i = 0; i < N; i++) cfg_to(cf[i], d4 + 4 * i);
        or_sparse_build_par(H->sp, H->ham, d4, N, diag);
        free(d4);
    } else {
        sparse_build(H->sp, H->ham, cf, N, H->n_stored_h, diag, H->builder, H->grouped_singles);
    }
    H->n_stored_h = N;
    double *init = NULL;
    if (init_last_iter) {
        init = malloc(sizeof(double) * N);
        for (size_t i = 0; i < N; i++) init[i] = H->wf.dets[i].coeff;
    }
    double ev;
    double *evec = malloc(sizeof(double) * N);
    DavStats st = {0};
    int r;
    if (H->parallel) r = or_davidson_par(H->sp, 1, init, coeff_eps, energy_eps, H->dav_max_iter, &ev, evec, NULL);
    else r = davidson(H->sp, sparse_mv_cb, H->sp->diag, N, 1, init, coeff_eps, energy_eps, H->dav_max_iter, &ev, evec, &st);
    if (r == 0) {
        H->wf.energy = ev;
        for (size_t i = 0; i < N; i++) H->wf.dets[i].coeff = evec[i];
    } else {
        fprintf(stderr, "oracle: Davidson Algorithm did not converge!\n");
    }
    if (davstats) { davstats[0] = st.iters; davstats[1] = st.n_sigma; davstats[2] = st.converged; davstats[3] = st.reason; }
    free(init); free(evec); free(cf); free(diag);
}

/* init_var_wf for z_sym == 1 (src/wf/mod.rs:1687-1740). */
OR_EXPORT Hci *or_hci_new(const Ham *h, int nup, int ndn, int z_sym, double eps_var, int builder, int grouped_singles) {
    if (z_sym != 1) return NULL; /* the antisymmetric start (:1714-1738) is outside this path */
    Hci *H = calloc(1, sizeof(Hci));
    H->ham = h;
    H->nup = nup; H->ndn = ndn; H->z_sym = z_sym; H->eps_var = eps_var;
    H->builder = builder; H->grouped_singles = grouped_singles;
    H->eg = excite_gen_new(h, nup, ndn);
    wf_init(&H->wf, 1024);
    Det hf;
    hf.config.up = bit128(nup) - 1;
    hf.config.dn = bit128(ndn) - 1;
    hf.coeff = 1.0;
    hf.diag = ham_diag(h, hf.config);
    hf.has_diag = 1;
    wf_append(&H->wf, hf);
    H->wf.energy = hf.diag;
    H->eps_iter = init_eps(&H->wf, eps_var, z_sym, H->eg);
    H->sp = or_sparse_new();
    H->n_stored_h = 0;
    H->dav_max_iter = 50; /* Config::new, algorithms/davidson.rs:73 */
    return H;
}

/* Davidson iteration cap of each solve (the reference fixes 50) and the
 * multi-threaded build / sigma (0 = the serial restatement). */
OR_EXPORT void or_hci_set_options(Hci *H, int dav_max_iter, int parallel) {
    H->dav_max_iter = dav_max_iter > 0 ? dav_max_iter : 50;
    H->parallel = parallel;
}

OR_EXPORT void or_hci_free(Hci *H) {
    if (!H) return;
    excite_gen_free(H->eg);
    wf_free(&H->wf);
    or_sparse_free(H->sp);
    free(H);
}

/* One pass of the loop body of variational (src/var/mod.rs:70-123).
 * Returns 1 when the loop would stop (converged), 0 otherwise. */
OR_EXPORT int or_hci_step(Hci *H) {
    int none = find_new_dets(H);
    if (H->eps == H->eps_var && none) { H->converged = 1; return 1; }
    int it = H->nlog + 1;
    int ds[4] = {0};
    sparse_optimize(H, 1e-4, 1e-8, it > 1, ds);
    if (H->nlog < 64) {
        H->log_eps[H->nlog] = H->eps;
        H->log_energy[H->nlog] = H->wf.energy;
        H->log_ndets[H->nlog] = H->wf.n;
        H->log_nnz[H->nlog] = or_sparse_nnz(H->sp);
        memcpy(H->log_dav[H->nlog], ds, sizeof(ds));
        H->nlog++;
    }
    H->eps = eps_next(&H->eps_iter); /* var/mod.rs:123 */
    return 0;
}

/* One loop pass that stops after the selection when the space would exceed max_dets:
 * returns 2 then (the new determinants are appended but not optimised, so the state
 * is only good for reading the earlier space, exported before the call). */
OR_EXPORT int or_hci_step_bounded(Hci *H, size_t max_dets) {
    int none = find_new_dets(H);
    if (H->eps == H->eps_var && none) { H->converged = 1; return 1; }
    if (H->wf.n > max_dets) return 2;
    int it = H->nlog + 1;
    int ds[4] = {0};
    sparse_optimize(H, 1e-4, 1e-8, it > 1, ds);
    if (H->nlog < 64) {
        H->log_eps[H->nlog] = H->eps;
        H->log_energy[H->nlog] = H->wf.energy;
        H->log_ndets[H->nlog] = H->wf.n;
        H->log_nnz[H->nlog] = or_sparse_nnz(H->sp);
        memcpy(H->log_dav[H->nlog], ds, sizeof(ds));
        H->nlog++;
    }
    H->eps = eps_next(&H->eps_iter); /* var/mod.rs:123 */
    return 0;
}

/* variational (src/var/mod.rs:59-134): at most 20 iterations. */
OR_EXPORT double or_hci_run(Hci *H, int max_iter) {
    int iter = 0;
    while (!H->converged) {
        iter++;
        if (iter > max_iter) break;
        if (or_hci_step(H)) break;
    }
    return H->wf.energy;
}

OR_EXPORT size_t or_hci_ndets(const Hci *H) { return H->wf.n; }
OR_EXPORT size_t or_hci_nstored(const Hci *H) { return H->n_stored_h; }
OR_EXPORT double or_hci_energy(const Hci *H) { return H->wf.energy; }
OR_EXPORT int or_hci_converged(const Hci *H) { return H->converged; }
OR_EXPORT double or_hci_eps(const Hci *H) { return H->eps; }
OR_EXPORT void or_hci_export(const Hci *H, uint64_t *dets, double *coeffs, double *diag) {
    for (size_t i = 0; i < H->wf.n; i++) {
        if (dets) cfg_to(H->wf.dets[i].config, dets + 4 * i);
        if (coeffs) coeffs[i] = H->wf.dets[i].coeff;
        if (diag) diag[i] = H->wf.dets[i].diag;
    }
}
OR_EXPORT const Sparse *or_hci_sparse(const Hci *H) { return H->sp; }
OR_EXPORT int or_hci_log(const Hci *H, double *eps, double *energy, uint64_t *ndets, uint64_t *nnz, int *dav) {
    for (int i = 0; i < H->nlog; i++) {
        eps[i] = H->log_eps[i]; energy[i] = H->log_energy[i];
        ndets[i] = H->log_ndets[i]; nnz[i] = H->log_nnz[i];
        memcpy(dav + 4 * i, H->log_dav[i], sizeof(int) * 4);
    }
    return H->nlog;
}

/* Excitation-generator introspection for tests. */
OR_EXPORT void or_excite_gen_max(const Hci *H, double *out3) {
    out3[0] = H->eg->max_opp_doub; out3[1] = H->eg->max_same_doub; out3[2] = H->eg->max_sing;
}
