// Determinant strings and Slater-Condon matrix elements on the device.
//
// A spin string of up to 64*W orbitals lives in W 64-bit words (W = 1 for
// norb <= 64, W = 2 up to the reference's u128 limit).  Every function below
// reproduces the reference's FP64 arithmetic operation for operation, so the
// elements it returns are bitwise equal to the CPU ones:
//   ham_sing          src/ham/mod.rs:135-168
//   ham_doub          src/ham/mod.rs:179-233
//   permute/permute_2 src/utils/ints.rs:76-97
//   combine_2/_4      src/utils/ints.rs:38-68
//   new_diag_*        src/wf/det.rs:271-420
// The sums contain no products, so no fused multiply-add can change them; the
// sign is applied as a multiplication by +-1.0, as in the reference.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace risq {

template <int W>
struct Bits {
    uint64_t w[W];

    __host__ __device__ __forceinline__ static Bits zero() {
        Bits b;
#pragma unroll
        for (int k = 0; k < W; k++) b.w[k] = 0;
        return b;
    }
    __device__ __forceinline__ Bits operator^(const Bits& o) const {
        Bits r;
#pragma unroll
        for (int k = 0; k < W; k++) r.w[k] = w[k] ^ o.w[k];
        return r;
    }
    __device__ __forceinline__ Bits operator&(const Bits& o) const {
        Bits r;
#pragma unroll
        for (int k = 0; k < W; k++) r.w[k] = w[k] & o.w[k];
        return r;
    }
    __device__ __forceinline__ Bits operator|(const Bits& o) const {
        Bits r;
#pragma unroll
        for (int k = 0; k < W; k++) r.w[k] = w[k] | o.w[k];
        return r;
    }
    // this & ~o
    __device__ __forceinline__ Bits andnot(const Bits& o) const {
        Bits r;
#pragma unroll
        for (int k = 0; k < W; k++) r.w[k] = w[k] & ~o.w[k];
        return r;
    }
    __device__ __forceinline__ bool operator==(const Bits& o) const {
        bool e = true;
#pragma unroll
        for (int k = 0; k < W; k++) e = e && (w[k] == o.w[k]);
        return e;
    }
    __device__ __forceinline__ bool operator!=(const Bits& o) const { return !(*this == o); }
    __device__ __forceinline__ bool is_zero() const {
        uint64_t a = 0;
#pragma unroll
        for (int k = 0; k < W; k++) a |= w[k];
        return a == 0;
    }
    __device__ __forceinline__ int popc() const {
        int c = 0;
#pragma unroll
        for (int k = 0; k < W; k++) c += __popcll(w[k]);
        return c;
    }
    // index of the lowest set bit (caller guarantees non-zero)
    __device__ __forceinline__ int ctz() const {
#pragma unroll
        for (int k = 0; k < W; k++)
            if (w[k]) return 64 * k + __ffsll((long long)w[k]) - 1;
        return 64 * W;
    }
    // clear the lowest set bit
    __device__ __forceinline__ void pop_lowest() {
#pragma unroll
        for (int k = 0; k < W; k++) {
            if (w[k]) { w[k] &= w[k] - 1; return; }
        }
    }
    __device__ __forceinline__ bool test(int b) const { return (w[b >> 6] >> (b & 63)) & 1ull; }
    __device__ __forceinline__ void set(int b) { w[b >> 6] |= 1ull << (b & 63); }
    __device__ __forceinline__ void clear(int b) { w[b >> 6] &= ~(1ull << (b & 63)); }
    // (1 << b) - 1 as a W-word string
    __device__ __forceinline__ static Bits below(int b) {
        Bits r;
#pragma unroll
        for (int k = 0; k < W; k++) {
            int lo = 64 * k;
            if (b >= lo + 64) r.w[k] = ~0ull;
            else if (b <= lo) r.w[k] = 0ull;
            else r.w[k] = (1ull << (b - lo)) - 1ull;
        }
        return r;
    }
};

// parity(n) of src/utils/bits.rs:171-180: +1 for an even popcount.
template <int W>
__device__ __forceinline__ int parity_sign(const Bits<W>& x) { return (x.popc() & 1) ? -1 : 1; }

// permute (src/utils/ints.rs:76-82).  For strings differing by one electron moved
// from i (in d1) to j (in d2), d1 & (d1 - d2) when d1 > d2 is the set of d1's
// occupied bits in [j, i), i.e. the common bits strictly between j and i; the
// d2 > d1 branch gives the same set.  That set is computed directly here.
template <int W>
__device__ __forceinline__ int permute1(const Bits<W>& d1, const Bits<W>& d2) {
    int i = d1.andnot(d2).ctz();
    int j = d2.andnot(d1).ctz();
    int lo = i < j ? i : j, hi = i < j ? j : i;
    Bits<W> m = Bits<W>::below(hi).andnot(Bits<W>::below(lo + 1));
    return parity_sign((d1 & d2) & m);
}

// permute_2 (src/utils/ints.rs:92-97).
template <int W>
__device__ __forceinline__ int permute2(const Bits<W>& d1, const Bits<W>& d2, int v0, int v1, int v2, int v3) {
    Bits<W> m = Bits<W>::below(v0) ^ Bits<W>::below(v1) ^ Bits<W>::below(v2) ^ Bits<W>::below(v3);
    return parity_sign((d1 & d2) & m);
}

// Packed 1-based integral indices (src/utils/ints.rs:38-68); indices here are
// the reference's 0-based orbital indices plus one, always positive.
__device__ __forceinline__ uint32_t c2(uint32_t i, uint32_t j) {
    return i > j ? (i * (i - 1)) / 2 + j : (j * (j - 1)) / 2 + i;
}
__device__ __forceinline__ uint32_t c4(uint32_t p, uint32_t q, uint32_t r, uint32_t s) {
    return c2(c2(p, q), c2(r, s));
}

// Integral tables in global memory, read through the read-only cache.
struct Ints {
    const double* __restrict__ h1;  // one_body, combine_2 layout
    const double* __restrict__ h2;  // two_body, combine_4 layout
    double nuc;
    __device__ __forceinline__ double ld1(uint32_t k) const { return __ldg(h1 + k); }
    __device__ __forceinline__ double ld2(uint32_t k) const { return __ldg(h2 + k); }
};

// The same tables staged in shared memory by the calling kernel.
struct IntsShared {
    const double* h1;
    const double* h2;
    double nuc;
    __device__ __forceinline__ double ld1(uint32_t k) const { return h1[k]; }
    __device__ __forceinline__ double ld2(uint32_t k) const { return h2[k]; }
};

// Ham::one_body (0-based p, q)          src/ham/mod.rs:65-67
template <class IT>
__device__ __forceinline__ double one_body(const IT& I, int p, int q) { return I.ld1(c2(p + 1, q + 1)); }
// Ham::direct(p,q,r,s) = (p r | q s)    src/ham/mod.rs:72-74
template <class IT>
__device__ __forceinline__ double direct(const IT& I, int p, int q, int r, int s) {
    return I.ld2(c4(p + 1, r + 1, q + 1, s + 1));
}
// Ham::direct_plus_exchange             src/ham/mod.rs:80-82
template <class IT>
__device__ __forceinline__ double dpe(const IT& I, int p, int q, int r, int s) {
    return __dsub_rn(I.ld2(c4(p + 1, r + 1, q + 1, s + 1)), I.ld2(c4(p + 1, s + 1, q + 1, r + 1)));
}

// <d1|H|d2> for one electron of spin sigma moved: s1/s2 are the two strings of
// that spin, opp the other spin's (equal) string.  ham_sing sums over d1's
// occupied orbitals k of spin sigma, which include the removed orbital i; that
// term is dpe(i,i,j,i) = (ij|ii) - (ii|ij), two reads of one packed entry, so
// exactly +0.0.  Adding +0.0 leaves every partial sum unchanged, hence the loop
// below runs over the common orbitals only and returns the same bits.  For the
// same reason the element is bitwise symmetric in (d1, d2).
template <int W, class IT = Ints>
__device__ __forceinline__ double sc_single(const IT& I, const Bits<W>& s1, const Bits<W>& s2, const Bits<W>& opp) {
    int i = s1.andnot(s2).ctz();
    int j = s2.andnot(s1).ctz();
    double out = one_body(I, i, j);
    Bits<W> com = s1 & s2;
    while (!com.is_zero()) {
        int k = com.ctz();
        com.pop_lowest();
        out = __dadd_rn(out, dpe(I, i, k, j, k));
    }
    Bits<W> o = opp;
    while (!o.is_zero()) {
        int k = o.ctz();
        o.pop_lowest();
        out = __dadd_rn(out, direct(I, i, k, j, k));
    }
    return __dmul_rn(out, (double)permute1(s1, s2));
}

// Same-spin double (ham_doub, src/ham/mod.rs:180-207): i<j removed from s1,
// k<l added in s2, value permute_2 * [(ik|jl) - (il|jk)].
template <int W, class IT = Ints>
__device__ __forceinline__ double sc_double_same(const IT& I, const Bits<W>& s1, const Bits<W>& s2) {
    Bits<W> rem = s1.andnot(s2), add = s2.andnot(s1);
    int i0 = rem.ctz();
    rem.pop_lowest();
    int i1 = rem.ctz();
    int i2 = add.ctz();
    add.pop_lowest();
    int i3 = add.ctz();
    return __dmul_rn((double)permute2(s1, s2, i0, i1, i2, i3), dpe(I, i0, i1, i2, i3));
}

// Opposite-spin double (ham_doub, src/ham/mod.rs:208-232).
template <int W, class IT = Ints>
__device__ __forceinline__ double sc_double_opp(const IT& I, const Bits<W>& a1, const Bits<W>& b1,
                                                const Bits<W>& a2, const Bits<W>& b2) {
    int ia = a1.andnot(a2).ctz(), aa = a2.andnot(a1).ctz();
    int ib = b1.andnot(b2).ctz(), ab = b2.andnot(b1).ctz();
    int sg = permute1(a1, a2) * permute1(b1, b2);
    return __dmul_rn((double)sg, direct(I, ia, ib, aa, ab));
}

// ham_diag (src/ham/mod.rs:92-124), same order of accumulation.
template <int W, class IT = Ints>
__device__ __forceinline__ double sc_diag(const IT& I, const Bits<W>& up, const Bits<W>& dn) {
    double d = I.nuc;
    Bits<W> t = up;
    while (!t.is_zero()) { int i = t.ctz(); t.pop_lowest(); d = __dadd_rn(d, one_body(I, i, i)); }
    t = dn;
    while (!t.is_zero()) { int i = t.ctz(); t.pop_lowest(); d = __dadd_rn(d, one_body(I, i, i)); }
    t = up;
    while (!t.is_zero()) {
        int i = t.ctz();
        t.pop_lowest();
        Bits<W> u = dn;
        while (!u.is_zero()) { int j = u.ctz(); u.pop_lowest(); d = __dadd_rn(d, direct(I, i, j, i, j)); }
    }
    for (int sp = 0; sp < 2; sp++) {
        Bits<W> x = sp == 0 ? up : dn;
        while (!x.is_zero()) {
            int i = x.ctz();
            x.pop_lowest();
            Bits<W> u = x;
            while (!u.is_zero()) { int j = u.ctz(); u.pop_lowest(); d = __dadd_rn(d, dpe(I, i, j, i, j)); }
        }
    }
    return d;
}

// <p|H|q> for a stored (connected, distinct) pair: the excitation class follows from
// the two popcounts, as in ham_off_diag_no_excite (src/ham/mod.rs:256-303).
template <int W, class IT = Ints>
__device__ __forceinline__ double sc_pair(const IT& I, const Bits<W>& a, const Bits<W>& b, const Bits<W>& aq,
                                          const Bits<W>& bq) {
    const int du = (a ^ aq).popc(), dd = (b ^ bq).popc();
    if (du == 0) return dd == 2 ? sc_single<W, IT>(I, b, bq, a) : sc_double_same<W, IT>(I, b, bq);
    if (dd == 0) return du == 2 ? sc_single<W, IT>(I, a, aq, b) : sc_double_same<W, IT>(I, a, aq);
    return sc_double_opp<W, IT>(I, a, b, aq, bq);
}

}  // namespace risq
