// Tiled upper-triangle storage and its sigma.
//
// The reference's SparseMatUpperTri (src/var/sparse.rs:24-36) holds every pair
// once and its matrix_vector_prod (src/var/sparse.rs:64-78) adds each element to
// two outputs: y_p += H_pq x_q and y_q += H_pq x_p.  On the GPU the second of
// these is a scattered atomic per pair, and a gather plus a scattered atomic per
// pair bound the plain kernel by L1/L2 request throughput, not by HBM.
//
// Here the stored pairs are regrouped after the build.  Rows are cut into panels
// of R = 2^rb consecutive rows and columns into windows of C = 2^cb.  A (panel,
// window) tile that holds enough pairs is "dense": sigma stages x of its window
// and zeroes a window of accumulators in shared memory, so that every pair costs
// two shared-memory updates and the global traffic per tile is one coalesced read
// of x and one coalesced flush of the accumulated column sums.  Pairs of sparse
// tiles stay as leftovers, kept in row order and summed per row by a warp with
// global gathers and atomics, as in the plain kernel.  Within a work unit (a run of
// one panel's tiles) the row sums gather in a shared accumulator that is flushed
// once.
//
// Shared windows sum in 32-bit fixed point (k_sigma_fx): each product is rounded,
// by a fixed rule, at a scale chosen per tile from the tile's largest row or column
// sum of |H|, and integer atomics are associative, so a window's sum does not depend
// on the order in which the pairs land.  The FP64 sigma (and the FP32 sigma when
// reproducible sums are asked for) then adds the window sums in 64-bit fixed point
// (scale 2^s per call, from max |x| and the largest row sum of |H| over both
// triangles, found during the conversion), so two runs give bitwise-equal vectors.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "internal.cuh"

namespace risq {

namespace {

constexpr int TT = 256;          // threads per CTA of the conversion and sigma kernels
constexpr int MAX_BINS = 16384;  // windows one panel may span during the conversion
constexpr unsigned FULL = 0xffffffffu;

// A tile is staged in shared memory when it holds at least max(DENSE_MIN, w >> DENSE_SHIFT)
// pairs (w = width of its window): staging w values of x, zeroing w accumulators and
// flushing them costs about as much as w >> DENSE_SHIFT scattered pairs.
constexpr int DENSE_MIN = 64;
constexpr int DENSE_SHIFT = 3;

__host__ __device__ __forceinline__ bool dense_tile(int count, int w) {
    return count >= DENSE_MIN && count >= (w >> DENSE_SHIFT);
}

__device__ __forceinline__ int window_width(int64_t N, int64_t J, int cb) {
    const int64_t c0 = J << cb;
    return (int)min((int64_t)1 << cb, N - c0);
}

// ---------------------------------------------------------------- conversion

// Per panel of the chunk [p_lo, p_hi): stored pairs, pairs in dense tiles, dense
// tiles, and per row the number of leftover pairs.  CSR input: row p's columns at
// cols[row_start[p] - base ...], row_len[p] of them.
__global__ void __launch_bounds__(TT) k_tile_count(int64_t N, int64_t p_lo, int64_t p_hi, int rb, int cb,
                                                   const int64_t* __restrict__ row_start, int64_t base,
                                                   const int32_t* __restrict__ row_len,
                                                   const int32_t* __restrict__ cols, int64_t* __restrict__ panel_nel,
                                                   int64_t* __restrict__ panel_dense_el,
                                                   int32_t* __restrict__ panel_ntiles,
                                                   int32_t* __restrict__ left_len) {
    extern __shared__ int32_t hist[];
    using BR = cub::BlockReduce<long long, TT>;
    __shared__ typename BR::TempStorage red;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t P = p_lo + blockIdx.x; P < p_hi; P += gridDim.x) {
        const int64_t r0 = P << rb, r1 = min(N, r0 + ((int64_t)1 << rb));
        const int64_t J0 = r0 >> cb;
        const int nb = (int)(((N - 1) >> cb) - J0 + 1);
        for (int b = threadIdx.x; b < nb; b += TT) hist[b] = 0;
        __syncthreads();
        long long my_nel = 0;
        for (int64_t r = r0 + warp; r < r1; r += TT / 32) {
            const int64_t s = row_start[r] - base;
            const int len = row_len[r];
            if (lane == 0) my_nel += len;
            for (int k = lane; k < len; k += 32) atomicAdd(&hist[(cols[s + k] >> cb) - J0], 1);
        }
        __syncthreads();
        long long my_tiles = 0, my_dense = 0;
        for (int b = threadIdx.x; b < nb; b += TT) {
            const int c = hist[b];
            if (c > 0 && dense_tile(c, window_width(N, J0 + b, cb))) {
                my_tiles++;
                my_dense += c;
            }
        }
        // leftover pairs of every row (pairs whose tile is not dense)
        for (int64_t r = r0 + warp; r < r1; r += TT / 32) {
            const int64_t s = row_start[r] - base;
            const int len = row_len[r];
            int nl = 0;
            for (int k = lane; k < len; k += 32) {
                const int64_t b = (cols[s + k] >> cb) - J0;
                nl += dense_tile(hist[b], window_width(N, J0 + b, cb)) ? 0 : 1;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) nl += __shfl_xor_sync(FULL, nl, o);
            if (lane == 0) left_len[r] = nl;
        }
        const long long t_nel = BR(red).Sum(my_nel);
        __syncthreads();
        const long long t_tiles = BR(red).Sum(my_tiles);
        __syncthreads();
        const long long t_dense = BR(red).Sum(my_dense);
        if (threadIdx.x == 0) {
            panel_nel[P - p_lo] = t_nel;
            panel_ntiles[P - p_lo] = (int32_t)t_tiles;
            panel_dense_el[P - p_lo] = t_dense;
        }
        __syncthreads();
    }
}

// Scatter the chunk's pairs into the tiled arrays.  panel_el_off / panel_tile_off:
// absolute first element / first tile of every panel of the chunk.  Also adds |H_pq|
// to the row sums of both p and q (row_abs, in units of 2^-32: integer sums are exact,
// so the sums and the fixed-point scale derived from them do not depend on the order
// of the additions, nor on how the rows are split between ranks).
template <typename VIN>
__global__ void __launch_bounds__(TT) k_tile_scatter(
    int64_t N, int64_t p_lo, int64_t p_hi, int rb, int cb, const int64_t* __restrict__ row_start, int64_t base,
    const int32_t* __restrict__ row_len, const int32_t* __restrict__ cols, const VIN* __restrict__ vin,
    const float* __restrict__ vlo_in, const int64_t* __restrict__ panel_el_off,
    const int64_t* __restrict__ panel_tile_off, const int64_t* __restrict__ panel_dense_el,
    const int32_t* __restrict__ left_len, int32_t* __restrict__ tile_win, int32_t* __restrict__ tile_len,
    int64_t* __restrict__ tile_off, int64_t* __restrict__ left_off, uint32_t* __restrict__ el_idx,
    VIN* __restrict__ vout, float* __restrict__ vlo_out, unsigned long long* __restrict__ row_abs, int64_t el_cap,
    int64_t tile_cap) {
    extern __shared__ int32_t sm_i[];
    int32_t* cursor = sm_i;              // per window: next dense slot (panel-relative), or -1
    int32_t* lcur = sm_i + MAX_BINS;     // per row of the panel: leftover start (panel-relative)
    using BS = cub::BlockScan<long long, TT>;
    __shared__ typename BS::TempStorage scan;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t cmask = (1u << cb) - 1u;
    for (int64_t P = p_lo + blockIdx.x; P < p_hi; P += gridDim.x) {
        const int64_t r0 = P << rb, r1 = min(N, r0 + ((int64_t)1 << rb));
        const int nr = (int)(r1 - r0);
        const int64_t J0 = r0 >> cb;
        const int nb = (int)(((N - 1) >> cb) - J0 + 1);
        const int64_t el0 = panel_el_off[P - p_lo];
        const int64_t t0 = panel_tile_off[P - p_lo];
        for (int b = threadIdx.x; b < nb; b += TT) cursor[b] = 0;
        __syncthreads();
        for (int64_t r = r0 + warp; r < r1; r += TT / 32) {
            const int64_t s = row_start[r] - base;
            const int len = row_len[r];
            for (int k = lane; k < len; k += 32) atomicAdd(&cursor[(cols[s + k] >> cb) - J0], 1);
        }
        __syncthreads();
        // dense windows in window order: element and tile prefix sums over contiguous
        // chunks of windows per thread
        const int per = (nb + TT - 1) / TT;
        const int b_lo = min(nb, (int)threadIdx.x * per), b_hi = min(nb, b_lo + per);
        long long my_el = 0, my_t = 0;
        for (int b = b_lo; b < b_hi; b++) {
            const int c = cursor[b];
            if (c > 0 && dense_tile(c, window_width(N, J0 + b, cb))) {
                my_el += c;
                my_t++;
            }
        }
        long long ex_el, ex_t;
        BS(scan).ExclusiveSum(my_el, ex_el);
        __syncthreads();
        BS(scan).ExclusiveSum(my_t, ex_t);
        __syncthreads();
        for (int b = b_lo; b < b_hi; b++) {
            const int c = cursor[b];
            if (c > 0 && dense_tile(c, window_width(N, J0 + b, cb))) {
                if (t0 + ex_t < tile_cap) {  // always true: the count pass sized the tile arrays
                    tile_win[t0 + ex_t] = (int32_t)(J0 + b);
                    tile_len[t0 + ex_t] = c;
                    tile_off[t0 + ex_t] = el0 + ex_el;
                }
                cursor[b] = (int32_t)ex_el;
                ex_el += c;
                ex_t++;
            } else {
                cursor[b] = -1;
            }
        }
        // leftover regions of the rows, in row order after the dense tiles
        {
            const int rper = (nr + TT - 1) / TT;
            const int q_lo = min(nr, (int)threadIdx.x * rper), q_hi = min(nr, q_lo + rper);
            long long my_l = 0;
            for (int i = q_lo; i < q_hi; i++) my_l += left_len[r0 + i];
            long long ex_l;
            BS(scan).ExclusiveSum(my_l, ex_l);
            const long long dense_total = panel_dense_el[P - p_lo];
            for (int i = q_lo; i < q_hi; i++) {
                lcur[i] = (int32_t)(dense_total + ex_l);
                left_off[r0 + i] = el0 + dense_total + ex_l;
                ex_l += left_len[r0 + i];
            }
        }
        __syncthreads();
        for (int64_t r = r0 + warp; r < r1; r += TT / 32) {
            const int64_t s = row_start[r] - base;
            const int len = row_len[r];
            const uint32_t lr = (uint32_t)(r - r0);
            int lnext = lcur[lr];
            unsigned long long rsum = 0ull;
            for (int k0 = 0; k0 < len; k0 += 32) {
                const int k = k0 + lane;
                const bool act = k < len;
                int q = 0;
                int32_t cur = -1;
                if (act) {
                    q = cols[s + k];
                    cur = cursor[(q >> cb) - J0];
                }
                const bool left = act && cur < 0;
                const unsigned ml = __ballot_sync(FULL, left);
                // this row's pairs that fall in one dense tile take consecutive slots, so
                // that sigma meets them as runs of one row
                const bool dense = act && !left;
                const int bin = (int)((q >> cb) - J0);
                const unsigned grp = __match_any_sync(FULL, dense ? bin : (int)(0x80000000u | (unsigned)lane));
                const int leader = __ffs(grp) - 1;
                int slot = 0;
                if (dense && lane == leader) slot = atomicAdd(&cursor[bin], __popc(grp));
                slot = __shfl_sync(FULL, slot, leader);
                int64_t pos = 0;
                uint32_t code = 0;
                if (act) {
                    if (left) {
                        pos = el0 + lnext + __popc(ml & lt);
                        code = (uint32_t)q;
                    } else {
                        pos = el0 + slot + __popc(grp & lt);
                        code = (lr << cb) | ((uint32_t)q & cmask);
                    }
                    const VIN v = vin[s + k];
                    const bool in = pos >= 0 && pos < el_cap;  // always true: see the count pass
                    if (in) {
                        el_idx[pos] = code;
                        vout[pos] = v;
                    }
                    double av = fabs((double)v);
                    if (vlo_in) {
                        if (in) vlo_out[pos] = vlo_in[s + k];
                        av = fabs((double)v + (double)vlo_in[s + k]);
                    }
                    const unsigned long long ai = (unsigned long long)llrint(av * 4294967296.0);
                    rsum += ai;
                    atomicAdd(row_abs + q, ai);
                }
                lnext += __popc(ml);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) rsum += __shfl_xor_sync(FULL, rsum, o);
            if (lane == 0 && rsum) atomicAdd(row_abs + r, rsum);
        }
        __syncthreads();
    }
}

__global__ void k_widen(const int32_t* __restrict__ a, int64_t n, int64_t* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

__global__ void k_max_u64(const unsigned long long* __restrict__ a, int64_t n, unsigned long long* __restrict__ out) {
    unsigned long long m = 0ull;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, a[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ---------------------------------------------------------------- sigma

template <typename X>
__global__ void k_absmax(const X* __restrict__ x, int64_t n, unsigned long long* __restrict__ out) {
    double m = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs((double)x[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// scalars[0]: max |x| (bits), scalars[1] <- 2^s, scalars[2] <- 2^-s, scalars[3]: work-unit counter
__global__ void k_fixed_scale(double* __restrict__ scalars, double row_abs_max, int smax, int top) {
    const double xmax = __longlong_as_double(*(const long long*)scalars);
    const double bound = row_abs_max * xmax;
    int s = 0;
    if (bound > 0.0 && isfinite(bound)) s = top - ilogb(bound);
    s = max(-smax, min(smax, s));
    scalars[1] = ldexp(1.0, s);
    scalars[2] = ldexp(1.0, -s);
    reinterpret_cast<unsigned long long*>(scalars)[3] = 0ull;
}

// FP32 / FP64 sums added with native global atomics (the window flushes).
template <typename X>
struct AccFloat {
    using T = X;
    __device__ __forceinline__ static void add(T* a, T v) { atomicAdd(a, v); }
};

// Four FP32 sums added to four consecutive global floats (16-byte aligned) by one
// vector reduction.
__device__ __forceinline__ void red_add_v4(float* a, const float4 v) {
    asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(a), "f"(v.x), "f"(v.y),
                 "f"(v.z), "f"(v.w)
                 : "memory");
}

// Adds the window sums src[0, n) (shared) to dst[0, n) (global), zeros skipped.  FP32
// sums into a 16-byte aligned destination go four at a time through vector reductions,
// a quarter of the L2 atomic operations.
template <typename A>
__device__ __forceinline__ void flush_window(typename A::T* __restrict__ dst, const typename A::T* __restrict__ src,
                                             int n) {
    using T = typename A::T;
    int i0 = 0;
    if constexpr (std::is_same<T, float>::value) {
        if ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0) {
            const int n4 = n >> 2;
            for (int i = threadIdx.x; i < n4; i += TT) {
                const float4 a = reinterpret_cast<const float4*>(src)[i];
                if (a.x != 0.f || a.y != 0.f || a.z != 0.f || a.w != 0.f) red_add_v4(dst + 4 * i, a);
            }
            i0 = 4 * n4;
        }
    }
    for (int i = i0 + threadIdx.x; i < n; i += TT) {
        const T a = src[i];
        if (a != 0) A::add(dst + i, a);
    }
}

// Stages x[0, n) into shared memory (16-byte vector loads when x is aligned).
template <typename X>
__device__ __forceinline__ void stage_window(X* __restrict__ dst, const X* __restrict__ x, int n) {
    constexpr int PER = 16 / sizeof(X);
    int i0 = 0;
    if ((reinterpret_cast<uintptr_t>(x) & 15u) == 0) {
        const int nv = n / PER;
        for (int i = threadIdx.x; i < nv; i += TT) reinterpret_cast<uint4*>(dst)[i] = __ldg(reinterpret_cast<const uint4*>(x) + i);
        i0 = nv * PER;
    }
    for (int i = i0 + threadIdx.x; i < n; i += TT) dst[i] = x[i];
}

// Four consecutive stored values (16-byte aligned element index e) as the vector type.
template <typename V, typename X, bool VLO>
__device__ __forceinline__ void load4(const V* __restrict__ vals, const float* __restrict__ vlo, int64_t e,
                                      X (&v)[4]) {
    if constexpr (std::is_same<V, double>::value) {
        const double2 a = __ldcs(reinterpret_cast<const double2*>(vals + e));
        const double2 b = __ldcs(reinterpret_cast<const double2*>(vals + e + 2));
        v[0] = (X)a.x; v[1] = (X)a.y; v[2] = (X)b.x; v[3] = (X)b.y;
    } else {
        const float4 a = __ldcs(reinterpret_cast<const float4*>(vals + e));
        v[0] = (X)a.x; v[1] = (X)a.y; v[2] = (X)a.z; v[3] = (X)a.w;
        if constexpr (VLO) {
            const float4 l = __ldcs(reinterpret_cast<const float4*>(vlo + e));
            v[0] += (X)l.x; v[1] += (X)l.y; v[2] += (X)l.z; v[3] += (X)l.w;
        }
    }
}

// Fixed-point tile sigma.  Shared-memory integer atomics are single instructions,
// where FP32 shared atomics are compare-and-swap loops and 64-bit ones slower still
// (measured on B200: 7.9, 2.6 and 1.5 per clock per SM), so each tile's row and column
// window sums are formed in 32-bit integers.  Every product is scaled by 2^s_t, s_t
// chosen from the tile's bound (its largest sum of |H| over one row or one column,
// times max |x|) so that no window sum exceeds 2^30, and rounded to an integer a
// (NP = 1), or to a + b 2^-20 with two integers (NP = 2: about 50 significant bits,
// for FP64 vectors).  Each product is rounded once, by a fixed rule, and integer sums
// do not depend on their order.  EXACT: the window sums are converted, again by a
// fixed rule, to the 64-bit fixed point of the whole sigma (scale 2^S, S from the row
// sums of |H|) and added with 64-bit global atomics, so sigma is bitwise reproducible
// and ranks' partial sums add exactly; otherwise (FP32 vectors) they are converted to
// FP32 and added with FP32 vector reductions.  Leftover pairs: one warp per row,
// private row sum, column sums by global atomics of the rounded products.
template <typename X, typename V, bool VLO, int NP, bool EXACT>
__global__ void __launch_bounds__(TT) k_sigma_fx(
    int64_t N, int64_t n_units, const int64_t* __restrict__ units, int rb, int cb,
    const int32_t* __restrict__ tile_win, const int32_t* __restrict__ tile_len, const int64_t* __restrict__ tile_off,
    const float* __restrict__ tile_bound, const int64_t* __restrict__ left_off, const int32_t* __restrict__ left_len,
    const uint32_t* __restrict__ el_idx, const V* __restrict__ vals, const float* __restrict__ vlo,
    const X* __restrict__ x, void* __restrict__ acc_out, double* __restrict__ scalars) {
    using Y = typename std::conditional<EXACT, long long, X>::type;  // unit row accumulator
    extern __shared__ __align__(16) unsigned char sm[];
    const int R = 1 << rb, C = 1 << cb;
    X* xP = reinterpret_cast<X*>(sm);
    X* xJ = xP + R;
    Y* yP = reinterpret_cast<Y*>(xJ + C);
    int* yPa = reinterpret_cast<int*>(yP + R);
    int* yPb = yPa + R;
    int* yJa = yPb + (NP == 2 ? R : 0);
    int* yJb = yJa + C;
    __shared__ long long s_unit;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t cmask = (uint32_t)C - 1u;
    const double xmax = __longlong_as_double(*reinterpret_cast<const long long*>(scalars));
    const double gscale = scalars[1];  // 2^S (EXACT)
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(scalars) + 3;
    long long* acc_ll = reinterpret_cast<long long*>(acc_out);
    X* acc_x = reinterpret_cast<X*>(acc_out);
    for (;;) {
        if (threadIdx.x == 0) s_unit = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const int64_t u = s_unit;
        if (u >= n_units) break;
        const int64_t tb = units[3 * u], te = units[3 * u + 1], pl = units[3 * u + 2];
        const int64_t P = pl >> 1;
        const bool with_left = (pl & 1) != 0;
        const int64_t r0 = P << rb;
        const int nr = (int)min((int64_t)R, N - r0);
        stage_window<X>(xP, x + r0, nr);
        for (int i = threadIdx.x; i < R; i += TT) {
            yP[i] = 0;
            yPa[i] = 0;
            if (NP == 2) yPb[i] = 0;
        }
        __syncthreads();
        for (int64_t t = tb; t < te; t++) {
            const int64_t c0 = (int64_t)tile_win[t] << cb;
            const int w = (int)min((int64_t)C, N - c0);
            const int64_t e0 = tile_off[t];
            const int len = tile_len[t];
            const double bt = (double)tile_bound[t] * xmax;
            int sh = 0;
            if (bt > 0.0 && isfinite(bt)) sh = 29 - ilogb(bt);
            sh = max(-200, min(200, sh));
            const X sc = (X)ldexp(1.0, sh);
            // a window sum (A, B) in the unit of the whole sigma: A 2^(S - s_t) + B 2^(S - s_t - 20)
            const double fa = ldexp(gscale, -sh), fb = ldexp(gscale, -sh - 20);
            const X inv = (X)ldexp(1.0, -sh);
            stage_window<X>(xJ, x + c0, w);
            for (int i = threadIdx.x; i < w; i += TT) {
                yJa[i] = 0;
                if (NP == 2) yJb[i] = 0;
            }
            __syncthreads();
            // one product to its integer parts
            auto split = [&](X p, int& a, int& b) {
                if constexpr (std::is_same<X, double>::value) {
                    a = __double2int_rn(p);
                    if (NP == 2) b = __double2int_rn((p - (double)a) * 1048576.0);
                } else {
                    a = __float2int_rn(p);
                    if (NP == 2) b = __float2int_rn((p - (float)a) * 1048576.f);
                }
            };
            auto add_col = [&](uint32_t lc, X p) {
                int a = 0, b = 0;
                split(p, a, b);
                atomicAdd(yJa + lc, a);
                if (NP == 2) atomicAdd(yJb + lc, b);
            };
            const int head = (int)min((int64_t)len, (4 - (e0 & 3)) & 3);
            const int64_t eb = e0 + head;
            const int nblk = (len - head) >> 2;
            const int rest = len - head - 4 * nblk;
            if ((int)threadIdx.x < head + rest) {
                const int64_t e = (int)threadIdx.x < head ? e0 + threadIdx.x : eb + 4 * nblk + (threadIdx.x - head);
                const uint32_t uu = __ldcs(el_idx + e);
                X v = (X)__ldcs(vals + e);
                if constexpr (VLO) v += (X)__ldcs(vlo + e);
                v *= sc;
                const uint32_t lr = uu >> cb, lc = uu & cmask;
                if (lr < (uint32_t)nr && lc < (uint32_t)w) {  // never false for a valid layout
                    int a = 0, b = 0;
                    split(v * xJ[lc], a, b);
                    atomicAdd(yPa + lr, a);
                    if (NP == 2) atomicAdd(yPb + lr, b);
                    add_col(lc, v * xP[lr]);
                }
            }
            auto sum_block = [&](const uint4 u4, const X (&v)[4]) {
                const uint32_t uq[4] = {u4.x, u4.y, u4.z, u4.w};
                uint32_t rcur = uq[0] >> cb;
                int ra = 0, rbb = 0;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const uint32_t lr = uq[j] >> cb, lc = uq[j] & cmask;
                    if (lr >= (uint32_t)nr || lc >= (uint32_t)w) continue;  // never taken for a valid layout
                    const X vs = v[j] * sc;
                    int a = 0, b = 0;
                    split(vs * xJ[lc], a, b);
                    add_col(lc, vs * xP[lr]);
                    if (lr != rcur) {
                        if ((ra | rbb) != 0 && rcur < (uint32_t)nr) {
                            atomicAdd(yPa + rcur, ra);
                            if (NP == 2) atomicAdd(yPb + rcur, rbb);
                        }
                        rcur = lr;
                        ra = rbb = 0;
                    }
                    ra += a;
                    rbb += b;
                }
                if ((ra | rbb) != 0 && rcur < (uint32_t)nr) {
                    atomicAdd(yPa + rcur, ra);
                    if (NP == 2) atomicAdd(yPb + rcur, rbb);
                }
            };
            for (int bk = threadIdx.x; bk < nblk; bk += 2 * TT) {
                const bool two = bk + TT < nblk;
                const int64_t e1 = eb + 4 * (int64_t)bk, e2 = e1 + 4 * (int64_t)TT;
                const uint4 u1 = __ldcs(reinterpret_cast<const uint4*>(el_idx + e1));
                X v1[4], v2[4];
                load4<V, X, VLO>(vals, vlo, e1, v1);
                uint4 u2 = make_uint4(0, 0, 0, 0);
                if (two) {
                    u2 = __ldcs(reinterpret_cast<const uint4*>(el_idx + e2));
                    load4<V, X, VLO>(vals, vlo, e2, v2);
                }
                sum_block(u1, v1);
                if (two) sum_block(u2, v2);
            }
            __syncthreads();
            // column window sums to the global accumulator
            if constexpr (EXACT) {
                for (int i = threadIdx.x; i < w; i += TT) {
                    const int a = yJa[i], b = NP == 2 ? yJb[i] : 0;
                    if ((a | b) != 0)
                        atomicAdd(reinterpret_cast<unsigned long long*>(acc_ll + c0 + i),
                                  (unsigned long long)llrint((double)a * fa + (double)b * fb));
                }
            } else {
                static_assert(EXACT || (std::is_same<X, float>::value && NP == 1), "FP32 sums: one part");
                if ((reinterpret_cast<uintptr_t>(acc_x + c0) & 15u) == 0) {
                    for (int i = threadIdx.x; i < (w >> 2); i += TT) {
                        const int4 a = reinterpret_cast<const int4*>(yJa)[i];
                        if (a.x | a.y | a.z | a.w)
                            red_add_v4(reinterpret_cast<float*>(acc_x) + c0 + 4 * i,
                                       make_float4((float)a.x * (float)inv, (float)a.y * (float)inv,
                                                   (float)a.z * (float)inv, (float)a.w * (float)inv));
                    }
                    for (int i = 4 * (w >> 2) + threadIdx.x; i < w; i += TT)
                        if (yJa[i] != 0) atomicAdd(acc_x + c0 + i, (X)yJa[i] * inv);
                } else {
                    for (int i = threadIdx.x; i < w; i += TT)
                        if (yJa[i] != 0) atomicAdd(acc_x + c0 + i, (X)yJa[i] * inv);
                }
            }
            // row window sums into the unit's accumulator (row i belongs to this thread here)
            for (int i = threadIdx.x; i < nr; i += TT) {
                const int a = yPa[i], b = NP == 2 ? yPb[i] : 0;
                if ((a | b) != 0) {
                    if constexpr (EXACT) yP[i] += llrint((double)a * fa + (double)b * fb);
                    else yP[i] += (X)a * inv;
                    yPa[i] = 0;
                    if (NP == 2) yPb[i] = 0;
                }
            }
            __syncthreads();
        }
        // leftover pairs: one warp per row, private row sum, column sums by global atomics
        for (int i = warp; with_left && i < nr; i += TT / 32) {
            const int64_t s = left_off[r0 + i];
            const int len = left_len[r0 + i];
            const X xr = xP[i];
            X rs = 0;
            for (int k = lane; k < len; k += 32) {
                const uint32_t q = __ldcs(el_idx + s + k);
                X v = (X)__ldcs(vals + s + k);
                if constexpr (VLO) v += (X)__ldcs(vlo + s + k);
                if (q >= (uint64_t)N) continue;  // never taken for a valid layout
                rs += v * __ldg(x + q);
                if constexpr (EXACT)
                    atomicAdd(reinterpret_cast<unsigned long long*>(acc_ll + q),
                              (unsigned long long)llrint((double)(v * xr) * gscale));
                else
                    atomicAdd(acc_x + q, v * xr);
            }
            // fixed lane order: the warp sum does not depend on timing
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) rs += __shfl_xor_sync(FULL, rs, o);
            if (lane == 0) {
                if constexpr (EXACT) yP[i] += llrint((double)rs * gscale);
                else yP[i] += rs;
            }
        }
        __syncthreads();
        if constexpr (EXACT) {
            for (int i = threadIdx.x; i < nr; i += TT)
                if (yP[i] != 0)
                    atomicAdd(reinterpret_cast<unsigned long long*>(acc_ll + r0 + i), (unsigned long long)yP[i]);
        } else {
            flush_window<AccFloat<X>>(acc_x + r0, yP, nr);
        }
        __syncthreads();
    }
}

// Per tile: the largest sum of |value| over one of its rows or columns, the bound that
// the fixed-point sigma scales each tile by (FP32 values of MIXED storage: the FP32
// remainder is below 2^-24 of the value, inside the bound's margin).
template <typename V>
__global__ void __launch_bounds__(TT) k_tile_bounds(int64_t n_tiles, int rb, int cb,
                                                   const int32_t* __restrict__ tile_len,
                                                   const int64_t* __restrict__ tile_off,
                                                   const uint32_t* __restrict__ el_idx,
                                                   const V* __restrict__ vals, float* __restrict__ bound) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int R = 1 << rb, C = 1 << cb;
    float* rs = reinterpret_cast<float*>(sm);
    float* cs = rs + R;
    __shared__ float s_max[TT / 32];
    const uint32_t cmask = (uint32_t)C - 1u;
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        for (int i = threadIdx.x; i < R + C; i += TT) rs[i] = 0.f;
        __syncthreads();
        const int64_t e0 = tile_off[t];
        const int len = tile_len[t];
        for (int k = threadIdx.x; k < len; k += TT) {
            const uint32_t u = el_idx[e0 + k];
            const float a = (float)fabs((double)vals[e0 + k]) * (1.f + 0x1p-20f);
            const uint32_t lr = u >> cb, lc = u & cmask;
            if (lr < (uint32_t)R) atomicAdd(rs + lr, a);
            atomicAdd(cs + lc, a);
        }
        __syncthreads();
        float m = 0.f;
        for (int i = threadIdx.x; i < R + C; i += TT) m = fmaxf(m, rs[i]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
        if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            float b = 0.f;
            for (int k = 0; k < TT / 32; k++) b = fmaxf(b, s_max[k]);
            // FP32 sums of |value| round down by at most a few ulps of the bound
            bound[t] = b * (1.f + 0x1p-16f);
        }
        __syncthreads();
    }
}

// y = diag x + acc (fixed point: acc 2^-s)
template <typename X, typename T>
__global__ void k_fixed_finish(int64_t N, const double* __restrict__ diag, const X* __restrict__ x,
                               const T* __restrict__ acc, const double* __restrict__ scalars,
                               X* __restrict__ y) {
    const double inv = std::is_same<T, long long>::value ? scalars[2] : 1.0;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
        y[p] = (X)(diag[p] * (double)x[p] + (double)acc[p] * inv);
}

// Calls f(p, q, v) for every stored pair (p < q, internal indices, FP64 value):
// one CTA per panel, its dense tiles and then its leftover rows.
template <typename V, bool VLO, typename F>
__global__ void __launch_bounds__(TT) k_tiles_each(int64_t N, int64_t p_lo, int64_t p_hi, int rb, int cb,
                                                  const int64_t* __restrict__ panel_tile,
                                                  const int32_t* __restrict__ tile_win,
                                                  const int32_t* __restrict__ tile_len,
                                                  const int64_t* __restrict__ tile_off,
                                                  const int64_t* __restrict__ left_off,
                                                  const int32_t* __restrict__ left_len,
                                                  const uint32_t* __restrict__ el_idx, const V* __restrict__ vals,
                                                  const float* __restrict__ vlo, F f) {
    const uint32_t cmask = (1u << cb) - 1u;
    for (int64_t P = p_lo + blockIdx.x; P < p_hi; P += gridDim.x) {
        const int64_t r0 = P << rb;
        for (int64_t t = panel_tile[P]; t < panel_tile[P + 1]; t++) {
            const int64_t c0 = (int64_t)tile_win[t] << cb, e0 = tile_off[t];
            for (int k = threadIdx.x; k < tile_len[t]; k += TT) {
                const uint32_t u = el_idx[e0 + k];
                double v = (double)vals[e0 + k];
                if constexpr (VLO) v += (double)vlo[e0 + k];
                f(r0 + (u >> cb), c0 + (u & cmask), v, e0 + k);
            }
        }
        const int nr = (int)min((int64_t)1 << rb, N - r0);
        for (int i = 0; i < nr; i++) {
            const int64_t s = left_off[r0 + i];
            for (int k = threadIdx.x; k < left_len[r0 + i]; k += TT) {
                double v = (double)vals[s + k];
                if constexpr (VLO) v += (double)vlo[s + k];
                f(r0 + i, (int64_t)el_idx[s + k], v, s + k);
            }
        }
    }
}

struct CooOut {
    int32_t* p;
    int32_t* q;
    double* v;
    __device__ void operator()(int64_t pp, int64_t qq, double vv, int64_t e) const {
        p[e] = (int32_t)pp;
        q[e] = (int32_t)qq;
        v[e] = vv;
    }
};

struct SelfEnergyAdd {
    const double* diag;
    double energy, gmin;
    double* out;
    __device__ void operator()(int64_t pp, int64_t qq, double vv, int64_t) const {
        const double v2 = vv * vv;
        atomicAdd(out + pp, -v2 / fmax(diag[qq] - energy, gmin));
        atomicAdd(out + qq, -v2 / fmax(diag[pp] - energy, gmin));
    }
};

// Stored pairs that touch a marked row (bitmap over internal indices), in the caller's
// indices, both orientations: (row, column, value) with the row marked.
struct RowFilter {
    const uint32_t* mark;
    const int32_t* orig;
    int64_t* out_r;
    int64_t* out_c;
    double* out_v;
    unsigned long long* count;
    unsigned long long cap;
    __device__ void emit(int64_t r, int64_t c, double v) const {
        const unsigned long long k = atomicAdd(count, 1ull);
        if (k < cap) {
            out_r[k] = orig[r];
            out_c[k] = orig[c];
            out_v[k] = v;
        }
    }
    __device__ void operator()(int64_t pp, int64_t qq, double vv, int64_t) const {
        if ((mark[pp >> 5] >> (pp & 31)) & 1u) emit(pp, qq, vv);
        if ((mark[qq >> 5] >> (qq & 31)) & 1u) emit(qq, pp, vv);
    }
};

template <typename F>
int tiles_each(risqgpu* h, F f) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(h->part_p_hi - h->part_p_lo, (int64_t)num_sms(h) * 8));
#define RQ_EACH(V, VLO, vals, lo)                                                                                   \
    k_tiles_each<V, VLO, F><<<grid, TT, 0, h->stream>>>((int64_t)h->N, h->part_p_lo, h->part_p_hi, h->tile_rb,      \
                                                         h->tile_cb,                                                  \
                                                         h->d_panel_tile, h->d_tile_win, h->d_tile_len,             \
                                                         h->d_tile_off, h->d_left_off, h->d_left_len, h->d_el_idx, \
                                                         vals, lo, f)
    if (h->precision == RISQGPU_FP64) RQ_EACH(double, false, h->d_val64, nullptr);
    else if (h->precision == RISQGPU_MIXED) RQ_EACH(float, true, h->d_val32, h->d_val_lo);
    else RQ_EACH(float, false, h->d_val32, nullptr);
#undef RQ_EACH
    return check_launch(h, "tiled pairs");
}

inline int grid_n(risqgpu* h, int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms(h) * 16));
}

template <typename X, typename V, bool VLO, int NP, bool EXACT>
int launch_fx(risqgpu* h, const X* x, X* y, const V* vals, const float* vlo) {
    using Y = typename std::conditional<EXACT, long long, X>::type;
    const int64_t N = (int64_t)h->N;
    const int R = 1 << h->tile_rb, C = 1 << h->tile_cb;
    const size_t smem = (size_t)(R + C) * sizeof(X) + (size_t)R * sizeof(Y) + (size_t)(R + C) * 4 * NP;
    auto kern = k_sigma_fx<X, V, VLO, NP, EXACT>;
    static int attr_set[64] = {0};
    const int dev = h->device & 63;
    if (attr_set[dev] < (int)smem) {
        RQ_CUDA(h, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set[dev] = (int)smem;
    }
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, TT, smem);
    const int grid =
        (int)std::max<int64_t>(1, std::min<int64_t>(h->n_units, (int64_t)num_sms(h) * std::max(occ, 1)));
    RQ_CUDA(h, cudaMemsetAsync(h->d_acc, 0, sizeof(long long) * N, h->stream));
    RQ_CUDA(h, cudaMemsetAsync(h->d_sig_scalars, 0, sizeof(double), h->stream));
    k_absmax<X><<<grid_n(h, N), 256, 0, h->stream>>>(x, N, reinterpret_cast<unsigned long long*>(h->d_sig_scalars));
    k_fixed_scale<<<1, 1, 0, h->stream>>>(h->d_sig_scalars, h->h_row_abs_max,
                                         std::is_same<X, float>::value ? 100 : 1000, 61);
    kern<<<grid, TT, smem, h->stream>>>(N, h->n_units, h->d_units, h->tile_rb, h->tile_cb, h->d_tile_win,
                                       h->d_tile_len, h->d_tile_off, h->d_tile_bound, h->d_left_off, h->d_left_len,
                                       h->d_el_idx, vals, vlo, x, h->d_acc, h->d_sig_scalars);
    RQ_TRY(check_launch(h, "sigma (tiles)"));
    // with a row-block partition every rank summed its own panels: the exact integer
    // sums are added across the ranks
    if (EXACT && h->part_n > 1) RQ_TRY(part_allreduce(h, h->d_acc, (size_t)N));
    k_fixed_finish<X, Y><<<grid_n(h, N), 256, 0, h->stream>>>(N, h->d_diag, x, reinterpret_cast<const Y*>(h->d_acc),
                                                             h->d_sig_scalars, y);
    return check_launch(h, "sigma (tiles)");
}

// FP32 vectors sum in 32-bit fixed point per tile and FP32 across tiles unless the
// handle asked for reproducible sums or is partitioned (the ranks' sums must add
// exactly); those, and FP64 vectors (two 32-bit parts), add in 64-bit fixed point.
template <typename V, typename X, bool VLO>
int launch_tiles(risqgpu* h, const X* x, X* y, const V* vals, const float* vlo) {
    if constexpr (std::is_same<X, float>::value) {
        if (!h->reproducible && h->part_n == 1)
            return launch_fx<float, float, false, 1, false>(h, x, y, h->d_val32, nullptr);
        return launch_fx<float, float, false, 1, true>(h, x, y, h->d_val32, nullptr);
    } else {
        return launch_fx<double, V, VLO, 2, true>(h, x, y, vals, vlo);
    }
}

// Grow a device array to hold `need` entries, keeping the first `keep`.
template <typename T>
int grow(risqgpu* h, T*& p, size_t& capacity, size_t need, size_t keep) {
    if (need <= capacity) return RISQGPU_OK;
    size_t nc = std::max(need, capacity + capacity / 2);
    T* q = nullptr;
    RQ_TRY(dalloc(h, q, nc));
    if (p && keep) RQ_CUDA(h, cudaMemcpyAsync(q, p, sizeof(T) * keep, cudaMemcpyDeviceToDevice, h->stream));
    RQ_TRY(sync(h, "tile arrays"));
    dfree(p);
    p = q;
    capacity = nc;
    return RISQGPU_OK;
}

}  // namespace

int part_allreduce(risqgpu* h, void* buf_dev, size_t count) {
    if (!h->part_reduce) {
        h->err = "partitioned handle without a reduce function";
        return RISQGPU_ERR_INVALID;
    }
    if (h->part_reduce(buf_dev, count, (void*)h->stream, h->part_user) != 0) {
        h->err = "the caller's all-reduce failed";
        return RISQGPU_ERR_CUDA;
    }
    return check_launch(h, "all-reduce");
}

int tile_shape(int64_t N, int& rb, int& cb) {
    // measured on the config-1 set (1.1e10 pairs): 1024 x 2048 tiles beat 512 x 4096,
    // 256 x 4096, 1024 x 4096 and 2048 x 4096 by 9-18 % (FP32) and 13-32 % (FP64)
    rb = 10;  // 1024 rows per panel
    cb = 11;  // 2048 columns per window
    while (cb < 16 && ((N + ((int64_t)1 << cb) - 1) >> cb) > MAX_BINS) cb++;
    return ((N + ((int64_t)1 << cb) - 1) >> cb) <= MAX_BINS ? RISQGPU_OK : RISQGPU_ERR_INVALID;
}

int TileBuilder::begin(risqgpu* h_, int64_t n_panels, int64_t element_capacity) {
    h = h_;
    el_cap = element_capacity;
    const int64_t N = (int64_t)h->N;
    // the build released the previous tiles (free_csr) and has already allocated the
    // element arrays (d_el_idx and the values), which must survive here
    h->tiled = false;
    h->n_tiles = 0;
    h->n_dense_el = 0;
    h->n_panels = n_panels;
    RQ_TRY(dalloc(h, h->d_panel_tile, (size_t)n_panels + 1));
    RQ_TRY(dalloc(h, h->d_left_off, (size_t)N));
    RQ_TRY(dalloc(h, h->d_left_len, (size_t)N));
    RQ_TRY(dalloc(h, row_abs, (size_t)N));
    RQ_TRY(dalloc(h, absmax, 1));
    RQ_CUDA(h, cudaMemsetAsync(row_abs, 0, sizeof(unsigned long long) * N, h->stream));
    RQ_CUDA(h, cudaMemsetAsync(absmax, 0, sizeof(unsigned long long), h->stream));
    tile_cap = 0;
    el_next = tile_next = 0;
    panel_el.assign((size_t)n_panels + 1, 0);
    return RISQGPU_OK;
}

template <typename VIN>
int TileBuilder::chunk(int64_t p_lo, int64_t p_hi, const int64_t* row_start, int64_t base, const int32_t* row_len,
                       const int32_t* cols, const VIN* vin, const float* vlo_in, VIN* vout, float* vlo_out) {
    const int64_t N = (int64_t)h->N;
    const int64_t np = p_hi - p_lo;
    if (np <= 0) return RISQGPU_OK;
    int64_t *nel = nullptr, *ndense = nullptr, *el_off = nullptr, *t_off = nullptr, *nt64 = nullptr;
    int32_t* nt = nullptr;
    char* tmp = nullptr;
    ScopedFree<7> release(nel, ndense, el_off, t_off, nt64, nt, tmp);
    RQ_TRY(dalloc(h, nel, np));
    RQ_TRY(dalloc(h, ndense, np));
    RQ_TRY(dalloc(h, el_off, np));
    RQ_TRY(dalloc(h, t_off, np));
    RQ_TRY(dalloc(h, nt64, np));
    RQ_TRY(dalloc(h, nt, np));
    const int rb = h->tile_rb, cb = h->tile_cb;
    const size_t smem_count = sizeof(int32_t) * MAX_BINS;
    const size_t smem_scatter = sizeof(int32_t) * (MAX_BINS + ((size_t)1 << rb));
    RQ_CUDA(h, cudaFuncSetAttribute(k_tile_count, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_count));
    RQ_CUDA(h, cudaFuncSetAttribute(k_tile_scatter<VIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_scatter));
    const int grid = (int)std::min<int64_t>(np, (int64_t)num_sms(h) * 2);
    k_tile_count<<<grid, TT, smem_count, h->stream>>>(N, p_lo, p_hi, rb, cb, row_start, base, row_len, cols, nel,
                                                      ndense, nt, h->d_left_len);
    RQ_TRY(check_launch(h, "tile count"));
    k_widen<<<grid_n(h, np), 256, 0, h->stream>>>(nt, np, nt64);
    size_t tb1 = 0, tb2 = 0;
    cub::DeviceScan::ExclusiveScan(nullptr, tb1, nel, el_off, cub::Sum(), (int64_t)el_next, (int)np, h->stream);
    cub::DeviceScan::ExclusiveScan(nullptr, tb2, nt64, t_off, cub::Sum(), (int64_t)tile_next, (int)np, h->stream);
    RQ_TRY(dalloc(h, tmp, std::max(tb1, tb2)));
    cub::DeviceScan::ExclusiveScan(tmp, tb1, nel, el_off, cub::Sum(), (int64_t)el_next, (int)np, h->stream);
    cub::DeviceScan::ExclusiveScan(tmp, tb2, nt64, t_off, cub::Sum(), (int64_t)tile_next, (int)np, h->stream);
    RQ_TRY(check_launch(h, "tile offsets"));
    int64_t last[4];
    RQ_CUDA(h, cudaMemcpyAsync(last + 0, el_off + np - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(last + 1, nel + np - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(last + 2, t_off + np - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(last + 3, nt64 + np - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
    RQ_CUDA(h, cudaMemcpyAsync(panel_el.data() + p_lo, el_off, sizeof(int64_t) * np, cudaMemcpyDeviceToHost,
                               h->stream));
    RQ_TRY(sync(h, "tile offsets"));
    const int64_t el_end = last[0] + last[1], t_end = last[2] + last[3];
    if (el_end > el_cap) {
        h->err = "tiled layout: " + std::to_string(el_end) + " elements exceed the " + std::to_string(el_cap) +
                 " slots counted";
        return RISQGPU_ERR_INVALID;
    }
    size_t c1 = tile_cap, c2 = tile_cap, c3 = tile_cap;
    RQ_TRY(grow(h, h->d_tile_win, c1, (size_t)t_end, (size_t)tile_next));
    RQ_TRY(grow(h, h->d_tile_len, c2, (size_t)t_end, (size_t)tile_next));
    RQ_TRY(grow(h, h->d_tile_off, c3, (size_t)t_end, (size_t)tile_next));
    tile_cap = c1;
    RQ_CUDA(h, cudaMemcpyAsync(h->d_panel_tile + p_lo, t_off, sizeof(int64_t) * np, cudaMemcpyDeviceToDevice,
                               h->stream));
    k_tile_scatter<VIN><<<grid, TT, smem_scatter, h->stream>>>(
        N, p_lo, p_hi, rb, cb, row_start, base, row_len, cols, vin, vlo_in, el_off, t_off, ndense, h->d_left_len,
        h->d_tile_win, h->d_tile_len, h->d_tile_off, h->d_left_off, h->d_el_idx, vout, vlo_out, row_abs,
        el_cap, (int64_t)tile_cap);
    RQ_TRY(check_launch(h, "tile scatter"));
    RQ_TRY(sync(h, "tile scatter"));
    el_next = el_end;
    tile_next = t_end;
    return RISQGPU_OK;
}

int TileBuilder::finish() {
    const int64_t N = (int64_t)h->N;
    // the tile range of this handle's last panel ends here (the panels of other ranks
    // are not held)
    RQ_CUDA(h, cudaMemcpyAsync(h->d_panel_tile + h->part_p_hi, &tile_next, sizeof(int64_t), cudaMemcpyHostToDevice,
                               h->stream));
    // row sums of |H| over both triangles: with a partition each rank holds part of every
    // row's sum, so the exact integer sums are added across the ranks first
    if (h->part_n > 1) RQ_TRY(part_allreduce(h, row_abs, (size_t)N));
    k_max_u64<<<grid_n(h, N), 256, 0, h->stream>>>(row_abs, N, absmax);
    unsigned long long mi = 0;
    RQ_CUDA(h, cudaMemcpyAsync(&mi, absmax, sizeof(mi), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "row sums"));
    // each |H_pq| was rounded to a multiple of 2^-32: the margin covers that rounding
    h->h_row_abs_max = 1.01 * ((double)mi / 4294967296.0) + 1e-6;
    h->n_tiles = tile_next;
    h->n_dense_el = 0;
    if (tile_next > 0) {
        int64_t* sum = nullptr;
        char* tmp = nullptr;
        ScopedFree<2> release(sum, tmp);
        RQ_TRY(dalloc(h, sum, 1));
        size_t tb = 0;
        cub::DeviceReduce::Sum(nullptr, tb, h->d_tile_len, sum, (int)tile_next, h->stream);
        RQ_TRY(dalloc(h, tmp, tb));
        cub::DeviceReduce::Sum(tmp, tb, h->d_tile_len, sum, (int)tile_next, h->stream);
        int64_t v = 0;
        RQ_CUDA(h, cudaMemcpyAsync(&v, sum, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
        RQ_TRY(sync(h, "dense pairs"));
        h->n_dense_el = (uint64_t)v;
    }
    RQ_TRY(make_units());
    if (tile_next > 0) {
        const int R = 1 << h->tile_rb, C = 1 << h->tile_cb;
        const size_t smem = (size_t)(R + C) * sizeof(float);
        RQ_TRY(dalloc(h, h->d_tile_bound, (size_t)tile_next));
        const int grid = (int)std::min<int64_t>(tile_next, (int64_t)num_sms(h) * 8);
        if (h->d_val64) {
            RQ_CUDA(h, cudaFuncSetAttribute(k_tile_bounds<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
            k_tile_bounds<double><<<grid, TT, smem, h->stream>>>(tile_next, h->tile_rb, h->tile_cb, h->d_tile_len,
                                                                 h->d_tile_off, h->d_el_idx, h->d_val64,
                                                                 h->d_tile_bound);
        } else {
            RQ_CUDA(h, cudaFuncSetAttribute(k_tile_bounds<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
            k_tile_bounds<float><<<grid, TT, smem, h->stream>>>(tile_next, h->tile_rb, h->tile_cb, h->d_tile_len,
                                                                h->d_tile_off, h->d_el_idx, h->d_val32,
                                                                h->d_tile_bound);
        }
        RQ_TRY(check_launch(h, "tile bounds"));
    }
    RQ_TRY(dalloc(h, h->d_acc, (size_t)N));
    RQ_TRY(dalloc(h, h->d_sig_scalars, 4));
    dfree(row_abs);
    dfree(absmax);
    h->tiled = true;
    return RISQGPU_OK;
}

// Sigma work units: each panel's tiles cut into runs of about `target` pairs (the
// panel's leftover pairs go with its last run), largest first, so that the CTAs that
// take units from a counter finish together even when a set has few, uneven panels.
int TileBuilder::make_units() {
    const int64_t p_lo = h->part_p_lo, p_hi = h->part_p_hi;
    panel_el[(size_t)p_hi] = el_next;
    std::vector<int64_t> pt((size_t)(p_hi - p_lo) + 1);
    std::vector<int32_t> tl((size_t)tile_next);
    RQ_CUDA(h, cudaMemcpyAsync(pt.data(), h->d_panel_tile + p_lo, sizeof(int64_t) * pt.size(), cudaMemcpyDeviceToHost,
                               h->stream));
    if (tile_next > 0)
        RQ_CUDA(h, cudaMemcpyAsync(tl.data(), h->d_tile_len, sizeof(int32_t) * tl.size(), cudaMemcpyDeviceToHost,
                                   h->stream));
    RQ_TRY(sync(h, "sigma units"));
    const int64_t total = el_next - panel_el[(size_t)p_lo];
    const int64_t target = std::max<int64_t>(32768, total / ((int64_t)num_sms(h) * 16));
    struct Unit { int64_t tb, te, pl, w; };
    std::vector<Unit> us;
    for (int64_t P = p_lo; P < p_hi; P++) {
        const int64_t tb = pt[(size_t)(P - p_lo)], te = pt[(size_t)(P - p_lo) + 1];
        const int64_t pairs = panel_el[(size_t)P + 1] - panel_el[(size_t)P];
        if (pairs == 0) continue;
        int64_t dense = 0;
        for (int64_t t = tb; t < te; t++) dense += tl[(size_t)t];
        int64_t start = tb, acc = 0;
        for (int64_t t = tb; t < te; t++) {
            acc += tl[(size_t)t];
            if (acc >= target && t + 1 < te) {
                us.push_back({start, t + 1, 2 * P, acc});
                start = t + 1;
                acc = 0;
            }
        }
        us.push_back({start, te, 2 * P + 1, acc + (pairs - dense)});
    }
    std::stable_sort(us.begin(), us.end(), [](const Unit& a, const Unit& b) { return a.w > b.w; });
    std::vector<int64_t> flat(3 * us.size());
    for (size_t i = 0; i < us.size(); i++) {
        flat[3 * i] = us[i].tb;
        flat[3 * i + 1] = us[i].te;
        flat[3 * i + 2] = us[i].pl;
    }
    h->n_units = (int64_t)us.size();
    if (!us.empty()) {
        RQ_TRY(dalloc(h, h->d_units, flat.size()));
        RQ_CUDA(h, cudaMemcpyAsync(h->d_units, flat.data(), sizeof(int64_t) * flat.size(), cudaMemcpyHostToDevice,
                                   h->stream));
        RQ_TRY(sync(h, "sigma units"));
    }
    return RISQGPU_OK;
}

TileBuilder::~TileBuilder() {
    dfree(row_abs);
    dfree(absmax);
}

template int TileBuilder::chunk<double>(int64_t, int64_t, const int64_t*, int64_t, const int32_t*, const int32_t*,
                                        const double*, const float*, double*, float*);
template int TileBuilder::chunk<float>(int64_t, int64_t, const int64_t*, int64_t, const int32_t*, const int32_t*,
                                       const float*, const float*, float*, float*);

// sigma over tiled storage; kind 0: FP64 vectors (FP64 values, or FP32 + remainder),
// 1: FP32 vectors with the FP32 values.
int sigma_tiles(risqgpu* h, const void* x, void* y, int kind) {
    if (kind == 0) {
        if (h->precision == RISQGPU_FP64)
            return launch_tiles<double, double, false>(h, (const double*)x, (double*)y, h->d_val64, nullptr);
        if (h->precision == RISQGPU_MIXED)
            return launch_tiles<float, double, true>(h, (const double*)x, (double*)y, h->d_val32, h->d_val_lo);
        h->err = "FP64 sigma needs FP64 or FP32 + remainder values";
        return RISQGPU_ERR_INVALID;
    }
    if (h->precision == RISQGPU_FP64) {
        h->err = "FP32 sigma needs FP32 values";
        return RISQGPU_ERR_INVALID;
    }
    return launch_tiles<float, float, false>(h, (const float*)x, (float*)y, h->d_val32, nullptr);
}

// Every stored pair of a tiled build as (p, q, value), internal indices, in storage order
// (nnz_upper entries each).
int tiles_coo(risqgpu* h, int32_t* p, int32_t* q, double* v) { return tiles_each(h, CooOut{p, q, v}); }

// out[i] -= sum_j H_ij^2 / max(H_jj - E, gmin) over the stored pairs (out zeroed by the caller).
int tiles_self_energy(risqgpu* h, double energy, double gmin, double* out) {
    return tiles_each(h, SelfEnergyAdd{h->d_diag, energy, gmin, out});
}

int tiles_rows(risqgpu* h, const uint32_t* mark, int64_t* out_r, int64_t* out_c, double* out_v,
               unsigned long long* count, unsigned long long cap) {
    return tiles_each(h, RowFilter{mark, h->d_orig, out_r, out_c, out_v, count, cap});
}

void free_tiles(risqgpu* h) {
    dfree(h->d_panel_tile);
    dfree(h->d_tile_bound);
    dfree(h->d_units);
    h->n_units = 0;
    dfree(h->d_tile_win);
    dfree(h->d_tile_len);
    dfree(h->d_tile_off);
    dfree(h->d_left_off);
    dfree(h->d_left_len);
    dfree(h->d_el_idx);
    dfree(h->d_acc);
    dfree(h->d_sig_scalars);
    h->tiled = false;
    h->n_panels = h->n_tiles = 0;
    h->n_dense_el = 0;
    h->h_row_abs_max = 0.0;
}

}  // namespace risq
