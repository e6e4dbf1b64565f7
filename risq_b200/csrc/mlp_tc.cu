// Learned-preconditioner inference on the fifth-generation tensor cores (tcgen05).
//
// Same function as k_mlp_scale (mlp.cu): per determinant, the network
// o = W3 relu(W2 relu(W1 x + b1) + b2) + b3 on the features x of both spin orders,
// f = clamp(exp((o(alpha, beta) + o(beta, alpha)) / 2), 0.25, 4), BF16 weights,
// FP32 accumulation, hidden activations rounded to BF16 between the layers.
//
// A CTA works on tiles of 64 determinants = 128 rows (row r < 64: determinant r in
// the (alpha, beta) order; row r + 64: the same determinant in the (beta, alpha)
// order), one row per thread of its four warps.
//   1. Each thread writes its row's occupation features (+1 / -1, BF16) into shared
//      memory as the A operand; the two continuous features stay FP32 and enter in
//      the epilogue (h1 += W1[:, 2n] dE + W1[:, 2n+1] sum_h on the CUDA cores).
//   2. One thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, M = N = 128,
//      K = 16 per instruction) against W1 staged once per CTA, accumulator in
//      TMEM; tcgen05.commit arrives on an mbarrier.
//   3. Each warp reads its 32 TMEM lanes (= its 32 rows) with tcgen05.ld, adds
//      the continuous terms and b1, applies ReLU, rounds to BF16 and writes the
//      row back to shared memory as the A operand of layer 2.
//   4. Layer 2 (K = 128) into the same TMEM columns; the epilogue folds bias,
//      ReLU and the W3 dot product per row; rows 64..127 hand their output to
//      rows 0..63 through shared memory, which write the factor.
// Operands use the K-major, no-swizzle canonical layout: 8 x 8 BF16 core matrices
// of 128 contiguous bytes, consecutive along K (leading byte offset 128 B), 8-row
// groups K/8 core matrices apart (stride byte offset).
// Every mbarrier wait is bounded in time; on a timeout the CTA records an error,
// stops, and still frees its TMEM.  The timeout path is exercised by a test-only
// switch (environment variable RISQGPU_TEST_MMA_STALL=1): the first completion wait
// then watches a barrier that nothing arrives on, with a 1 ms limit, and the call
// must come back with an error status while the handle stays usable.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "internal.cuh"

namespace risq {

namespace {

constexpr int TC_ROWS = 128;   // MMA M
constexpr int TC_DETS = 64;    // determinants per tile
constexpr int TC_H = 128;      // hidden width = MMA N
constexpr int TC_THREADS = 128;
constexpr unsigned long long WAIT_NS = 2000000000ull;  // 2 s per MMA completion wait
constexpr unsigned long long STALL_PROBE_NS = 1000000ull;  // 1 ms: the test-only stalled wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// byte offset of element (row, k) of a K-major, no-swizzle operand with K columns
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int K) {
    return (uint32_t)((row & 7) * 16 + (row >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (k & 7) * 2);
}

// tcgen05 shared-memory matrix descriptor: start address, leading / stride byte
// offsets (all >> 4), descriptor version 1 at bits 46-47, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9,
// 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at 24-28.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_H >> 3) << 17) |
                           ((uint32_t)(TC_ROWS >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(IDESC), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// wait for completion of phase `parity` of the mbarrier, at most limit_ns
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, unsigned long long limit_ns = WAIT_NS) {
    const unsigned long long t0 = global_ns();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// 32 consecutive FP32 accumulator columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint16_t to_bf16(float f) {  // round to nearest even (finite values)
    uint32_t u = __float_as_uint(f);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
__device__ __forceinline__ float from_bf16(uint16_t b) { return __uint_as_float(((uint32_t)b) << 16); }

// bit o of a W-word string without dynamic indexing (keeps the words in registers)
template <int W>
__device__ __forceinline__ bool bit_of(const uint64_t (&x)[W], int o) {
    uint64_t w = x[0];
#pragma unroll
    for (int i = 1; i < W; i++)
        if ((o >> 6) == i) w = x[i];
    return (w >> (o & 63)) & 1ull;
}

struct TcSmem {
    // byte offsets inside the dynamic shared memory block (operands 128-byte aligned)
    uint32_t a1, b1, a2, b2, fl, total;
    __host__ __device__ static TcSmem make(int K1, int norb) {
        TcSmem s;
        s.a1 = 0;
        s.b1 = s.a1 + TC_ROWS * K1 * 2;
        s.a2 = s.b1 + TC_H * K1 * 2;
        s.b2 = s.a2 + TC_ROWS * TC_H * 2;
        s.fl = s.b2 + TC_H * TC_H * 2;
        // floats: wc0, wc1, b1, b2, w3 (5 x 128), hpp (norb), partner outputs (64)
        s.total = s.fl + 4 * (5 * TC_H + ((norb + 3) & ~3) + TC_DETS) + 16;
        return s;
    }
};

template <int W>
__global__ void __launch_bounds__(TC_THREADS) k_mlp_scale_tc(
    const uint64_t* __restrict__ up, const uint64_t* __restrict__ dn, const double* __restrict__ diag, int64_t N,
    int norb, int K1, const double* __restrict__ h1, double energy, const uint16_t* __restrict__ w1,
    const float* __restrict__ bias1, const uint16_t* __restrict__ w2, const float* __restrict__ bias2,
    const uint16_t* __restrict__ w3, const float* __restrict__ bias3, float4 fnorm, float* __restrict__ out,
    int* __restrict__ err, int stall_probe) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ __align__(8) uint64_t never_bar;  // nothing arrives on it (stall probe)
    __shared__ uint32_t tmem_slot;
    const TcSmem L = TcSmem::make(K1, norb);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int n_in = 2 * norb + 2;
    float* wc0 = reinterpret_cast<float*>(sm + L.fl);
    float* wc1 = wc0 + TC_H;
    float* fb1 = wc1 + TC_H;
    float* fb2 = fb1 + TC_H;
    float* fw3 = fb2 + TC_H;
    float* hpp = fw3 + TC_H;
    float* partner = hpp + ((norb + 3) & ~3);

    // stage the weights: W1 occupation columns and W2 as BF16 B operands, the rest as FP32
    for (int i = tid; i < TC_H * K1; i += TC_THREADS) {
        const int j = i / K1, k = i % K1;
        const uint16_t v = k < 2 * norb ? w1[j * n_in + k] : (uint16_t)0;
        *reinterpret_cast<uint16_t*>(sm + L.b1 + kmajor_off(j, k, K1)) = v;
    }
    for (int i = tid; i < TC_H * TC_H; i += TC_THREADS) {
        const int j = i / TC_H, k = i % TC_H;
        *reinterpret_cast<uint16_t*>(sm + L.b2 + kmajor_off(j, k, TC_H)) = w2[i];
    }
    for (int j = tid; j < TC_H; j += TC_THREADS) {
        wc0[j] = from_bf16(w1[j * n_in + 2 * norb]);
        wc1[j] = from_bf16(w1[j * n_in + 2 * norb + 1]);
        fb1[j] = bias1[j];
        fb2[j] = bias2[j];
        fw3[j] = from_bf16(w3[j]);
    }
    for (int k = tid; k < norb; k += TC_THREADS) {
        const uint32_t i = k + 1;
        hpp[k] = (float)h1[(i * (i - 1)) / 2 + i];
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&never_bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TC_H));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_proxy_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t mb = smem_u32(&mbar);
    const uint32_t a1 = smem_u32(sm + L.a1), b1 = smem_u32(sm + L.b1);
    const uint32_t a2 = smem_u32(sm + L.a2), b2 = smem_u32(sm + L.b2);
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    const float b3 = bias3[0];
    const uint16_t ONE = 0x3F80u, MONE = 0xBF80u;
    uint32_t phase = 0;
    const int64_t ntiles = (N + TC_DETS - 1) / TC_DETS;

    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        // ---- features of this thread's row -> A1 ----
        const int r = tid;
        const int64_t d = tile * TC_DETS + (r & (TC_DETS - 1));
        const bool valid = d < N;
        uint64_t a[W], b[W];
        float dE = 0.f, sum_h = 0.f;
#pragma unroll
        for (int k = 0; k < W; k++) { a[k] = 0; b[k] = 0; }
        if (valid) {
#pragma unroll
            for (int k = 0; k < W; k++) { a[k] = up[k * N + d]; b[k] = dn[k * N + d]; }
            for (int o = 0; o < norb; o++) {
                if (bit_of<W>(a, o)) sum_h += hpp[o];
                if (bit_of<W>(b, o)) sum_h += hpp[o];
            }
            dE = ((float)(diag[d] - energy) - fnorm.x) * fnorm.y;
            sum_h = (sum_h - fnorm.z) * fnorm.w;
        }
        const bool ab = r < TC_DETS;  // (alpha, beta) order for rows 0..63
        for (int q = 0; q < K1 / 8; q++) {
            uint32_t pk[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                uint16_t lo, hi;
#pragma unroll
                for (int hlf = 0; hlf < 2; hlf++) {
                    const int k = q * 8 + e * 2 + hlf;
                    uint16_t v = 0;
                    if (valid && k < 2 * norb) {
                        const bool lead = k < norb;
                        const int o = lead ? k : k - norb;
                        const bool set = (lead == ab) ? bit_of<W>(a, o) : bit_of<W>(b, o);
                        v = set ? ONE : MONE;
                    }
                    if (hlf == 0) lo = v; else hi = v;
                }
                pk[e] = (uint32_t)lo | ((uint32_t)hi << 16);
            }
            *reinterpret_cast<uint4*>(sm + L.a1 + kmajor_off(r, q * 8, K1)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
        fence_proxy_async();
        __syncthreads();
        // ---- layer 1 on the tensor cores ----
        if (tid == 0) {
            fence_after();
            const uint32_t sbo = (uint32_t)(K1 / 8) * 128;
            for (int ks = 0; ks < K1 / 16; ks++)
                mma_bf16(tmem, smem_desc(a1 + ks * 256, 128, sbo), smem_desc(b1 + ks * 256, 128, sbo), ks > 0);
            mma_commit(mb);
        }
        // the stall probe waits on a barrier whose phase never completes, so the bounded
        // wait runs out; the MMA issued above completes on `mb` and is awaited below
        bool ok = stall_probe ? mbar_wait(smem_u32(&never_bar), 0, STALL_PROBE_NS) : mbar_wait(mb, phase);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) atomicExch(err, 1);
            mbar_wait(mb, phase);  // let the MMA in flight finish (bounded) before TMEM is freed
            break;
        }
        phase ^= 1;
        fence_after();
        // ---- epilogue 1: + continuous features + b1, ReLU, BF16 -> A2 ----
#pragma unroll 1
        for (int c = 0; c < TC_H / 32; c++) {
            float v[32];
            tmem_ld32(taddr + c * 32, v);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint32_t pk[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int j0 = c * 32 + q * 8 + e * 2;
                    const float x0 = fmaxf(v[q * 8 + e * 2] + fb1[j0] + wc0[j0] * dE + wc1[j0] * sum_h, 0.f);
                    const float x1 = fmaxf(v[q * 8 + e * 2 + 1] + fb1[j0 + 1] + wc0[j0 + 1] * dE + wc1[j0 + 1] * sum_h, 0.f);
                    pk[e] = (uint32_t)to_bf16(x0) | ((uint32_t)to_bf16(x1) << 16);
                }
                *reinterpret_cast<uint4*>(sm + L.a2 + kmajor_off(r, c * 32 + q * 8, TC_H)) =
                    make_uint4(pk[0], pk[1], pk[2], pk[3]);
            }
        }
        fence_proxy_async();
        fence_before();
        __syncthreads();
        // ---- layer 2 on the tensor cores (same TMEM columns) ----
        if (tid == 0) {
            fence_after();
            const uint32_t sbo = (uint32_t)(TC_H / 8) * 128;
            for (int ks = 0; ks < TC_H / 16; ks++)
                mma_bf16(tmem, smem_desc(a2 + ks * 256, 128, sbo), smem_desc(b2 + ks * 256, 128, sbo), ks > 0);
            mma_commit(mb);
        }
        ok = mbar_wait(mb, phase);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) atomicExch(err, 1);
            mbar_wait(mb, phase);
            break;
        }
        phase ^= 1;
        fence_after();
        // ---- epilogue 2: + b2, ReLU, W3 dot, b3 ----
        float o = b3;
#pragma unroll 1
        for (int c = 0; c < TC_H / 32; c++) {
            float v[32];
            tmem_ld32(taddr + c * 32, v);
#pragma unroll
            for (int j = 0; j < 32; j++) o += fw3[c * 32 + j] * fmaxf(v[j] + fb2[c * 32 + j], 0.f);
        }
        if (r >= TC_DETS) partner[r - TC_DETS] = o;
        fence_before();
        __syncthreads();
        if (r < TC_DETS && valid) {
            const float f = __expf(0.5f * (o + partner[r]));
            out[d] = fminf(fmaxf(f, 0.25f), 4.0f);
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_H));
}

}  // namespace

// Tensor-core path of mlp_scale_impl for hidden = 128 (every trained network) and
// 2n <= 128; returns RISQGPU_ERR_INVALID when the network does not fit it.
int mlp_scale_tc(risqgpu* h, double energy, float* out) {
    if (h->mlp.hidden != TC_H || 2 * h->norb > 128 || h->W != 1) return RISQGPU_ERR_INVALID;
    const int K1 = ((2 * h->norb + 15) / 16) * 16;
    const TcSmem L = TcSmem::make(K1, h->norb);
    const int64_t N = (int64_t)h->N;
    int* err = nullptr;
    ScopedFree<1> release(err);
    RQ_TRY(dalloc(h, err, 1));
    const char* probe_env = std::getenv("RISQGPU_TEST_MMA_STALL");
    const int stall_probe = (probe_env && std::strcmp(probe_env, "1") == 0) ? 1 : 0;
    RQ_CUDA(h, cudaMemsetAsync(err, 0, sizeof(int), h->stream));
    auto kern = k_mlp_scale_tc<1>;  // 2n <= 128: one word per spin string
    RQ_CUDA(h, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, TC_THREADS, L.total);
    occ = std::max(1, std::min(occ, 4));  // TMEM: 4 x 128 columns per SM at most
    const int64_t ntiles = (N + TC_DETS - 1) / TC_DETS;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)num_sms(h) * occ));
    kern<<<grid, TC_THREADS, L.total, h->stream>>>(h->d_up, h->d_dn, h->d_diag, N, h->norb, K1, h->d_h1, energy,
                                                   h->mlp.w1, h->mlp.b1, h->mlp.w2, h->mlp.b2, h->mlp.w3, h->mlp.b3,
                                                   h->mlp.fnorm, out, err, stall_probe);
    RQ_TRY(check_launch(h, "mlp scale (tensor cores)"));
    int herr = 0;
    RQ_CUDA(h, cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    RQ_TRY(sync(h, "mlp scale (tensor cores)"));
    if (herr) {
        h->err = "tensor-core MLP: an MMA completion wait timed out";
        return RISQGPU_ERR_CUDA;
    }
    return RISQGPU_OK;
}

}  // namespace risq
