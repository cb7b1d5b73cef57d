// mlp.cuh -- the learned con2prim initial guess: a 5 -> 64 -> 64 -> 64 -> 2
// ReLU MLP evaluated and trained with 5th-generation tensor cores
// (tcgen05.mma, kind::f16, BF16 operands in shared memory, FP32 accumulators
// in tensor memory).  Outputs (normalised): log(Z / (D + tau + B^2)), the
// Newton variable Z = rho h W^2 relative to the analytic start, and log W (an
// auxiliary target, trained but not used by the solver).  No counterpart in
// the reference, which starts its Newton iteration from a hydro fixed point
// (core/rmhd_core.py:255-266).
//
// One CTA of 128 threads owns a tile of 128 samples: thread t <-> sample
// (row) t <-> TMEM lane t.  Every GEMM is issued as M = 128:
//   forward      H_l[128 x out] = H_{l-1}[128 x in] . W_l^T           (A, B K-major)
//   data grad    dH_{l-1}[128 x in] = dZ_l[128 x out] . W_l           (A K-major, B MN-major)
//   weight grad  dW_l[out(pad 128) x in] = dZ_l^T . H_{l-1}           (A, B MN-major)
// Operands use the SWIZZLE_NONE canonical layout: 8x8 core matrices of 8
// rows x 16 bytes; element (r, c) of an R-row operand lives at byte
//   (c/8)*(R/8)*128 + (r/8)*128 + (r%8)*16 + (c%8)*2,
// so the same bytes serve as a K-major operand (rows = M/N, cols = K: SBO =
// 128, LBO = (R/8)*128) or as an MN-major one (rows = K, cols = M/N: SBO =
// (R/8)*128, LBO = 128).  dZ^T is padded to M = 128 by keeping the dZ buffer
// 16 column groups wide with zeros beyond the layer's outputs.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mlp {

constexpr int TILE = 128;  // samples per CTA (= MMA M)
constexpr int NIN = 5, KIN = 16, H = 64, NOUT = 2, NOUTP = 16;

// FP32 master parameters, W[out][in] row-major, then the feature / target
// normalisation constants.
struct Params {
    float W1[H * NIN], b1[H], W2[H * H], b2[H], W3[H * H], b3[H], W4[NOUT * H], b4[NOUT];
    float xmu[NIN], xsd[NIN], ymu[NOUT], ysd[NOUT];
};
constexpr int kTrainable = H * NIN + H + 2 * (H * H + H) + NOUT * H + NOUT;  // 8834

// shared-memory map (bytes) of the training kernel; the inference kernel
// uses the first kInferSmem bytes (weights + H0 + one activation buffer)
constexpr int OFF_W1 = 0;                      // [64 x 16]  bf16  2 KB
constexpr int OFF_W2 = OFF_W1 + 64 * 16 * 2;   // [64 x 64]         8 KB
constexpr int OFF_W3 = OFF_W2 + 64 * 64 * 2;   // [64 x 64]         8 KB
constexpr int OFF_W4 = OFF_W3 + 64 * 64 * 2;   // [16 x 64]         2 KB
constexpr int OFF_BIAS = OFF_W4 + 16 * 64 * 2; // b1 b2 b3 b4 f32   1 KB (read by every row)
constexpr int OFF_H0 = OFF_BIAS + 1024;        // [128 x 16]        4 KB
constexpr int OFF_H1 = OFF_H0 + 128 * 16 * 2;  // [128 x 64]       16 KB each
constexpr int OFF_H2 = OFF_H1 + 128 * 64 * 2;
constexpr int OFF_H3 = OFF_H2 + 128 * 64 * 2;
constexpr int kInferSmem = OFF_H2;             // W + H0 + H1 (H1 reused per layer)
constexpr int OFF_DZ = OFF_H3 + 128 * 64 * 2;  // [128 x 128] bf16, 32 KB (16 col groups)
constexpr int OFF_DS1 = OFF_DZ + 128 * 128 * 2;  // ReLU'(z) of layers 1..3, bf16 16 KB each
constexpr int OFF_DS2 = OFF_DS1 + 128 * 64 * 2;
constexpr int OFF_DS3 = OFF_DS2 + 128 * 64 * 2;
constexpr int OFF_RED = OFF_DS3 + 128 * 64 * 2;  // [128][65] f32 bias-gradient reduction
constexpr int OFF_BAR = OFF_RED + 128 * 65 * 4;  // mbarrier (8 B) + TMEM address (4 B)
constexpr int kTrainSmem = OFF_BAR + 16;
static_assert(kTrainSmem <= 227 * 1024, "training tile exceeds shared memory");

// byte offset of element (r, c) in an operand with R rows
__device__ __forceinline__ uint32_t elem_off(int R, int r, int c) {
    return (uint32_t)((c >> 3) * (R >> 3) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// ------------------------------------------------------------- PTX glue ---
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// SWIZZLE_NONE shared-memory matrix descriptor (Blackwell version bit 46 = 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;  // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor: kind::f16, A = B = BF16, D = F32, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int N, int a_mn_major, int b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn_major << 15) |
           ((uint32_t)b_mn_major << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
    const uint32_t mask = 0;  // no output lanes disabled
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(mbar), "r"(count) : "memory");
}

// init + make the initialisation visible to the async proxy (tcgen05.commit)
__device__ __forceinline__ void mbar_init_fenced(uint32_t mbar, uint32_t count) {
    mbar_init(mbar, count);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// warp-wide: allocate ncols TMEM columns, address written to smem
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(dst_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(taddr), "r"(ncols)
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp-collective);
// the wait is in the same asm statement so no use of the registers can be
// scheduled before the load has completed
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// polls of an MMA-completion wait before it gives up (~seconds)
constexpr long kPollLimit = 1L << 26;

// Bounded wait on the MMA-completion barrier.  Returns false (and records a
// status) if the MMAs did not complete within `limit` polls; the caller then
// stops issuing work for this tile and exits cleanly.
__device__ __forceinline__ bool mbar_test_wait(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity, int* status,
                                                  long limit = kPollLimit) {
    if (limit < 1024) {
        // a test limit of a few polls: non-blocking probes, since one
        // try_wait may itself suspend the thread until the phase completes
        for (long it = 0; it < limit; ++it)
            if (mbar_test_wait(mbar, parity)) return true;
    } else {
        for (long it = 0; it < limit; ++it)
            if (mbar_try_wait(mbar, parity)) return true;
    }
    if (status) atomicExch(status, 1);
    return false;
}

// After a wait gave up at `phase` (already flipped by the caller), the MMAs
// it waited for may still be running and writing TMEM: wait for them once
// more, again bounded, before the block frees its TMEM and exits.
__device__ __forceinline__ void drain_after_timeout(uint32_t mbar, uint32_t phase) {
    mbar_wait_bounded(mbar, phase ^ 1u, nullptr);
}

// ReLU of two float32 values rounded to a packed bfloat16 pair (the ReLU is
// the conversion's .relu modifier: one instruction for two columns).  The
// first value lands in the low half, i.e. at the lower address.
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// 16 accumulator columns plus their biases -> ReLU -> 16 bfloat16 values
// (8 packed pairs): the bias adds as packed float32x2 adds (sm_100 FADD2)
__device__ __forceinline__ void bias_relu16(const float* z, const float* bias, uint32_t* h) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float2 b = *reinterpret_cast<const float2*>(bias + 2 * i);
        const float2 s = __fadd2_rn(make_float2(z[2 * i], z[2 * i + 1]), b);
        h[i] = relu_bf16x2(s.x, s.y);
    }
}

// write 8 consecutive columns [c0, c0+8) of row r as bf16 (16-byte store)
__device__ __forceinline__ void st_row8(unsigned char* base, int R, int r, int c0, const float* v) {
    __nv_bfloat162 p[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4*>(base + elem_off(R, r, c0)) = *reinterpret_cast<uint4*>(p);
}

// the same store from 4 packed bfloat16 pairs
__device__ __forceinline__ void st_row8_packed(unsigned char* base, int R, int r, int c0, const uint32_t* p) {
    *reinterpret_cast<uint4*>(base + elem_off(R, r, c0)) = make_uint4(p[0], p[1], p[2], p[3]);
}

// FP32 master weights -> bf16 K-major operands in shared memory (all
// threads), biases in float32.
__device__ __forceinline__ void load_weights(unsigned char* sm, const Params* P) {
    for (int e = threadIdx.x; e < 64 * 16; e += blockDim.x) {  // W1 [64 x 16], in 5..15 = 0
        int o = e / 16, i = e % 16;
        float w = i < NIN ? P->W1[o * NIN + i] : 0.f;
        *reinterpret_cast<__nv_bfloat16*>(sm + OFF_W1 + elem_off(64, o, i)) = __float2bfloat16_rn(w);
    }
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
        int o = e / 64, i = e % 64;
        *reinterpret_cast<__nv_bfloat16*>(sm + OFF_W2 + elem_off(64, o, i)) =
            __float2bfloat16_rn(P->W2[o * H + i]);
        *reinterpret_cast<__nv_bfloat16*>(sm + OFF_W3 + elem_off(64, o, i)) =
            __float2bfloat16_rn(P->W3[o * H + i]);
    }
    for (int e = threadIdx.x; e < 16 * 64; e += blockDim.x) {  // W4 [16 x 64], rows 2..15 = 0
        int o = e / 64, i = e % 64;
        float w = o < NOUT ? P->W4[o * H + i] : 0.f;
        *reinterpret_cast<__nv_bfloat16*>(sm + OFF_W4 + elem_off(16, o, i)) = __float2bfloat16_rn(w);
    }
    float* bs = reinterpret_cast<float*>(sm + OFF_BIAS);
    for (int e = threadIdx.x; e < 3 * H + NOUT; e += blockDim.x)
        bs[e] = e < H ? P->b1[e]
                      : (e < 2 * H ? P->b2[e - H] : (e < 3 * H ? P->b3[e - 2 * H] : P->b4[e - 3 * H]));
}

// Issue D[128 x N] (+)= A[128 x K] . B for K = 16*ksteps, both operands
// K-major with the layout above (thread 0 only).
__device__ __forceinline__ void mma_kmajor(uint32_t tmem_d, uint32_t a_addr, int a_rows,
                                           uint32_t b_addr, int b_rows, int N, int ksteps) {
    const uint32_t idesc = idesc_bf16(N, 0, 0);
    const uint32_t a_lbo = (a_rows / 8) * 128, b_lbo = (b_rows / 8) * 128;
    for (int kb = 0; kb < ksteps; ++kb) {
        uint64_t a = sdesc(a_addr + 2 * kb * a_lbo, a_lbo, 128);
        uint64_t b = sdesc(b_addr + 2 * kb * b_lbo, b_lbo, 128);
        mma_bf16(tmem_d, a, b, idesc, kb > 0 ? 1u : 0u);
    }
}

// ---- the forward pass in steps, for kernels that run several tiles per
// block or put other work between the tensor-core waits ----

// H0 row `row` of the activation buffer h: 5 normalised features, zeros up
// to 16
__device__ __forceinline__ void store_h0(unsigned char* h, int row, const float* h0) {
    float v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = i < NIN ? h0[i] : 0.f;
    st_row8(h, 128, row, 0, v);
    st_row8(h, 128, row, 8, v + 8);
}

// one thread, after a barrier preceded by fence_async_smem() and
// tc_fence_before(): the MMAs of layer l with the activations at shared
// address `in` (H0 for l = 0) into the accumulator columns at tmem_d,
// committed to mbar
__device__ __forceinline__ void issue_layer(const unsigned char* sm, uint32_t tmem_d, uint32_t mbar,
                                            int l, uint32_t in) {
    tc_fence_after();
    if (l == 0) mma_kmajor(tmem_d, in, 128, smem_u32(sm + OFF_W1), 64, 64, 1);
    else if (l < 3) mma_kmajor(tmem_d, in, 128, smem_u32(sm + (l == 1 ? OFF_W2 : OFF_W3)), 64, 64, 4);
    else mma_kmajor(tmem_d, in, 128, smem_u32(sm + OFF_W4), 16, NOUTP, 4);
    mma_commit(mbar);
}

// all threads of the tile, after layer l's MMAs completed (and
// tc_fence_after): the ReLU activations of row `row` into h (l < 3), or its
// two outputs (l == 3).  tmem_row: the accumulator columns at this thread's
// TMEM lane.
__device__ __forceinline__ void finish_layer(const unsigned char* sm, unsigned char* h, uint32_t tmem_row,
                                             int row, int l, float* out) {
    const float* bsm = reinterpret_cast<const float*>(sm + OFF_BIAS);
    if (l < 3) {
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
            float z[16];
            uint32_t hv[8];
            tmem_ld16(tmem_row + cb * 16, z);
            bias_relu16(z, bsm + l * H + cb * 16, hv);
            st_row8_packed(h, 128, row, cb * 16, hv);
            st_row8_packed(h, 128, row, cb * 16 + 8, hv + 4);
        }
    } else {
        float y[16];
        tmem_ld16(tmem_row, y);
        out[0] = y[0] + bsm[3 * H];
        out[1] = y[1] + bsm[3 * H + 1];
    }
}

// forward pass of one tile, in shared memory / TMEM.  Thread t owns row t.
// h0: normalised features of this thread's row.  When TRAIN, keeps H1..H3 and
// ReLU'(z) for the backward pass; otherwise H1 is reused for every layer.
// Returns false if an MMA wait timed out (uniform across the block).
template <bool TRAIN>
__device__ __forceinline__ bool forward_tile(unsigned char* sm, uint32_t tmem, uint32_t mbar, uint32_t& phase,
                             const Params* P, const float* h0, float* out, int* status,
                             long poll_limit = kPollLimit) {
    const int t = threadIdx.x;
    const uint32_t lane_base = (uint32_t)((t >> 5) * 32) << 16;
    store_h0(sm + OFF_H0, t, h0);
    const float* bsm = reinterpret_cast<const float*>(sm + OFF_BIAS);
    const int offDS[3] = {OFF_DS1, OFF_DS2, OFF_DS3};
    for (int l = 0; l < 4; ++l) {
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0)
            issue_layer(sm, tmem, mbar, l,
                        smem_u32(sm + (l == 0 ? OFF_H0 : (TRAIN ? OFF_H1 + (l - 1) * 128 * 64 * 2 : OFF_H1))));
        bool ok = mbar_wait_bounded(mbar, phase, status, poll_limit);
        phase ^= 1u;
        if (!__syncthreads_and(ok)) return false;
        tc_fence_after();
        if (TRAIN && l < 3) {
            unsigned char* dst = sm + OFF_H1 + l * 128 * 64 * 2;
#pragma unroll
            for (int cb = 0; cb < 4; ++cb) {
                float z[16], g[16];
                uint32_t h[8];
                tmem_ld16(tmem + lane_base + cb * 16, z);
                bias_relu16(z, bsm + l * H + cb * 16, h);
                st_row8_packed(dst, 128, t, cb * 16, h);
                st_row8_packed(dst, 128, t, cb * 16 + 8, h + 4);
                // ReLU'(z) = 1 where the activation is positive
#pragma unroll
                for (int i = 0; i < 16; ++i) g[i] = z[i] + bsm[l * H + cb * 16 + i] > 0.f ? 1.f : 0.f;
                st_row8(sm + offDS[l], 128, t, cb * 16, g);
                st_row8(sm + offDS[l], 128, t, cb * 16 + 8, g + 8);
            }
        } else {
            finish_layer(sm, sm + OFF_H1, tmem + lane_base, t, l, out);
        }
    }
    return true;
}

__device__ __forceinline__ void features_norm(const Params* P, const float* xr, float* h0) {
#pragma unroll
    for (int i = 0; i < NIN; ++i) h0[i] = __fdividef(xr[i] - P->xmu[i], P->xsd[i]);
}

}  // namespace mlp
