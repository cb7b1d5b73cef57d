// mlp.cu -- forward, backward and optimiser kernels of the learned con2prim
// initial-guess network (see mlp.cuh for the tensor-core data layout).
//
//   k_mlp_forward   batched inference: raw invariants -> (log(Z / (D + tau + B^2)), log W)
//   k_mlp_train     forward + backward of one 128-sample tile per CTA step,
//                   gradients of the mean-squared error summed into a float32
//                   buffer (atomics), loss summed alongside
//   k_mlp_adam      Adam update of the float32 master weights
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/astrofd.h"
#include "mlp.cuh"

using namespace mlp;

namespace {

__global__ void __launch_bounds__(128) k_mlp_forward(const Params* P, const float* x, float* y,
                                                     long n, int* status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kInferSmem);
    uint32_t* taddr_s = reinterpret_cast<uint32_t*>(sm + kInferSmem + 8);
    const int t = threadIdx.x;
    if (t < 32) tmem_alloc(smem_u32(taddr_s), 64);
    if (t == 0) mbar_init_fenced(smem_u32(bar), 1);
    load_weights(sm, P);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *taddr_s;
    uint32_t phase = 0;
    const long ntiles = (n + TILE - 1) / TILE;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long row = tile * TILE + t;
        float xr[NIN] = {0, 0, 0, 0, 0}, h0[NIN], o[2];
        if (row < n)
            for (int i = 0; i < NIN; ++i) xr[i] = x[row * NIN + i];
        features_norm(P, xr, h0);
        if (!forward_tile<false>(sm, tmem, smem_u32(bar), phase, P, h0, o, status)) {
            drain_after_timeout(smem_u32(bar), phase);
            break;
        }
        if (row < n) {
            y[row * 2 + 0] = o[0] * P->ysd[0] + P->ymu[0];
            y[row * 2 + 1] = o[1] * P->ysd[1] + P->ymu[1];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (t < 32) tmem_free(tmem, 64);
}

// gradient buffer layout == the trainable prefix of Params
struct GradOff {
    static constexpr int W1 = 0, b1 = W1 + H * NIN, W2 = b1 + H, b2 = W2 + H * H, W3 = b2 + H,
                         b3 = W3 + H * H, W4 = b3 + H, b4 = W4 + NOUT * H;
};

// MMAs of one backward layer: dW (cols 64..127 of TMEM) = dZ^T . Hin and,
// when want_dh, dH (cols 0..63) = dZ . W.  Thread 0 only.
__device__ void backward_mmas(unsigned char* sm, uint32_t tmem, int out_cols, int hin_off,
                              int hin_cols, bool want_dh, int w_off, int w_rows, int w_cols) {
    const uint32_t dz = smem_u32(sm + OFF_DZ);
    // dW[out(pad 128) x in] += dZ^T[128 x 128 batch] . Hin[128 batch x in]:
    // both operands MN-major; K = batch in 8 steps of 16 rows
    {
        const uint32_t idesc = idesc_bf16(hin_cols, 1, 1);
        const uint32_t hin = smem_u32(sm + hin_off);
        for (int kb = 0; kb < 8; ++kb) {
            uint64_t a = sdesc(dz + kb * 256, 128, 16 * 128);
            uint64_t b = sdesc(hin + kb * 256, 128, 16 * 128);
            mma_bf16(tmem + 64, a, b, idesc, kb > 0 ? 1u : 0u);
        }
    }
    if (want_dh) {
        // dH[128 x in] = dZ[128 x out] . W[out x in]: A K-major (K = out),
        // B = W read MN-major (K = out rows, N = in cols)
        const uint32_t idesc = idesc_bf16(w_cols, 0, 1);
        const uint32_t w = smem_u32(sm + w_off);
        const int ksteps = out_cols / 16;
        for (int kb = 0; kb < ksteps; ++kb) {
            uint64_t a = sdesc(dz + 2 * kb * 2048, 2048, 128);
            uint64_t b = sdesc(w + kb * 256, 128, (w_rows / 8) * 128);
            mma_bf16(tmem, a, b, idesc, kb > 0 ? 1u : 0u);
        }
    }
}

__global__ void __launch_bounds__(128) k_mlp_train(const Params* P, const float* x, const float* tg,
                                                   long n, float* grad, float* loss, int* status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
    uint32_t* taddr_s = reinterpret_cast<uint32_t*>(sm + OFF_BAR + 8);
    float* red = reinterpret_cast<float*>(sm + OFF_RED);
    const int t = threadIdx.x, warp = t >> 5;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    if (t < 32) tmem_alloc(smem_u32(taddr_s), 128);
    if (t == 0) mbar_init_fenced(smem_u32(bar), 1);
    load_weights(sm, P);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *taddr_s;
    const uint32_t mbar = smem_u32(bar);
    uint32_t phase = 0;
    const float inv_n = 1.0f / (float)(n * NOUT);
    const long ntiles = (n + TILE - 1) / TILE;
    float my_loss = 0.f;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long row = tile * TILE + t;
        const bool valid = row < n;
        float xr[NIN] = {0, 0, 0, 0, 0}, h0[NIN], o[2];
        if (valid)
            for (int i = 0; i < NIN; ++i) xr[i] = x[row * NIN + i];
        features_norm(P, xr, h0);
        if (!forward_tile<true>(sm, tmem, mbar, phase, P, h0, o, status)) {
            drain_after_timeout(mbar, phase);
            break;
        }
        // d(mean squared error)/d(output) in normalised target units
        float dy[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) dy[i] = 0.f;
        if (valid) {
            for (int j = 0; j < NOUT; ++j) {
                float target = (tg[row * NOUT + j] - P->ymu[j]) / P->ysd[j];
                float e = o[j] - target;
                my_loss += e * e;
                dy[j] = 2.0f * e * inv_n;
            }
        }
        // dZ4 into the dZ buffer: columns 0..15, zeros in column groups 2..15
        {
            float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int g = 2; g < 16; ++g) st_row8(sm + OFF_DZ, 128, t, g * 8, zero);
            st_row8(sm + OFF_DZ, 128, t, 0, dy);
            st_row8(sm + OFF_DZ, 128, t, 8, dy + 8);
        }
        // layer l = 4..1 backward: dW_l, db_l and (l > 1) dZ_{l-1}
        bool ok = true;
        for (int l = 4; l >= 1 && ok; --l) {
            const int out_cols = l == 4 ? NOUTP : H;
            const int hin_off = l == 1 ? OFF_H0 : OFF_H1 + (l - 2) * 128 * 64 * 2;
            const int hin_cols = l == 1 ? KIN : H;
            const int w_off = l == 4 ? OFF_W4 : (l == 3 ? OFF_W3 : OFF_W2);
            const int w_rows = l == 4 ? 16 : 64;
            // bias gradient: column sums of dZ (this thread's row -> smem)
            {
                float dzr[64];
                for (int c = 0; c < out_cols; ++c) {
                    __nv_bfloat16 b = *reinterpret_cast<const __nv_bfloat16*>(
                        sm + OFF_DZ + elem_off(128, t, c));
                    dzr[c] = __bfloat162float(b);
                }
                for (int c = 0; c < out_cols; ++c) red[t * 65 + c] = dzr[c];
            }
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            if (t == 0) {
                tc_fence_after();
                backward_mmas(sm, tmem, out_cols, hin_off, hin_cols, l > 1, w_off, w_rows, H);
                mma_commit(mbar);
            }
            if (t < out_cols) {
                const int nreal = l == 4 ? NOUT : H;
                if (t < nreal) {
                    float s = 0.f;
                    for (int r = 0; r < TILE; ++r) s += red[r * 65 + t];
                    const int boff = l == 4 ? GradOff::b4 : (l == 3 ? GradOff::b3 : (l == 2 ? GradOff::b2 : GradOff::b1));
                    atomicAdd(grad + boff + t, s);
                }
            }
            bool w = mbar_wait_bounded(mbar, phase, status);
            phase ^= 1u;
            ok = __syncthreads_and(w);
            if (!ok) {
                drain_after_timeout(mbar, phase);
                break;
            }
            tc_fence_after();
            // weight gradient rows (out features) live in TMEM lanes 0..63
            if (warp < 2) {
                const int o = t;
                const int nreal_out = l == 4 ? NOUT : H;
                const int nin = l == 1 ? NIN : H;
                const int woff = l == 4 ? GradOff::W4 : (l == 3 ? GradOff::W3 : (l == 2 ? GradOff::W2 : GradOff::W1));
                for (int cb = 0; cb < hin_cols / 16; ++cb) {
                    float g[16];
                    tmem_ld16(tmem + lane_base + 64 + cb * 16, g);
                    if (o < nreal_out)
                        for (int i = 0; i < 16; ++i)
                            if (cb * 16 + i < nin) atomicAdd(grad + woff + o * nin + cb * 16 + i, g[i]);
                }
            }
            if (l > 1) {
                // dZ_{l-1} = dH_{l-1} * ReLU'(z_{l-1}) -> dZ buffer columns 0..63
                const int ds = l == 4 ? OFF_DS3 : (l == 3 ? OFF_DS2 : OFF_DS1);
#pragma unroll
                for (int cb = 0; cb < 4; ++cb) {
                    float dh[16];
                    tmem_ld16(tmem + lane_base + cb * 16, dh);
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        __nv_bfloat16 b = *reinterpret_cast<const __nv_bfloat16*>(
                            sm + ds + elem_off(128, t, cb * 16 + i));
                        dh[i] *= __bfloat162float(b);
                    }
                    st_row8(sm + OFF_DZ, 128, t, cb * 16, dh);
                    st_row8(sm + OFF_DZ, 128, t, cb * 16 + 8, dh + 8);
                }
            }
            tc_fence_before();
            __syncthreads();
        }
        if (!ok) break;
    }
    // loss: warp reduce then one atomic per warp
    for (int s = 16; s > 0; s >>= 1) my_loss += __shfl_xor_sync(0xffffffffu, my_loss, s);
    if ((t & 31) == 0 && loss) atomicAdd(loss, my_loss * inv_n);
    tc_fence_before();
    __syncthreads();
    if (t < 32) tmem_free(tmem, 128);
}

__global__ void k_mlp_adam(float* w, float* g, float* m, float* v, int n, float lr, float b1,
                           float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.f - b1) * gi;
        float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        g[i] = 0.f;
    }
}

bool g_attr_done = false;

cudaError_t ensure_smem_attrs() {
    if (g_attr_done) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kTrainSmem);
    if (e != cudaSuccess) return e;
    cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    g_attr_done = true;
    return cudaSuccess;
}

int sm_count() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

}  // namespace

extern "C" {

size_t astro_mlp_param_bytes(void) { return sizeof(Params); }
int astro_mlp_trainable(void) { return kTrainable; }

int astro_mlp_forward(const void* params, const float* x, float* y, int64_t n, int* status,
                      void* stream) {
    if (!params || n < 0) return ASTRO_E_INVALID;
    if (n == 0) return ASTRO_OK;  // an empty batch may pass null arrays
    if (!x || !y) return ASTRO_E_INVALID;
    const long ntiles = (n + TILE - 1) / TILE;
    const int grid = (int)(ntiles < 4L * sm_count() ? ntiles : 4L * sm_count());
    k_mlp_forward<<<grid, TILE, kInferSmem + 16, (cudaStream_t)stream>>>((const Params*)params, x, y,
                                                                        n, status);
    return cudaGetLastError() == cudaSuccess ? ASTRO_OK : ASTRO_E_CUDA;
}

int astro_mlp_train_grad(const void* params, const float* x, const float* t, int64_t n, float* grad,
                         float* loss, int* status, void* stream) {
    if (!params || !x || !t || !grad || n <= 0) return ASTRO_E_INVALID;
    if (ensure_smem_attrs() != cudaSuccess) return ASTRO_E_CUDA;
    const long ntiles = (n + TILE - 1) / TILE;
    const int grid = (int)(ntiles < sm_count() ? ntiles : sm_count());
    k_mlp_train<<<grid, TILE, kTrainSmem, (cudaStream_t)stream>>>((const Params*)params, x, t, n, grad,
                                                                loss, status);
    return cudaGetLastError() == cudaSuccess ? ASTRO_OK : ASTRO_E_CUDA;
}

int astro_mlp_adam(void* params, float* grad, float* m, float* v, float lr, float beta1, float beta2,
                   float eps, int step, void* stream) {
    if (!params || !grad || !m || !v || step < 1) return ASTRO_E_INVALID;
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    k_mlp_adam<<<(kTrainable + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        (float*)params, grad, m, v, kTrainable, lr, beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? ASTRO_OK : ASTRO_E_CUDA;
}

}  // extern "C"
