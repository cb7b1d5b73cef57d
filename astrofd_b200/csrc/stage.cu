// stage.cu -- the fused SSPRK stage kernel (see stage.cuh).
//
// Thread block: TY x TZ = 4 x 32 cells of a (y, z) column, 4 warps, warp w
// owning row w.  The block marches along x over TX planes.  Per plane i:
//   1. wait for the halo box of plane i (TMA, 9 x 10 x 40 floats: the cells
//      and their 3-cell y/z halo) and for ring plane i+3 (TMA, the column's
//      own 4 x 36 cells of each of the six planes i-2 .. i+3);
//   2. one loop of face jobs, 32 faces each: the (TY+1) rows of TZ y faces
//      and the TY x (TZ+1) z faces from the halo box (fluxes to shared
//      memory), spread over the warps, then each warp's own row of x faces
//      i+1/2 from the ring (flux in registers).  The face code exists once:
//      the vector components are rotated so every face is evaluated as an x
//      face;
//   3. barrier; the halo box of plane i+1 and ring plane i+4 go out;
//   4. per cell: divergence (x fluxes of i-1/2 and i+1/2 in registers, y and z
//      fluxes from shared memory), GLM damping, the resistive Laplacian (from
//      the float32 tiles, differences in float64), the float64 SSPRK
//      combination; U_k to global memory.
// A float32 face whose result is not finite (float32 overflow) marks its two
// cells: they are not updated here but listed, and k_stage_fix redoes them
// with that face in float64 from the float64 stage input.  Cells outside
// [lo, hi)^3 (ghosts and the loop-bound frame) are updated by the caller.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "physics.cuh"
#include "stage.cuh"

using namespace astro;

namespace astro_stage {
namespace {

constexpr int NM = 9;                 // RMHD primitives
constexpr int HY = TY + 6, HZ = 40;   // halo box: rows, columns (16-byte multiple)
constexpr int CZ = 36;                // ring box columns: k0-3 .. k0+32 (aligned start)
constexpr int NRING = 6;
constexpr int HALO_FLOATS = NM * HY * HZ;
constexpr int CORE_FLOATS = NM * TY * CZ;
constexpr int FY_FLOATS = NM * (TY + 1) * TZ;
constexpr int FZ_FLOATS = NM * TY * (TZ + 1);
constexpr uint32_t HALO_BYTES = HALO_FLOATS * 4;
constexpr uint32_t CORE_BYTES = CORE_FLOATS * 4;
constexpr int CORE_STRIDE = (CORE_FLOATS + 31) & ~31;  // ring slot, 128-byte multiple
// shared memory map (bytes); TMA destinations 128-byte aligned
constexpr int OFF_HALO = 0;
constexpr int OFF_RING = (OFF_HALO + HALO_FLOATS * 4 + 127) & ~127;
constexpr int OFF_FY = OFF_RING + NRING * CORE_STRIDE * 4;
constexpr int OFF_FZ = OFF_FY + FY_FLOATS * 4;
constexpr int OFF_BAR = (OFF_FZ + FZ_FLOATS * 4 + 7) & ~7;
constexpr int OFF_CNT = OFF_BAR + 8 * (NRING + 1);
// y-face jobs: rows 0..TY; z-face jobs: the TY x (TZ+1) faces in chunks of 32;
// one more mark word for the x faces
constexpr int kYJobs = TY + 1;
constexpr int kZJobs = (TY * (TZ + 1) + 31) / 32;
constexpr int kJobs = kYJobs + kZJobs;  // y/z jobs; index kJobs is a warp's x row
constexpr int OFF_FAIL = OFF_CNT + 4 * (NRING + 1);
constexpr int kSmem = OFF_FAIL + 4 * 3 * kJobs;
static_assert(OFF_RING % 128 == 0 && CORE_STRIDE * 4 % 128 == 0, "TMA alignment");
static_assert(kSmem <= 56 * 1024, "four blocks per SM");
constexpr long kPollLimit = kTilePollLimit;  // polls of a tile-load wait before it gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void bar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool bar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool bar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait; false if the load did not land within `limit` polls.  A
// limit of a few polls (a test setting) uses non-blocking probes, since one
// try_wait may itself suspend the thread until the phase completes.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, long limit = kPollLimit) {
    if (limit < 1024) {
        for (long it = 0; it < limit; ++it)
            if (bar_test(bar, parity)) return true;
        return false;
    }
    for (long it = 0; it < limit; ++it)
        if (bar_try(bar, parity)) return true;
    return false;
}
// 4-d tiled TMA load (box of the map) at (k, j, i, v) into shared memory
__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap* map, int k, int j, int i,
                                         uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(k), "r"(j), "r"(i), "r"(0), "r"(bar)
        : "memory");
}

// Rotate the vector components of a primitive state so that direction `dir`
// becomes the first (cyclic: the face's normal, then the next two axes), or
// back.  The face physics is then always evaluated as an x face, so one copy
// of its code serves all three directions (runtime selects instead of three
// inlined variants); the arithmetic is the same up to the order of the
// three-term sums (v^2, B^2, v.B), i.e. float32 rounding.
__device__ __forceinline__ void rot3(float* c, int dir) {
    const float a = c[0], b = c[1], d = c[2];
    c[0] = dir == 0 ? a : (dir == 1 ? b : d);
    c[1] = dir == 0 ? b : (dir == 1 ? d : a);
    c[2] = dir == 0 ? d : (dir == 1 ? a : b);
}
__device__ __forceinline__ void unrot3(float* c, int dir) {
    const float a = c[0], b = c[1], d = c[2];  // components (n, n+1, n+2)
    c[0] = dir == 0 ? a : (dir == 1 ? d : b);
    c[1] = dir == 0 ? b : (dir == 1 ? a : d);
    c[2] = dir == 0 ? d : (dir == 1 ? b : a);
}

// One float32 face of direction `dir`: rows[o] points at stencil cell o
// (cell c-3+o) of variable 0 in shared memory, sv is the variable stride
// (floats).  Returns false when the flux or the wave speeds are not finite.
template <int RECON, int RIEMANN>
__device__ __forceinline__ bool face_any(const Phys<float>& P, int lim, const float* const* rows,
                                         int sv, int dir, float* F) {
    float qL[NM], qR[NM];
#pragma unroll
    for (int v = 0; v < NM; ++v) {
        float st[6];
#pragma unroll
        for (int o = 0; o < 6; ++o) st[o] = rows[o][v * sv];
        recon_face<RECON>(st, lim, qL[v], qR[v]);
    }
    rot3(qL + 1, dir); rot3(qR + 1, dir);
    rot3(qL + 5, dir); rot3(qR + 5, dir);
    float sL = -1.f, sR = 1.f;
    r_face<RIEMANN, false, false>(P, 0, qL, qR, F, sL, sR);
    unrot3(F + 1, dir);
    unrot3(F + 5, dir);
    bool ok = isfinite(sL) && isfinite(sR);
#pragma unroll
    for (int v = 0; v < NM; ++v) ok &= isfinite(F[v]);
    return ok;
}

// The same face in float64 from the float64 stage input (a face whose float32
// evaluation overflowed); the flux is returned as float32 like the others.
template <int RECON, int RIEMANN, int DIR>
__device__ __forceinline__ void face_f64(const StageArgs& a, int i, int j, int k, float* Fo) {
    const Phys<double> P = Phys<double>::from(a.p);
    const size_t nc = (size_t)a.nx * a.ny * a.nz;
    const size_t cell = ((size_t)i * a.ny + j) * a.nz + k;
    const long stride = DIR == 0 ? (long)a.ny * a.nz : (DIR == 1 ? (long)a.nz : 1L);
    double qL[NM], qR[NM];
    for (int v = 0; v < NM; ++v) {
        double st[6];
        for (int o = 0; o < 6; ++o) st[o] = a.pr[(size_t)v * nc + cell + (o - 3) * stride];
        recon_face<RECON>(st, a.p.limiter, qL[v], qR[v]);
    }
    double F[NM], sL = -1.0, sR = 1.0;
    r_face<RIEMANN, false, false>(P, DIR, qL, qR, F, sL, sR);
    for (int v = 0; v < NM; ++v) Fo[v] = (float)F[v];
}

// The update of cell (i, j, k) from its six face fluxes (low and high x, y,
// z): divergence, GLM damping, resistive Laplacian, the float64 SSPRK
// combination (the split path's k_update, operation for operation), U_k and
// the passive rows of dst.
// lap: the cell's resistive Laplacian of B (3 values) when the caller has it
// (the fused kernel, from its float32 tiles), else null: from the float64
// stage input.
__device__ __forceinline__ void update_cell(const StageArgs& a, int i, int j, int k,
                                            const float* fxl, const float* fxh, const float* fyl,
                                            const float* fyh, const float* fzl, const float* fzh,
                                            const double* lap = nullptr) {
    const size_t nc = (size_t)a.nx * a.ny * a.nz;
    const size_t cell = ((size_t)i * a.ny + j) * a.nz + k;
    const double i0d = a.idd[0], i1d = a.idd[1], i2d = a.idd[2];
    double rhs[NM];
#pragma unroll
    for (int v = 0; v < NM; ++v) {
        double r = 0.0;
        r -= ((double)fxh[v] - (double)fxl[v]) * i0d;
        r -= ((double)fyh[v] - (double)fyl[v]) * i1d;
        r -= ((double)fzh[v] - (double)fzl[v]) * i2d;
        rhs[v] = r;
    }
    const double* q = a.pr;
    rhs[8] -= a.p.glm_cp * a.p.glm_cp * q[8 * nc + cell];
    if (a.p.resistive && a.p.resistivity > 0.0 && lap) {
#pragma unroll
        for (int c = 0; c < 3; ++c) rhs[5 + c] += a.p.resistivity * lap[c];
    } else if (a.p.resistive && a.p.resistivity > 0.0) {
        const long sty = a.nz, stx = (long)a.ny * a.nz;
        const double ix2 = a.idd2[0], iy2 = a.idd2[1], iz2 = a.idd2[2];
#pragma unroll
        for (int c = 5; c < 8; ++c) {
            const double* B = q + (size_t)c * nc + cell;
            const double b0 = B[0];
            const double lap = (B[stx] - 2.0 * b0 + B[-stx]) * ix2 +
                               (B[sty] - 2.0 * b0 + B[-sty]) * iy2 +
                               (B[1] - 2.0 * b0 + B[-1]) * iz2;
            rhs[c] += a.p.resistivity * lap;
        }
    }
    const Phys<double> PD = Phys<double>::from(a.p);
    double q0[NM], U0[NM];
#pragma unroll
    for (int v = 0; v < NM; ++v) q0[v] = a.pr0[(size_t)v * nc + cell];
    r_p2c(PD, q0, U0);
    const double dt = a.dt;
#pragma unroll
    for (int v = 0; v < NM; ++v) {
        const double r = rhs[v], u0 = U0[v];
        double un;
        if (a.stage == 0) un = __dadd_rn(u0, __dmul_rn(dt, r));
        else {
            const double uk = a.U[(size_t)v * nc + cell];
            if (a.nstages == 2)
                un = __dmul_rn(0.5, __dadd_rn(__dadd_rn(u0, uk), __dmul_rn(dt, r)));
            else if (a.stage == 1)
                un = __dadd_rn(__dmul_rn(0.75, u0), __dmul_rn(0.25, __dadd_rn(uk, __dmul_rn(dt, r))));
            else
                un = __dadd_rn(__dmul_rn(1.0 / 3.0, u0),
                               __dmul_rn(2.0 / 3.0, __dadd_rn(uk, __dmul_rn(dt, r))));
        }
        a.U[(size_t)v * nc + cell] = un;
    }
    // rows past the 9 primitives: the passive scalars (no fluxes for RMHD
    // WENO/PPM, rmhd_core.py:1440-1557) get the SSPRK combination of the step
    // input and the stage input, any other row 0
    for (int v = NM; v < a.nv; ++v) {
        const size_t o = (size_t)v * nc + cell;
        const int tt = v - a.p.passive_offset;
        double out = 0.0;
        if (tt < 0 || tt >= a.p.n_passive) {
        } else if (a.stage == 0) out = __dadd_rn(a.pr0[o], __dmul_rn(dt, 0.0));
        else {
            const double t0 = a.pr0[o], tk = a.pr[o];
            if (a.nstages == 2)
                out = __dmul_rn(0.5, __dadd_rn(__dadd_rn(t0, tk), __dmul_rn(dt, 0.0)));
            else if (a.stage == 1)
                out = __dadd_rn(__dmul_rn(0.75, t0), __dmul_rn(0.25, __dadd_rn(tk, __dmul_rn(dt, 0.0))));
            else
                out = __dadd_rn(__dmul_rn(1.0 / 3.0, t0),
                                __dmul_rn(2.0 / 3.0, __dadd_rn(tk, __dmul_rn(dt, 0.0))));
        }
        a.dst[o] = out;
    }
}

__device__ __forceinline__ bool finite9(const float* F) {
    bool ok = true;
#pragma unroll
    for (int v = 0; v < NM; ++v) ok &= isfinite(F[v]);
    return ok;
}

template <int RECON, int RIEMANN>
__global__ void __launch_bounds__(kThreads, 4)
    k_stage(const __grid_constant__ CUtensorMap tm_halo, const __grid_constant__ CUtensorMap tm_core,
            const __grid_constant__ StageArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    float* halo = reinterpret_cast<float*>(sm + OFF_HALO);
    float* ring = reinterpret_cast<float*>(sm + OFF_RING);
    float* Fy = reinterpret_cast<float*>(sm + OFF_FY);
    float* Fz = reinterpret_cast<float*>(sm + OFF_FZ);
    unsigned* issued = reinterpret_cast<unsigned*>(sm + OFF_CNT);   // loads per barrier
    unsigned* failed = reinterpret_cast<unsigned*>(sm + OFF_FAIL);  // [2][kJobs]: lanes
    const uint32_t bar0 = smem_u32(sm + OFF_BAR);  // ring slots 0..5, then the halo box
    const uint32_t hbar = bar0 + 8 * NRING;

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    // tile origin; blockIdx.x: z tiles fastest, then y tiles; blockIdx.y: x chunks
    const int nzt = (a.hi[2] - a.lo + TZ - 1) / TZ;
    const int k0 = a.lo + (int)(blockIdx.x % nzt) * TZ;
    const int j0 = a.lo + (int)(blockIdx.x / nzt) * TY;
    const int i0 = a.lo + (int)blockIdx.y * TX;
    const int i1 = min(i0 + TX, a.hi[0]);
    if (i0 >= i1) return;
    const int j = j0 + warp, k = k0 + lane;
    const bool mine = j < a.hi[1] && k < a.hi[2];  // this thread's column holds a cell

    const Phys<float> P = Phys<float>::from(a.p);
    const int lim = a.p.limiter;
    const int base = i0 - 3;  // plane of ring index 0
    auto slot_of = [&](int plane) { return (plane - base) % NRING; };
    auto parity_of = [&](int plane) { return (uint32_t)(((plane - base) / NRING) & 1); };
    auto ring_at = [&](int plane) { return ring + slot_of(plane) * CORE_STRIDE; };

    if (t == 0) {
        for (int s = 0; s <= NRING; ++s) {
            bar_init(bar0 + 8 * s);
            issued[s] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (t < 3 * kJobs) failed[t] = 0;
    __syncthreads();
    auto load_ring = [&](int pl) {
        const int s = slot_of(pl);
        bar_expect(bar0 + 8 * s, CORE_BYTES);
        tma_load(smem_u32(ring_at(pl)), &tm_core, k0 - 3, j0, pl, bar0 + 8 * s);
        ++issued[s];
    };
    auto load_halo = [&](int pl) {
        bar_expect(hbar, HALO_BYTES);
        tma_load(smem_u32(halo), &tm_halo, k0 - 3, j0 - 3, pl, hbar);
        ++issued[NRING];
    };
    // the x faces' stencil of the first plane (planes i0-3 .. i0+2); the first
    // halo box goes out after the pass for plane i0 - 1, like every later one
    if (t == 0)
        for (int pl = i0 - 3; pl <= i0 + 2; ++pl) load_ring(pl);
    // planes i0-3 .. i0+1 here; the loop's first pass waits for i0+2
    bool w0 = true;
    for (int pl = i0 - 3; pl <= i0 + 1; ++pl)
        w0 &= bar_wait(bar0 + 8 * slot_of(pl), parity_of(pl), a.poll_limit);
    bool ok = __syncthreads_and(w0);

    float Flo[NM], Fhi[NM];
    // Per plane i, two barriers: (1) the waits for the halo box of plane i and
    // ring plane i+3, which also separate the previous plane's update (reads
    // of Fy / Fz) from this plane's face writes; (2) after the face jobs: the
    // y and z faces of plane i from the halo box (fluxes to shared memory)
    // and this thread's x face i + 1/2 from the ring (to Fhi), one loop so the
    // face code exists once.  Then the next loads go out and the cells of
    // plane i are updated.  The pass for "plane i0 - 1" computes only the x
    // face i0 - 1/2.  A face whose float32 result is not finite is marked; the
    // cells next to it are not updated here but listed for k_stage_fix, which
    // redoes them with that face in float64.  Marks rotate over three buffers
    // (written by plane i's jobs, read by its update, cleared during the next
    // plane's update).
#pragma unroll 1
    for (int i = i0 - 1; i < i1 && ok; ++i) {
        unsigned* fail = failed + (i % 3) * kJobs;  // i >= 2: no negative modulo
        const bool cells = i >= i0;
        if (cells && mine) {
            // L2 prefetch of this cell's float64 update operands
            const size_t nc = (size_t)a.nx * a.ny * a.nz;
            const size_t cell = ((size_t)i * a.ny + j) * a.nz + k;
#pragma unroll
            for (int v = 0; v < NM; ++v) {
                asm volatile("prefetch.global.L2 [%0];" ::"l"(a.pr0 + (size_t)v * nc + cell));
                if (a.stage > 0)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a.U + (size_t)v * nc + cell));
            }
        }
        bool w = bar_wait(bar0 + 8 * slot_of(i + 3), parity_of(i + 3), a.poll_limit);
        if (cells) w &= bar_wait(hbar, (uint32_t)((i - i0) & 1), a.poll_limit);
        ok = __syncthreads_and(w);
        if (!ok) break;
        // jobs: y and z faces warp-strided (none for plane i0 - 1), then the
        // warp's own x row
        int job = cells ? warp : kJobs;
#pragma unroll 1
        while (job <= kJobs) {
            const float* rows[6];
            int sv, dir, r, c;
            bool need;
            if (job == kJobs) {
                // x face of this thread's column, planes i-2 .. i+3 (every lane
                // computes it; only the lanes that own a cell use it)
#pragma unroll
                for (int o = 0; o < 6; ++o) rows[o] = ring_at(i - 2 + o) + warp * CZ + lane + 3;
                sv = TY * CZ;
                dir = 0;
                r = warp;
                c = lane;
                need = true;
            } else if (job < kYJobs) {
                // face between rows j0+job-1 and j0+job at column k0+lane
                r = job;
                c = lane;
                const float* s0 = halo + r * HZ + lane + 3;
#pragma unroll
                for (int o = 0; o < 6; ++o) rows[o] = s0 + o * HZ;
                sv = HY * HZ;
                dir = 1;
                need = k0 + c < a.hi[2] && j0 + r <= a.hi[1];
            } else {
                // the TY x (TZ+1) z faces, row-major, 32 per job
                const int f = (job - kYJobs) * 32 + lane;
                r = f / (TZ + 1);
                c = f - r * (TZ + 1);
                const float* s0 = halo + (r + 3) * HZ + c;
#pragma unroll
                for (int o = 0; o < 6; ++o) rows[o] = s0 + o;
                sv = HY * HZ;
                dir = 2;
                need = f < TY * (TZ + 1) && j0 + r < a.hi[1] && k0 + c <= a.hi[2];
            }
            if (need) {
                float F[NM];
                const bool fin = face_any<RECON, RIEMANN>(P, lim, rows, sv, dir, F);
                if (dir == 0) {
#pragma unroll
                    for (int v = 0; v < NM; ++v) Fhi[v] = fin ? F[v] : __int_as_float(0x7fc00000);
                } else if (dir == 1) {
#pragma unroll
                    for (int v = 0; v < NM; ++v) Fy[(v * (TY + 1) + r) * TZ + c] = F[v];
                    if (!fin) atomicOr(&fail[job], 1u << lane);
                } else {
#pragma unroll
                    for (int v = 0; v < NM; ++v) Fz[(v * TY + r) * (TZ + 1) + c] = F[v];
                    if (!fin) atomicOr(&fail[job], 1u << lane);
                }
            }
            job = job == kJobs ? kJobs + 1 : (job + TY < kJobs ? job + TY : kJobs);
        }
        // the resistive Laplacian of B of this thread's cell from the tiles (the
        // float32 copy; plane i in the halo box, planes i +- 1 in the ring),
        // differences in float64 -- before the tiles are refilled
        double lap[3];
        const bool resist = a.p.resistive && a.p.resistivity > 0.0;
        if (cells && mine && resist) {
            const double ix2 = a.idd2[0], iy2 = a.idd2[1], iz2 = a.idd2[2];
            const float* hc = halo + (warp + 3) * HZ + lane + 3;
            const float* rm = ring_at(i - 1) + warp * CZ + lane + 3;
            const float* rp = ring_at(i + 1) + warp * CZ + lane + 3;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int v = 5 + c;
                const double b0 = (double)hc[v * HY * HZ];
                lap[c] = ((double)rp[v * TY * CZ] - 2.0 * b0 + (double)rm[v * TY * CZ]) * ix2 +
                         ((double)hc[v * HY * HZ + HZ] - 2.0 * b0 + (double)hc[v * HY * HZ - HZ]) * iy2 +
                         ((double)hc[v * HY * HZ + 1] - 2.0 * b0 + (double)hc[v * HY * HZ - 1]) * iz2;
            }
        }
        __syncthreads();  // halo box and ring plane i-2 consumed; fluxes and marks complete
        if (t == 0 && i + 1 < i1) {
            load_halo(i + 1);
            load_ring(i + 4);
        }
        if (cells && mine) {
            // the cell's y and z faces: marks, then fluxes
            const int fz = warp * (TZ + 1) + lane;
            const bool bad = !finite9(Flo) || !finite9(Fhi) || ((fail[warp] >> lane) & 1u) ||
                             ((fail[warp + 1] >> lane) & 1u) ||
                             ((fail[kYJobs + (fz >> 5)] >> (fz & 31)) & 1u) ||
                             ((fail[kYJobs + ((fz + 1) >> 5)] >> ((fz + 1) & 31)) & 1u);
            if (bad) {
                const unsigned slot = atomicAdd(a.defer_count, 1u);
                a.defer_list[slot] = (unsigned)(((size_t)i * a.ny + j) * a.nz + k);
            } else {
                float fyl[NM], fyh[NM], fzl[NM], fzh[NM];
#pragma unroll
                for (int v = 0; v < NM; ++v) {
                    fyl[v] = Fy[(v * (TY + 1) + warp) * TZ + lane];
                    fyh[v] = Fy[(v * (TY + 1) + warp + 1) * TZ + lane];
                    fzl[v] = Fz[v * TY * (TZ + 1) + fz];
                    fzh[v] = Fz[v * TY * (TZ + 1) + fz + 1];
                }
                update_cell(a, i, j, k, Flo, Fhi, fyl, fyh, fzl, fzh, resist ? lap : nullptr);
            }
        }
        // the marks of plane i + 2 (last read by the update of plane i - 1)
        if (t < kJobs) failed[((i + 2) % 3) * kJobs + t] = 0;
#pragma unroll
        for (int v = 0; v < NM; ++v) Flo[v] = Fhi[v];
    }
    if (!ok) {
        // a tile load did not land in time: before the block's shared memory
        // goes away, wait (bounded again, with the full budget whatever the
        // tile waits had) for the last load issued on every barrier (at most
        // one per barrier is ever outstanding), and report
        if (t == 0) {
            for (int s = 0; s <= NRING; ++s)
                if (issued[s] > 0) bar_wait(bar0 + 8 * s, (issued[s] - 1) & 1u);
            if (a.timeouts) atomicAdd(a.timeouts, 1ull);
        }
        __syncthreads();
    }
}

// The cells k_stage listed: all six faces again from global memory, float32
// from the padded copy (the same face code) and, where that is not finite,
// float64 from the stage input; then the update.
template <int RECON, int RIEMANN>
__global__ void __launch_bounds__(128) k_stage_fix(const __grid_constant__ StageArgs a) {
    const unsigned n = *a.defer_count;
    const Phys<float> P = Phys<float>::from(a.p);
    const size_t vs = (size_t)a.nx * a.ny * a.pitch;  // variable stride of the copy
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const unsigned cell = a.defer_list[e];
        const int k = (int)(cell % (unsigned)a.nz);
        const unsigned rr = cell / (unsigned)a.nz;
        const int j = (int)(rr % (unsigned)a.ny), i = (int)(rr / (unsigned)a.ny);
        float F[6][NM];
#pragma unroll 1
        for (int f = 0; f < 6; ++f) {
            const int dir = f >> 1, hi = f & 1;
            const int fi = i + (dir == 0 ? hi : 0), fj = j + (dir == 1 ? hi : 0),
                      fk = k + (dir == 2 ? hi : 0);
            const long st = dir == 0 ? (long)a.ny * a.pitch : (dir == 1 ? (long)a.pitch : 1L);
            const float* c0 = a.prf + ((size_t)fi * a.ny + fj) * a.pitch + fk;
            const float* rows[6];
            for (int o = 0; o < 6; ++o) rows[o] = c0 + (o - 3) * st;
            float G[NM];
            bool fin = face_any<RECON, RIEMANN>(P, a.p.limiter, rows, (int)vs, dir, G);
            if (!fin) {
                if (dir == 0) face_f64<RECON, RIEMANN, 0>(a, fi, fj, fk, G);
                else if (dir == 1) face_f64<RECON, RIEMANN, 1>(a, fi, fj, fk, G);
                else face_f64<RECON, RIEMANN, 2>(a, fi, fj, fk, G);
            }
            for (int v = 0; v < NM; ++v) F[f][v] = G[v];
        }
        update_cell(a, i, j, k, F[0], F[1], F[2], F[3], F[4], F[5]);
    }
}

// cuTensorMapEncodeTiled from the driver, without linking libcuda
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)f;
    });
    return fn;
}

// The float32 copy as a 4-d tensor (k, j, i, v), rows padded to `pitch`
// floats (a multiple of 16 bytes, as the TMA strides must be).
bool make_map(CUtensorMap* m, const float* prf, int pitch, int ny, int nx, uint32_t box_k,
              uint32_t box_j) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)pitch, (cuuint64_t)ny, (cuuint64_t)nx, (cuuint64_t)NM};
    const cuuint64_t strides[3] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * ny * 4,
                                   (cuuint64_t)pitch * ny * nx * 4};
    const cuuint32_t box[4] = {box_k, box_j, 1, NM};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void*)prf, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

template <int RE, int RI>
cudaError_t launch_t(const CUtensorMap& mh, const CUtensorMap& mc, const StageArgs& a, dim3 grid,
                     cudaStream_t s) {
    // the shared-memory attributes are per device: set once on each
    static unsigned long long done = 0;  // bit d: set on device d (d < 64)
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return cudaErrorInvalidDevice;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (!(done & bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_stage<RE, RI>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
        if (e != cudaSuccess) return e;
        cudaFuncSetAttribute(k_stage<RE, RI>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        done |= bit;
    }
    cudaError_t e = cudaMemsetAsync(a.defer_count, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    k_stage<RE, RI><<<grid, kThreads, kSmem, s>>>(mh, mc, a);
    k_stage_fix<RE, RI><<<148, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

bool supported(const AstroParams& p, const AstroGrid& g) {
    if (p.physics != ASTRO_RMHD || p.precision != ASTRO_PREC_MIXED) return false;
    if (p.flux_mode != ASTRO_FLUX_CONSERVATIVE || !p.fused_stage) return false;
    // WENO5 / PPM: stencil radius 3 and first updated cell 3, so every tile's
    // boxes start on a 16-byte boundary (k0 - 3 = 32 t)
    if (p.recon != ASTRO_RECON_WENO && p.recon != ASTRO_RECON_PPM) return false;
    if (p.riemann != ASTRO_RIEMANN_HLLE && p.riemann != ASTRO_RIEMANN_HLLD) return false;
    // the updated range [3, n-3) must be non-empty in every direction; the
    // TMA boxes start at lo - 3 = 0 plus whole tiles (16-byte aligned)
    return g.nx >= 7 && g.ny >= 7 && g.nz >= 7 && g.nv >= NM;
}

cudaError_t launch(const StageArgs& a, cudaStream_t s) {
    CUtensorMap mh, mc;
    memset(&mh, 0, sizeof(mh));
    memset(&mc, 0, sizeof(mc));
    if (!make_map(&mh, a.prf, a.pitch, a.ny, a.nx, HZ, HY) ||
        !make_map(&mc, a.prf, a.pitch, a.ny, a.nx, CZ, TY))
        return cudaErrorInvalidValue;
    const int nzt = (a.hi[2] - a.lo + TZ - 1) / TZ;
    const int nyt = (a.hi[1] - a.lo + TY - 1) / TY;
    const int nxc = (a.hi[0] - a.lo + TX - 1) / TX;
    if (nzt <= 0 || nyt <= 0 || nxc <= 0) return cudaSuccess;
    const dim3 grid((unsigned)(nzt * nyt), (unsigned)nxc);
    if (a.p.recon == ASTRO_RECON_WENO) {
        if (a.p.riemann == ASTRO_RIEMANN_HLLD) return launch_t<ASTRO_RECON_WENO, ASTRO_RIEMANN_HLLD>(mh, mc, a, grid, s);
        return launch_t<ASTRO_RECON_WENO, ASTRO_RIEMANN_HLLE>(mh, mc, a, grid, s);
    }
    if (a.p.riemann == ASTRO_RIEMANN_HLLD) return launch_t<ASTRO_RECON_PPM, ASTRO_RIEMANN_HLLD>(mh, mc, a, grid, s);
    return launch_t<ASTRO_RECON_PPM, ASTRO_RIEMANN_HLLE>(mh, mc, a, grid, s);
}

}  // namespace astro_stage
