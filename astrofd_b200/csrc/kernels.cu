// kernels.cu -- sm_100a kernels and the C ABI of libastrofd_b200.so.
//
// Per SSPRK stage the right-hand side is built face by face:
//   k_face    one thread per cell face in one direction: reconstruct the
//             left/right primitive states from the 4- or 6-point stencil,
//             floor, p2c, physical flux, wave speeds, Riemann flux.  Every face
//             is evaluated once (the reference evaluates each face twice, once
//             from each neighbour).  The result lands in a per-direction face
//             buffer F[v][cell], indexed by the cell on the high side.
//   k_update  one thread per cell (ghosts included): flux divergence, GLM
//             damping, resistive Laplacian, passive-scalar fluxes, the SSPRK
//             combination in float64 and con2prim, writing U_k and the next
//             stage's primitives.  Cells outside the reference's loop bounds get
//             rhs = 0, i.e. the reference's p2c -> c2p round trip.
// The reference's RMHD PPM/WENO x faces use the wave speeds left over from the
// previous cell's z face (core/rmhd_core.py:1285,1314,1445,1468).  In
// ASTRO_FLUX_REFERENCE mode those faces are evaluated a second time with the
// carried speeds (k_face<GIVEN=true>), read from the z-face speed buffer; in
// ASTRO_FLUX_CONSERVATIVE mode every face uses its own speeds, so each face
// flux enters both neighbours and the scheme conserves D, S, tau exactly.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <vector>

#include "mlp.cuh"
#include "physics.cuh"
#include "stage.cuh"

using namespace astro;

namespace {

// process-wide count of kernels this library has launched (diagnostic only)
std::atomic<unsigned long long> g_launches{0};
// polls per MMA-completion wait of the learned con2prim (test hook)
std::atomic<long long> g_mma_poll_limit{0};
inline long mma_poll_limit() {
    const long long v = g_mma_poll_limit.load(std::memory_order_relaxed);
    return v > 0 ? (long)v : mlp::kPollLimit;
}
// polls per tile-load wait of the fused stage kernel (test hook)
std::atomic<long long> g_tile_poll_limit{0};
inline long tile_poll_limit() {
    const long long v = g_tile_poll_limit.load(std::memory_order_relaxed);
    return v > 0 ? (long)v : astro_stage::kTilePollLimit;
}
// Newton polish steps of the learned con2prim in the steps (test hook; -1:
// the default of 2)
std::atomic<int> g_step_polish{-1};
inline int step_polish() {
    const int v = g_step_polish.load(std::memory_order_relaxed);
    return v >= 0 ? v : 2;
}

// Optional per-launch CUDA-event timing (astro_step_profiled, and the
// astro_prof_start/stop sessions): an event is recorded after every launch;
// the gap to the previous event is charged to the launch's kernel class.
struct Prof {
    std::vector<cudaEvent_t> ev;  // cap + 1
    std::vector<int> kind;        // cap
    int n = 0;
    bool on = false;
    int create(int cap) {
        ev.assign((size_t)cap + 1, nullptr);
        kind.assign((size_t)cap, 0);
        for (auto& e : ev)
            if (cudaEventCreate(&e) != cudaSuccess) return ASTRO_E_CUDA;
        return ASTRO_OK;
    }
    int cap() const { return (int)kind.size(); }
    void sum(AstroKernelTimes* t) const {
        memset(t, 0, sizeof(*t));
        for (int i = 0; i < n; ++i) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
            const int k = kind[i] < 5 ? kind[i] : 2;
            t->ms[k] += ms;
            t->launches[k] += 1;
        }
    }
    ~Prof() {
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    }
};
thread_local Prof* t_prof = nullptr;

inline void mark(int kind, cudaStream_t s) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    Prof* P = t_prof;
    if (P && P->on && P->n < P->cap()) {
        cudaEventRecord(P->ev[P->n + 1], s);
        P->kind[P->n++] = kind;
    }
}

constexpr int kMaxPassive = 8;
constexpr int kMaxNV = 64;

struct Bounds {
    int lo, hi[3];  // cells updated: [lo, hi[d]) per dimension
};

// loop bounds of the reference right-hand sides (ghost-inclusive indices)
__host__ Bounds bounds_of(const AstroParams& p, const AstroGrid& g) {
    Bounds b;
    b.lo = (p.recon == ASTRO_RECON_MUSCL) ? 2 : 3;
    int off = (p.recon != ASTRO_RECON_MUSCL) ? 3 : (p.physics == ASTRO_SRHD ? 3 : 2);
    b.hi[0] = g.nx - off;
    b.hi[1] = g.ny - off;
    b.hi[2] = g.nz - off;
    return b;
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Layout {
    size_t prA, prB, U, F[3], FxC, aux[3], Sz, fix, c2pfb, prf, dfr, total;
    bool fused;  // stages run as the fused kernel (stage.cu): no face buffers,
                 // the float32 copy in padded rows of `pitch` floats
    int pitch;
};

inline bool carried_mode(const AstroParams& p) {
    return p.physics == ASTRO_RMHD && p.recon != ASTRO_RECON_MUSCL &&
           p.flux_mode == ASTRO_FLUX_REFERENCE;
}

inline bool passive_fluxes(const AstroParams& p) {
    if (p.n_passive <= 0) return false;
    if (p.physics == ASTRO_SRHD) return p.recon != ASTRO_RECON_WENO;
    return p.recon == ASTRO_RECON_MUSCL;
}

// capacity of the float64 fix-up list: a fraction of one face pass; faces
// beyond it keep their float32 result (counted, never written out of bounds)
inline size_t fix_capacity(const AstroGrid& g) {
    const size_t nc = (size_t)g.nx * g.ny * g.nz;
    return nc / 16 + 1024;
}

// learned con2prim: cells whose Newton polish fails are listed (one slot per
// cell, so the list cannot overflow) and solved by a second kernel in dense
// warps; the listing kernel then carries no copy of the full solver
inline size_t c2p_fb_capacity(const AstroGrid& g) { return (size_t)g.nx * g.ny * g.nz; }

// fused: the step's stages run as the fused kernel (astro_stage::supported;
// steps only, not the GR wrappers)
Layout layout_of(const AstroParams& p, const AstroGrid& g, bool with_state, bool fused = false) {
    Layout L;
    memset(&L, 0, sizeof(L));
    const size_t nc = (size_t)g.nx * g.ny * g.nz;
    const int nm = p.physics == ASTRO_SRHD ? 5 : 9;
    const size_t rs = p.precision == ASTRO_PREC_MIXED ? 4 : 8;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t r = o; o += align256(bytes); return r; };
    L.fused = fused && with_state;
    L.pitch = g.nz;
    L.prA = with_state ? take((size_t)g.nv * nc * 8) : 0;
    L.prB = with_state ? take((size_t)g.nv * nc * 8) : 0;
    L.U = with_state ? take((size_t)nm * nc * 8) : 0;
    if (L.fused) {
        L.pitch = astro_stage::pitch_of(g.nz);
        L.prf = take((size_t)nm * g.nx * g.ny * L.pitch * sizeof(float));
        // cells whose float32 faces overflowed (a slot for every cell)
        L.dfr = take(256 + nc * sizeof(unsigned));
        L.c2pfb = p.c2p_guess == ASTRO_GUESS_LEARNED ? take(256 + c2p_fb_capacity(g) * sizeof(unsigned)) : 0;
        L.total = o;
        return L;
    }
    for (int d = 0; d < 3; ++d) L.F[d] = take((size_t)nm * nc * rs);
    L.FxC = carried_mode(p) ? take((size_t)nm * nc * rs) : 0;
    for (int d = 0; d < 3; ++d) L.aux[d] = passive_fluxes(p) ? take(4 * nc * rs) : 0;
    L.Sz = carried_mode(p) ? take(2 * nc * rs) : 0;
    // float32 passes: counter + list of faces to recompute in float64
    L.fix = p.precision == ASTRO_PREC_MIXED ? take(256 + fix_capacity(g) * sizeof(unsigned)) : 0;
    // float32 copy of the nm primitives the float32 face passes read
    L.prf = p.precision == ASTRO_PREC_MIXED ? take((size_t)nm * nc * sizeof(float)) : 0;
    L.c2pfb = (with_state && p.c2p_guess == ASTRO_GUESS_LEARNED)
                  ? take(256 + c2p_fb_capacity(g) * sizeof(unsigned))
                  : 0;
    L.total = o;
    return L;
}

int validate(const AstroParams* p, const AstroGrid* g) {
    if (!p || !g) return ASTRO_E_INVALID;
    if (p->physics != ASTRO_SRHD && p->physics != ASTRO_RMHD) return ASTRO_E_INVALID;
    if (p->recon < 0 || p->recon > 2 || p->limiter < 0 || p->limiter > 2) return ASTRO_E_INVALID;
    if (p->riemann < 0 || p->riemann > (p->physics == ASTRO_SRHD ? 1 : 2)) return ASTRO_E_INVALID;
    if (p->precision != ASTRO_PREC_FP64 && p->precision != ASTRO_PREC_MIXED) return ASTRO_E_INVALID;
    if (p->flux_mode != ASTRO_FLUX_REFERENCE && p->flux_mode != ASTRO_FLUX_CONSERVATIVE)
        return ASTRO_E_INVALID;
    const int nm = p->physics == ASTRO_SRHD ? 5 : 9;
    if (g->nv < nm || g->nv > kMaxNV) return ASTRO_E_SHAPE;
    if (p->n_passive < 0 || p->n_passive > kMaxPassive) return ASTRO_E_UNSUPPORTED;
    if (p->n_passive > 0 && (p->passive_offset < nm || p->passive_offset + p->n_passive > g->nv))
        return ASTRO_E_SHAPE;
    // the bulk pressure the SRHD MUSCL faces add sits in variable 5
    if (p->physics == ASTRO_SRHD && p->passive_offset > 5 && g->nv < 6) return ASTRO_E_SHAPE;
    // any block size: where a small block leaves a scheme's cell range
    // [lo, n - off) empty, nothing is updated there, as in the reference's
    // loops; every stencil read of a cell in the range stays inside the block
    if (g->nx < 1 || g->ny < 1 || g->nz < 1) return ASTRO_E_SHAPE;
    // cell indices are 32-bit in the kernels; 2^31 cells of even 5 float64
    // variables exceed the device memory
    if ((double)g->nx * g->ny * g->nz >= 2147483648.0) return ASTRO_E_SHAPE;
    if (!(g->dx > 0) || !(g->dy > 0) || !(g->dz > 0)) return ASTRO_E_INVALID;
    return ASTRO_OK;
}

// ------------------------------------------------------------ face pass ---
struct FaceArgs {
    const double* pr;
    const float* prf;    // float32 copy of the nm primitives (float32 passes)
    int nx, ny, nz;
    int dir;
    int org[3], ext[3];  // first cell and extents of the face block
    Bounds b;
    void* F;             // R[nm][nc]
    void* aux;           // R[4][nc]: sL, sR, vL, vR (or null)
    void* speeds_out;    // R[2][nc]: sL, sR (z faces, carried mode) or null
    const void* carried; // R[2][nc]: z-face speeds read by the carried x faces
    int ndiss;           // SRHD Israel-Stewart blocks: dissipation fluxes per face
    AstroParams p;
    // float32 passes: faces whose float32 result is not finite are listed here
    // and recomputed in float64 by k_face_fix
    unsigned* fix_count;
    unsigned* fix_list;
    unsigned fix_cap;
};

// One face: reconstruct, floor, p2c, flux, speeds, Riemann in arithmetic R,
// stored as RS.  Returns false when the stored flux or speeds are not finite.
template <int PHYS, int RECON, int RIEMANN, typename R, typename RS, bool GIVEN, int DIR>
__device__ __forceinline__ bool face_at(const FaceArgs& a, int i, int j, int k) {
    constexpr int NM = PHYS == ASTRO_SRHD ? 5 : 9;
    const size_t nc = (size_t)a.nx * a.ny * a.nz;
    const size_t cell = ((size_t)i * a.ny + j) * a.nz + k;
    const long stride = DIR == 0 ? (long)a.ny * a.nz : (DIR == 1 ? (long)a.nz : 1L);
    const Phys<R> P = Phys<R>::from(a.p);

    R qL[NM], qR[NM];
    constexpr int o0 = RECON == ASTRO_RECON_MUSCL ? -2 : -3;
    constexpr int o1 = RECON == ASTRO_RECON_MUSCL ? 1 : 2;
#pragma unroll
    for (int v = 0; v < NM; ++v) {
        R st[6];
        if constexpr (sizeof(R) == 4) {
            // the float32 copy: one conversion per cell and stage instead of
            // one per stencil use
            const float* base = a.prf + (size_t)v * nc + cell;
#pragma unroll
            for (int o = o0; o <= o1; ++o) st[o + 3] = __ldg(base + o * stride);
        } else {
            const double* base = a.pr + (size_t)v * nc + cell;
#pragma unroll
            for (int o = o0; o <= o1; ++o) st[o + 3] = (R)__ldg(base + o * stride);
        }
        recon_face<RECON>(st, a.p.limiter, qL[v], qR[v]);
    }
    R F[NM];
    R sL = R(-1), sR = R(1);
    if (GIVEN) {
        // previous cell of the reference's i-j-k loop, whose z-low face speeds
        // are still in (sL, sR) when this cell's x-low face is evaluated
        int pi = i, pj = j, pk = k;
        bool first = false;
        if (k > a.b.lo) pk = k - 1;
        else if (j > a.b.lo) { pj = j - 1; pk = a.b.hi[2] - 1; }
        else if (i > a.b.lo) { pi = i - 1; pj = a.b.hi[1] - 1; pk = a.b.hi[2] - 1; }
        else first = true;
        if (!first) {
            const RS* S = (const RS*)a.carried;
            const size_t pc = ((size_t)pi * a.ny + pj) * a.nz + pk;
            sL = (R)S[pc];
            sR = (R)S[nc + pc];
        }
    }
    if (PHYS == ASTRO_SRHD) {
        if (RECON == ASTRO_RECON_MUSCL && a.p.passive_offset > 5) {
            // add_pi_lr (srhd_core.py:394-398): the cells' bulk pressure on
            // the reconstructed face pressures, before the floor
            qL[4] += (R)__ldg(a.pr + 5 * nc + cell - stride);
            qR[4] += (R)__ldg(a.pr + 5 * nc + cell);
        }
        if (a.ndiss > 0) {
            R isL[10], isR[10];
#pragma unroll
            for (int m = 0; m < 10; ++m) {
                isL[m] = (R)__ldg(a.pr + (size_t)(5 + m) * nc + cell - stride);
                isR[m] = (R)__ldg(a.pr + (size_t)(5 + m) * nc + cell);
            }
            s_face<RIEMANN>(P, DIR, qL, qR, F, sL, sR, a.ndiss, isL, isR);
        } else {
            s_face<RIEMANN>(P, DIR, qL, qR, F, sL, sR);
        }
    } else {
        r_face<RIEMANN, RECON == ASTRO_RECON_MUSCL, GIVEN>(P, DIR, qL, qR, F, sL, sR);
    }
    RS* Fo = (RS*)a.F;
    bool finite = true;
#pragma unroll
    for (int v = 0; v < NM; ++v) {
        const RS f = (RS)F[v];
        finite &= isfinite(f);
        Fo[(size_t)v * nc + cell] = f;
    }
    finite &= isfinite((RS)sL) && isfinite((RS)sR);
    if (a.aux) {
        RS* A = (RS*)a.aux;
        A[cell] = (RS)sL;
        A[nc + cell] = (RS)sR;
        A[2 * nc + cell] = (RS)qL[1 + DIR];
        A[3 * nc + cell] = (RS)qR[1 + DIR];
    }
    if (a.speeds_out) {
        RS* S = (RS*)a.speeds_out;
        S[cell] = (RS)sL;
        S[nc + cell] = (RS)sR;
    }
    return finite;
}

template <int PHYS, int RECON, int RIEMANN, typename R, bool GIVEN, int DIR>
__global__ void __launch_bounds__(128) k_face(FaceArgs a) {
    // grid: x over the (j, k) plane of the face block, y over its x layers;
    // one 32-bit split of the in-plane index per thread
    const unsigned e2 = (unsigned)a.ext[2];
    const unsigned plane = (unsigned)a.ext[1] * e2;
    const unsigned tp = blockIdx.x * blockDim.x + threadIdx.x;
    if (tp >= plane) return;
    const int c = (int)(tp % e2), bb = (int)(tp / e2);
    for (int aa = blockIdx.y; aa < a.ext[0]; aa += gridDim.y) {
        const int i = a.org[0] + aa, j = a.org[1] + bb, k = a.org[2] + c;
        const bool ok = face_at<PHYS, RECON, RIEMANN, R, R, GIVEN, DIR>(a, i, j, k);
        if (sizeof(R) == 4 && !ok && a.fix_list) {
            const unsigned slot = atomicAdd(a.fix_count, 1u);
            if (slot < a.fix_cap) a.fix_list[slot] = (unsigned)aa * plane + tp;
        }
    }
}

// whether everything face_at stored for this face (fluxes, and the speeds
// and face velocities where the pass keeps them) is finite
template <int NM>
__device__ __forceinline__ bool face_stored_finite(const FaceArgs& a, size_t nc, size_t cell) {
    bool ok = true;
    const float* F = (const float*)a.F;
#pragma unroll
    for (int v = 0; v < NM; ++v) ok &= isfinite(F[(size_t)v * nc + cell]);
    if (a.aux) {
        const float* A = (const float*)a.aux;
#pragma unroll
        for (int m = 0; m < 4; ++m) ok &= isfinite(A[(size_t)m * nc + cell]);
    }
    if (a.speeds_out) {
        const float* S = (const float*)a.speeds_out;
        ok &= isfinite(S[cell]) && isfinite(S[nc + cell]);
    }
    return ok;
}

// float64 recomputation of the faces a float32 pass listed as non-finite
// (float32 overflows where float64 does not, e.g. squared WENO smoothness
// indicators of a state whose fields have grown past ~1e9).  If more faces
// failed than the list holds (the counter keeps counting past its capacity),
// the list is incomplete: every face of the pass is then checked and the
// non-finite ones are recomputed, so no float32 failure is left in place.
template <int PHYS, int RECON, int RIEMANN, bool GIVEN, int DIR>
__global__ void __launch_bounds__(128) k_face_fix(FaceArgs a) {
    constexpr int NM = PHYS == ASTRO_SRHD ? 5 : 9;
    const unsigned cnt = *a.fix_count;
    if (cnt <= a.fix_cap) {
        for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt;
             q += gridDim.x * blockDim.x) {
            const long t = a.fix_list[q];
            const int c = (int)(t % a.ext[2]);
            const long r = t / a.ext[2];
            const int bb = (int)(r % a.ext[1]);
            const int aa = (int)(r / a.ext[1]);
            face_at<PHYS, RECON, RIEMANN, double, float, GIVEN, DIR>(a, a.org[0] + aa,
                                                                    a.org[1] + bb, a.org[2] + c);
        }
        return;
    }
    const size_t nc = (size_t)a.nx * a.ny * a.nz;
    const size_t plane = (size_t)a.ext[1] * a.ext[2];
    const size_t total = (size_t)a.ext[0] * plane;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (size_t)gridDim.x * blockDim.x) {
        const int aa = (int)(q / plane);
        const size_t tp = q % plane;
        const int bb = (int)(tp / a.ext[2]), c = (int)(tp % a.ext[2]);
        const int i = a.org[0] + aa, j = a.org[1] + bb, k = a.org[2] + c;
        const size_t cell = ((size_t)i * a.ny + j) * a.nz + k;
        if (!face_stored_finite<NM>(a, nc, cell))
            face_at<PHYS, RECON, RIEMANN, double, float, GIVEN, DIR>(a, i, j, k);
    }
}

// ---------------------------------------------------------- update pass ---
struct UpdArgs {
    const double* pr0;   // step input primitives (U0 = p2c(pr0), passives t0)
    const double* prk;   // this stage's input primitives
    double* U;           // U_{k-1} in, U_k out (may be null for rhs-only)
    double* dst;         // next primitives (stage mode) or rhs (rhs mode)
    float* dstf;         // optional float32 copy of the next nm primitives
    const void* F[3];
    const void* FxL;     // x-low-face fluxes (== F[0] unless carried mode)
    const void* aux[3];
    int nv, nx, ny, nz;
    Bounds b;
    double dd[3], dt;
    // 1/dd and 1/(dd^2 + 1e-12), the IEEE quotients the kernel would form
    // per cell, computed once on the host (the same values)
    double idd[3], idd2[3];
    int stage, nstages, rhs_only;
    int defer_c2p;       // learned con2prim: write U every stage, primitives later
    int frame_only;      // only the cells outside the updated range (the fused
                         // stage kernel updates the others)
    AstroParams p;
    AstroC2PStats* stats;
};

// Numba's addressing for the passive stencils of the MUSCL right-hand sides:
// negative indices wrap per axis, positive overruns alias the next row of the
// C-contiguous block (core/srhd_core.py:550-560, core/rmhd_core.py:832-940).
// A read past the end of the block is undefined in the reference; NaN here.
__device__ __forceinline__ double pget(const double* pr, int nv, int nx, int ny, int nz, int v,
                                       int i, int j, int k) {
    if (i < 0) i += nx;
    if (j < 0) j += ny;
    if (k < 0) k += nz;
    const size_t flat = (((size_t)v * nx + i) * ny + j) * nz + k;
    if (flat >= (size_t)nv * nx * ny * nz) return __longlong_as_double(0x7ff8000000000000LL);
    return __ldg(pr + flat);
}

enum { PK_WENO = 0, PK_PPM = 1, PK_MC = 2 };

__device__ double passive_face(const UpdArgs& a, int idx, int kind, int n, int i, int j, int k,
                               double vL, double vR, double sL, double sR) {
    const int di = n == 0, dj = n == 1, dk = n == 2;
    double s[6];
#pragma unroll
    for (int o = -3; o <= 2; ++o)
        s[o + 3] = pget(a.prk, a.nv, a.nx, a.ny, a.nz, idx, i + o * di, j + o * dj, k + o * dk);
    double tL, tR;
    if (kind == PK_WENO) recon_face<ASTRO_RECON_WENO>(s, 0, tL, tR);
    else if (kind == PK_PPM) recon_face<ASTRO_RECON_PPM>(s, 0, tL, tR);
    else recon_face<ASTRO_RECON_MUSCL>(s, a.p.limiter, tL, tR);
    return hlle_scalar(tL, tR, tL * vL, tR * vR, sL, sR);
}

template <typename RF> __device__ __forceinline__ double ldf(const void* p, size_t i) {
    return (double)__ldg((const RF*)p + i);
}

constexpr int kUpdateBlock = 128;

// DEFER: the learned con2prim runs in its own kernel, so this one only writes
// U (the con2prim code is compiled out).  Every load is a plain coalesced
// load with no dependence on an earlier one, so a thread's loads overlap each
// other; 8 blocks of 128 threads per SM (64 registers, a few spilled) keep
// more of them in flight than 6 blocks at 80 registers (3.81 against 3.96
// ms/step; 10 and 12 blocks spill too much).  Staging the loads through
// shared memory with per-thread cp.async streamed more slowly on B200 (4.2
// against 6.4 TB/s for the same bytes).
template <int PHYS, typename RF, bool DEFER, bool PASSIVE>
__global__ void __launch_bounds__(kUpdateBlock, PASSIVE ? 1 : 8) k_update(UpdArgs a) {
    constexpr int NM = PHYS == ASTRO_SRHD ? 5 : 9;
    constexpr int T = kUpdateBlock;
    const unsigned nc32 = (unsigned)a.nx * (unsigned)a.ny * (unsigned)a.nz;
    const size_t nc = nc32;
    const unsigned cell32 = blockIdx.x * T + threadIdx.x;
    const size_t cell = cell32;
    const int np = a.p.n_passive, po = a.p.passive_offset;
    C2PCount cnt;
    if (cell32 < nc32) {
        const unsigned k = cell32 % (unsigned)a.nz;
        const unsigned r32 = cell32 / (unsigned)a.nz;
        const unsigned j = r32 % (unsigned)a.ny;
        const unsigned i = r32 / (unsigned)a.ny;
        const bool in = (int)i >= a.b.lo && (int)i < a.b.hi[0] && (int)j >= a.b.lo &&
                        (int)j < a.b.hi[1] && (int)k >= a.b.lo && (int)k < a.b.hi[2];
        if (DEFER && a.frame_only && in) return;
        const long st[3] = {(long)a.ny * a.nz, (long)a.nz, 1L};
        int nres = 0;
        if (PHYS == ASTRO_RMHD && a.p.resistive && a.p.resistivity > 0.0) {
            // conservative mode applies eta*Laplacian(B) exactly once for
            // every reconstruction (the reference adds it twice for PPM and
            // not at all for WENO, rmhd_core.py:1414-1435,1440-1557)
            nres = a.p.flux_mode == ASTRO_FLUX_CONSERVATIVE
                       ? 1
                       : (a.p.recon == ASTRO_RECON_MUSCL ? 1 : (a.p.recon == ASTRO_RECON_PPM ? 2 : 0));
        }
        auto flux = [&](int d, int v, int hi) -> double {
            const size_t o = (size_t)v * nc + cell;
            if (hi) return ldf<RF>(a.F[d], o + st[d]);
            return ldf<RF>(d == 0 ? a.FxL : a.F[d], o);
        };
        double rhs[NM];
        double rp[kMaxPassive];
#pragma unroll
        for (int v = 0; v < NM; ++v) rhs[v] = 0.0;
        for (int t = 0; t < np; ++t) rp[t] = 0.0;
        if (in) {
            if constexpr (sizeof(RF) == 4) {
                // float32 fluxes: multiply by 1/dx (the float64 path divides
                // as the reference does)
                const double i0 = a.idd[0], i1 = a.idd[1], i2 = a.idd[2];
#pragma unroll
                for (int v = 0; v < NM; ++v) {
                    double r = 0.0;
                    r -= (flux(0, v, 1) - flux(0, v, 0)) * i0;
                    r -= (flux(1, v, 1) - flux(1, v, 0)) * i1;
                    r -= (flux(2, v, 1) - flux(2, v, 0)) * i2;
                    rhs[v] = r;
                }
            } else {
#pragma unroll
                for (int v = 0; v < NM; ++v) {
                    double r = 0.0;
                    r -= (flux(0, v, 1) - flux(0, v, 0)) / a.dd[0];
                    r -= (flux(1, v, 1) - flux(1, v, 0)) / a.dd[1];
                    r -= (flux(2, v, 1) - flux(2, v, 0)) / a.dd[2];
                    rhs[v] = r;
                }
            }
            if (PHYS == ASTRO_RMHD) {
                const double* q = a.prk;
                const double psi = q[8 * nc + cell];
                rhs[8] -= a.p.glm_cp * a.p.glm_cp * psi;
                for (int rep = 0; rep < nres; ++rep) {
                    const double ix2 = a.idd2[0], iy2 = a.idd2[1], iz2 = a.idd2[2];
#pragma unroll
                    for (int c = 5; c < 8; ++c) {
                        const double* B = q + (size_t)c * nc + cell;
                        const double b0 = B[0];
                        double lap = (B[st[0]] - 2.0 * b0 + B[-st[0]]) * ix2 +
                                     (B[st[1]] - 2.0 * b0 + B[-st[1]]) * iy2 +
                                     (B[st[2]] - 2.0 * b0 + B[-st[2]]) * iz2;
                        rhs[c] += a.p.resistivity * lap;
                    }
                }
            }
            // passive scalars: the reference's triple evaluation (see header)
            if (PASSIVE && np > 0) {
                for (int n = 0; n < 3; ++n) {
                    int kinds[3], nk = 0, lkind = PK_MC;
                    if (PHYS == ASTRO_SRHD) {
                        if (a.p.recon == ASTRO_RECON_MUSCL && n == 0) { kinds[0] = PK_WENO; kinds[1] = PK_PPM; kinds[2] = PK_MC; nk = 3; }
                        if (a.p.recon == ASTRO_RECON_MUSCL && n == 2) { kinds[0] = PK_MC; nk = 1; }
                        if (a.p.recon == ASTRO_RECON_PPM && n == 1) { kinds[0] = PK_WENO; kinds[1] = PK_PPM; kinds[2] = PK_MC; nk = 3; }
                        if (a.p.recon == ASTRO_RECON_PPM && n == 2) { kinds[0] = PK_WENO; kinds[1] = PK_PPM; nk = 2; lkind = PK_PPM; }
                    } else if (a.p.recon == ASTRO_RECON_MUSCL) {
                        kinds[0] = PK_WENO; kinds[1] = PK_PPM; kinds[2] = PK_MC; nk = 3;
                    }
                    if (nk == 0) continue;
                    const size_t lo = cell, hi = cell + st[n];
                    const double sLl = ldf<RF>(a.aux[n], lo), sRl = ldf<RF>(a.aux[n], nc + lo);
                    const double vLl = ldf<RF>(a.aux[n], 2 * nc + lo), vRl = ldf<RF>(a.aux[n], 3 * nc + lo);
                    double sLh = ldf<RF>(a.aux[n], hi), sRh = ldf<RF>(a.aux[n], nc + hi);
                    const double vLh = ldf<RF>(a.aux[n], 2 * nc + hi), vRh = ldf<RF>(a.aux[n], 3 * nc + hi);
                    if (PHYS == ASTRO_RMHD) { sLh = sLl; sRh = sRl; }  // low-face speeds reused
                    const int i2 = i + (n == 0), j2 = j + (n == 1), k2 = k + (n == 2);
                    for (int t = 0; t < np; ++t) {
                        const int idx = po + t;
                        const double FLt = passive_face(a, idx, lkind, n, i, j, k, vLl, vRl, sLl, sRl);
                        double acc = 0.0;
                        for (int q = 0; q < nk; ++q) {
                            const double FRt = passive_face(a, idx, kinds[q], n, i2, j2, k2, vLh, vRh, sLh, sRh);
                            acc -= (FRt - FLt) / a.dd[n];
                        }
                        rp[t] += acc;
                    }
                }
            }
        }
        if (a.rhs_only) {
#pragma unroll
            for (int v = 0; v < NM; ++v) a.dst[(size_t)v * nc + cell] = rhs[v];
            for (int t = 0; t < np; ++t) a.dst[(size_t)(NM + t) * nc + cell] = rp[t];
        } else {
            const Phys<double> P = Phys<double>::from(a.p);
            double q0[NM], U0[NM], Un[NM], q[NM];
#pragma unroll
            for (int v = 0; v < NM; ++v) q0[v] = a.pr0[(size_t)v * nc + cell];
            if (PHYS == ASTRO_SRHD) s_p2c(P, q0, U0);
            else r_p2c(P, q0, U0);
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
                Un[v] = un;
            }
            if (a.stage != a.nstages - 1 || DEFER) {
#pragma unroll
                for (int v = 0; v < NM; ++v) a.U[(size_t)v * nc + cell] = Un[v];
            }
            if (!DEFER) {
                if (PHYS == ASTRO_SRHD) s_c2p(P, Un, q);
                else r_c2p(P, Un, q, cnt);
#pragma unroll
                for (int v = 0; v < NM; ++v) a.dst[(size_t)v * nc + cell] = q[v];
                if (a.dstf)
#pragma unroll
                    for (int v = 0; v < NM; ++v) a.dstf[(size_t)v * nc + cell] = (float)q[v];
            }
            for (int v = NM; v < a.nv; ++v) {
                double out = 0.0;
                const int t = v - po;
                if (PHYS == ASTRO_SRHD && v < po) {
                    // Israel-Stewart fields 5..PASSIVE_OFFSET-1: carried from
                    // the stage input (srhd_core.py:1309-1310)
                    out = a.prk[(size_t)v * nc + cell];
                } else if (np > 0 && t >= 0 && t < np) {
                    const size_t o = (size_t)v * nc + cell;
                    const double t0 = a.pr0[o], r = rp[t];
                    if (a.stage == 0) out = __dadd_rn(t0, __dmul_rn(dt, r));
                    else {
                        const double tk = a.prk[o];
                        if (a.nstages == 2)
                            out = __dmul_rn(0.5, __dadd_rn(__dadd_rn(t0, tk), __dmul_rn(dt, r)));
                        else if (a.stage == 1)
                            out = __dadd_rn(__dmul_rn(0.75, t0), __dmul_rn(0.25, __dadd_rn(tk, __dmul_rn(dt, r))));
                        else
                            out = __dadd_rn(__dmul_rn(1.0 / 3.0, t0),
                                            __dmul_rn(2.0 / 3.0, __dadd_rn(tk, __dmul_rn(dt, r))));
                    }
                }
                a.dst[(size_t)v * nc + cell] = out;
            }
        }
    }
    if (!DEFER && a.stats && !a.rhs_only) {
        // warp-aggregated counters, one atomic per warp and counter
        unsigned n1 = __reduce_add_sync(0xffffffffu, cell < nc ? 1u : 0u);
        unsigned n2 = __reduce_add_sync(0xffffffffu, cnt.newton);
        unsigned n3 = __reduce_add_sync(0xffffffffu, cnt.bisect);
        unsigned n4 = __reduce_add_sync(0xffffffffu, cnt.hydro_fallback);
        if ((threadIdx.x & 31) == 0) {
            if (n1) atomicAdd(&a.stats->cells, (unsigned long long)n1);
            if (n2) atomicAdd(&a.stats->newton, (unsigned long long)n2);
            if (n3) atomicAdd(&a.stats->bisection, (unsigned long long)n3);
            if (n4) atomicAdd(&a.stats->hydro_fallback, (unsigned long long)n4);
        }
    }
}

// ------------------------------------------------- learned con2prim ---
// Five invariants of a conserved RMHD state (log D, |S|/D, tau/D, B^2/D,
// (S.B)^2/D^3), the last four through log1p so the inputs stay O(1).
__device__ __forceinline__ void c2p_features(const double* U, float* x) {
    const double S2 = U[1] * U[1] + U[2] * U[2] + U[3] * U[3];
    const double B2 = U[5] * U[5] + U[6] * U[6] + U[7] * U[7];
    const double SB = U[1] * U[5] + U[2] * U[6] + U[3] * U[7];
    // the features feed a bfloat16 network (8-bit mantissa): the ratios in
    // float32 with the approximate reciprocal and square root, and the fast
    // float32 logarithm (one MUFU operation each), are far more accurate than
    // that; overflowing ratios saturate at the 1e30 clamp
    const float Df = fminf(fmaxf((float)U[0], 1e-30f), 1e30f);
    const float iD = rcp_(Df);
    const float sb = (float)SB * iD;
    const float r[4] = {sqrtf((float)S2) * iD, fmaxf((float)U[4], 0.f) * iD, (float)B2 * iD,
                        sb * sb * iD};
    x[0] = __logf(Df);
#pragma unroll
    for (int i = 0; i < 4; ++i) x[1 + i] = __logf(1.0f + fminf(r[i], 1e30f));
}

struct C2PArgs {
    const double* U;   // [9][count]
    double* q;         // [>=9][count]: rows 0..8 written
    float* qf = nullptr;  // optional float32 copy of rows 0..8 (next stage's faces)
    int qf_nz = 0, qf_pitch = 0;  // qf rows of qf_pitch floats per qf_nz cells
                                  // (padded copy of the fused stages), else flat
    long count;
    AstroParams p;
    const mlp::Params* net;
    AstroC2PStats* stats;
    int* status;
    int max_polish;
    unsigned* fb_count = nullptr;  // null: every cell is solved in k_c2p_learned
    unsigned* fb_list = nullptr;   // cell indices
    unsigned fb_cap = 0;
    long poll_limit = mlp::kPollLimit;  // polls per MMA-completion wait
};

// the float32 copy's index of (variable v, cell): flat, or rows padded to
// qf_pitch floats
__device__ __forceinline__ size_t qf_index(const C2PArgs& a, int v, long cell) {
    if (a.qf_pitch == a.qf_nz) return (size_t)v * a.count + cell;
    const unsigned c = (unsigned)cell, nz = (unsigned)a.qf_nz;
    const size_t rows = (size_t)(a.count / a.qf_nz);
    return ((size_t)v * rows + c / nz) * a.qf_pitch + c % nz;
}

__device__ __forceinline__ bool c2p_defer(const C2PArgs& a, long cell) {
    if (!a.fb_list) return false;
    const unsigned slot = atomicAdd(a.fb_count, 1u);
    if (slot >= a.fb_cap) return false;
    a.fb_list[slot] = (unsigned)cell;
    return true;
}

// Learned con2prim: per 128-cell tile the MLP (tcgen05, BF16, FP32 accumulate)
// predicts log(Z / (D + tau + B^2)); Newton on the reference's equation
// continues from that guess or, where its first step is not already short,
// from the better of it and the analytic start D + tau + B^2
// (r_newton_polish2), for at most max_polish steps; cells that do not meet
// |f| < 1e-10 max(1, tau) then (or whose primitives from Z are invalid) get
// the reference's complete con2prim, so their result is the reference's.
// LISTED: a fallback list with a slot for every cell (fb_cap >= count);
// otherwise every failing cell is solved inline.
template <bool LISTED>
__global__ void __launch_bounds__(128, 5) k_c2p_learned(C2PArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + mlp::kInferSmem);
    uint32_t* taddr_s = reinterpret_cast<uint32_t*>(sm + mlp::kInferSmem + 8);
    const int t = threadIdx.x;
    // uniform across the block; without a network: Z = D + tau + B^2.  If a
    // tensor-core wait gives up, the block finishes its tiles without the
    // network (same solver, analytic start), so no cell is left unsolved.
    bool net = a.net != nullptr;
    bool timed_out = false;
    if (net) {
        if (t < 32) mlp::tmem_alloc(mlp::smem_u32(taddr_s), 64);
        if (t == 0) mlp::mbar_init_fenced(mlp::smem_u32(bar), 1);
        mlp::load_weights(sm, a.net);
        mlp::fence_async_smem();
        mlp::tc_fence_before();
    }
    __syncthreads();
    if (net) mlp::tc_fence_after();
    const uint32_t tmem = net ? *taddr_s : 0u;
    uint32_t phase = 0;
    const Phys<double> P = Phys<double>::from(a.p);
    C2PCount cnt;
    unsigned n_cells = 0, n_polish = 0, n_fallback = 0, polish_steps = 0;
    const long ntiles = (a.count + mlp::TILE - 1) / mlp::TILE;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long cell = tile * mlp::TILE + t;
        const bool valid = cell < a.count;
        {
            // the next tile's conserved rows into L2 while this tile runs:
            // its loads then wait on L2, not DRAM
            const long nxt = cell + (long)gridDim.x * mlp::TILE;
            if (nxt < a.count)
#pragma unroll
                for (int v = 0; v < 9; ++v)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a.U + (size_t)v * a.count + nxt));
        }
        double U[9] = {1, 0, 0, 0, 1, 0, 0, 0, 0};
        if (valid)
#pragma unroll
            for (int v = 0; v < 9; ++v) U[v] = a.U[(size_t)v * a.count + cell];
        float o[2] = {0.f, 0.f};
        if (net) {
            float xr[5], h0[5];
            c2p_features(U, xr);
            mlp::features_norm(a.net, xr, h0);
            if (!mlp::forward_tile<false>(sm, tmem, mlp::smem_u32(bar), phase, a.net, h0, o,
                                          a.status, a.poll_limit)) {
                net = false;
                timed_out = true;
            }
        }
        if (!valid) continue;
        ++n_cells;
        const double D = U[0], tau = U[4];
        const double B2 = U[5] * U[5] + U[6] * U[6] + U[7] * U[7];
        const double SB = U[1] * U[5] + U[2] * U[6] + U[3] * U[7];
        const double S2 = U[1] * U[1] + U[2] * U[2] + U[3] * U[3];
        // the analytic start D + tau + B^2 (the reference's second Newton
        // start) and the network's Z = that start x exp(output 0)
        const double Za = rmax(D + tau + B2, 1e-12);
        double Z = Za;
        bool polished;
        double q[9];
        int steps = 0;
        bool done = false;
        if (net) {
            // the guess only has to start Newton: a float32 exponential
            const float lz = o[0] * a.net->ysd[0] + a.net->ymu[0];
            Z = Za * (double)__expf(fmaxf(fminf(lz, 40.f), -40.f));
            polished = isfinite(Z) && r_newton_polish2(P, Z, Za, a.max_polish, D, tau, B2, SB, S2, &steps);
        } else {
            polished = isfinite(Z) && r_newton_polish(P, Z, a.max_polish, D, tau, B2, SB, S2, &steps);
        }
        if (polished) {
            ++n_polish;
            polish_steps += steps;
            done = r_prims_from_Z_checked(P, Z, U, q);
            if (LISTED && !done && c2p_defer(a, cell)) continue;
        } else {
            ++n_fallback;
            polish_steps += a.max_polish;
            // the reference's complete con2prim, in k_c2p_fallback so that the
            // long solves do not hold up the 31 other cells of this warp
            if (LISTED && c2p_defer(a, cell)) continue;
        }
        if constexpr (!LISTED) {
            if (!done) r_c2p<true>(P, U, q, cnt);
        }
#pragma unroll
        for (int v = 0; v < 9; ++v) a.q[(size_t)v * a.count + cell] = q[v];
        if (a.qf)
#pragma unroll
            for (int v = 0; v < 9; ++v) a.qf[qf_index(a, v, cell)] = (float)q[v];
    }
    if (a.net) {
        if (timed_out) mlp::drain_after_timeout(mlp::smem_u32(bar), phase);
        mlp::tc_fence_before();
        __syncthreads();
        if (t < 32) mlp::tmem_free(tmem, 64);
    }
    if (a.stats) {
        if (timed_out && t == 0) atomicAdd(&a.stats->wait_timeouts, 1ull);
        atomicAdd(&a.stats->cells, (unsigned long long)n_cells);
        if (n_polish) atomicAdd(&a.stats->learned_polish, (unsigned long long)n_polish);
        if (n_fallback) atomicAdd(&a.stats->learned_fallback, (unsigned long long)n_fallback);
        if (polish_steps) atomicAdd(&a.stats->polish_steps, (unsigned long long)polish_steps);
        if (cnt.newton) atomicAdd(&a.stats->newton, (unsigned long long)cnt.newton);
        if (cnt.bisect) atomicAdd(&a.stats->bisection, (unsigned long long)cnt.bisect);
        if (cnt.hydro_fallback) atomicAdd(&a.stats->hydro_fallback, (unsigned long long)cnt.hydro_fallback);
    }
}

// The cells k_c2p_learned listed: the reference's complete con2prim, one cell
// per thread.
__global__ void __launch_bounds__(128) k_c2p_fallback(C2PArgs a) {
    const unsigned n = min(*a.fb_count, a.fb_cap);
    const Phys<double> P = Phys<double>::from(a.p);
    C2PCount cnt;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const size_t cell = a.fb_list[e];
        double U[9], q[9];
#pragma unroll
        for (int v = 0; v < 9; ++v) U[v] = a.U[(size_t)v * a.count + cell];
        r_c2p<true>(P, U, q, cnt);
#pragma unroll
        for (int v = 0; v < 9; ++v) a.q[(size_t)v * a.count + cell] = q[v];
        if (a.qf)
#pragma unroll
            for (int v = 0; v < 9; ++v) a.qf[qf_index(a, (int)v, (long)cell)] = (float)q[v];
    }
    if (a.stats) {
        if (cnt.newton) atomicAdd(&a.stats->newton, (unsigned long long)cnt.newton);
        if (cnt.bisect) atomicAdd(&a.stats->bisection, (unsigned long long)cnt.bisect);
        if (cnt.hydro_fallback) atomicAdd(&a.stats->hydro_fallback, (unsigned long long)cnt.hydro_fallback);
    }
}

__global__ void k_c2p_features(const double* U, float* x, long count) {
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long)gridDim.x * blockDim.x) {
        double u[9];
        for (int v = 0; v < 9; ++v) u[v] = U[(size_t)v * count + t];
        float f[5];
        c2p_features(u, f);
        for (int i = 0; i < 5; ++i) x[t * 5 + i] = f[i];
    }
}

// the learned polish's float64 reciprocal over an array (test hook)
__global__ void k_rcp_f64(const double* x, double* y, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        y[i] = rcp_nr(x[i]);
}

int g_sm_count = 0;
int sm_count_cached() {
    if (!g_sm_count) {
        int dev = 0, n = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        g_sm_count = n;
    }
    return g_sm_count;
}

int g_c2p_blocks_per_sm[2] = {0, 0};

template <bool LISTED>
cudaError_t launch_c2p_learned_t(const C2PArgs& a, cudaStream_t s) {
    const long ntiles = (a.count + mlp::TILE - 1) / mlp::TILE;
    int& bps = g_c2p_blocks_per_sm[LISTED ? 1 : 0];
    if (!bps) {
        // prefer the largest shared-memory carveout and size the persistent
        // grid by what is resident per SM: shared memory (one 42 KB tile
        // each), registers, and TMEM (8 blocks x 64 columns)
        cudaFuncSetAttribute(k_c2p_learned<LISTED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        int dev = 0, smem_sm = 0, reserved = 0, regs_sm = 65536;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
        cudaFuncAttributes fa;
        int nb = 4;
        if (cudaFuncGetAttributes(&fa, k_c2p_learned<LISTED>) == cudaSuccess && smem_sm > 0) {
            const int per_block = mlp::kInferSmem + 16 + (int)fa.sharedSizeBytes + reserved;
            const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
            const int by_smem = smem_sm / per_block;
            const int by_regs = regs_sm / (regs_warp > 0 ? regs_warp * (mlp::TILE / 32) : 1);
            nb = by_smem < by_regs ? by_smem : by_regs;
        }
        bps = nb < 1 ? 1 : (nb > 8 ? 8 : nb);
    }
    const long cap = (long)bps * sm_count_cached();
    const int grid = (int)(ntiles < cap ? ntiles : cap);
    if (grid <= 0) return cudaSuccess;
    if (a.fb_list && cudaMemsetAsync(a.fb_count, 0, sizeof(unsigned), s) != cudaSuccess)
        return cudaGetLastError();
    k_c2p_learned<LISTED><<<grid, mlp::TILE, mlp::kInferSmem + 16, s>>>(a);
    mark(3, s);
    if (LISTED) {
        k_c2p_fallback<<<sm_count_cached() * 4, 128, 0, s>>>(a);
        mark(4, s);
    }
    return cudaGetLastError();
}

// with a fallback list (a slot for every cell) or with inline solves
cudaError_t launch_c2p_learned(const C2PArgs& a, cudaStream_t s) {
    if (a.fb_list) {
        if (a.fb_cap < (unsigned long)a.count) return cudaErrorInvalidValue;
        return launch_c2p_learned_t<true>(a, s);
    }
    return launch_c2p_learned_t<false>(a, s);
}

// float32 copy of the first nm primitive rows (stage inputs that no
// con2prim kernel of this library produced)
__global__ void k_prim_f32(const double* __restrict__ pr, float* __restrict__ prf, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        prf[i] = (float)pr[i];
}

// the same into rows padded to `pitch` floats (n = variables x nx x ny rows)
__global__ void k_prim_f32_rows(const double* __restrict__ pr, float* __restrict__ prf, size_t rows,
                                int nz, int pitch) {
    const size_t n = rows * (size_t)nz;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / (unsigned)nz, k = i % (unsigned)nz;
        prf[r * pitch + k] = (float)pr[i];
    }
}

// ------------------------------------------------------------- dispatch ---
// direction is a template parameter so the per-direction component indices
// fold to constants and the face state stays in registers
template <int PH, int RE, int RI, typename R>
cudaError_t launch_face_dir(const FaceArgs& a, bool given, dim3 grd, dim3 blk, cudaStream_t s) {
    constexpr bool F32 = sizeof(R) == 4;
    const dim3 fgrd(148 * 4);
    // the fix-up counter starts every float32 pass at zero (the workspace, or
    // the shared static scratch, holds the previous pass's count)
    if (F32) {
        const cudaError_t e = cudaMemsetAsync(a.fix_count, 0, sizeof(unsigned), s);
        if (e != cudaSuccess) return e;
    }
    if constexpr (PH == ASTRO_RMHD && RE != ASTRO_RECON_MUSCL) {
        if (given) {
            k_face<PH, RE, RI, R, true, 0><<<grd, blk, 0, s>>>(a);
            if (F32) k_face_fix<PH, RE, RI, true, 0><<<fgrd, blk, 0, s>>>(a);
            return cudaSuccess;
        }
    }
    if (a.dir == 0) {
        k_face<PH, RE, RI, R, false, 0><<<grd, blk, 0, s>>>(a);
        if (F32) k_face_fix<PH, RE, RI, false, 0><<<fgrd, blk, 0, s>>>(a);
    } else if (a.dir == 1) {
        k_face<PH, RE, RI, R, false, 1><<<grd, blk, 0, s>>>(a);
        if (F32) k_face_fix<PH, RE, RI, false, 1><<<fgrd, blk, 0, s>>>(a);
    } else {
        k_face<PH, RE, RI, R, false, 2><<<grd, blk, 0, s>>>(a);
        if (F32) k_face_fix<PH, RE, RI, false, 2><<<fgrd, blk, 0, s>>>(a);
    }
    return cudaSuccess;
}

template <typename R>
cudaError_t launch_face_t(const FaceArgs& a, bool given, cudaStream_t s) {
    // an empty cell range in any direction: no faces (checked per extent,
    // since two negative extents would give a positive product)
    if (a.ext[0] <= 0 || a.ext[1] <= 0 || a.ext[2] <= 0) return cudaSuccess;
    const unsigned plane = (unsigned)a.ext[1] * (unsigned)a.ext[2];
    const dim3 blk(128), grd((plane + 127) / 128, (unsigned)(a.ext[0] < 65535 ? a.ext[0] : 65535));
    const AstroParams& p = a.p;
    cudaError_t me = cudaSuccess;
#define FACE(PH, RE, RI) me = launch_face_dir<PH, RE, RI, R>(a, given, grd, blk, s)
#define RECONS(PH, RI)                                                          \
    do {                                                                        \
        if (p.recon == 0) FACE(PH, 0, RI);                                      \
        else if (p.recon == 1) FACE(PH, 1, RI);                                 \
        else FACE(PH, 2, RI);                                                   \
    } while (0)
    if (p.physics == ASTRO_SRHD) {
        if (p.riemann == 1) RECONS(ASTRO_SRHD, 1);
        else RECONS(ASTRO_SRHD, 0);
    } else {
        if (p.riemann == 2) RECONS(ASTRO_RMHD, 2);
        else if (p.riemann == 1) RECONS(ASTRO_RMHD, 1);
        else RECONS(ASTRO_RMHD, 0);
    }
#undef RECONS
#undef FACE
    if (me != cudaSuccess) return me;
    mark(0, s);
    return cudaGetLastError();
}

template <int PH, typename RF, bool DEF, bool PAS>
void launch_update_t(const UpdArgs& a, dim3 grd, dim3 blk, cudaStream_t s) {
    k_update<PH, RF, DEF, PAS><<<grd, blk, 0, s>>>(a);
}

cudaError_t launch_update(const UpdArgs& a, cudaStream_t s) {
    const size_t nc = (size_t)a.nx * a.ny * a.nz;
    const dim3 blk(kUpdateBlock), grd((unsigned)((nc + kUpdateBlock - 1) / kUpdateBlock));
    const bool mixed = a.p.precision == ASTRO_PREC_MIXED;
    const bool pas = passive_fluxes(a.p);
#define UPD(PH, DEF)                                                               \
    do {                                                                           \
        if (pas) {                                                                 \
            if (mixed) launch_update_t<PH, float, DEF, true>(a, grd, blk, s);      \
            else launch_update_t<PH, double, DEF, true>(a, grd, blk, s);           \
        } else {                                                                   \
            if (mixed) launch_update_t<PH, float, DEF, false>(a, grd, blk, s);     \
            else launch_update_t<PH, double, DEF, false>(a, grd, blk, s);          \
        }                                                                          \
    } while (0)
    if (a.p.physics == ASTRO_SRHD) {
        if (a.defer_c2p) UPD(ASTRO_SRHD, true);  // GR steps: con2prim after the sources
        else UPD(ASTRO_SRHD, false);
    } else if (a.defer_c2p) UPD(ASTRO_RMHD, true);
    else UPD(ASTRO_RMHD, false);
#undef UPD
    mark(1, s);
    return cudaGetLastError();
}

// All face passes of one stage: z (with speeds in carried mode), x, carried x, y.
// prf_ready: the float32 copy of pr was written by the kernel that produced pr
// SRHD blocks of 15+ variables carry Israel-Stewart fields whose fluxes the
// reference adds to every MUSCL face once and to every PPM face twice
// (srhd_core.py:543-544, 958-961) and not in WENO; conservative mode adds
// them once for PPM too.
int dissipation_fluxes(const AstroParams& p, const AstroGrid& g) {
    if (p.physics != ASTRO_SRHD || g.nv < 15) return 0;
    if (p.recon == ASTRO_RECON_MUSCL) return 1;
    if (p.recon == ASTRO_RECON_PPM) return p.flux_mode == ASTRO_FLUX_CONSERVATIVE ? 1 : 2;
    return 0;
}

cudaError_t face_passes(const AstroParams& p, const AstroGrid& g, const Bounds& b,
                        const double* pr, char* work, const Layout& L, cudaStream_t s,
                        bool prf_ready = false) {
    const bool carried = carried_mode(p);
    const bool mixed = p.precision == ASTRO_PREC_MIXED;
    const int order[3] = {2, 0, 1};
    float* prf = mixed ? (float*)(work + L.prf) : nullptr;
    if (mixed && !prf_ready) {
        const size_t n = (size_t)(p.physics == ASTRO_SRHD ? 5 : 9) * g.nx * g.ny * g.nz;
        k_prim_f32<<<sm_count_cached() * 8, 256, 0, s>>>(pr, prf, n);
        mark(2, s);
    }
    for (int oi = 0; oi < 3; ++oi) {
        const int d = order[oi];
        FaceArgs a;
        memset(&a, 0, sizeof(a));
        a.pr = pr; a.prf = prf; a.nx = g.nx; a.ny = g.ny; a.nz = g.nz; a.dir = d; a.b = b; a.p = p;
        a.ndiss = dissipation_fluxes(p, g);
        for (int e = 0; e < 3; ++e) {
            a.org[e] = b.lo;
            a.ext[e] = b.hi[e] - b.lo + (e == d ? 1 : 0);
        }
        a.F = work + L.F[d];
        a.aux = passive_fluxes(p) ? (void*)(work + L.aux[d]) : nullptr;
        if (mixed) {
            a.fix_count = (unsigned*)(work + L.fix);
            a.fix_list = (unsigned*)(work + L.fix + 256);
            a.fix_cap = (unsigned)fix_capacity(g);
        }
        a.speeds_out = (carried && d == 2) ? (void*)(work + L.Sz) : nullptr;
        cudaError_t e = mixed ? launch_face_t<float>(a, false, s) : launch_face_t<double>(a, false, s);
        if (e != cudaSuccess) return e;
        if (carried && d == 0) {
            FaceArgs c = a;
            c.ext[0] = b.hi[0] - b.lo;  // x-low faces of the updated cells
            c.F = work + L.FxC;
            c.aux = nullptr;
            c.speeds_out = nullptr;
            c.carried = work + L.Sz;
            e = mixed ? launch_face_t<float>(c, true, s) : launch_face_t<double>(c, true, s);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

UpdArgs update_args(const AstroParams& p, const AstroGrid& g, const Bounds& b, char* work,
                    const Layout& L) {
    UpdArgs u;
    memset(&u, 0, sizeof(u));
    for (int d = 0; d < 3; ++d) {
        u.F[d] = work + L.F[d];
        u.aux[d] = passive_fluxes(p) ? (const void*)(work + L.aux[d]) : nullptr;
    }
    u.FxL = carried_mode(p) ? (const void*)(work + L.FxC) : u.F[0];
    u.nv = g.nv; u.nx = g.nx; u.ny = g.ny; u.nz = g.nz;
    u.b = b;
    u.dd[0] = g.dx; u.dd[1] = g.dy; u.dd[2] = g.dz;
    for (int d = 0; d < 3; ++d) {
        u.idd[d] = 1.0 / u.dd[d];
        u.idd2[d] = 1.0 / (u.dd[d] * u.dd[d] + 1e-12);
    }
    u.p = p;
    return u;
}

int cuda_status(cudaError_t e) { return e == cudaSuccess ? ASTRO_OK : ASTRO_E_CUDA; }

// ------------------------------------------------------- CFL reduction ---
__global__ void k_max_char_speed(const double* pr, int nx, int ny, int nz, double srhd_gamma,
                                 unsigned long long* out) {
    const size_t n = (size_t)(nx - 2) * (ny - 2) * (nz - 2);
    const size_t nc = (size_t)nx * ny * nz;
    Phys<double> P;
    P.srhd_gamma = srhd_gamma;
    double loc = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int k = 1 + (int)(t % (nz - 2));
        const int j = 1 + (int)((t / (nz - 2)) % (ny - 2));
        const int i = 1 + (int)(t / ((size_t)(nz - 2) * (ny - 2)));
        const size_t c = ((size_t)i * ny + j) * nz + k;
        const double cs = s_sound_speed(P, pr[c], pr[4 * nc + c]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double lm, lp;
            eig_speeds(pr[(1 + d) * nc + c], cs, lm, lp);
            loc = rmax(loc, rmax(fabs(lm), fabs(lp)));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loc = rmax(loc, __shfl_xor_sync(0xffffffffu, loc, o));
    __shared__ double wmax[32];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = loc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? wmax[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = rmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        // non-negative doubles order like their bit patterns
        if (threadIdx.x == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
    }
}

__global__ void k_floor_small(double* out) {
    if (*out < 1e-12) *out = 1e-12;
}

// ------------------------------------------------------------ ghosts -----
__global__ void k_periodic_yz(double* pr, int nv, int nx, int ny, int nz, int ng) {
    // every cell with a y or z ghost index receives orig[i, my(j), mz(k)];
    // the sources all have interior j and k, so the gather is race free and
    // equals the reference's sequential y-then-z slab copies
    const size_t nc = (size_t)nx * ny * nz;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < nc;
         t += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % nz);
        const int j = (int)((t / nz) % ny);
        const int i = (int)(t / ((size_t)nz * ny));
        const bool gy = j < ng || j >= ny - ng, gz = k < ng || k >= nz - ng;
        if (!gy && !gz) continue;
        const int sj = j < ng ? j + (ny - 2 * ng) : (j >= ny - ng ? j - (ny - 2 * ng) : j);
        const int sk = k < ng ? k + (nz - 2 * ng) : (k >= nz - ng ? k - (nz - 2 * ng) : k);
        const size_t src = ((size_t)i * ny + sj) * nz + sk;
        for (int v = 0; v < nv; ++v) pr[(size_t)v * nc + t] = pr[(size_t)v * nc + src];
    }
}

__global__ void k_outflow_right_x(double* pr, int nv, int nx, int ny, int nz, int ng) {
    const size_t plane = (size_t)ny * nz, nc = plane * nx;
    const size_t n = plane * ng;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t g = t / plane, jk = t % plane;
        const size_t dst = (nx - ng + g) * plane + jk, src = (size_t)(nx - ng - 1) * plane + jk;
        for (int v = 0; v < nv; ++v) pr[(size_t)v * nc + dst] = pr[(size_t)v * nc + src];
    }
}

__device__ double nozzle_weight(double r, double radius, double shear, int profile) {
    if (radius <= 0.0) return 0.0;
    if (profile == 1) return r >= radius ? 0.0 : 0.5 * (1.0 + cos(M_PI * r / radius));
    if (profile == 2) {
        if (r >= radius) return 0.0;
        double x = r / radius;
        return rmax(0.0, 1.0 - x * x);
    }
    if (shear > 0.0) return 0.5 * (1.0 - tanh((r - radius) / shear));
    return r <= radius ? 1.0 : 0.0;
}

// zero-gradient y/z ghost fill: each ghost cell of the y/z frame of every x
// plane gathers the nearest interior cell (race-free: sources are interior)
__global__ void k_outflow_yz(double* pr, int nv, int nx, int ny, int nz, int ng) {
    const int nyi = ny - 2 * ng;
    const size_t frame = (size_t)ny * nz - (size_t)nyi * (nz - 2 * ng);
    const size_t n = (size_t)nx * frame, nc = (size_t)nx * ny * nz;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / frame);
        const size_t q = t % frame;
        int j, k;
        const size_t rows = (size_t)2 * ng * nz;  // the 2 ng full y-ghost rows first
        if (q < rows) {
            const int r = (int)(q / nz);
            j = r < ng ? r : ny - 2 * ng + r;
            k = (int)(q % nz);
        } else {  // then the z-ghost columns of the interior rows
            const size_t u = q - rows;
            j = ng + (int)(u / (2 * ng));
            const int c = (int)(u % (2 * ng));
            k = c < ng ? c : nz - 2 * ng + c;
        }
        const int js = j < ng ? ng : (j >= ny - ng ? ny - ng - 1 : j);
        const int ks = k < ng ? ng : (k >= nz - ng ? nz - ng - 1 : k);
        const size_t dst = ((size_t)i * ny + j) * nz + k, src = ((size_t)i * ny + js) * nz + ks;
        for (int v = 0; v < nv; ++v) pr[(size_t)v * nc + dst] = pr[(size_t)v * nc + src];
    }
}

__global__ void k_nozzle(double* pr, int nv, int nx, int ny, int nz, AstroNozzle c,
                         const double* draws, const int32_t* rank_map, int n_weighted) {
    const int ng = c.ng, nyl = ny - 2 * ng, nzl = nz - 2 * ng;
    const size_t n = (size_t)ng * nyl * nzl, nc = (size_t)nx * ny * nz;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int kk = (int)(t % nzl), jj = (int)((t / nzl) % nyl), g = (int)(t / ((size_t)nzl * nyl));
        const int j = jj + ng, k = kk + ng;
        const double y = (j - ng + 0.5) * c.dy, z = (k - ng + 0.5) * c.dz;
        const double rr = sqrt((y - c.y0) * (y - c.y0) + (z - c.z0) * (z - c.z0));
        const double s = nozzle_weight(rr, c.radius, c.shear_thick, c.profile);
        if (c.ambient_bc == 1 && !(s > 0.0)) {
            // outside the nozzle: zero-gradient from the first interior layer
            const size_t cell = ((size_t)g * ny + j) * nz + k, src = ((size_t)ng * ny + j) * nz + k;
            for (int v = 0; v < nv; ++v) pr[(size_t)v * nc + cell] = pr[(size_t)v * nc + src];
            continue;
        }
        double rho = c.eta_rho * c.rho_amb * s + c.rho_amb * (1.0 - s);
        double p = c.p_eq;
        const double beta = sqrt(1.0 - 1.0 / (c.gamma_jet * c.gamma_jet));
        double vx = beta * s + c.vx_amb * (1.0 - s);
        double vy = c.vy_amb, vz = c.vz_amb;
        // which cells draw random numbers is decided on the host with the
        // reference's own Python math (the rank map), so the draw order and
        // count match rng.random() calls in core/nozzle.py:50-53 exactly
        if (c.perturb && draws && rank_map) {
            const int rk = rank_map[(size_t)jj * nzl + kk];
            if (rk >= 0) {
                const double* d = draws + 3 * ((size_t)g * n_weighted + rk);
                vy += c.turb_vamp * (2.0 * d[0] - 1.0);
                vz += c.turb_vamp * (2.0 * d[1] - 1.0);
                p *= (1.0 + c.turb_pamp * (2.0 * d[2] - 1.0));
            }
        }
        const size_t cell = ((size_t)g * ny + j) * nz + k;
        pr[cell] = rho;
        pr[nc + cell] = vx;
        pr[2 * nc + cell] = vy;
        pr[3 * nc + cell] = vz;
        pr[4 * nc + cell] = p;
        if (nv >= 15)
            for (int v = 5; v < 15; ++v) pr[(size_t)v * nc + cell] = 0.0;
        for (int tt = 0; tt < c.n_tracers && tt < 8; ++tt) {
            const double tn = c.tracer_nozzle[tt], ta = c.tracer_amb[tt];
            pr[(size_t)(c.tracer_offset + tt) * nc + cell] = ta + (tn - ta) * s;
        }
        if (c.two_temperature && nv > c.thermo_offset + 1) {
            pr[(size_t)c.thermo_offset * nc + cell] = c.te;
            pr[(size_t)(c.thermo_offset + 1) * nc + cell] = c.ti;
        }
        // the inflow's ionisation fractions (core/nozzle.py:77-82)
        if (c.chemistry && nv > c.chem_offset + 2)
            for (int m = 0; m < 3; ++m) pr[(size_t)(c.chem_offset + m) * nc + cell] = c.chem_x[m];
        if (c.physics == 1) {
            double Bx = 0.0, By = 0.0, Bz = 0.0;
            if (c.b_init == 1) Bx = c.b0 * s;
            else if (c.b_init == 2) By = c.b0 * s;
            else if (c.b_init == 3) {
                // toroidal B_phi(r) around the jet axis, on the ambient axial field
                const double bphi = rr < c.radius ? c.b0 * rr / c.radius : c.b0 * c.radius / rr;
                const double f = rr > 0.0 ? s * bphi / rr : 0.0;
                Bx = c.b_amb_x;
                By = -f * (z - c.z0);
                Bz = f * (y - c.y0);
            }
            pr[5 * nc + cell] = Bx;
            pr[6 * nc + cell] = By;
            pr[7 * nc + cell] = Bz;
            pr[8 * nc + cell] = 0.0;
        }
    }
}

// -------------------------------------------------------- conversions ---
__global__ void k_p2c(AstroParams p, const double* q, double* U, long count) {
    const Phys<double> P = Phys<double>::from(p);
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long)gridDim.x * blockDim.x) {
        double a[9], b[9];
        const int nm = p.physics == ASTRO_SRHD ? 5 : 9;
        for (int v = 0; v < nm; ++v) a[v] = q[(size_t)v * count + t];
        if (p.physics == ASTRO_SRHD) s_p2c(P, a, b);
        else r_p2c(P, a, b);
        for (int v = 0; v < nm; ++v) U[(size_t)v * count + t] = b[v];
    }
}

// qf: optional float32 copy of the result in rows of `pitch` floats per nz
// cells (the fused stages' input)
__global__ void k_c2p(AstroParams p, const double* U, double* q, long count, AstroC2PStats* stats,
                      float* qf = nullptr, int nz = 1, int pitch = 1) {
    const Phys<double> P = Phys<double>::from(p);
    C2PCount cnt;
    unsigned mine = 0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long)gridDim.x * blockDim.x) {
        double a[9], b[9];
        const int nm = p.physics == ASTRO_SRHD ? 5 : 9;
        for (int v = 0; v < nm; ++v) a[v] = U[(size_t)v * count + t];
        if (p.physics == ASTRO_SRHD) s_c2p(P, a, b);
        else r_c2p(P, a, b, cnt);
        for (int v = 0; v < nm; ++v) q[(size_t)v * count + t] = b[v];
        if (qf) {
            const size_t rows = (size_t)(count / nz);
            const size_t r = (size_t)t / (unsigned)nz, k = (size_t)t % (unsigned)nz;
            for (int v = 0; v < nm; ++v) qf[((size_t)v * rows + r) * pitch + k] = (float)b[v];
        }
        ++mine;
    }
    if (stats) {
        atomicAdd(&stats->cells, (unsigned long long)mine);
        if (cnt.newton) atomicAdd(&stats->newton, (unsigned long long)cnt.newton);
        if (cnt.bisect) atomicAdd(&stats->bisection, (unsigned long long)cnt.bisect);
        if (cnt.hydro_fallback) atomicAdd(&stats->hydro_fallback, (unsigned long long)cnt.hydro_fallback);
    }
}

// ------------------------------------------------------------ sources ---
__global__ void k_cooling(double* pr, int nx, int ny, int nz, int ng, double dt, double cool,
                          double heat, double pmax) {
    const size_t nc = (size_t)nx * ny * nz;
    const int ex = nx - 2 * ng, ey = ny - 2 * ng, ez = nz - 2 * ng;
    const size_t n = (size_t)ex * ey * ez;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int k = ng + (int)(t % ez), j = ng + (int)((t / ez) % ey), i = ng + (int)(t / ((size_t)ez * ey));
        const size_t c = ((size_t)i * ny + j) * nz + k;
        const double rho = pr[c], p = pr[4 * nc + c];
        const double dp = __dmul_rn(dt, heat - __dmul_rn(__dmul_rn(cool, rho), p));
        double pn = __dadd_rn(p, dp);
        if (pn < 1e-12) pn = 1e-12;
        if (pn > pmax) pn = pmax;
        pr[4 * nc + c] = pn;
    }
}

__global__ void k_two_temperature(double* pr, int nx, int ny, int nz, int ng, double dt,
                                  double tau, int off) {
    const size_t nc = (size_t)nx * ny * nz;
    const int ex = nx - 2 * ng, ey = ny - 2 * ng, ez = nz - 2 * ng;
    const size_t n = (size_t)ex * ey * ez;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int k = ng + (int)(t % ez), j = ng + (int)((t / ez) % ey), i = ng + (int)(t / ((size_t)ez * ey));
        const size_t c = ((size_t)i * ny + j) * nz + k;
        const double rho = pr[c], p = pr[4 * nc + c];
        const double T = p / rmax(rho, 1e-12);
        double Te = pr[(size_t)off * nc + c], Ti = pr[(size_t)(off + 1) * nc + c];
        Te = __dadd_rn(Te, __dmul_rn(dt, T - Te) / tau);
        Ti = __dadd_rn(Ti, __dmul_rn(dt, T - Ti) / tau);
        pr[(size_t)off * nc + c] = Te;
        pr[(size_t)(off + 1) * nc + c] = Ti;
    }
}

// H/He ionisation (core/chemistry.py:43-139): rates are the reference's
// fits; operation order follows its expressions
__device__ __forceinline__ double chem_clamp(double x, double lo, double hi) {
    return x < lo ? lo : (x > hi ? hi : x);
}
__device__ __forceinline__ double chem_ci(double a, double e, double T) {
    return a * sqrt(T) * exp(-e / rmax(T, 1.0)) / (1.0 + sqrt(T / 1.0e5));
}

__global__ void k_ion_chemistry(double* pr, int nx, int ny, int nz, AstroChemistry c, double dt) {
    const double SMALL = 1e-20;
    const size_t nc = (size_t)nx * ny * nz;
    const int ng = c.ng, ex = nx - 2 * ng, ey = ny - 2 * ng, ez = nz - 2 * ng;
    const size_t n = (size_t)ex * ey * ez;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int k = ng + (int)(t % ez), j = ng + (int)((t / ez) % ey), i = ng + (int)(t / ((size_t)ez * ey));
        const size_t cl = ((size_t)i * ny + j) * nz + k;
        const double rho = pr[cl], p = pr[4 * nc + cl];
        if (!(rho > 0.0) || !(p > 0.0)) continue;
        double T = (p / rmax(rho, SMALL)) * c.tunit_k;
        if (T < c.tmin_k) T = c.tmin_k;
        const double nH = c.x * rho, nHe = c.y * rho / 4.0;
        double* s = pr + (size_t)c.chem_offset * nc + cl;
        const double xHII = chem_clamp(s[0], 0.0, 1.0);
        double xHeII = chem_clamp(s[nc], 0.0, 1.0);
        const double xHeIII = chem_clamp(s[2 * nc], 0.0, 1.0);
        xHeII = rmin(xHeII, 1.0 - xHeIII);
        const double xHeI = rmax(0.0, 1.0 - xHeII - xHeIII);
        const double xHI = 1.0 - xHII;
        const double ne = rmax(nH * xHII + nHe * (xHeII + 2.0 * xHeIII), SMALL);
        const double C_H = c.rate_scale * chem_ci(5.85e-11, 157809.1, T);
        const double C_HeI = c.rate_scale * chem_ci(2.38e-11, 285335.4, T);
        const double C_HeII = c.rate_scale * chem_ci(5.68e-12, 631515.0, T);
        const double A_H = c.rate_scale * (2.59e-13 * pow(T / 1.0e4, -0.7));
        const double A_HeII = c.rate_scale * (1.50e-10 * pow(T / 1.0e4, -0.6353));
        const double A_HeIII = c.rate_scale * (3.36e-10 * pow(T / 1.0e4, -0.5));
        double xHII_n = (xHII + dt * ne * C_H * xHI) / (1.0 + dt * ne * A_H);
        const double xHeIII_n =
            chem_clamp((xHeIII + dt * ne * C_HeII * xHeII) / (1.0 + dt * ne * A_HeIII), 0.0, 1.0);
        double xHeII_n = (xHeII + dt * ne * (C_HeI * xHeI + A_HeIII * xHeIII_n)) /
                         (1.0 + dt * ne * (A_HeII + C_HeII));
        xHII_n = chem_clamp(xHII_n, 0.0, 1.0);
        xHeII_n = chem_clamp(xHeII_n, 0.0, 1.0 - xHeIII_n);
        const double dE = c.energy_scale * (nH * 157809.1 * (xHII_n - xHII) +
                                            nHe * 285335.4 * (xHeII_n - xHeII) +
                                            nHe * 631515.0 * (xHeIII_n - xHeIII));
        double pn = p + (-(c.gamma - 1.0) * dE / rmax(c.tunit_k, SMALL));
        if (pn < SMALL) pn = SMALL;
        pr[4 * nc + cl] = pn;
        s[0] = xHII_n;
        s[nc] = xHeII_n;
        s[2 * nc] = xHeIII_n;
    }
}

// Causal dissipation (core/dissipation.py:5-215), interior cells.  Pass 1:
// first-order upwind advection of the 10 dissipative variables from the old
// values into scratch (the reference's copies).  Pass 2: relaxation from the
// advected values (or pr without advection), writing all 10 back.
__global__ void k_dissip_advect(const double* pr, double* adv, int nx, int ny, int nz, int ng,
                                double dt, double dx, double dy, double dz) {
    const size_t nc = (size_t)nx * ny * nz;
    const int ex = nx - 2 * ng, ey = ny - 2 * ng, ez = nz - 2 * ng;
    const size_t n = (size_t)ex * ey * ez;
    const long sx = (long)ny * nz, sy = nz;
    const double hx = rmax(dx, 1e-12), hy = rmax(dy, 1e-12), hz = rmax(dz, 1e-12);
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int k = ng + (int)(t % ez), j = ng + (int)((t / ez) % ey), i = ng + (int)(t / ((size_t)ez * ey));
        const size_t c = ((size_t)i * ny + j) * nz + k;
        const double vx = pr[nc + c], vy = pr[2 * nc + c], vz = pr[3 * nc + c];
        for (int v = 0; v < 10; ++v) {
            const double* a = pr + (size_t)(5 + v) * nc + c;
            const double u0 = a[0];
            const double ddx = vx > 0.0 ? (u0 - a[-sx]) / hx : (a[sx] - u0) / hx;
            const double ddy = vy > 0.0 ? (u0 - a[-sy]) / hy : (a[sy] - u0) / hy;
            const double ddz = vz > 0.0 ? (u0 - a[-1]) / hz : (a[1] - u0) / hz;
            adv[(size_t)v * nc + c] = u0 - dt * (vx * ddx + vy * ddy + vz * ddz);
        }
    }
}

__device__ __forceinline__ double dcap(double x, double cap) {
    return x > cap ? cap : (x < -cap ? -cap : x);
}

__global__ void k_dissip_relax(double* pr, const double* adv, int nx, int ny, int nz,
                               AstroDissipation c, double dt, double dx, double dy, double dz) {
    const size_t nc = (size_t)nx * ny * nz;
    const int ng = c.ng, ex = nx - 2 * ng, ey = ny - 2 * ng, ez = nz - 2 * ng;
    const size_t n = (size_t)ex * ey * ez;
    const long sx = (long)ny * nz, sy = nz;
    const double i2x = 0.5 / rmax(dx, 1e-12), i2y = 0.5 / rmax(dy, 1e-12), i2z = 0.5 / rmax(dz, 1e-12);
    const double cap = c.cap_frac * c.p_max;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int k = ng + (int)(t % ez), j = ng + (int)((t / ez) % ey), i = ng + (int)(t / ((size_t)ez * ey));
        const size_t cl = ((size_t)i * ny + j) * nz + k;
        double d[10];
        for (int v = 0; v < 10; ++v) d[v] = adv ? adv[(size_t)v * nc + cl] : pr[(size_t)(5 + v) * nc + cl];
        auto g = [&](int var, long off) { return pr[(size_t)var * nc + cl + off]; };
        const double dvx_dx = (g(1, sx) - g(1, -sx)) * i2x, dvx_dy = (g(1, sy) - g(1, -sy)) * i2y,
                     dvx_dz = (g(1, 1) - g(1, -1)) * i2z;
        const double dvy_dx = (g(2, sx) - g(2, -sx)) * i2x, dvy_dy = (g(2, sy) - g(2, -sy)) * i2y,
                     dvy_dz = (g(2, 1) - g(2, -1)) * i2z;
        const double dvz_dx = (g(3, sx) - g(3, -sx)) * i2x, dvz_dy = (g(3, sy) - g(3, -sy)) * i2y,
                     dvz_dz = (g(3, 1) - g(3, -1)) * i2z;
        const double divv = dvx_dx + dvy_dy + dvz_dz;
        if (c.zeta != 0.0) {
            const double pi_eq = -c.zeta * divv;
            d[0] = dcap((d[0] + dt * pi_eq / c.tau_bulk) / (1.0 + dt / c.tau_bulk), cap);
        }
        if (c.eta != 0.0) {
            const double sxx = dvx_dx - (1.0 / 3.0) * divv, syy = dvy_dy - (1.0 / 3.0) * divv;
            const double szz = dvz_dz - (1.0 / 3.0) * divv;
            const double sxy = 0.5 * (dvx_dy + dvy_dx), sxz = 0.5 * (dvx_dz + dvz_dx);
            const double syz = 0.5 * (dvy_dz + dvz_dy);
            const double e2 = -2.0 * c.eta, ts = c.tau_shear;
            const double eq[6] = {e2 * sxx, e2 * syy, e2 * szz, e2 * sxy, e2 * sxz, e2 * syz};
            double s6[6];
            for (int m = 0; m < 6; ++m) s6[m] = (d[1 + m] + dt * eq[m] / ts) / (1.0 + dt / ts);
            s6[2] = -(s6[0] + s6[1]);  // traceless
            for (int m = 0; m < 6; ++m) d[1 + m] = dcap(s6[m], cap);
        }
        if (c.kappa != 0.0) {
            auto T = [&](long off) { return g(4, off) / rmax(g(0, off), 1e-12); };
            const double dTdx = (T(sx) - T(-sx)) * i2x, dTdy = (T(sy) - T(-sy)) * i2y,
                         dTdz = (T(1) - T(-1)) * i2z;
            const double eq[3] = {-c.kappa * dTdx, -c.kappa * dTdy, -c.kappa * dTdz};
            for (int m = 0; m < 3; ++m)
                d[7 + m] = dcap((d[7 + m] + dt * eq[m] / c.tau_heat) / (1.0 + dt / c.tau_heat), cap);
        }
        for (int v = 0; v < 10; ++v) pr[(size_t)(5 + v) * nc + cl] = d[v];
    }
}

// run diagnostics (utils/diagnostics.py:5-57, 128-183)
__device__ __forceinline__ void atomic_max_pos(double* dst, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax((unsigned long long*)dst, (unsigned long long)__double_as_longlong(v));
}

__global__ void k_diagnostics(AstroParams p, const double* pr, int nv, int nx, int ny, int nz,
                              int ng, double dx, double dy, double dz, double gamma,
                              double* out) {
    // cell counts below 2^31 (checked by the host), so 32-bit index arithmetic
    const unsigned nc = (unsigned)nx * ny * nz;
    const unsigned ey = ny - 2 * ng, ez = nz - 2 * ng;
    const unsigned n = (unsigned)(nx - 2 * ng) * ey * ez;
    const bool mhd = p.physics == ASTRO_RMHD, divb = nv >= 8;
    double gmax = 0.0, sx = 0.0, bmax = 0.0, bsum = 0.0, bsq = 0.0, cnt = 0.0;
    const int sX = ny * nz, sY = nz;
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const unsigned k = ng + t % ez, j = ng + (t / ez) % ey, i = ng + t / (ez * ey);
        const size_t c = ((size_t)i * ny + j) * nz + k;
        const double vx = pr[nc + c], vy = pr[2 * nc + c], vz = pr[3 * nc + c];
        double v2 = vx * vx + vy * vy + vz * vz;
        if (v2 >= 1.0) v2 = 1.0 - 1e-14;
        gmax = rmax(gmax, 1.0 / sqrt(1.0 - v2));
        if (i == (unsigned)ng) {
            double q[9], U[9];
            for (int v = 0; v < (mhd ? 9 : 5); ++v) q[v] = pr[(size_t)v * nc + c];
            Phys<double> P = Phys<double>::from(p);
            P.gamma = P.srhd_gamma = gamma;
            if (mhd) r_p2c(P, q, U);
            else s_p2c(P, q, U);
            sx += U[1];
        }
        if (divb) {
            const double* B = pr + 5 * nc + c;
            const double d = (B[sX] - B[-sX]) / (2.0 * dx) + (B[nc + sY] - B[nc - sY]) / (2.0 * dy) +
                             (B[2 * nc + 1] - B[2 * nc - 1]) / (2.0 * dz);
            bmax = rmax(bmax, fabs(d));
            bsum += d;
            bsq += d * d;
            cnt += 1.0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        gmax = rmax(gmax, __shfl_down_sync(0xffffffffu, gmax, o));
        bmax = rmax(bmax, __shfl_down_sync(0xffffffffu, bmax, o));
        sx += __shfl_down_sync(0xffffffffu, sx, o);
        bsum += __shfl_down_sync(0xffffffffu, bsum, o);
        bsq += __shfl_down_sync(0xffffffffu, bsq, o);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomic_max_pos(out, gmax);
        if (sx != 0.0) atomicAdd(out + 1, sx);
        if (divb) {
            atomic_max_pos(out + 2, bmax);
            atomicAdd(out + 3, bsum);
            atomicAdd(out + 4, bsq);
            atomicAdd(out + 5, cnt);
        }
    }
}

// ------------------------------------------------- fixed-metric GR ---
// lapse helpers of gr_metric.py:6-38 (r offset by 1e-12 as there)
__device__ __forceinline__ double gr_radius(double x, double y, double z) {
    return sqrt(x * x + y * y + z * z) + 1e-12;
}

__device__ __forceinline__ double gr_ks_alpha(double x, double y, double z, double M) {
    const double H = M / gr_radius(x, y, z);
    return 1.0 / sqrt(1.0 + 2.0 * H);
}

// grad ln(alpha): isotropic Schwarzschild lapse, or Kerr-Schild (spin 0)
__device__ __forceinline__ void gr_dlna(int metric, double x, double y, double z, double M,
                                        double* g) {
    const double r = gr_radius(x, y, z);
    double dlnadr;
    if (metric == ASTRO_GR_SCHWARZSCHILD) {
        const double a = M / (2.0 * r);
        const double denom = 1.0 - a * a;
        dlnadr = denom == 0.0 ? 0.0 : (2.0 * a) / (r * denom);
    } else {
        const double H = M / r;
        dlnadr = H / (r * (1.0 + 2.0 * H));
    }
    g[0] = dlnadr * (x / r);
    g[1] = dlnadr * (y / r);
    g[2] = dlnadr * (z / r);
}

struct GRGeom {
    int nx, ny, nz, ng, offs_x;
    double dx, dy, dz, mass;
    __device__ bool interior(unsigned c, int& i, int& j, int& k, double& x, double& y,
                             double& z) const {
        k = (int)(c % (unsigned)nz);
        const unsigned r = c / (unsigned)nz;
        j = (int)(r % (unsigned)ny);
        i = (int)(r / (unsigned)ny);
        if (i < ng || i >= nx - ng || j < ng || j >= ny - ng || k < ng || k >= nz - ng)
            return false;
        x = (offs_x + (i - ng) + 0.5) * dx;
        y = (j - ng + 0.5) * dy;
        z = (k - ng + 0.5) * dz;
        return true;
    }
};

// copy of the block with the interior velocities divided by max(alpha_KS,
// 1e-12): what the flux passes see (grhd_core.py:22-37)
__global__ void k_gr_rescale(const double* __restrict__ pr, double* __restrict__ out, int nv,
                             GRGeom G) {
    const unsigned nc = (unsigned)G.nx * G.ny * G.nz;
    for (unsigned c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        int i, j, k;
        double x, y, z;
        const bool in = G.interior(c, i, j, k, x, y, z);
        const double ax = in ? rmax(gr_ks_alpha(x, y, z, G.mass), 1e-12) : 1.0;
        for (int v = 0; v < nv; ++v) {
            const double q = pr[(size_t)v * nc + c];
            out[(size_t)v * nc + c] = (in && v >= 1 && v <= 3) ? q / ax : q;
        }
    }
}

// out[1..4] += coef * source over the interior (grhd_core.py:47-78,
// grmhd_core.py:47-80); out is a right-hand side (coef 1) or the stage's
// conserved state (coef = the stage's weight of dt * rhs)
__global__ void k_gr_source(AstroParams p, int metric, const double* __restrict__ pr,
                            double* __restrict__ out, GRGeom G, double coef) {
    const unsigned nc = (unsigned)G.nx * G.ny * G.nz;
    const bool mhd = p.physics == ASTRO_RMHD;
    const Phys<double> P = Phys<double>::from(p);
    const double gfac = p.gamma / (p.gamma - 1.0);
    for (unsigned c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        int i, j, k;
        double x, y, z;
        if (!G.interior(c, i, j, k, x, y, z)) continue;
        double g[3];
        gr_dlna(metric, x, y, z, G.mass, g);
        double q[9], U[9];
        for (int v = 0; v < (mhd ? 9 : 5); ++v) q[v] = pr[(size_t)v * nc + c];
        double v2 = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        if (v2 >= 1.0) v2 = 1.0 - 1e-14;
        const double W = 1.0 / sqrt(1.0 - v2);
        const double h = 1.0 + gfac * q[4] / rmax(q[0], 1e-12);
        double w = q[0] * h * W * W;
        if (mhd) {
            w = w + (q[5] * q[5] + q[6] * q[6] + q[7] * q[7]);
            r_p2c(P, q, U);
        } else {
            s_p2c(P, q, U);
        }
        w = w + q[4];
        double* o = out + c;
        o[(size_t)1 * nc] += coef * (w * g[0]);
        o[(size_t)2 * nc] += coef * (w * g[1]);
        o[(size_t)3 * nc] += coef * (w * g[2]);
        o[(size_t)4 * nc] += coef * (U[1] * g[0] + U[2] * g[1] + U[3] * g[2]);
    }
}

int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    if (g > 148 * 32) g = 148 * 32;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

// ------------------------------------------------- allocation-free rhs ---
// Scratch for astro_rhs_static: a fixed-size array in the module's device
// memory.  Every device that loads this library holds it (32 MiB) until the
// process exits.  Host code must not use the symbol's name as a device
// pointer: the device address is looked up with cudaGetSymbolAddress while
// the caller's context is current, once per CUDA context, and cached under
// that context's unique ID (cuCtxGetId, never reused within a process).  A
// primary context re-created after cudaDeviceReset, or a driver-API context
// the caller made current, is a new context with its own copy of the module,
// so it gets its own lookup instead of a stale address.
static constexpr size_t kStaticScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {
typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*CtxGetIdFn)(void* ctx, unsigned long long* id);

struct ScratchEntry {
    unsigned long long ctx_id;
    void* ptr;
};
constexpr int kScratchEntries = 64;
ScratchEntry g_scratch_cache[kScratchEntries];
int g_scratch_used = 0, g_scratch_next = 0;
std::mutex g_static_scratch_mu;

// unique ID of the calling thread's current context, or 0 when the driver
// entry points are unavailable (then every call looks the address up)
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_cur = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = (CtxGetCurrentFn)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)f;
    });
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_cur || !get_id || get_cur(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of g_static_scratch in the current context (nullptr on
// error).  The first call in a context may load the module; made while the
// stream is being captured it is refused (ASTRO_E_INVALID), since a module
// load inside a capture can invalidate it.
void* static_scratch_address(cudaStream_t s, int* err) {
    // a runtime call first, so that a thread with no current context gets the
    // device's primary context before the driver is asked for it
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
        *err = ASTRO_E_CUDA;
        return nullptr;
    }
    const unsigned long long id = current_context_id();
    std::lock_guard<std::mutex> lock(g_static_scratch_mu);
    if (id != 0)
        for (int e = 0; e < g_scratch_used; ++e)
            if (g_scratch_cache[e].ctx_id == id) return g_scratch_cache[e].ptr;
    if (cs != cudaStreamCaptureStatusNone) {
        *err = ASTRO_E_INVALID;
        return nullptr;
    }
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_static_scratch) != cudaSuccess || !ptr) {
        *err = ASTRO_E_CUDA;
        return nullptr;
    }
    if (id != 0) {
        int slot = g_scratch_used < kScratchEntries ? g_scratch_used++ : g_scratch_next;
        if (slot == g_scratch_next) g_scratch_next = (g_scratch_next + 1) % kScratchEntries;
        g_scratch_cache[slot] = ScratchEntry{id, ptr};
    }
    return ptr;
}
}  // namespace

// =================================================================== C ABI ==
extern "C" {

int astro_version(void) { return 10000; }

const char* astro_error_string(int code) {
    switch (code) {
        case ASTRO_OK: return "ok";
        case ASTRO_E_INVALID: return "invalid argument";
        case ASTRO_E_SHAPE: return "grid shape incompatible with the stencil/ghost layers";
        case ASTRO_E_WORKSPACE: return "workspace missing or too small";
        case ASTRO_E_UNSUPPORTED: return "configuration not supported";
        case ASTRO_E_CUDA: return "CUDA error";
        default: return "unknown error";
    }
}

size_t astro_rhs_workspace_bytes(const AstroParams* p, const AstroGrid* g) {
    if (validate(p, g) != ASTRO_OK) return 0;
    return layout_of(*p, *g, false).total;
}

int astro_rhs(const AstroParams* p, const AstroGrid* g, const double* pr, double* rhs,
              void* work, size_t work_bytes, void* stream) {
    int v = validate(p, g);
    if (v != ASTRO_OK) return v;
    if (!pr || !rhs) return ASTRO_E_INVALID;
    const Layout L = layout_of(*p, *g, false);
    if (!work || work_bytes < L.total) return ASTRO_E_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    const Bounds b = bounds_of(*p, *g);
    cudaError_t e = face_passes(*p, *g, b, pr, (char*)work, L, s);
    if (e != cudaSuccess) return ASTRO_E_CUDA;
    UpdArgs u = update_args(*p, *g, b, (char*)work, L);
    u.pr0 = pr; u.prk = pr; u.dst = rhs; u.rhs_only = 1;
    return cuda_status(launch_update(u, s));
}

// the layout of astro_step / astro_step_stage (fused stages where supported)
static Layout step_layout(const AstroParams& p, const AstroGrid& g) {
    return layout_of(p, g, true, astro_stage::supported(p, g));
}

size_t astro_step_workspace_bytes(const AstroParams* p, const AstroGrid* g) {
    if (validate(p, g) != ASTRO_OK) return 0;
    return step_layout(*p, *g).total;
}

// argument checks shared by astro_step and astro_step_stage
static int step_check(const AstroParams* p, const AstroGrid* g, int rk_order, void* work,
                      size_t work_bytes) {
    int v = validate(p, g);
    if (v != ASTRO_OK) return v;
    if (rk_order != 2 && rk_order != 3) return ASTRO_E_INVALID;
    const bool learned = p->c2p_guess == ASTRO_GUESS_LEARNED;
    if (p->c2p_guess != ASTRO_GUESS_REFERENCE && !learned) return ASTRO_E_INVALID;
    if (learned && (p->physics != ASTRO_RMHD || !p->mlp)) return ASTRO_E_UNSUPPORTED;
    if (!work || work_bytes < step_layout(*p, *g).total) return ASTRO_E_WORKSPACE;
    return ASTRO_OK;
}

// One SSPRK stage: faces of cur, update (U_{st-1} -> U_st in the workspace),
// con2prim into dst.  prf_ready: the float32 copy of cur is already in the
// workspace; dstf: where the con2prim also writes dst's float32 copy.
// The fused version: the float32 copy of cur (padded rows) if it is not in
// the workspace yet, the fused kernel over the updated cells, the update of
// the frame outside them, then con2prim of every cell (writing the next
// stage's float32 copy).
static int run_stage_fused(const AstroParams* p, const AstroGrid* g, const Layout& L, char* w,
                           const double* pr_in, const double* cur, double* dst, double dt,
                           int nst, int st, bool prf_ready, bool want_dstf,
                           AstroC2PStats* stats, cudaStream_t s) {
    const bool learned = p->c2p_guess == ASTRO_GUESS_LEARNED;
    const Bounds b = bounds_of(*p, *g);
    const size_t nc = (size_t)g->nx * g->ny * g->nz;
    float* prf = (float*)(w + L.prf);
    double* U = (double*)(w + L.U);
    if (!prf_ready) {
        k_prim_f32_rows<<<sm_count_cached() * 8, 256, 0, s>>>(cur, prf, (size_t)9 * g->nx * g->ny,
                                                               g->nz, L.pitch);
        mark(2, s);
    }
    astro_stage::StageArgs a;
    memset(&a, 0, sizeof(a));
    a.prf = prf; a.pr = cur; a.pr0 = pr_in; a.U = U; a.dst = dst;
    a.timeouts = stats ? &stats->wait_timeouts : nullptr;
    a.defer_count = (unsigned*)(w + L.dfr);
    a.defer_list = (unsigned*)(w + L.dfr + 256);
    a.nv = g->nv; a.nx = g->nx; a.ny = g->ny; a.nz = g->nz; a.pitch = L.pitch;
    a.lo = b.lo; a.hi[0] = b.hi[0]; a.hi[1] = b.hi[1]; a.hi[2] = b.hi[2];
    a.dd[0] = g->dx; a.dd[1] = g->dy; a.dd[2] = g->dz; a.dt = dt;
    for (int d = 0; d < 3; ++d) {
        a.idd[d] = 1.0 / a.dd[d];
        a.idd2[d] = 1.0 / (a.dd[d] * a.dd[d] + 1e-12);
    }
    a.stage = st; a.nstages = nst; a.p = *p;
    a.poll_limit = tile_poll_limit();
    cudaError_t e = astro_stage::launch(a, s);
    if (e != cudaSuccess) return ASTRO_E_CUDA;
    mark(0, s);
    UpdArgs u = update_args(*p, *g, b, w, L);
    u.pr0 = pr_in; u.prk = cur; u.U = U; u.dst = dst; u.dstf = nullptr;
    u.dt = dt; u.stage = st; u.nstages = nst; u.rhs_only = 0; u.stats = stats;
    u.defer_c2p = 1; u.frame_only = 1;
    e = launch_update(u, s);
    if (e != cudaSuccess) return ASTRO_E_CUDA;
    float* dstf = want_dstf ? prf : nullptr;
    if (learned) {
        C2PArgs c;
        c.U = U; c.q = dst;
        c.count = (long)nc;
        c.p = *p; c.net = (const mlp::Params*)p->mlp; c.stats = stats;
        c.status = nullptr; c.max_polish = step_polish();
        c.poll_limit = mma_poll_limit();
        c.fb_count = (unsigned*)(w + L.c2pfb);
        c.fb_list = (unsigned*)(w + L.c2pfb + 256);
        c.fb_cap = (unsigned)c2p_fb_capacity(*g);
        c.qf = dstf; c.qf_nz = g->nz; c.qf_pitch = L.pitch;
        e = launch_c2p_learned(c, s);
    } else {
        k_c2p<<<sm_count_cached() * 8, 128, 0, s>>>(*p, U, dst, (long)nc, stats, dstf, g->nz,
                                                    L.pitch);
        mark(1, s);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? ASTRO_OK : ASTRO_E_CUDA;
}

static int run_stage(const AstroParams* p, const AstroGrid* g, const Layout& L, char* w,
                     const double* pr_in, const double* cur, double* dst, double dt, int nst,
                     int st, bool prf_ready, float* dstf, AstroC2PStats* stats, cudaStream_t s) {
    if (L.fused)
        return run_stage_fused(p, g, L, w, pr_in, cur, dst, dt, nst, st, prf_ready,
                               dstf != nullptr, stats, s);
    const bool learned = p->c2p_guess == ASTRO_GUESS_LEARNED;
    const Bounds b = bounds_of(*p, *g);
    cudaError_t e = face_passes(*p, *g, b, cur, w, L, s, prf_ready);
    if (e != cudaSuccess) return ASTRO_E_CUDA;
    UpdArgs u = update_args(*p, *g, b, w, L);
    u.pr0 = pr_in; u.prk = cur; u.U = (double*)(w + L.U); u.dst = dst;
    u.dstf = learned ? nullptr : dstf;
    u.dt = dt; u.stage = st; u.nstages = nst; u.rhs_only = 0; u.stats = stats;
    u.defer_c2p = learned ? 1 : 0;
    e = launch_update(u, s);
    if (e != cudaSuccess) return ASTRO_E_CUDA;
    if (learned) {
        C2PArgs c;
        c.U = (const double*)(w + L.U); c.q = dst;
        c.count = (long)g->nx * g->ny * g->nz;
        c.p = *p; c.net = (const mlp::Params*)p->mlp; c.stats = stats;
        c.status = nullptr; c.max_polish = step_polish();
        c.poll_limit = mma_poll_limit();
        c.fb_count = (unsigned*)(w + L.c2pfb);
        c.fb_list = (unsigned*)(w + L.c2pfb + 256);
        c.fb_cap = (unsigned)c2p_fb_capacity(*g);
        c.qf = dstf;
        e = launch_c2p_learned(c, s);
        if (e != cudaSuccess) return ASTRO_E_CUDA;
    }
    return ASTRO_OK;
}

int astro_step(const AstroParams* p, const AstroGrid* g, const double* pr_in, double* pr_out,
               double dt, int rk_order, void* work, size_t work_bytes, AstroC2PStats* stats,
               void* stream) {
    int v = step_check(p, g, rk_order, work, work_bytes);
    if (v != ASTRO_OK) return v;
    if (!pr_in || !pr_out || pr_in == pr_out) return ASTRO_E_INVALID;
    const Layout L = step_layout(*p, *g);
    cudaStream_t s = (cudaStream_t)stream;
    char* w = (char*)work;
    const int nst = rk_order;
    const double* cur = pr_in;
    double* bufs[2] = {(double*)(w + L.prA), (double*)(w + L.prB)};
    const bool mixed = p->precision == ASTRO_PREC_MIXED;
    for (int st = 0; st < nst; ++st) {
        // stage 0 converts its input to the float32 copy; later stages get the
        // copy from the kernel that produced their primitives
        double* dst = (st == nst - 1) ? pr_out : bufs[st % 2];
        float* dstf = (mixed && st < nst - 1) ? (float*)(w + L.prf) : nullptr;
        v = run_stage(p, g, L, w, pr_in, cur, dst, dt, nst, st, st > 0, dstf, stats, s);
        if (v != ASTRO_OK) return v;
        cur = dst;
    }
    return ASTRO_OK;
}

int astro_step_stage(const AstroParams* p, const AstroGrid* g, const double* pr_in,
                     const double* pr_stage, double* pr_out, double dt, int rk_order, int stage,
                     void* work, size_t work_bytes, AstroC2PStats* stats, void* stream) {
    int v = step_check(p, g, rk_order, work, work_bytes);
    if (v != ASTRO_OK) return v;
    if (stage < 0 || stage >= rk_order) return ASTRO_E_INVALID;
    if (!pr_in || !pr_stage || !pr_out || pr_out == pr_in || pr_out == pr_stage)
        return ASTRO_E_INVALID;
    if (stage == 0 && pr_stage != pr_in) return ASTRO_E_INVALID;
    const Layout L = step_layout(*p, *g);
    // the caller may have changed pr_stage's ghosts since it was written: the
    // float32 copy is made from it here
    return run_stage(p, g, L, (char*)work, pr_in, pr_stage, pr_out, dt, rk_order, stage, false,
                     nullptr, stats, (cudaStream_t)stream);
}

unsigned long long astro_launch_count(void) { return g_launches.load(); }

int astro_debug_set_mma_poll_limit(long long polls) {
    if (polls < 0) return ASTRO_E_INVALID;
    g_mma_poll_limit.store(polls, std::memory_order_relaxed);
    return ASTRO_OK;
}

int astro_debug_rcp_f64(const double* x, double* y, int64_t n, void* stream) {
    if (n < 0) return ASTRO_E_INVALID;
    if (n == 0) return ASTRO_OK;
    if (!x || !y) return ASTRO_E_INVALID;
    const int grid = (int)((n + 255) / 256 < 65535 ? (n + 255) / 256 : 65535);
    k_rcp_f64<<<grid, 256, 0, (cudaStream_t)stream>>>(x, y, (long)n);
    return cudaGetLastError() == cudaSuccess ? ASTRO_OK : ASTRO_E_CUDA;
}

int astro_debug_set_tile_poll_limit(long long polls) {
    if (polls < 0) return ASTRO_E_INVALID;
    g_tile_poll_limit.store(polls, std::memory_order_relaxed);
    return ASTRO_OK;
}

int astro_debug_set_step_polish(int steps) {
    if (steps < -1 || steps > 50) return ASTRO_E_INVALID;
    g_step_polish.store(steps, std::memory_order_relaxed);
    return ASTRO_OK;
}

int astro_step_profiled(const AstroParams* p, const AstroGrid* g, const double* pr_in,
                        double* pr_out, double dt, int rk_order, void* work, size_t work_bytes,
                        AstroC2PStats* stats, void* stream, AstroKernelTimes* times) {
    if (!times) return ASTRO_E_INVALID;
    if (t_prof) return ASTRO_E_INVALID;  // a profiling session is running
    Prof P;
    if (P.create(64) != ASTRO_OK) return ASTRO_E_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEventRecord(P.ev[0], s);
    P.on = true;
    t_prof = &P;
    int rc = astro_step(p, g, pr_in, pr_out, dt, rk_order, work, work_bytes, stats, stream);
    t_prof = nullptr;
    if (rc == ASTRO_OK && cudaEventSynchronize(P.ev[P.n]) != cudaSuccess) rc = ASTRO_E_CUDA;
    memset(times, 0, sizeof(*times));
    if (rc == ASTRO_OK) P.sum(times);
    return rc;
}

int astro_prof_start(int max_launches, void* stream) {
    if (max_launches < 1 || max_launches > (1 << 20) || t_prof) return ASTRO_E_INVALID;
    Prof* P = new Prof();
    if (P->create(max_launches) != ASTRO_OK) {
        delete P;
        return ASTRO_E_CUDA;
    }
    cudaEventRecord(P->ev[0], (cudaStream_t)stream);
    P->on = true;
    t_prof = P;
    return ASTRO_OK;
}

int astro_prof_stop(AstroKernelTimes* times) {
    Prof* P = t_prof;
    if (!P || !times) return ASTRO_E_INVALID;
    t_prof = nullptr;
    int rc = cudaEventSynchronize(P->ev[P->n]) == cudaSuccess ? ASTRO_OK : ASTRO_E_CUDA;
    memset(times, 0, sizeof(*times));
    if (rc == ASTRO_OK) P->sum(times);
    delete P;
    return rc;
}

size_t astro_max_char_speed_workspace_bytes(void) { return 0; }

int astro_max_char_speed(const AstroParams* p, const AstroGrid* g, const double* pr,
                         double* out, void* work, size_t work_bytes, void* stream) {
    (void)work; (void)work_bytes;
    if (!p || !g || !pr || !out) return ASTRO_E_INVALID;
    if (g->nv < 5 || g->nx < 3 || g->ny < 3 || g->nz < 3) return ASTRO_E_SHAPE;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(out, 0, sizeof(double), s) != cudaSuccess) return ASTRO_E_CUDA;
    const size_t n = (size_t)(g->nx - 2) * (g->ny - 2) * (g->nz - 2);
    k_max_char_speed<<<grid_for(n, 256), 256, 0, s>>>(pr, g->nx, g->ny, g->nz, p->srhd_gamma,
                                                     (unsigned long long*)out);
    mark(2, s);
    k_floor_small<<<1, 1, 0, s>>>(out);
    mark(2, s);
    return cuda_status(cudaGetLastError());
}

int astro_periodic_yz(double* pr, const AstroGrid* g, int ng, void* stream) {
    if (!pr || !g || ng < 1) return ASTRO_E_INVALID;
    if (g->ny - 2 * ng < ng || g->nz - 2 * ng < ng) return ASTRO_E_SHAPE;
    const size_t nc = (size_t)g->nx * g->ny * g->nz;
    k_periodic_yz<<<grid_for(nc, 256), 256, 0, (cudaStream_t)stream>>>(pr, g->nv, g->nx, g->ny,
                                                                      g->nz, ng);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

int astro_outflow_right_x(double* pr, const AstroGrid* g, int ng, void* stream) {
    if (!pr || !g || ng < 1 || g->nx < 2 * ng + 1) return ASTRO_E_INVALID;
    const size_t n = (size_t)g->ny * g->nz * ng;
    k_outflow_right_x<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(pr, g->nv, g->nx,
                                                                         g->ny, g->nz, ng);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

int astro_nozzle_left_x(double* pr, const AstroGrid* g, const AstroNozzle* nz,
                        const double* draws, const int32_t* rank_map, int32_t n_weighted,
                        void* stream) {
    if (!pr || !g || !nz || nz->ng < 1) return ASTRO_E_INVALID;
    if (nz->perturb && (!draws || !rank_map) && n_weighted > 0) return ASTRO_E_INVALID;
    if (g->ny - 2 * nz->ng < 1 || g->nz - 2 * nz->ng < 1 || g->nx < nz->ng) return ASTRO_E_SHAPE;
    if (g->nv < 5 || (nz->physics == 1 && g->nv < 9)) return ASTRO_E_SHAPE;
    if (nz->n_tracers > 8) return ASTRO_E_UNSUPPORTED;
    if (nz->n_tracers > 0 && (nz->tracer_offset < 0 || nz->tracer_offset + nz->n_tracers > g->nv))
        return ASTRO_E_SHAPE;
    if (nz->two_temperature && nz->thermo_offset < 0) return ASTRO_E_SHAPE;
    if (nz->chemistry && nz->chem_offset < 0) return ASTRO_E_SHAPE;
    if (nz->b_init < 0 || nz->b_init > 3 || nz->ambient_bc < 0 || nz->ambient_bc > 1)
        return ASTRO_E_INVALID;
    if (nz->ambient_bc == 1 && g->nx <= nz->ng) return ASTRO_E_SHAPE;
    const size_t n = (size_t)nz->ng * (g->ny - 2 * nz->ng) * (g->nz - 2 * nz->ng);
    k_nozzle<<<grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(pr, g->nv, g->nx, g->ny, g->nz,
                                                                *nz, draws, rank_map, n_weighted);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

int astro_outflow_yz(double* pr, const AstroGrid* g, int ng, void* stream) {
    if (!pr || !g || ng < 1) return ASTRO_E_INVALID;
    if (g->ny - 2 * ng < 1 || g->nz - 2 * ng < 1 || g->nx < 1) return ASTRO_E_SHAPE;
    const size_t frame = (size_t)g->ny * g->nz - (size_t)(g->ny - 2 * ng) * (g->nz - 2 * ng);
    const size_t n = (size_t)g->nx * frame;
    k_outflow_yz<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(pr, g->nv, g->nx, g->ny,
                                                                     g->nz, ng);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

int astro_p2c(const AstroParams* p, const double* prim, double* cons, int64_t count, void* stream) {
    if (!p || count < 0) return ASTRO_E_INVALID;
    if (count == 0) return ASTRO_OK;  // an empty batch may pass null arrays
    if (!prim || !cons) return ASTRO_E_INVALID;
    k_p2c<<<grid_for(count, 128), 128, 0, (cudaStream_t)stream>>>(*p, prim, cons, count);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

int astro_c2p(const AstroParams* p, const double* cons, double* prim, int64_t count,
              AstroC2PStats* stats, void* stream) {
    if (!p || count < 0) return ASTRO_E_INVALID;
    if (count == 0) return ASTRO_OK;  // an empty batch may pass null arrays
    if (!prim || !cons) return ASTRO_E_INVALID;
    k_c2p<<<grid_for(count, 128), 128, 0, (cudaStream_t)stream>>>(*p, cons, prim, count, stats);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

int astro_cooling_heating(double* pr, const AstroGrid* g, int ng, double dt, double cool,
                          double heat, double p_max, void* stream) {
    if (!pr || !g || ng < 0 || g->nv < 5) return ASTRO_E_INVALID;
    if (cool == 0.0 && heat == 0.0) return ASTRO_OK;
    if (g->nx <= 2 * ng || g->ny <= 2 * ng || g->nz <= 2 * ng) return ASTRO_OK;
    const size_t n = (size_t)(g->nx - 2 * ng) * (g->ny - 2 * ng) * (g->nz - 2 * ng);
    k_cooling<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(pr, g->nx, g->ny, g->nz, ng, dt,
                                                                 cool, heat, p_max);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

int astro_two_temperature(double* pr, const AstroGrid* g, int ng, double dt, double tau,
                          int thermo_offset, void* stream) {
    if (!pr || !g || ng < 0 || thermo_offset < 0) return ASTRO_E_INVALID;
    if (g->nv < thermo_offset + 2 || tau <= 0.0) return ASTRO_OK;
    if (g->nx <= 2 * ng || g->ny <= 2 * ng || g->nz <= 2 * ng) return ASTRO_OK;
    const size_t n = (size_t)(g->nx - 2 * ng) * (g->ny - 2 * ng) * (g->nz - 2 * ng);
    k_two_temperature<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        pr, g->nx, g->ny, g->nz, ng, dt, tau, thermo_offset);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

int astro_ion_chemistry(double* pr, const AstroGrid* g, const AstroChemistry* c, double dt,
                        void* stream) {
    if (!pr || !g || !c || c->ng < 0 || c->chem_offset < 5) return ASTRO_E_INVALID;
    if (g->nv < c->chem_offset + 3) return ASTRO_E_SHAPE;
    if (g->nx <= 2 * c->ng || g->ny <= 2 * c->ng || g->nz <= 2 * c->ng) return ASTRO_OK;
    const size_t n = (size_t)(g->nx - 2 * c->ng) * (g->ny - 2 * c->ng) * (g->nz - 2 * c->ng);
    k_ion_chemistry<<<grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(pr, g->nx, g->ny, g->nz,
                                                                        *c, dt);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

size_t astro_causal_dissipation_workspace_bytes(const AstroGrid* g) {
    if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1) return 0;
    return (size_t)10 * g->nx * g->ny * g->nz * sizeof(double);
}

int astro_causal_dissipation(double* pr, const AstroGrid* g, const AstroDissipation* c, double dt,
                             void* work, size_t work_bytes, void* stream) {
    if (!pr || !g || !c || c->ng < 1) return ASTRO_E_INVALID;
    if (g->nv < 15) return ASTRO_E_SHAPE;
    if (c->tau_bulk <= 0.0 || c->tau_shear <= 0.0 || c->tau_heat <= 0.0) return ASTRO_E_INVALID;
    if (g->nx <= 2 * c->ng || g->ny <= 2 * c->ng || g->nz <= 2 * c->ng) return ASTRO_OK;
    if (c->advect && (!work || work_bytes < astro_causal_dissipation_workspace_bytes(g)))
        return ASTRO_E_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n = (size_t)(g->nx - 2 * c->ng) * (g->ny - 2 * c->ng) * (g->nz - 2 * c->ng);
    double* adv = c->advect ? (double*)work : nullptr;
    if (adv) {
        k_dissip_advect<<<grid_for(n, 128), 128, 0, s>>>(pr, adv, g->nx, g->ny, g->nz, c->ng, dt,
                                                         g->dx, g->dy, g->dz);
        mark(2, s);
    }
    k_dissip_relax<<<grid_for(n, 128), 128, 0, s>>>(pr, adv, g->nx, g->ny, g->nz, *c, dt, g->dx,
                                                    g->dy, g->dz);
    mark(2, s);
    return cuda_status(cudaGetLastError());
}

static int gr_check(const AstroParams* p, const AstroGrid* g, const AstroGR* gr) {
    int v = validate(p, g);
    if (v != ASTRO_OK) return v;
    if (!gr || gr->metric < ASTRO_GR_MINKOWSKI || gr->metric > ASTRO_GR_OTHER) return ASTRO_E_INVALID;
    if (gr->ng < 0 || 2 * gr->ng >= g->nx || 2 * gr->ng >= g->ny || 2 * gr->ng >= g->nz)
        return ASTRO_E_SHAPE;
    if (!(gr->mass == gr->mass)) return ASTRO_E_INVALID;
    return ASTRO_OK;
}

static bool gr_rescales(const AstroGR& gr) {
    return gr.orthonormal_flux &&
           (gr.metric == ASTRO_GR_SCHWARZSCHILD || gr.metric == ASTRO_GR_KERR_SCHILD);
}

static GRGeom gr_geom(const AstroGrid& g, const AstroGR& gr) {
    GRGeom G;
    G.nx = g.nx; G.ny = g.ny; G.nz = g.nz; G.ng = gr.ng; G.offs_x = gr.offs_x;
    G.dx = g.dx; G.dy = g.dy; G.dz = g.dz; G.mass = gr.mass;
    return G;
}

size_t astro_gr_workspace_bytes(const AstroParams* p, const AstroGrid* g, const AstroGR* gr,
                                int step) {
    if (gr_check(p, g, gr) != ASTRO_OK) return 0;
    const size_t nc = (size_t)g->nx * g->ny * g->nz;
    return layout_of(*p, *g, step != 0).total +
           (gr_rescales(*gr) ? align256((size_t)g->nv * nc * 8) : 0);
}

// the flux passes' input: pr, or its rescaled copy at the end of the workspace
static const double* gr_flux_input(const AstroGR& gr, const AstroGrid& g, const double* pr,
                                   char* w, size_t off, cudaStream_t s) {
    if (!gr_rescales(gr)) return pr;
    double* out = (double*)(w + off);
    const size_t nc = (size_t)g.nx * g.ny * g.nz;
    k_gr_rescale<<<grid_for(nc, 256), 256, 0, s>>>(pr, out, g.nv, gr_geom(g, gr));
    mark(2, s);
    return out;
}

int astro_rhs_gr(const AstroParams* p, const AstroGrid* g, const AstroGR* gr, const double* pr,
                 double* rhs, void* work, size_t work_bytes, void* stream) {
    int v = gr_check(p, g, gr);
    if (v != ASTRO_OK) return v;
    if (!pr || !rhs) return ASTRO_E_INVALID;
    const Layout L = layout_of(*p, *g, false);
    if (!work || work_bytes < astro_gr_workspace_bytes(p, g, gr, 0)) return ASTRO_E_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    char* w = (char*)work;
    const Bounds b = bounds_of(*p, *g);
    const double* fin = gr_flux_input(*gr, *g, pr, w, L.total, s);
    cudaError_t e = face_passes(*p, *g, b, fin, w, L, s);
    if (e != cudaSuccess) return ASTRO_E_CUDA;
    UpdArgs u = update_args(*p, *g, b, w, L);
    u.pr0 = pr; u.prk = pr; u.dst = rhs; u.rhs_only = 1;
    e = launch_update(u, s);
    if (e != cudaSuccess) return ASTRO_E_CUDA;
    if (gr->metric != ASTRO_GR_MINKOWSKI) {
        const size_t nc = (size_t)g->nx * g->ny * g->nz;
        k_gr_source<<<grid_for(nc, 256), 256, 0, s>>>(*p, gr->metric, pr, rhs, gr_geom(*g, *gr),
                                                      1.0);
        mark(2, s);
    }
    return cuda_status(cudaGetLastError());
}

int astro_step_gr(const AstroParams* p, const AstroGrid* g, const AstroGR* gr,
                  const double* pr_in, double* pr_out, double dt, int rk_order, void* work,
                  size_t work_bytes, AstroC2PStats* stats, void* stream) {
    int v = gr_check(p, g, gr);
    if (v != ASTRO_OK) return v;
    if (!pr_in || !pr_out || pr_in == pr_out) return ASTRO_E_INVALID;
    if (rk_order != 2 && rk_order != 3) return ASTRO_E_INVALID;
    const bool learned = p->c2p_guess == ASTRO_GUESS_LEARNED;
    if (p->c2p_guess != ASTRO_GUESS_REFERENCE && !learned) return ASTRO_E_INVALID;
    if (learned && (p->physics != ASTRO_RMHD || !p->mlp)) return ASTRO_E_UNSUPPORTED;
    const Layout L = layout_of(*p, *g, true);
    if (!work || work_bytes < astro_gr_workspace_bytes(p, g, gr, 1)) return ASTRO_E_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    char* w = (char*)work;
    const Bounds b = bounds_of(*p, *g);
    const int nst = rk_order;
    const size_t nc = (size_t)g->nx * g->ny * g->nz;
    const double* cur = pr_in;
    double* bufs[2] = {(double*)(w + L.prA), (double*)(w + L.prB)};
    double* U = (double*)(w + L.U);
    for (int st = 0; st < nst; ++st) {
        // the update writes U only; the sources are added to U with the
        // stage's weight of dt * rhs, then con2prim gives the primitives
        const double* fin = gr_flux_input(*gr, *g, cur, w, L.total, s);
        cudaError_t e = face_passes(*p, *g, b, fin, w, L, s);
        if (e != cudaSuccess) return ASTRO_E_CUDA;
        double* dst = (st == nst - 1) ? pr_out : bufs[st % 2];
        UpdArgs u = update_args(*p, *g, b, w, L);
        u.pr0 = pr_in; u.prk = cur; u.U = U; u.dst = dst; u.dstf = nullptr;
        u.dt = dt; u.stage = st; u.nstages = nst; u.rhs_only = 0; u.stats = stats;
        u.defer_c2p = 1;
        e = launch_update(u, s);
        if (e != cudaSuccess) return ASTRO_E_CUDA;
        if (gr->metric != ASTRO_GR_MINKOWSKI) {
            const double wgt = st == 0 ? 1.0 : (nst == 2 ? 0.5 : (st == 1 ? 0.25 : 2.0 / 3.0));
            k_gr_source<<<grid_for(nc, 256), 256, 0, s>>>(*p, gr->metric, cur, U,
                                                          gr_geom(*g, *gr), wgt * dt);
            mark(2, s);
        }
        if (learned) {
            C2PArgs c;
            c.U = U; c.q = dst; c.count = (long)nc;
            c.p = *p; c.net = (const mlp::Params*)p->mlp; c.stats = stats;
            c.status = nullptr; c.max_polish = step_polish();
        c.poll_limit = mma_poll_limit();
            c.fb_count = (unsigned*)(w + L.c2pfb);
            c.fb_list = (unsigned*)(w + L.c2pfb + 256);
            c.fb_cap = (unsigned)c2p_fb_capacity(*g);
            e = launch_c2p_learned(c, s);
        } else {
            k_c2p<<<sm_count_cached() * 8, 128, 0, s>>>(*p, U, dst, (long)nc, stats);
            mark(2, s);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return ASTRO_E_CUDA;
        cur = dst;
    }
    return ASTRO_OK;
}

int astro_diagnostics(const AstroParams* p, const AstroGrid* g, int ng, const double* pr,
                      double gamma, double* out, void* stream) {
    if (!p || !g || !pr || !out || ng < 1) return ASTRO_E_INVALID;
    if (g->nv < 5 || (p->physics == ASTRO_RMHD && g->nv < 9)) return ASTRO_E_SHAPE;
    if ((double)g->nv * g->nx * g->ny * g->nz >= 2147483648.0) return ASTRO_E_SHAPE;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(out, 0, 6 * sizeof(double), s) != cudaSuccess) return ASTRO_E_CUDA;
    if (g->nx <= 2 * ng || g->ny <= 2 * ng || g->nz <= 2 * ng) return ASTRO_OK;
    const size_t n = (size_t)(g->nx - 2 * ng) * (g->ny - 2 * ng) * (g->nz - 2 * ng);
    const int grid = grid_for(n, 256) < sm_count_cached() * 8 ? grid_for(n, 256) : sm_count_cached() * 8;
    k_diagnostics<<<grid, 256, 0, s>>>(*p, pr, g->nv, g->nx, g->ny, g->nz, ng, g->dx, g->dy, g->dz,
                                       gamma, out);
    mark(2, s);
    return cuda_status(cudaGetLastError());
}

size_t astro_c2p_learned_workspace_bytes(int64_t count) {
    if (count < 0) return 0;
    return 256 + (size_t)count * sizeof(unsigned);
}

int astro_c2p_learned(const AstroParams* p, const double* cons, double* prim, int64_t count,
                      int max_polish, void* work, size_t work_bytes, AstroC2PStats* stats,
                      int* status, void* stream) {
    if (!p || count < 0 || p->physics != ASTRO_RMHD) return ASTRO_E_INVALID;
    if (max_polish < 0 || max_polish > 50) return ASTRO_E_INVALID;
    if (count == 0) return ASTRO_OK;  // an empty batch may pass null arrays
    if (!cons || !prim) return ASTRO_E_INVALID;
    C2PArgs c;
    c.U = cons; c.q = prim; c.count = count; c.p = *p;
    c.net = (const mlp::Params*)p->mlp; c.stats = stats; c.status = status;
    c.max_polish = max_polish;
    c.poll_limit = mma_poll_limit();
    if (work) {
        // fallback list: cell indices are 32-bit
        if (work_bytes < astro_c2p_learned_workspace_bytes(count)) return ASTRO_E_WORKSPACE;
        if (count >= (int64_t)UINT32_MAX) return ASTRO_E_SHAPE;
        c.fb_count = (unsigned*)work;
        c.fb_list = (unsigned*)((char*)work + 256);
        c.fb_cap = (unsigned)count;
    }
    return cuda_status(launch_c2p_learned(c, (cudaStream_t)stream));
}

int astro_c2p_features(const double* cons, float* x, int64_t count, void* stream) {
    if (count < 0) return ASTRO_E_INVALID;
    if (count == 0) return ASTRO_OK;  // an empty batch may pass null arrays
    if (!cons || !x) return ASTRO_E_INVALID;
    k_c2p_features<<<grid_for(count, 256), 256, 0, (cudaStream_t)stream>>>(cons, x, count);
    mark(2, (cudaStream_t)stream);
    return cuda_status(cudaGetLastError());
}

size_t astro_rhs_static_max_bytes(void) { return kStaticScratchBytes; }

int astro_rhs_static(const AstroParams* p, const AstroGrid* g, const double* pr, double* rhs,
                     void* stream) {
    int v = validate(p, g);
    if (v != ASTRO_OK) return v;
    if (!pr || !rhs) return ASTRO_E_INVALID;
    const Layout L = layout_of(*p, *g, false);
    if (L.total > kStaticScratchBytes) return ASTRO_E_WORKSPACE;  // grid too large
    int err = ASTRO_OK;
    cudaStream_t s = (cudaStream_t)stream;
    char* w = (char*)static_scratch_address(s, &err);
    if (!w) return err;
    const Bounds b = bounds_of(*p, *g);
    // every scratch value the update reads is written by the face passes of
    // this same call; the one counter that must start at zero (the float32
    // fix-up list's) is cleared by each face pass
    cudaError_t e = face_passes(*p, *g, b, pr, w, L, s);
    if (e != cudaSuccess) return ASTRO_E_CUDA;
    UpdArgs u = update_args(*p, *g, b, w, L);
    u.pr0 = pr; u.prk = pr; u.dst = rhs; u.rhs_only = 1;
    return cuda_status(launch_update(u, s));
}

}  // extern "C"
