// stage.cuh -- the fused SSPRK stage kernel (internal interface between
// stage.cu and kernels.cu; not part of the C ABI).
//
// One kernel per RK stage replaces the three per-direction face passes, the
// face-flux buffers and the update pass of the split path: each thread block
// owns a 4 x 32 (y, z) column of cells and marches along x through a chunk
// of planes.  The float32 primitives arrive by TMA (cp.async.bulk.tensor) into
// shared memory: for every plane a box with the 3-cell y/z halo (the y and z
// faces' stencils) and, six planes deep, a ring of the column's own cells (the
// x faces' stencils).  Every face of the block is evaluated once from shared
// memory, the y/z fluxes stay in shared memory, the x fluxes in registers,
// and the divergence, GLM damping, resistive term and the float64 SSPRK
// combination follow in the same thread, which writes U_k.  The reference's
// per-cell loop (core/rmhd_core.py:1440-1557) evaluates the same faces twice.
// The split path (per-direction face kernels + update) stays the default: on
// B200 at 256^3 the fused kernel takes 3.85-3.93 ms per stage against the
// split path's 3.6 ms (16 resident warps per SM, set by its 56 KB of shared
// memory and 128 registers, against the face kernels' 32).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/astrofd.h"

namespace astro_stage {

// cells owned by one thread block: TY rows (y) x TZ columns (z); planes per
// block along x
constexpr int TY = 4, TZ = 32, TX = 32;
constexpr int kThreads = TY * TZ;

struct StageArgs {
    const float* prf;     // float32 copy of the stage input, padded rows (pitch)
    const double* pr;     // stage input (float64): resistive term, psi, fix-ups
    const double* pr0;    // step input: U0 = p2c(pr0), passives
    double* U;            // U_{k-1} in (stages 1, 2), U_k out
    double* dst;          // next primitives: passive rows written here
    unsigned long long* timeouts;  // AstroC2PStats.wait_timeouts or null
    unsigned* defer_count;  // cells whose float32 faces overflowed: counter
    unsigned* defer_list;   // and list (a slot for every cell), redone by a
                            // second kernel with those faces in float64
    int nv, nx, ny, nz, pitch;
    int lo, hi[3];        // updated cells [lo, hi[d]) per direction
    double dd[3], dt;
    double idd[3], idd2[3];  // 1/dd and 1/(dd^2 + 1e-12), computed on the host
    int stage, nstages;
    long poll_limit;      // polls per tile-load wait (the default, or a test setting)
    AstroParams p;
};
// polls per tile-load wait unless a test sets fewer
constexpr long kTilePollLimit = 1L << 24;

// whether the fused kernel covers this configuration: RMHD, float32 faces,
// conservative fluxes, WENO5 or PPM, HLLE or "hlld", no passive fluxes
bool supported(const AstroParams& p, const AstroGrid& g);
// row pitch (floats) of the padded float32 primitive copy: rows of 16 bytes
inline int pitch_of(int nz) { return (nz + 3) & ~3; }
// launches the fused kernel over the updated cells; the caller updates the
// cells outside them (ghosts and the reference's loop-bound frame)
cudaError_t launch(const StageArgs& a, cudaStream_t s);

}  // namespace astro_stage
