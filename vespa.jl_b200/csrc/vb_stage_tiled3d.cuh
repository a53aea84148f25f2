// vb_stage_tiled3d.cuh -- shared pieces of the tiled, z-marching fused RK2
// stage kernels for 3D uniform meshes (the hot path of the 256^3 benchmark):
// the tile geometry and the TMA stage-buffer layout (a block owns a 16 x 16
// column tile and marches z, loading each plane's interior and its four 2-cell
// halo strips NS planes ahead of use), halo indexing, the per-cell LO_* order
// classes, the CFL terms, the box lookup and the persistent-grid sizing.  The
// kernels are k_stage_tiled3d_f64 (VB_FP64, vb_stage_tiled3d_f64.cuh) and
// k_stage_tiled3d_mixed (VB_MIXED, vb_stage_tiled3d_mixed.cuh).
//
// Requirements (checked on the host): nx % 16 == 0, ny % 16 == 0, nz >= 2, and
// a periodic axis is periodic on both sides.  The BF instantiations record the
// domain-boundary faces' fluxes in the boundary-flux register (bflux_add).
#pragma once

#include <cstring>

#include "vb_launch.h"
#include "vb_stage_generic.cuh"

namespace vb {

namespace t3 {

constexpr int TX = 16, TY = 16, NT = TX * TY;
constexpr int NH = 4 * TY + 4 * TX;  // halo cells: two 2-wide x strips, two 2-high y strips
constexpr int UPLANE = (NT + NH) * 5;  // float64 values per staged plane
// TMA box regions inside a staged plane (float64 offsets), each [5][..] field-major
constexpr int U_XLO = NT * 5;
constexpr int U_XHI = U_XLO + 2 * TY * 5;
constexpr int U_YLO = U_XHI + 2 * TY * 5;
constexpr int U_YHI = U_YLO + 2 * TX * 5;
constexpr uint32_t PLANE_BYTES = UPLANE * 8;
constexpr int TMA_ISSUER = 5 * 32;  // the thread that issues a block's stage loads
// every TMA destination in shared memory is 128-byte aligned
static_assert((U_XLO * 8) % 128 == 0 && (U_XHI * 8) % 128 == 0 && (U_YLO * 8) % 128 == 0 &&
                  (U_YHI * 8) % 128 == 0 && (UPLANE * 8) % 128 == 0,
              "TMA destinations must be 128-byte aligned");

// halo index -> staged-plane offset of field 0 (add f * region field stride)
__device__ __forceinline__ int halo_uoff(int h, int f)
{
    if (h < 32) return U_XLO + f * (2 * TY) + (h >> 1) * 2 + (h & 1);
    if (h < 64) { h -= 32; return U_XHI + f * (2 * TY) + (h >> 1) * 2 + (h & 1); }
    if (h < 96) { h -= 64; return U_YLO + f * (2 * TX) + (h >> 4) * TX + (h & 15); }
    h -= 96;
    return U_YHI + f * (2 * TX) + (h >> 4) * TX + (h & 15);
}
// halo index of local cell (lx, ly) outside the interior (star stencil only)
__device__ __forceinline__ int halo_idx(int lx, int ly)
{
    if (lx < 0) return ly * 2 + (lx + 2);
    if (lx >= TX) return 32 + ly * 2 + (lx - TX);
    if (ly < 0) return 64 + (ly + 2) * TX + lx;
    return 96 + (ly - TY) * TX + lx;
}

}  // namespace t3

// The float64 HLLC of the tiled 3D kernel, one non-inlined body per face
// orientation.  The kernel solves faces at seven call sites; inlined at each,
// its code outgrew the instruction cache (no_instruction stalls), and as a
// call it runs about 5 % faster.  The operations, hence the bits, are the same.
struct F64x5 {
    double v[5];
};
template <int DIM>
__device__ __noinline__ F64x5 hllc_f64_call(F64x5 L, F64x5 R, double gamma)
{
    F64x5 F;
    hllc_flux<double, DIM>(L.v, R.v, gamma, F.v);
    return F;
}
template <int DIM>
__device__ __forceinline__ void tiled_hllc(const double WL[5], const double WR[5], double gamma,
                                           double F[5])
{
    F64x5 L, R;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        L.v[k] = WL[k];
        R.v[k] = WR[k];
    }
    const F64x5 r = hllc_f64_call<DIM>(L, R, gamma);
#pragma unroll
    for (int k = 0; k < 5; ++k) F[k] = r.v[k];
}

// A stage load's bounded wait gave up (a block-uniform decision, taken after
// the barrier that follows the wait): the block issues no further load and
// skips the rest of its work.  Thread 0 waits, each wait bounded again, for
// the item's stage loads that may still be in flight -- stage planes q .. q +
// NS - 1 below nplanes, pipeline position qb -- so that no copy lands in the
// block's shared memory after it has exited, and flags the box; every thread
// waits for its own cp.async copies.  The caller then returns from the kernel.
template <int NS>
__device__ __noinline__ void stage_abandon(uint64_t *bars, int qb, int q, int nplanes, Ctrl *ctrl)
{
    cp_async_wait_all();
    if (threadIdx.x != 0) return;
    for (int j = q; j < q + NS && j < nplanes; ++j)
        mbar_wait(&bars[(qb + j) % NS], ((qb + j) / NS) & 1, WAIT_LIMIT_NS);
    atomicOr(&ctrl->flags, CTRL_F_TIMEOUT);
}

// _bflux_capture!, src/reflux.jl:125-132, for the tiled kernels: the thread
// that solved domain-boundary face (axis d, side) adds (scale * F) * area to
// entry `idx` of that plane (the other axes column-major, lowest fastest).
// Each entry belongs to one face, hence to one thread of the launch, and the
// launches of a step are ordered, so the sum is the serial one; the add is a
// fire-and-forget reduction (no value returned), so the solving warp does not
// wait for the register's memory before the block's next barrier.
static __device__ __forceinline__ void bflux_add(const Geom &g, double *bf, int d, int side,
                                                 int64_t idx, double scale, double area,
                                                 const double F[5])
{
    // plane sizes as products of the other axes (ncell / n[e] without a division)
    const int64_t P0 = g.n[1] * g.n[2], P1 = g.n[0] * g.n[2], P2 = g.n[0] * g.n[1];
    const int64_t P = d == 0 ? P0 : (d == 1 ? P1 : P2);
    int64_t off = d == 0 ? 0 : (d == 1 ? 10 * P0 : 10 * (P0 + P1));
    off += (int64_t)side * 5 * P + idx;
    if (!VB_DCHECK(idx >= 0 && idx < P)) return;  // check build only
#pragma unroll
    for (int k = 0; k < 5; ++k) atomicAdd(bf + off + k * P, scale * F[k] * area);
}

__device__ __forceinline__ int lo_class(int64_t c, int64_t n, bool periodic)
{
    if (c > 0) return LO_BEFORE;
    return (periodic && n > 1) ? LO_AFTER : LO_SELF;
}

__device__ __forceinline__ void prefetch_l1(const void *p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// compute_dt's per-cell term of a new state, exactly as src/driver.jl:178-185;
// GRAV: then the free-fall rate of the cell (src/gravity.jl:439-441)
template <bool GRAV = false>
__device__ __forceinline__ double cfl_term_exact(const double un[5], const Geom &g, double m)
{
    double W[5];
    cons2prim(un, g.gamma, W);
    const double cs = sound_speed(W, g.gamma);
    m = nan_max(m, (fabs(W[1]) + cs) / g.w[0]);
    m = nan_max(m, (fabs(W[2]) + cs) / g.w[1]);
    m = nan_max(m, (fabs(W[3]) + cs) / g.w[2]);
    if constexpr (GRAV) m = nan_max(m, gravity_invdt(g.grav_G, W[0]));
    return m;
}

// The same over x and y only (2D grids: compute_dt loops d in 1:N)
__device__ __forceinline__ double cfl_term2d_exact(const double un[5], const Geom &g, double m)
{
    double W[5];
    cons2prim(un, g.gamma, W);
    const double cs = sound_speed(W, g.gamma);
    m = nan_max(m, (fabs(W[1]) + cs) / g.w[0]);
    return nan_max(m, (fabs(W[2]) + cs) / g.w[1]);
}

// Persistent: a grid of (2 x SMs) blocks pulls work items from work[STAGE-1].
// An item is a column tile and a z chunk of one box (within a box, item =
// chunk * ntiles + tile, so concurrently processed items are spatial
// neighbours and share halo planes in L2).
//
// BATCH = false: one box, passed by value as a kernel parameter (its geometry
// and tensor maps are then read from the constant bank); BATCH = true: the box
// of each item is looked up in the device table.
template <bool BATCH>
__device__ __forceinline__ const BoxDesc &box_of(const BoxDesc &box0, const BoxDesc *boxes,
                                                 const int *item_box, int item)
{
    if constexpr (BATCH)
        return boxes[item_box[item]];
    else
        return box0;
}

}  // namespace vb

namespace vb {

// Resident blocks of a persistent kernel on the current device (all SMs), with
// its dynamic shared memory opted in once.
template <typename K>
int persistent_blocks(K kernel1, K kernel2, size_t smem)
{
    if (cudaFuncSetAttribute(kernel1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(kernel2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
        return -1;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel2, t3::NT, smem) != cudaSuccess ||
        per_sm < 1)
        return -1;
    return sms * per_sm;
}

}  // namespace vb
