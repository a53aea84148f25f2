// vb_common.cuh -- device-side geometry, control block and small helpers
// shared by every kernel translation unit of libvespa_b200.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace vb {

// Device bounds checks of the check build (`make -C vespa.jl_b200/csrc check`:
// -DVB_CHECK, libvespa_b200_check.so).  VB_DCHECK(cond) is true when cond
// holds; otherwise it records the source line of the check in its
// translation unit's word (the first failure wins) and the caller skips the
// access it guards, so a bad index becomes a status instead of a fault.
// vb_check_read collects and clears the words through readers that each
// translation unit registers at load time.  In the normal build VB_DCHECK is
// the constant true and generates no code.
#ifdef VB_CHECK
void check_register(unsigned (*read_and_clear)());  // vb_api.cu
namespace {
__device__ unsigned int vb_check_word = 0;
__device__ __noinline__ bool vb_dcheck_fail(unsigned line)
{
    atomicCAS(&vb_check_word, 0u, line);
    return false;
}
unsigned vb_check_take()
{
    unsigned w = 0;
    const unsigned z = 0;
    if (cudaMemcpyFromSymbol(&w, vb_check_word, sizeof w) != cudaSuccess) return 0;
    cudaMemcpyToSymbol(vb_check_word, &z, sizeof z);
    return w;
}
struct VbCheckRegistrar {
    VbCheckRegistrar() { check_register(&vb_check_take); }
} vb_check_registrar;
}  // namespace
#define VB_DCHECK(cond) ((cond) ? true : vb_dcheck_fail(__LINE__))
#else
#define VB_DCHECK(cond) true
#endif

enum { BC_OUTFLOW = 0, BC_PERIODIC = 1, BC_REFLECTING = 2 };
enum { PREC_FP64 = 0, PREC_MIXED = 1 };

// Uniform-mesh geometry (lib/RefMesh/src/RefMesh.jl:122-142), passed by value
// to kernels.  Unused axes have n = 1.
struct Geom {
    int nd;
    int bc_lo[3];
    int bc_hi[3];
    int64_t n[3];
    int64_t stride[3];
    int64_t ncell;
    double w[3];     // cell widths (hi - lo) / n
    double invw[3];  // 1 / w (VB_MIXED CFL term only)
    double area[3];  // face areas: product of the other axes' widths
    double vol;      // cell volume: left-fold product of the widths
    double gamma;
    double cfl;
    double aexp;
    // self-gravity (src/gravity.jl), set while a grid has gravity enabled:
    // grav_g = g = -grad phi per cell (nd * ncell doubles, axis-major), held
    // over a step; grav_G = the constant G of the free-fall dt limiter
    const double *grav_g;
    double grav_G;
    // slab of a z-split domain (vb_grid_set_zwindow): planes zw0 <= z < zw1
    // are this rank's own, the others ghost copies of its neighbours'.  The
    // CFL maximum and the totals cover cells act0 <= lin < act1 only, and
    // the tiled kernels give plane zw0 the lo-face order class zcls0 (its
    // class in the whole domain; -1: the slab's own).  Defaults: all planes.
    int zw0, zw1, zcls0;
    int64_t act0, act1;
};

// Coordinates of cell `lin` (x fastest, strides 1, n0, n0*n1): 32-bit
// unsigned divisions while the grid has fewer than 2^31 cells, 64-bit ones
// beyond (a 64-bit division is a long instruction sequence).
__device__ __forceinline__ void cell_coords(const Geom &g, int64_t lin, int64_t cc[3])
{
    if (g.ncell <= 0x7fffffffLL) {
        const unsigned l = (unsigned)lin, n0 = (unsigned)g.n[0], n1 = (unsigned)g.n[1];
        const unsigned q = l / n0, r = q / n1;
        cc[0] = (int64_t)(l - q * n0);
        cc[1] = (int64_t)(q - r * n1);
        cc[2] = (int64_t)r;
    } else {
        cc[0] = lin % g.n[0];
        cc[1] = (lin / g.n[0]) % g.n[1];
        cc[2] = lin / (g.n[0] * g.n[1]);
    }
}

// 4 pi, as FOURPI in src/gravity.jl:21
constexpr double VB_FOURPI = 4.0 * 3.14159265358979323846;

// _gravity_invdt, src/gravity.jl:439-441: the free-fall rate bound sqrt(4 pi G rho) / 0.5
__device__ __forceinline__ double gravity_invdt(double G, double rho)
{
    return rho > 0.0 ? __dsqrt_rn(__dmul_rn(__dmul_rn(VB_FOURPI, G), rho)) / 0.5 : 0.0;
}

// apply_gravity_source! for one cell (src/gravity.jl:371-382, 419-437):
// acc += (0, -rho g V, -(rho v . g) V) from the stage state u, with g zero on
// the axes beyond ND.  Every product and sum rounded separately, in the
// reference's order.
template <int ND>
__device__ __forceinline__ void gravity_source(const Geom &g, int64_t lin, const double u[5],
                                               double acc[5])
{
    double gv[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < ND; ++d) gv[d] = g.grav_g[d * g.ncell + lin];
    const double rho = u[0], V = g.vol;
    double es = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) es = __dadd_rn(es, __dmul_rn(u[1 + d], gv[d]));
    const double esV = __dmul_rn(es, V);
    acc[0] = __dadd_rn(acc[0], 0.0);
#pragma unroll
    for (int d = 0; d < 3; ++d)
        acc[1 + d] = __dadd_rn(acc[1 + d], -__dmul_rn(__dmul_rn(rho, gv[d]), V));
    acc[4] = __dadd_rn(acc[4], -esV);
}

// Per-grid control block in device memory.  The stepping kernels read dt and
// invV from here so a whole evolve! loop can run without host round trips.
struct Ctrl {
    double t;                       // simulation clock (sim.t)
    double dt;                      // dt of the step in flight
    double invV;                    // dt / (aexp * V)
    double tfinal;                  // evolve target; +Inf for fixed-count runs
    unsigned long long invdt_bits;  // running max of (|v_d| + c) / w_d (bit pattern)
    long long step;                 // sim.step
    long long step_limit;           // evolve: stop after this many steps
    int active;                     // 1 while the step in flight must run
    int flags;                      // error bits, CTRL_F_*
    unsigned int work[2];           // work-queue cursors of the two stage kernels
};

enum { CTRL_F_NONFINITE = 1, CTRL_F_TIMEOUT = 2 };

// min/max: fmin/fmax (one instruction).  They differ from Julia's Base.min /
// Base.max only in the sign of a zero result and in NaN handling.  Where they
// are used (the HLLC wave speeds SL/SR, the pressure floor, the dt clip) a
// zero's sign never reaches later arithmetic: SL and SR only feed the
// SL >= 0 / SR <= 0 tests when they are zero.  NaN is caught separately by the
// CFL reduction below.

// NaN-propagating max used by the CFL reduction: any NaN wins.
__device__ __forceinline__ double nan_max(double m, double x) { return (x > m || x != x) ? x : m; }

// Non-negative doubles order like their unsigned bit patterns; a NaN (either
// sign) has a larger pattern than +Inf, so a u64 max keeps NaN visible.
__device__ __forceinline__ unsigned long long order_bits(double x)
{
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    // a negative NaN has the sign bit set: still larger than +Inf's pattern
    return b;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide max folded into the control block's running max.  The read of
// the current value skips atomics that cannot raise it (the value only grows).
__device__ __forceinline__ void block_max_to(unsigned long long *dst, double v, double *smem32)
{
    v = warp_max(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) smem32[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double x = lane < nw ? smem32[lane] : 0.0;
        x = warp_max(x);
        if (lane == 0) {
            unsigned long long b = order_bits(x);
            if (b > *((volatile unsigned long long *)dst)) atomicMax(dst, b);
        }
    }
}

}  // namespace vb
