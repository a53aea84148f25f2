// vb_gravity.cu -- self-gravity on uniform grids (src/gravity.jl): the
// Poisson solve nabla^2 phi = 4 pi G rho by matrix-free conjugate gradients on
// the device, and the field g = -grad phi that the stage kernels add as a
// source (gravity_source in vb_common.cuh) while the grid has gravity enabled.
//
// Compiled with -fmad=false: the operator row, the field and the CG vector
// updates round every product and sum separately, like the reference's Julia
// loops.  The operator row is summed in the reference's CSR order
// (_assemble_poisson_struct, src/gravity.jl:514-545), so A x is bit-identical
// to the reference's _lap_csr_cpu! (325-334).  The CG inner products are
// deterministic block-tree sums (fixed partial count and order) rather than
// the reference's serial sums, so a solve matches the reference's to the
// solver tolerance, not bit for bit.
//
// Every pass streams the CG vectors from HBM over a fixed grid of GP blocks
// (the stencil's neighbours come from L1/L2); the stencil passes walk rows of
// x so that a cell's coordinates cost no division.  One
// CG iteration is five launches (matvec + p.Ap partials, alpha, vector update
// + r.r partials, beta, direction update); groups of iterations replay as one
// CUDA graph, each launch returning at once after convergence, and the host
// reads the stop flag between groups.
#include <cmath>
#include <cstring>
#include <vector>

#include "vb_internal.h"

namespace vb {
namespace {

constexpr int GB = 256;  // threads per block
constexpr int GP = 592;  // blocks (= partial sums) per reduction pass: 4 per SM, fixed
constexpr int GP_SM = 4;  // the GP blocks fit in one wave only at <= 64 registers a thread
constexpr int GRAPH_ITERS = 8;

struct GravCtrl {
    double rhobar, rsold, pAp, alpha, beta, bnorm, relres, mu, mgmu;
    long long iters, maxiter;
    int done, pad;
    double tol;
};

// phi's boundary codes and the operator's per-axis coefficient area / distance
struct GravP {
    int per_lo[3], per_hi[3];  // 1: periodic side
    double coef[3];
    double G;
    int project_mean;
};

// neighbour of `lin` (coordinate c on axis d) across its lo or hi face under
// phi's codes; -1 at a wall (homogeneous Neumann)
__device__ __forceinline__ int64_t gnb(const Geom &g, const GravP &P, int64_t lin, int64_t c,
                                       int d, bool hi)
{
    const int64_t n = g.n[d];
    const int64_t j = hi ? c + 1 : c - 1;
    if (j >= 0 && j < n) return hi ? lin + g.stride[d] : lin - g.stride[d];
    if (hi ? P.per_hi[d] : P.per_lo[d]) return lin + ((j < 0 ? n - 1 : 0) - c) * g.stride[d];
    return -1;
}

// Visit this block's cells: rows of x (coordinates derived once per row), rows
// strided over the GP blocks and x over the block's threads; a row shorter
// than half the block is shared with the next rows (thread t takes x = t % n0
// of row t / n0 of each group of GB / n0 rows), so no thread idles on a short
// row.  1D grids stride cells directly.  A fixed order per thread, so the
// partial sums are deterministic.
template <int ND, typename F>
__device__ __forceinline__ void for_cells(const Geom &g, F &&f)
{
    if constexpr (ND == 1) {
        for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < g.ncell; i += (int64_t)GP * GB) {
            const int64_t cc[3] = {i, 0, 0};
            f(i, cc);
        }
    } else {
        const int64_t n0 = g.n[0], nrow = g.ncell / n0;
        const int rpg = n0 >= GB / 2 ? 1 : GB / (int)n0;  // rows per group
        const int rsub = rpg == 1 ? 0 : (int)threadIdx.x / (int)n0;
        const int64_t cx0 = rpg == 1 ? threadIdx.x : (int)threadIdx.x - rsub * (int)n0;
        if (rsub >= rpg) return;
        // row = cz * n1 + cy, advanced by `step` rows without a division per row
        const int64_t n1 = g.n[1], step = (int64_t)GP * rpg, sy = step % n1, sz = step / n1;
        int64_t row = (int64_t)blockIdx.x * rpg + rsub, cy = row % n1, cz = row / n1;
        if (n0 <= GB) {
            // one cell per row and thread: two rows per pass, in the same
            // order, so that the loads of both are in flight together
            if (cx0 >= n0) return;
            for (; row + step < nrow; row += 2 * step) {
                int64_t cy2 = cy + sy, cz2 = cz + sz;
                if (cy2 >= n1) {
                    cy2 -= n1;
                    ++cz2;
                }
                const int64_t c1[3] = {cx0, cy, cz}, c2[3] = {cx0, cy2, cz2};
                f(row * n0 + cx0, c1);
                f((row + step) * n0 + cx0, c2);
                cy = cy2 + sy;
                cz = cz2 + sz;
                if (cy >= n1) {
                    cy -= n1;
                    ++cz;
                }
            }
            if (row < nrow) {
                const int64_t c1[3] = {cx0, cy, cz};
                f(row * n0 + cx0, c1);
            }
            return;
        }
        for (; row < nrow; row += step) {
            for (int64_t cx = cx0; cx < n0; cx += GB) {
                const int64_t cc[3] = {cx, cy, cz};
                f(row * n0 + cx, cc);
            }
            cy += sy;
            cz += sz;
            if (cy >= n1) {
                cy -= n1;
                ++cz;
            }
        }
    }
}

// (A x)[lin], A = -nabla^2 V: sum over the row's faces of coef * (x_c - x_nb),
// in the order the reference's CSR row lists them: lo faces emitted by a lower
// cell (z, y, x), the cell's own hi faces (x, y, z; a 1-cell periodic axis
// lists its self face twice), lo faces emitted by a periodic partner above
// (x, y, z).
template <int ND>
__device__ __forceinline__ double lap_row(const Geom &g, const GravP &P, const double *__restrict__ x,
                                          int64_t lin, const int64_t cc[3])
{
    const double xc = x[lin];
    double s = 0.0;
    bool inner = true;  // every neighbour inside the grid: the row lists the lo
#pragma unroll          // faces z, y, x, then the hi faces x, y, z
    for (int d = 0; d < ND; ++d) inner = inner && cc[d] >= 1 && cc[d] + 1 < g.n[d];
    if (inner) {
#pragma unroll
        for (int d = ND - 1; d >= 0; --d) s = s + P.coef[d] * (xc - x[lin - g.stride[d]]);
#pragma unroll
        for (int d = 0; d < ND; ++d) s = s + P.coef[d] * (xc - x[lin + g.stride[d]]);
        return s;
    }
#pragma unroll
    for (int d = ND - 1; d >= 0; --d) {
        const int64_t nb = gnb(g, P, lin, cc[d], d, false);
        if (nb >= 0 && nb < lin) s = s + P.coef[d] * (xc - x[nb]);
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        const int64_t nb = gnb(g, P, lin, cc[d], d, true);
        if (nb < 0) continue;
        s = s + P.coef[d] * (xc - x[nb]);
        if (nb == lin) s = s + P.coef[d] * (xc - x[nb]);
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        const int64_t nb = gnb(g, P, lin, cc[d], d, false);
        if (nb > lin) s = s + P.coef[d] * (xc - x[nb]);
    }
    return s;
}

// (A x)[i] on a periodic n^3 grid (the multigrid preconditioner's, and the CG
// matvec's when the grid is such a cube), in the
// same CSR row order as lap_row (lo faces of lower cells z, y, x; hi faces
// x, y, z, a 1-cell axis twice; lo faces wrapped to a higher index x, y, z),
// with 32-bit indices: the same bits as lap_row<3> on that grid.
// (x, y, z) of cell i of a periodic n^3 cube, x fastest: masks and shifts
// when n is a power of two, else two unsigned divisions
__device__ __forceinline__ void cube_coords(int n, int i, int c[3])
{
    const unsigned u = (unsigned)i, un = (unsigned)n;
    if ((un & (un - 1u)) == 0u) {
        const int sh = __ffs(n) - 1;
        c[0] = (int)(u & (un - 1u));
        c[1] = (int)((u >> sh) & (un - 1u));
        c[2] = (int)(u >> (2 * sh));
    } else {
        const unsigned q = u / un, r = q / un;
        c[0] = (int)(u - q * un);
        c[1] = (int)(q - r * un);
        c[2] = (int)r;
    }
}

__device__ __forceinline__ double lap_cube(int n, const GravP &P, const double *__restrict__ x, int i)
{
    int c[3];
    cube_coords(n, i, c);
    const int st[3] = {1, n, n * n};
    const double xc = x[i];
    double s = 0.0;
#pragma unroll
    for (int d = 2; d >= 0; --d)
        if (c[d] > 0) s = s + P.coef[d] * (xc - x[i - st[d]]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int nb = c[d] < n - 1 ? i + st[d] : i - (n - 1) * st[d];
        s = s + P.coef[d] * (xc - x[nb]);
        if (nb == i) s = s + P.coef[d] * (xc - x[nb]);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
        if (c[d] == 0 && n > 1) s = s + P.coef[d] * (xc - x[i + (n - 1) * st[d]]);
    return s;
}

// Deterministic sum over the block's threads (fixed tree: a shuffle tree in
// each warp, then one over the warp sums), returned to every thread.  `sh`
// holds at least NW + 1 doubles.
template <int NTH>
__device__ __forceinline__ double tree_sum(double v, double *sh)
{
    constexpr int NW = NTH / 32;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        double r = l < NW ? sh[l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r = r + __shfl_down_sync(0xffffffffu, r, o);
        if (l == 0) sh[NW] = r;
    }
    __syncthreads();
    const double r = sh[NW];
    __syncthreads();  // sh is free for the next sum
    return r;
}

__device__ __forceinline__ double block_sum(double v, double *sh) { return tree_sum<GB>(v, sh); }

// Sum of the GP partials part[0..GP) by one block of 1024 threads (fixed tree).
__device__ __forceinline__ double final_sum(const double *part, double *sh)
{
    const int t = threadIdx.x;
    return tree_sum<1024>(t < GP ? part[t] : 0.0, sh);
}

// partials of sum(x * V) and sum(V) (the volume-weighted mean of a field)
__global__ void __launch_bounds__(GB, GP_SM) k_meanpart(Geom g, const double *__restrict__ x, double *part)
{
    __shared__ double sh[GB];
    double s = 0.0, v = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < g.ncell; i += (int64_t)GP * GB) {
        s = s + x[i] * g.vol;
        v = v + g.vol;
    }
    s = block_sum(s, sh);
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
        part[GP + blockIdx.x] = v;
    }
}

// which = 0: rhobar; 1: mu (the potential's mean)
__global__ void __launch_bounds__(1024) k_mean_final(const double *part, GravCtrl *gc, int which)
{
    __shared__ double sh[1024];
    const double s = final_sum(part, sh);
    const double v = final_sum(part + GP, sh);
    if (threadIdx.x == 0) {
        if (which == 0) gc->rhobar = s / v;
        else gc->mu = s / v;
    }
}

// _rhs_flat_kernel!, src/gravity.jl:215-231: b = -4 pi G (rho - rhobar) V
__global__ void __launch_bounds__(GB, GP_SM) k_rhs(Geom g, GravP P, const double *__restrict__ U, double *b,
                                           const GravCtrl *gc)
{
    const double rhobar = P.project_mean ? gc->rhobar : 0.0;
    for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < g.ncell; i += (int64_t)GP * GB)
        b[i] = -VB_FOURPI * P.G * (U[i] - rhobar) * g.vol * 1.0;
}

// CG start, src/gravity.jl:272-279: r = b - A phi, p = r; partials of r.r and b.b
template <int ND>
__global__ void __launch_bounds__(GB, GP_SM) k_cg_init(Geom g, GravP P, const double *__restrict__ phi,
                                               const double *__restrict__ b, double *r, double *p,
                                               double *part)
{
    __shared__ double sh[GB];
    double rr = 0.0, bb = 0.0;
    for_cells<ND>(g, [&](int64_t i, const int64_t cc[3]) {
        const double ri = b[i] - lap_row<ND>(g, P, phi, i, cc);
        r[i] = ri;
        p[i] = ri;
        rr = rr + ri * ri;
        bb = bb + b[i] * b[i];
    });
    rr = block_sum(rr, sh);
    bb = block_sum(bb, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = rr;
        part[GP + blockIdx.x] = bb;
    }
}

__global__ void __launch_bounds__(1024) k_cg_init_final(const double *part, GravCtrl *gc)
{
    __shared__ double sh[1024];
    const double rr = final_sum(part, sh);
    const double bb = final_sum(part + GP, sh);
    if (threadIdx.x == 0) {
        double bnorm = sqrt(bb);
        if (bnorm == 0.0) bnorm = 1.0;
        gc->rsold = rr;
        gc->bnorm = bnorm;
        gc->relres = sqrt(rr) / bnorm;
        gc->iters = 0;
        gc->done = gc->maxiter <= 0 ? 1 : 0;
    }
}

// Ap = A p; partials of p.Ap
template <int ND>
__global__ void __launch_bounds__(GB, GP_SM) k_cg_matvec(Geom g, GravP P, const double *__restrict__ p,
                                                 double *__restrict__ Ap, double *part, const GravCtrl *gc)
{
    __shared__ double sh[GB];
    if (gc->done) return;
    double s = 0.0;
    for_cells<ND>(g, [&](int64_t i, const int64_t cc[3]) {
        const double a = lap_row<ND>(g, P, p, i, cc);
        Ap[i] = a;
        s = s + p[i] * a;
    });
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// k_cg_matvec on the periodic cube (lap_cube, the same row sums), one thread
// per cell; each block's p.Ap partial goes to cpart[block]
__global__ void __launch_bounds__(GB) k_cg_matvec_cube(int n, GravP P, const double *__restrict__ p,
                                                      double *__restrict__ Ap, double *cpart,
                                                      const GravCtrl *gc)
{
    __shared__ double sh[GB / 32 + 1];
    if (gc->done) return;
    const int i = blockIdx.x * GB + threadIdx.x;
    double s = 0.0;
    if (i < n * n * n) {
        const double a = lap_cube(n, P, p, i);
        Ap[i] = a;
        s = p[i] * a;
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) cpart[blockIdx.x] = s;
}

// fold nb block partials into the GP partials the one-block final sums read:
// block b sums its fixed contiguous range of cpart (a fixed tree)
__global__ void __launch_bounds__(GB, GP_SM) k_fold_parts(const double *__restrict__ cpart, int nb,
                                                         double *part, const GravCtrl *gc)
{
    __shared__ double sh[GB / 32 + 1];
    if (gc->done) return;
    const int per = (nb + GP - 1) / GP, lo = blockIdx.x * per, hi = min(nb, lo + per);
    double s = 0.0;
    for (int j = lo + (int)threadIdx.x; j < hi; j += GB) s = s + cpart[j];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// iters = k; stop when p.Ap <= 0, else alpha = rsold / p.Ap
__global__ void __launch_bounds__(1024) k_cg_alpha(const double *part, GravCtrl *gc)
{
    __shared__ double sh[1024];
    if (gc->done) return;
    const double pAp = final_sum(part, sh);
    if (threadIdx.x == 0) {
        gc->iters += 1;
        gc->pAp = pAp;
        if (pAp <= 0.0) gc->done = 1;
        else gc->alpha = gc->rsold / pAp;
    }
}

// phi += alpha p; r -= alpha Ap; partials of r.r
__global__ void __launch_bounds__(GB, GP_SM) k_cg_update(Geom g, double *phi, const double *__restrict__ p,
                                                 double *r, const double *__restrict__ Ap,
                                                 double *part, const GravCtrl *gc)
{
    __shared__ double sh[GB];
    if (gc->done) return;
    const double alpha = gc->alpha;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < g.ncell; i += (int64_t)GP * GB) {
        phi[i] = phi[i] + alpha * p[i];
        const double ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        s = s + ri * ri;
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// relres; stop at tol, else beta = rsnew / rsold; stop after maxiter
__global__ void __launch_bounds__(1024) k_cg_beta(const double *part, GravCtrl *gc)
{
    __shared__ double sh[1024];
    if (gc->done) return;
    const double rsnew = final_sum(part, sh);
    if (threadIdx.x == 0) {
        gc->relres = sqrt(rsnew) / gc->bnorm;
        if (gc->relres <= gc->tol) {
            gc->done = 1;
            return;
        }
        gc->beta = rsnew / gc->rsold;
        gc->rsold = rsnew;
        if (gc->iters >= gc->maxiter) gc->done = 1;
    }
}

// p = r + beta p
__global__ void __launch_bounds__(GB, GP_SM) k_cg_dir(Geom g, double *p, const double *__restrict__ r,
                                              const GravCtrl *gc)
{
    if (gc->done) return;
    const double beta = gc->beta;
    for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < g.ncell; i += (int64_t)GP * GB)
        p[i] = r[i] + beta * p[i];
}

__global__ void __launch_bounds__(GB, GP_SM) k_sub_mean(Geom g, double *phi, const GravCtrl *gc)
{
    const double mu = gc->mu;
    for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < g.ncell; i += (int64_t)GP * GB)
        phi[i] = phi[i] - mu;
}

// g = -grad phi, _gax (src/gravity.jl:387-394): central difference over the two
// face distances; across a wall the neighbour value is the cell's own and the
// distance half a width
template <int ND>
__global__ void __launch_bounds__(GB, GP_SM) k_accel(Geom g, GravP P, const double *__restrict__ phi,
                                             double *gacc)
{
    for_cells<ND>(g, [&](int64_t i, const int64_t cc[3]) {
        const double pc = phi[i];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const int64_t lo = gnb(g, P, i, cc[d], d, false), hi = gnb(g, P, i, cc[d], d, true);
            const double wlo = lo < 0 ? pc : phi[lo], whi = hi < 0 ? pc : phi[hi];
            const double fd = 0.5 * (g.w[d] + g.w[d]);  // _face_distance
            const double dlo = lo < 0 ? 0.5 * g.w[d] : fd, dhi = hi < 0 ? 0.5 * g.w[d] : fd;
            gacc[d * g.ncell + i] = -(whi - wlo) / (dlo + dhi);
        }
    });
}

template <int ND>
__global__ void __launch_bounds__(GB, GP_SM) k_lap(Geom g, GravP P, const double *__restrict__ x, double *out)
{
    for_cells<ND>(g, [&](int64_t i, const int64_t cc[3]) { out[i] = lap_row<ND>(g, P, x, i, cc); });
}

// ---------------------------------------------------------------------------
// Multigrid-preconditioned CG (precond = VB_GRAV_PRECOND_MG), after the
// reference's ext/mg_pcg.jl: the outer CG runs on the exact operator A; the
// preconditioner z = M^-1 r is one composite-smoothed two-level cycle
// (_amg_cycle!, mg_pcg.jl:152-174): two damped-Jacobi sweeps on A from z = 0,
// the residual moved to the base grid (on a uniform mesh the cells
// themselves), one periodic cell-centred V-cycle of -lap there (_mg_vcycle!,
// 123-145: damped Jacobi 2 + 2, full-weighting restriction, trilinear
// prolongation, 30 sweeps on the coarsest level), the correction de-meaned,
// scaled by 1/V and added, two more Jacobi sweeps on A.

constexpr double MG_OMEGA = 0.8;

// diag(A): the row's coefficients summed in the row's order; 1 for an empty row
template <int ND>
__global__ void __launch_bounds__(GB, GP_SM) k_diag(Geom g, GravP P, double *diag)
{
    for_cells<ND>(g, [&](int64_t i, const int64_t cc[3]) {
        double s = 0.0;
#pragma unroll
        for (int d = ND - 1; d >= 0; --d) {
            const int64_t nb = gnb(g, P, i, cc[d], d, false);
            if (nb >= 0 && nb < i) s = s + P.coef[d];
        }
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const int64_t nb = gnb(g, P, i, cc[d], d, true);
            if (nb < 0) continue;
            s = s + P.coef[d];
            if (nb == i) s = s + P.coef[d];
        }
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const int64_t nb = gnb(g, P, i, cc[d], d, false);
            if (nb > i) s = s + P.coef[d];
        }
        diag[i] = s == 0.0 ? 1.0 : s;
    });
}

// one damped-Jacobi sweep on A (_matvec! then _csr_jacobi!, mg_pcg.jl:148-150):
// xout = x + omega (rhs - A x) / diag, xin == nullptr standing for x = 0; one
// thread per cell of the periodic cube
__global__ void __launch_bounds__(GB) k_ajac_cube(int n, GravP P, const double *__restrict__ xin,
                                                 const double *__restrict__ rhs,
                                                 const double *__restrict__ diag,
                                                 double *__restrict__ xout, const GravCtrl *gc)
{
    if (gc->done) return;
    const int i = blockIdx.x * GB + threadIdx.x;
    if (i >= n * n * n) return;
    const double ax = xin ? lap_cube(n, P, xin, i) : 0.0;
    const double xv = xin ? xin[i] : 0.0;
    xout[i] = xv + MG_OMEGA * (rhs[i] - ax) / diag[i];
}

// mr = rhs - A x, and the base-grid right-hand side (0 + mr: the scatter onto
// a zeroed base grid, one base cell per cell on a uniform mesh), whose
// correction e starts at zero; one thread per cell of the periodic cube
__global__ void __launch_bounds__(GB) k_aresid_cube(int n, GravP P, const double *__restrict__ x,
                                                   const double *__restrict__ rhs,
                                                   double *__restrict__ mr, double *__restrict__ tb,
                                                   double *__restrict__ te, const GravCtrl *gc)
{
    if (gc->done) return;
    const int i = blockIdx.x * GB + threadIdx.x;
    if (i >= n * n * n) return;
    const double m = rhs[i] - lap_cube(n, P, x, i);
    mr[i] = m;
    tb[i] = 0.0 + m;
    te[i] = 0.0;
}

__device__ __forceinline__ int mg_wrap(int a, int n) { return a < 0 ? n - 1 : (a >= n ? 0 : a); }

// _mgk_jacobi! (mg_pcg.jl:21-31): phi = (1 - w) phiold + w (sum_nb + h^2 b) / 6
// for cell i of the periodic n^3 level
__device__ __forceinline__ double mg_jacobi_cell(int n, int i, double h2, const double *phiold,
                                                 const double *__restrict__ b)
{
    int c[3];
    cube_coords(n, i, c);
    const int x = c[0], y = c[1], z = c[2];
    const int nn = n * n;
    const double s = phiold[i - x + mg_wrap(x - 1, n)] + phiold[i - x + mg_wrap(x + 1, n)] +
                     phiold[i - y * n + mg_wrap(y - 1, n) * n] + phiold[i - y * n + mg_wrap(y + 1, n) * n] +
                     phiold[i - z * nn + mg_wrap(z - 1, n) * nn] + phiold[i - z * nn + mg_wrap(z + 1, n) * nn];
    return (1.0 - MG_OMEGA) * phiold[i] + MG_OMEGA * (s + h2 * b[i]) / 6.0;
}

__global__ void __launch_bounds__(GB, GP_SM) k_mg_jacobi(int n, double h2, const double *__restrict__ phiold,
                                                 const double *__restrict__ b, double *phi,
                                                 const GravCtrl *gc)
{
    if (gc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * n * n) return;
    phi[i] = mg_jacobi_cell(n, i, h2, phiold, b);
}

// `sweeps` (even) Jacobi sweeps of a small level in one block, alternating
// e -> t -> e, with a block barrier between sweeps: the same values as
// `sweeps` launches of k_mg_jacobi
__global__ void __launch_bounds__(GB, GP_SM) k_mg_jacobi_block(int n, double h2, int sweeps, double *e,
                                                       const double *__restrict__ b, double *t,
                                                       const GravCtrl *gc)
{
    if (gc->done) return;
    const int nc = n * n * n;
    for (int k = 0; k < sweeps; ++k) {
        const double *src = (k & 1) ? t : e;
        double *dst = (k & 1) ? e : t;
        for (int i = threadIdx.x; i < nc; i += GB) dst[i] = mg_jacobi_cell(n, i, h2, src, b);
        __syncthreads();
    }
}

// _mgk_residual! (33-43): r = b - (6 phi - sum_nb) / h^2
__global__ void __launch_bounds__(GB, GP_SM) k_mg_residual(int n, double invh2, const double *__restrict__ phi,
                                                   const double *__restrict__ b, double *r,
                                                   const GravCtrl *gc)
{
    if (gc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * n * n) return;
    int c[3];
    cube_coords(n, i, c);
    const int x = c[0], y = c[1], z = c[2];
    const int nn = n * n;
    const double s = phi[i - x + mg_wrap(x - 1, n)] + phi[i - x + mg_wrap(x + 1, n)] +
                     phi[i - y * n + mg_wrap(y - 1, n) * n] + phi[i - y * n + mg_wrap(y + 1, n) * n] +
                     phi[i - z * nn + mg_wrap(z - 1, n) * nn] + phi[i - z * nn + mg_wrap(z + 1, n) * nn];
    r[i] = b[i] - (6.0 * phi[i] - s) * invh2;
}

// _mgk_restrict! (45-53): coarse = mean of the 8 fine children; coarse e = 0
__global__ void __launch_bounds__(GB, GP_SM) k_mg_restrict(int nc, const double *__restrict__ rf, double *bc,
                                                   double *ec, const GravCtrl *gc)
{
    if (gc->done) return;
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= nc * nc * nc) return;
    int C[3];
    cube_coords(nc, I, C);
    const int n = 2 * nc, x = 2 * C[0], y = 2 * C[1], z = 2 * C[2];
    auto f = [&](int a, int b_, int c) { return rf[a + n * (b_ + n * c)]; };
    bc[I] = 0.125 * (f(x, y, z) + f(x + 1, y, z) + f(x, y + 1, z) + f(x + 1, y + 1, z) + f(x, y, z + 1) +
                     f(x + 1, y, z + 1) + f(x, y + 1, z + 1) + f(x + 1, y + 1, z + 1));
    ec[I] = 0.0;
}

// _mgk_prolong_add! (55-66): trilinear cell-centred prolongation (weights 3/4,
// 1/4, periodic) added into the fine level
__global__ void __launch_bounds__(GB, GP_SM) k_mg_prolong_add(int nc, const double *__restrict__ phic,
                                                      double *phif, const GravCtrl *gc)
{
    if (gc->done) return;
    const int n = 2 * nc;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * n * n) return;
    int c[3];
    cube_coords(n, i, c);
    const int x = c[0], y = c[1], z = c[2];
    const int ic[2] = {x / 2, mg_wrap(x / 2 + ((x & 1) ? 1 : -1), nc)};
    const int jc[2] = {y / 2, mg_wrap(y / 2 + ((y & 1) ? 1 : -1), nc)};
    const int kc[2] = {z / 2, mg_wrap(z / 2 + ((z & 1) ? 1 : -1), nc)};
    const double w[2] = {0.75, 0.25};
    double v = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < 2; ++c)
                v = v + w[a] * w[b] * w[c] * phic[ic[a] + nc * (jc[b] + nc * kc[c])];
    phif[i] = phif[i] + v;
}

// partials of sum(e) over the base grid (the correction's mean)
__global__ void __launch_bounds__(GB, GP_SM) k_sumpart(int64_t n, const double *__restrict__ e, double *part,
                                               const GravCtrl *gc)
{
    __shared__ double sh[GB];
    if (gc->done) return;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < n; i += (int64_t)GP * GB) s = s + e[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(1024) k_sum_final(const double *part, int64_t n, GravCtrl *gc)
{
    __shared__ double sh[1024];
    if (gc->done) return;
    const double s = final_sum(part, sh);
    if (threadIdx.x == 0) gc->mgmu = s / (double)n;
}

// z += (e - mean) / Vbase + 0 * mr / diag  (_mgk_gather! with gamma = 0, then x .+= mc)
__global__ void __launch_bounds__(GB, GP_SM) k_mg_gather_add(int64_t n, const double *__restrict__ e,
                                                     const double *__restrict__ mr,
                                                     const double *__restrict__ diag, double Vbase,
                                                     double *z, const GravCtrl *gc)
{
    if (gc->done) return;
    const double mu = gc->mgmu;
    for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < n; i += (int64_t)GP * GB) {
        const double mc = (e[i] - mu) / Vbase + 0.0 * mr[i] / diag[i];
        z[i] = z[i] + mc;
    }
}

// PCG start after z = M^-1 r: p = z; partials of r.z
__global__ void __launch_bounds__(GB, GP_SM) k_pcg_start(Geom g, const double *__restrict__ r,
                                                 const double *__restrict__ z, double *p, double *part)
{
    __shared__ double sh[GB];
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < g.ncell; i += (int64_t)GP * GB) {
        p[i] = z[i];
        s = s + r[i] * z[i];
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// rz of the start (r.z): held in rsold, as the reference's rz
__global__ void __launch_bounds__(1024) k_pcg_start_final(const double *part, GravCtrl *gc)
{
    __shared__ double sh[1024];
    const double rz = final_sum(part, sh);
    if (threadIdx.x == 0) gc->rsold = rz;
}

// relres from r.r; stop at tol (mg_pcg.jl:202-203)
__global__ void __launch_bounds__(1024) k_pcg_check(const double *part, GravCtrl *gc)
{
    __shared__ double sh[1024];
    if (gc->done) return;
    const double rr = final_sum(part, sh);
    if (threadIdx.x == 0) {
        gc->relres = sqrt(rr) / gc->bnorm;
        if (gc->relres <= gc->tol) gc->done = 1;
    }
}

// partials of r.z (after the preconditioner)
__global__ void __launch_bounds__(GB, GP_SM) k_pcg_rz(Geom g, const double *__restrict__ r,
                                              const double *__restrict__ z, double *part,
                                              const GravCtrl *gc)
{
    __shared__ double sh[GB];
    if (gc->done) return;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * GB + threadIdx.x; i < g.ncell; i += (int64_t)GP * GB)
        s = s + r[i] * z[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// beta = rznew / rz; rz = rznew; stop after maxiter
__global__ void __launch_bounds__(1024) k_pcg_beta(const double *part, GravCtrl *gc)
{
    __shared__ double sh[1024];
    if (gc->done) return;
    const double rz = final_sum(part, sh);
    if (threadIdx.x == 0) {
        gc->beta = rz / gc->rsold;
        gc->rsold = rz;
        if (gc->iters >= gc->maxiter) gc->done = 1;
    }
}

}  // namespace
}  // namespace vb

using vb::detail::fail;
using vb::detail::use;

struct vb_gravity {
    vb::GravP P{};
    double *phi = nullptr, *b = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr;
    double *gacc = nullptr, *part = nullptr;
    // periodic cube (n^3, n <= 1024, phi periodic on every side): the
    // one-thread-per-cell matvec and its per-block partials
    int cube_n = 0;
    double *cpart = nullptr;
    vb::GravCtrl *gc = nullptr;   // device
    vb::GravCtrl *hgc = nullptr;  // pinned host mirror
    cudaGraphExec_t gexec = nullptr;
    int64_t maxiter = 500;
    double tol = 1e-8;
    // multigrid preconditioner (precond = VB_GRAV_PRECOND_MG)
    int precond = VB_GRAV_PRECOND_NONE;
    double *z = nullptr, *z2 = nullptr, *mr = nullptr, *diag = nullptr;
    struct Level {
        int n;
        double h;
        double *e, *b, *r, *t;
    };
    std::vector<Level> lev;  // base grid first, then each coarsening
    double hbase = 0.0, vbase = 0.0;
    int64_t graph_launches = 0;  // kernels per replay of the iteration graph
};

namespace {

// launch kern<ND> on the grid-stride grid; evaluates to 1 (one launch)
#define ND_DISPATCH(nd, kern, ...)                                        \
    ((nd) == 1   ? (kern<1><<<vb::GP, vb::GB, 0, s>>>(__VA_ARGS__), 1)   \
     : (nd) == 2 ? (kern<2><<<vb::GP, vb::GB, 0, s>>>(__VA_ARGS__), 1)   \
                 : (kern<3><<<vb::GP, vb::GB, 0, s>>>(__VA_ARGS__), 1))

// One CG iteration (five launches; each returns at once after convergence).
inline unsigned mg_blocks(int64_t n) { return (unsigned)((n + vb::GB - 1) / vb::GB); }

// Ap = A p and the GP partials of p.Ap; evaluates to the launch count
int queue_matvec(vb_grid *gr, vb_gravity *gv)
{
    cudaStream_t s = gr->ctx->stream;
    const vb::Geom &g = gr->g;
    if (gv->cube_n) {
        const int n = gv->cube_n;
        const unsigned nb = mg_blocks((int64_t)n * n * n);
        vb::k_cg_matvec_cube<<<nb, vb::GB, 0, s>>>(n, gv->P, gv->p, gv->Ap, gv->cpart, gv->gc);
        vb::k_fold_parts<<<vb::GP, vb::GB, 0, s>>>(gv->cpart, (int)nb, gv->part, gv->gc);
        return 2;
    }
    return ND_DISPATCH(g.nd, vb::k_cg_matvec, g, gv->P, gv->p, gv->Ap, gv->part, gv->gc);
}

int queue_iteration(vb_grid *gr, vb_gravity *gv)
{
    cudaStream_t s = gr->ctx->stream;
    const vb::Geom &g = gr->g;
    VB_CHECK_LAUNCH(gr->ctx, queue_matvec(gr, gv));
    vb::k_cg_alpha<<<1, 1024, 0, s>>>(gv->part, gv->gc);
    VB_CHECK_LAUNCH(gr->ctx, 1);
    vb::k_cg_update<<<vb::GP, vb::GB, 0, s>>>(g, gv->phi, gv->p, gv->r, gv->Ap, gv->part, gv->gc);
    VB_CHECK_LAUNCH(gr->ctx, 1);
    vb::k_cg_beta<<<1, 1024, 0, s>>>(gv->part, gv->gc);
    VB_CHECK_LAUNCH(gr->ctx, 1);
    vb::k_cg_dir<<<vb::GP, vb::GB, 0, s>>>(g, gv->p, gv->r, gv->gc);
    VB_CHECK_LAUNCH(gr->ctx, 1);
    return VB_OK;
}

// z = M^-1 r (one composite-smoothed two-level cycle)
int queue_precond(vb_grid *gr, vb_gravity *gv)
{
    cudaStream_t s = gr->ctx->stream;
    const vb::Geom &g = gr->g;
    const vb::GravP &P = gv->P;
    // the preconditioner runs on periodic cubes only: one thread per cell
    const int n = (int)g.n[0];
    const unsigned nb = mg_blocks((int64_t)n * n * n);
    auto ajac = [&](const double *xin, double *xout) {
        vb::k_ajac_cube<<<nb, vb::GB, 0, s>>>(n, P, xin, gv->r, gv->diag, xout, gv->gc);
        return 1;
    };
    VB_CHECK_LAUNCH(gr->ctx, ajac(nullptr, gv->z2));  // pre-smooth from z = 0
    VB_CHECK_LAUNCH(gr->ctx, ajac(gv->z2, gv->z));
    auto &top = gv->lev[0];
    vb::k_aresid_cube<<<nb, vb::GB, 0, s>>>(n, P, gv->z, gv->r, gv->mr, top.b, top.e, gv->gc);
    VB_CHECK_LAUNCH(gr->ctx, 1);
    // V-cycle: down the levels, then back up
    const int L = (int)gv->lev.size();
    auto jacobi = [&](const vb_gravity::Level &l, int sweeps) {
        const double h2 = l.h * l.h;
        const unsigned nb = mg_blocks((int64_t)l.n * l.n * l.n);
        for (int k = 0; k < sweeps; k += 2) {  // even counts end in e
            vb::k_mg_jacobi<<<nb, vb::GB, 0, s>>>(l.n, h2, l.e, l.b, l.t, gv->gc);
            vb::k_mg_jacobi<<<nb, vb::GB, 0, s>>>(l.n, h2, l.t, l.b, l.e, gv->gc);
        }
        return sweeps;
    };
    for (int k = 0; k + 1 < L; ++k) {
        const auto &l = gv->lev[k], &c = gv->lev[k + 1];
        VB_CHECK_LAUNCH(gr->ctx, jacobi(l, 2));
        vb::k_mg_residual<<<mg_blocks((int64_t)l.n * l.n * l.n), vb::GB, 0, s>>>(
            l.n, 1.0 / (l.h * l.h), l.e, l.b, l.r, gv->gc);
        vb::k_mg_restrict<<<mg_blocks((int64_t)c.n * c.n * c.n), vb::GB, 0, s>>>(c.n, l.r, c.b, c.e, gv->gc);
        VB_CHECK_LAUNCH(gr->ctx, 2);
    }
    {  // coarsest: 2 pre + 30 sweeps, in one block when the level is small
        const auto &l = gv->lev[L - 1];
        if ((int64_t)l.n * l.n * l.n <= 16 * vb::GB) {
            vb::k_mg_jacobi_block<<<1, vb::GB, 0, s>>>(l.n, l.h * l.h, 32, l.e, l.b, l.t, gv->gc);
            VB_CHECK_LAUNCH(gr->ctx, 1);
        } else {
            VB_CHECK_LAUNCH(gr->ctx, jacobi(l, 32));
        }
    }
    for (int k = L - 2; k >= 0; --k) {
        const auto &l = gv->lev[k], &c = gv->lev[k + 1];
        vb::k_mg_prolong_add<<<mg_blocks((int64_t)l.n * l.n * l.n), vb::GB, 0, s>>>(c.n, c.e, l.e, gv->gc);
        VB_CHECK_LAUNCH(gr->ctx, 1);
        VB_CHECK_LAUNCH(gr->ctx, jacobi(l, 2));
    }
    const int64_t nt = (int64_t)top.n * top.n * top.n;
    vb::k_sumpart<<<vb::GP, vb::GB, 0, s>>>(nt, top.e, gv->part + 2 * vb::GP, gv->gc);
    vb::k_sum_final<<<1, 1024, 0, s>>>(gv->part + 2 * vb::GP, nt, gv->gc);
    vb::k_mg_gather_add<<<vb::GP, vb::GB, 0, s>>>(nt, top.e, gv->mr, gv->diag, gv->vbase, gv->z, gv->gc);
    VB_CHECK_LAUNCH(gr->ctx, 3);
    VB_CHECK_LAUNCH(gr->ctx, ajac(gv->z, gv->z2));  // post-smooth
    VB_CHECK_LAUNCH(gr->ctx, ajac(gv->z2, gv->z));
    return VB_OK;
}

// One preconditioned CG iteration (mg_pcg.jl:194-209).
int queue_pcg_iteration(vb_grid *gr, vb_gravity *gv)
{
    cudaStream_t s = gr->ctx->stream;
    const vb::Geom &g = gr->g;
    VB_CHECK_LAUNCH(gr->ctx, queue_matvec(gr, gv));
    vb::k_cg_alpha<<<1, 1024, 0, s>>>(gv->part, gv->gc);
    vb::k_cg_update<<<vb::GP, vb::GB, 0, s>>>(g, gv->phi, gv->p, gv->r, gv->Ap, gv->part, gv->gc);
    vb::k_pcg_check<<<1, 1024, 0, s>>>(gv->part, gv->gc);
    VB_CHECK_LAUNCH(gr->ctx, 4);
    int rc = queue_precond(gr, gv);
    if (rc) return rc;
    vb::k_pcg_rz<<<vb::GP, vb::GB, 0, s>>>(g, gv->r, gv->z, gv->part, gv->gc);
    vb::k_pcg_beta<<<1, 1024, 0, s>>>(gv->part, gv->gc);
    vb::k_cg_dir<<<vb::GP, vb::GB, 0, s>>>(g, gv->p, gv->z, gv->gc);  // p = z + beta p
    VB_CHECK_LAUNCH(gr->ctx, 3);
    return VB_OK;
}

int capture_iterations(vb_grid *gr, vb_gravity *gv)
{
    cudaStream_t s = gr->ctx->stream;
    VB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int64_t before = gr->ctx->launches;
    int rc = VB_OK;
    gv->graph_launches = 0;
    for (int k = 0; k < vb::GRAPH_ITERS && !rc; ++k)
        rc = gv->precond == VB_GRAV_PRECOND_MG ? queue_pcg_iteration(gr, gv) : queue_iteration(gr, gv);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    gv->graph_launches = gr->ctx->launches - before;
    gr->ctx->launches = before;  // counted per replay
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(VB_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&gv->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        gv->gexec = nullptr;
        return fail(VB_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    return VB_OK;
}

int refresh_accel(vb_grid *gr, vb_gravity *gv)
{
    cudaStream_t s = gr->ctx->stream;
    const vb::Geom &g = gr->g;
    VB_CHECK_LAUNCH(gr->ctx, ND_DISPATCH(g.nd, vb::k_accel, g, gv->P, gv->phi, gv->gacc));
    return VB_OK;
}

void free_gravity(vb_gravity *gv)
{
    if (!gv) return;
    if (gv->gexec) cudaGraphExecDestroy(gv->gexec);
    cudaFree(gv->phi);
    cudaFree(gv->b);
    cudaFree(gv->r);
    cudaFree(gv->p);
    cudaFree(gv->Ap);
    cudaFree(gv->gacc);
    cudaFree(gv->part);
    cudaFree(gv->cpart);
    cudaFree(gv->gc);
    cudaFreeHost(gv->hgc);
    cudaFree(gv->z);
    cudaFree(gv->z2);
    cudaFree(gv->mr);
    cudaFree(gv->diag);
    for (auto &l : gv->lev) {
        cudaFree(l.e);
        cudaFree(l.b);
        cudaFree(l.r);
        cudaFree(l.t);
    }
    delete gv;
}

int check_grid(vb_grid *gr)
{
    if (!gr) return fail(VB_EINVAL, "null grid");
    if (!gr->grav) return fail(VB_EINVAL, "gravity is not enabled on this grid");
    return use(gr->ctx);
}

}  // namespace

// solve_poisson! (src/gravity.jl:251-300) for the grid's current density,
// warm-started from the stored potential; then g = -grad phi for the stages.
int vb::detail::gravity_solve(vb_grid *gr, int64_t *iters, double *relres)
{
    vb_gravity *gv = gr->grav;
    cudaStream_t s = gr->ctx->stream;
    const Geom &g = gr->g;
    gv->hgc->maxiter = gv->maxiter;
    gv->hgc->tol = gv->tol;
    VB_CUDA(cudaMemcpyAsync(&gv->gc->maxiter, &gv->hgc->maxiter, sizeof(long long),
                            cudaMemcpyHostToDevice, s));
    VB_CUDA(cudaMemcpyAsync(&gv->gc->tol, &gv->hgc->tol, sizeof(double), cudaMemcpyHostToDevice, s));
    if (gv->P.project_mean) {
        k_meanpart<<<GP, GB, 0, s>>>(g, gr->U, gv->part);
        VB_CHECK_LAUNCH(gr->ctx, 1);
        k_mean_final<<<1, 1024, 0, s>>>(gv->part, gv->gc, 0);
        VB_CHECK_LAUNCH(gr->ctx, 1);
    }
    k_rhs<<<GP, GB, 0, s>>>(g, gv->P, gr->U, gv->b, gv->gc);
    VB_CHECK_LAUNCH(gr->ctx, 1);
    VB_CHECK_LAUNCH(gr->ctx, ND_DISPATCH(g.nd, k_cg_init, g, gv->P, gv->phi, gv->b, gv->r, gv->p, gv->part));
    k_cg_init_final<<<1, 1024, 0, s>>>(gv->part, gv->gc);
    VB_CHECK_LAUNCH(gr->ctx, 1);
    if (gv->precond == VB_GRAV_PRECOND_MG) {  // z = M^-1 r, p = z, rz (mg_pcg.jl:188-191)
        int rc = queue_precond(gr, gv);
        if (rc) return rc;
        k_pcg_start<<<GP, GB, 0, s>>>(g, gv->r, gv->z, gv->p, gv->part);
        k_pcg_start_final<<<1, 1024, 0, s>>>(gv->part, gv->gc);
        VB_CHECK_LAUNCH(gr->ctx, 2);
    }
    if (!gv->gexec) {
        int rc = capture_iterations(gr, gv);
        if (rc) return rc;
    }
    // the stop flag is set by convergence, p.Ap <= 0 or maxiter, so this ends
    for (;;) {
        VB_CUDA(cudaGraphLaunch(gv->gexec, s));
        gr->ctx->launches += gv->graph_launches;
        VB_CUDA(cudaMemcpyAsync(gv->hgc, gv->gc, sizeof(GravCtrl), cudaMemcpyDeviceToHost, s));
        VB_CUDA(cudaStreamSynchronize(s));
        if (gv->hgc->done) break;
    }
    if (gv->P.project_mean) {
        k_meanpart<<<GP, GB, 0, s>>>(g, gv->phi, gv->part);
        VB_CHECK_LAUNCH(gr->ctx, 1);
        k_mean_final<<<1, 1024, 0, s>>>(gv->part, gv->gc, 1);
        VB_CHECK_LAUNCH(gr->ctx, 1);
        k_sub_mean<<<GP, GB, 0, s>>>(g, gv->phi, gv->gc);
        VB_CHECK_LAUNCH(gr->ctx, 1);
    }
    int rc = refresh_accel(gr, gv);
    if (rc) return rc;
    if (iters) *iters = gv->hgc->iters;
    if (relres) *relres = gv->hgc->relres;
    return VB_OK;
}

void vb::detail::gravity_free(vb_gravity *gv) { free_gravity(gv); }

extern "C" {

int vb_gravity_enable(vb_grid *gr, const vb_gravity_desc *d)
{
    if (!gr || !d) return fail(VB_EINVAL, "null argument");
    if (d->flags != 0) return fail(VB_EINVAL, "flags must be 0");
    if (!(d->tol >= 0.0) || d->maxiter < 0) return fail(VB_EINVAL, "tol and maxiter must be non-negative");
    if (!std::isfinite(d->G)) return fail(VB_EINVAL, "G must be finite");
    int rc = use(gr->ctx);
    if (rc) return rc;
    const vb::Geom &g = gr->g;
    vb::GravP P{};
    for (int a = 0; a < 3; ++a) {
        if (a < g.nd) {
            for (int side = 0; side < 2; ++side) {
                const int bc = side ? d->bc_hi[a] : d->bc_lo[a];
                if (bc < VB_BC_OUTFLOW || bc > VB_BC_REFLECTING)
                    return fail(VB_EINVAL, "unknown boundary condition");
            }
            if ((d->bc_lo[a] == VB_BC_PERIODIC) != (d->bc_hi[a] == VB_BC_PERIODIC))
                return fail(VB_EINVAL, "a periodic axis must be periodic on both sides");
            P.per_lo[a] = d->bc_lo[a] == VB_BC_PERIODIC;
            P.per_hi[a] = d->bc_hi[a] == VB_BC_PERIODIC;
            P.coef[a] = g.area[a] / (0.5 * (g.w[a] + g.w[a]));  // area / _face_distance
        } else {
            P.per_lo[a] = P.per_hi[a] = 1;
            P.coef[a] = 0.0;
        }
    }
    P.G = d->G;
    P.project_mean = d->project_mean ? 1 : 0;
    if (d->precond != VB_GRAV_PRECOND_NONE && d->precond != VB_GRAV_PRECOND_MG)
        return fail(VB_EINVAL, "unknown preconditioner");
    if (d->precond == VB_GRAV_PRECOND_MG) {
        // the base-grid V-cycle is periodic and cubic (mg_pcg.jl:88-89)
        bool ok = g.nd == 3 && g.n[0] == g.n[1] && g.n[1] == g.n[2] && g.n[0] <= 1024;
        for (int a = 0; a < 3; ++a) ok = ok && P.per_lo[a] && P.per_hi[a];
        if (!ok)
            return fail(VB_ENOTSUP, "the multigrid preconditioner needs a 3D cubic grid (n <= 1024) "
                                    "with periodic phi on every side");
    }
    vb_gravity *gv = gr->grav;
    if (!gv) {
        gv = new vb_gravity;
        const size_t n = (size_t)g.ncell * sizeof(double);
        cudaError_t e = cudaSuccess;
        for (double **buf : {&gv->phi, &gv->b, &gv->r, &gv->p, &gv->Ap})
            if (e == cudaSuccess) e = cudaMalloc(buf, n);
        if (e == cudaSuccess) e = cudaMalloc(&gv->gacc, n * g.nd);
        if (e == cudaSuccess) e = cudaMalloc(&gv->part, sizeof(double) * 3 * vb::GP);
        if (e == cudaSuccess) e = cudaMalloc(&gv->gc, sizeof(vb::GravCtrl));
        if (e == cudaSuccess) e = cudaMallocHost(&gv->hgc, sizeof(vb::GravCtrl));
        if (e == cudaSuccess) e = cudaMemsetAsync(gv->phi, 0, n, gr->ctx->stream);  // phi starts at 0
        if (e == cudaSuccess) e = cudaMemsetAsync(gv->gacc, 0, n * g.nd, gr->ctx->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(gv->gc, 0, sizeof(vb::GravCtrl), gr->ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(gr->ctx->stream);
        if (e != cudaSuccess) {
            free_gravity(gv);
            return fail(e == cudaErrorMemoryAllocation ? VB_ENOMEM : VB_ECUDA,
                        std::string("gravity allocation: ") + cudaGetErrorString(e));
        }
        std::memset(gv->hgc, 0, sizeof(vb::GravCtrl));
    }
    gv->P = P;
    {
        bool cube = g.nd == 3 && g.n[0] == g.n[1] && g.n[1] == g.n[2] && g.n[0] <= 1024;
        for (int a = 0; a < 3; ++a) cube = cube && P.per_lo[a] && P.per_hi[a];
        gv->cube_n = cube ? (int)g.n[0] : 0;
        if (cube && !gv->cpart) {
            const cudaError_t e = cudaMalloc(&gv->cpart, sizeof(double) * mg_blocks(g.ncell));
            if (e != cudaSuccess) {
                gv->cube_n = 0;
                if (!gr->grav) free_gravity(gv);
                return fail(e == cudaErrorMemoryAllocation ? VB_ENOMEM : VB_ECUDA,
                            std::string("gravity allocation: ") + cudaGetErrorString(e));
            }
        }
    }
    gv->maxiter = d->maxiter;
    gv->tol = d->tol;
    gr->grav = gv;
    if (gv->gexec) {  // the iteration graph depends on the preconditioner
        cudaGraphExecDestroy(gv->gexec);
        gv->gexec = nullptr;
    }
    gv->precond = d->precond;
    if (gv->precond == VB_GRAV_PRECOND_MG && !gv->z) {
        // levels: coarsen while even and > 4 (mg_pcg.jl:111-116)
        const size_t n = (size_t)g.ncell * sizeof(double);
        cudaError_t e = cudaSuccess;
        for (double **buf : {&gv->z, &gv->z2, &gv->mr, &gv->diag})
            if (e == cudaSuccess) e = cudaMalloc(buf, n);
        gv->hbase = g.w[0];
        gv->vbase = gv->hbase * gv->hbase * gv->hbase;
        int nl = (int)g.n[0];
        double h = gv->hbase;
        for (;;) {
            vb_gravity::Level l{nl, h, nullptr, nullptr, nullptr, nullptr};
            const size_t bytes = sizeof(double) * (size_t)nl * nl * nl;
            for (double **buf : {&l.e, &l.b, &l.r, &l.t})
                if (e == cudaSuccess) e = cudaMalloc(buf, bytes);
            gv->lev.push_back(l);
            if (!(nl > 4 && nl % 2 == 0)) break;
            nl /= 2;
            h *= 2.0;
        }
        if (e == cudaSuccess) {
            cudaStream_t s = gr->ctx->stream;
            vb::k_diag<3><<<vb::GP, vb::GB, 0, s>>>(g, P, gv->diag);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        }
        if (e != cudaSuccess) {
            gr->grav = nullptr;
            free_gravity(gv);
            return fail(e == cudaErrorMemoryAllocation ? VB_ENOMEM : VB_ECUDA,
                        std::string("multigrid allocation: ") + cudaGetErrorString(e));
        }
    }
    gr->g.grav_g = gv->gacc;
    gr->g.grav_G = d->G;
    gr->box_kz = -1;          // the tiled kernels' box descriptor carries the geometry
    gr->invdt_valid = false;  // the free-fall limiter joins the CFL maximum
    return VB_OK;
}

int vb_gravity_disable(vb_grid *gr)
{
    if (!gr) return fail(VB_EINVAL, "null grid");
    if (!gr->grav) return VB_OK;
    int rc = use(gr->ctx);
    if (rc) return rc;
    cudaStreamSynchronize(gr->ctx->stream);
    free_gravity(gr->grav);
    gr->grav = nullptr;
    gr->g.grav_g = nullptr;
    gr->g.grav_G = 0.0;
    gr->box_kz = -1;
    gr->invdt_valid = false;
    return VB_OK;
}

int vb_gravity_solve(vb_grid *gr, int64_t *iters, double *relres)
{
    VB_RANGE("vb_gravity_solve");
    int rc = check_grid(gr);
    if (rc) return rc;
    return vb::detail::gravity_solve(gr, iters, relres);
}

int vb_gravity_phi(vb_grid *gr, double *phi)
{
    int rc = check_grid(gr);
    if (rc) return rc;
    if (!phi) return fail(VB_EINVAL, "null output");
    VB_CUDA(cudaMemcpyAsync(phi, gr->grav->phi, sizeof(double) * gr->g.ncell, cudaMemcpyDeviceToHost,
                            gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    return VB_OK;
}

int vb_gravity_set_phi(vb_grid *gr, const double *phi)
{
    int rc = check_grid(gr);
    if (rc) return rc;
    if (!phi) return fail(VB_EINVAL, "null input");
    VB_CUDA(cudaMemcpyAsync(gr->grav->phi, phi, sizeof(double) * gr->g.ncell, cudaMemcpyHostToDevice,
                            gr->ctx->stream));
    rc = refresh_accel(gr, gr->grav);
    if (rc) return rc;
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    return VB_OK;
}

int vb_gravity_accel(vb_grid *gr, double *gout)
{
    int rc = check_grid(gr);
    if (rc) return rc;
    if (!gout) return fail(VB_EINVAL, "null output");
    VB_CUDA(cudaMemcpyAsync(gout, gr->grav->gacc, sizeof(double) * gr->g.ncell * gr->g.nd,
                            cudaMemcpyDeviceToHost, gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    return VB_OK;
}

int vb_gravity_laplacian(vb_grid *gr, const double *x, double *Ax)
{
    VB_RANGE("vb_gravity_laplacian");
    int rc = check_grid(gr);
    if (rc) return rc;
    if (!x || !Ax) return fail(VB_EINVAL, "null argument");
    vb_gravity *gv = gr->grav;
    cudaStream_t s = gr->ctx->stream;
    const size_t n = sizeof(double) * gr->g.ncell;
    // the CG scratch r (input) and Ap (output) are free between solves
    VB_CUDA(cudaMemcpyAsync(gv->r, x, n, cudaMemcpyHostToDevice, s));
    VB_CHECK_LAUNCH(gr->ctx, ND_DISPATCH(gr->g.nd, vb::k_lap, gr->g, gv->P, gv->r, gv->Ap));
    VB_CUDA(cudaMemcpyAsync(Ax, gv->Ap, n, cudaMemcpyDeviceToHost, s));
    VB_CUDA(cudaStreamSynchronize(s));
    return VB_OK;
}

}  // extern "C"
