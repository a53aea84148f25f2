// vb_muscl.cu -- lib/PPMKernels' unsplit MUSCL step (muscl_step_3d!,
// lib/PPMKernels/src/muscl_grid.jl:314-380; Enzo HydroMethod=3): PLM with the
// minmod-theta limiter on (rho, eint, v), the HLL Riemann flux, SSP-RK2, on
// five conserved arrays (D, S1, S2, S3, Tau = rho * specific total energy)
// with ng ghost zones per side.  The second scheme behind the library, beside
// the hydro step of the main path.
//
// The reference sweeps the three axes over transposed slabs and adds each
// axis's flux divergence into one zeroed dU.  Here a CTA owns a 32 x 8 column
// of cells (ghost cells included) and marches it along z.  The primitives of
// five z-planes (the current one, its two stencil neighbours each side)
// sit in a shared-memory ring with a two-cell x/y halo, filled by cp.async one
// plane ahead.  Each plane, every interface flux the tile needs is evaluated
// once: the x and y faces into shared memory, the z face in registers, where
// it becomes the next plane's lower z face.  Each cell then sums
// dU = ((0 + du_x) + du_y) + du_z exactly as the reference's accumulation
// reaches it (x in place; y and z through zero-filled slabs added over the
// whole grid).  A flux depends only on its four stencil cells, so evaluating
// it once instead of twice changes no bit.  Compiled with -fmad=false:
// bit-identical to the oracle's restatement.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "vb_internal.h"
#include "vb_tma.cuh"

namespace vb {
namespace {

constexpr int MB = 256;

struct MusclFields {
    double *f[5];  // D, S1, S2, S3, Tau
};

struct MusclGeom {
    int64_t n[3], stride[3], N;
    int ng;
    double gamma, theta, dtdx, small_rho;
};

// Julia's Base.min / max for floats: NaN propagates, the sign of x - y decides
__device__ __forceinline__ double jmin(double x, double y)
{
    const double d = x - y;
    if (isnan(x) || isnan(y)) return d;
    return signbit(d) ? x : y;
}
__device__ __forceinline__ double jmax(double x, double y)
{
    const double d = x - y;
    if (isnan(x) || isnan(y)) return d;
    return signbit(d) ? y : x;
}

// _msign / _minmod3 / _plm_pt, muscl.jl:13-26 (Enzo's sign(0) = -1; NaN -> -1)
// 0.25 (sa + sb) |sa + sc| with signs sa, sb, sc = +-1 (sign(x) = x > 0 ? 1 :
// -1) is exactly +-1 when the three signs agree, a zero carrying sa's sign
// when sa = sb != sc, and +0 when sa != sb; multiplying that factor by the
// smallest magnitude rounds exactly as the reference's product does.
__device__ __forceinline__ double minmod3(double a, double b, double c)
{
    const bool pa = a > 0.0, pb = b > 0.0, pc = c > 0.0;
    const double f = pa != pb ? 0.0 : pa != pc ? (pa ? 0.0 : -0.0) : (pa ? 1.0 : -1.0);
    return f * jmin(fabs(a), jmin(fabs(b), fabs(c)));
}
__device__ __forceinline__ double plm_pt(double vm1, double v, double vp1, double th)
{
    return v + 0.5 * minmod3((v - vm1) * th, (vp1 - v) * th, 0.5 * (vp1 - vm1));
}

// _hll, muscl.jl:29-30
__device__ __forceinline__ double hll1(double ap, double am, double fl, double fr, double ul, double ur)
{
    return (ap * fl + am * fr - ap * am * (ur - ul)) / (ap + am);
}

// HLL flux of primitive L/R states (rho, eint, u_normal, v, w): the first five
// components of _hll6 (muscl.jl:57-78; identical to _hll5)
__device__ __forceinline__ void hll5(const double L[5], const double R[5], double g, double gm1,
                                     double F[5])
{
    const double h = 0.5;
    const double rl = L[0], el = L[1], ul = L[2], vl = L[3], wl = L[4];
    const double rr = R[0], er = R[1], ur = R[2], vr = R[3], wr = R[4];
    const double v2l = ul * ul + vl * vl + wl * wl, pl = gm1 * rl * el, csl = sqrt(g * pl / rl);
    const double etl = el + h * v2l;
    const double UlS1 = rl * ul, UlS2 = rl * vl, UlS3 = rl * wl, UlE = rl * etl;
    const double FlD = rl * ul, FlS1 = UlS1 * ul + pl, FlS2 = UlS2 * ul, FlS3 = UlS3 * ul;
    const double FlE = (UlE + pl) * ul;
    const double lpl = ul + csl, lml = ul - csl;
    const double v2r = ur * ur + vr * vr + wr * wr, pr = gm1 * rr * er, csr = sqrt(g * pr / rr);
    const double etr = er + h * v2r;
    const double UrS1 = rr * ur, UrS2 = rr * vr, UrS3 = rr * wr, UrE = rr * etr;
    const double FrD = rr * ur, FrS1 = UrS1 * ur + pr, FrS2 = UrS2 * ur, FrS3 = UrS3 * ur;
    const double FrE = (UrE + pr) * ur;
    const double lpr = ur + csr, lmr = ur - csr;
    const double ap = jmax(0.0, jmax(lpl, lpr)), am = jmax(0.0, jmax(-lml, -lmr));
    F[0] = hll1(ap, am, FlD, FrD, rl, rr);
    F[1] = hll1(ap, am, FlS1, FrS1, UlS1, UrS1);
    F[2] = hll1(ap, am, FlS2, FrS2, UlS2, UrS2);
    F[3] = hll1(ap, am, FlS3, FrS3, UlS3, UrS3);
    F[4] = hll1(ap, am, FlE, FrE, UlE, UrE);
}

// Per stage, before the tile pass, one pass over every cell (block 32 x 8,
// grid z = planes):
//  - COPY: U0 = U (the step-start state, ghosts as they were);
//  - FILL: a ghost takes the value of its periodic image, the cell whose
//    every ghost coordinate p moved by +-active into the active range (what
//    the three axis fills x, y, z in turn leave in it; the image is active,
//    so no thread reads a cell another thread writes);
//  - primitives of the resulting U (_cons2prim_k!, muscl_grid.jl:23-34):
//    prim = (rho, eint, vx, vy, vz), eint floored at small_rho.
template <bool COPY, bool FILL>
__global__ void __launch_bounds__(MB) k_muscl_prep(MusclGeom m, MusclFields U, double *U0, double *prim)
{
    const int64_t c[3] = {(int64_t)blockIdx.x * 32 + threadIdx.x % 32,
                          (int64_t)blockIdx.y * 8 + threadIdx.x / 32, (int64_t)blockIdx.z};
    if (c[0] >= m.n[0] || c[1] >= m.n[1]) return;
    const int64_t N = m.N, i = c[0] + c[1] * m.stride[1] + c[2] * m.stride[2];
    int64_t src = i;
    if constexpr (FILL) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int64_t act = m.n[a] - 2 * m.ng;
            if (c[a] < m.ng) src += act * m.stride[a];
            else if (c[a] >= m.ng + act) src -= act * m.stride[a];
        }
    }
    double u[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) u[f] = U.f[f][src];
    if constexpr (COPY) {
#pragma unroll
        for (int f = 0; f < 5; ++f) U0[f * N + i] = src == i ? u[f] : U.f[f][i];
    }
    if (src != i)
#pragma unroll
        for (int f = 0; f < 5; ++f) U.f[f][i] = u[f];
    const double d = u[0], vx = u[1] / d, vy = u[2] / d, vz = u[3] / d;
    prim[i] = d;
    prim[2 * N + i] = vx;
    prim[3 * N + i] = vy;
    prim[4 * N + i] = vz;
    prim[N + i] = jmax(u[4] / d - 0.5 * (vx * vx + vy * vy + vz * vz), m.small_rho);
}

// Tile of one CTA: TX x TY cells of one z-plane, one thread per cell column.
constexpr int TX = 32, TY = 8, NT = TX * TY;
constexpr int PW = TX + 4, PH = TY + 4;  // plane window: 2-cell halo in x and y
constexpr int PF = PW * PH;              // one primitive field of one plane
constexpr int PS = 5 * PF;               // one ring slot: the five primitive fields
constexpr int NSLOT = 5;                 // planes k-1 .. k+2 in use, k+3 landing
constexpr int FXN = (TX + 1) * TY;       // x faces of one plane tile
constexpr int FYN = TX * (TY + 1);       // y faces of one plane tile
constexpr size_t TILE_SMEM = sizeof(double) * (NSLOT * PS + 5 * FXN + 5 * FYN);

// HLL flux through one interface from the primitives of its four stencil
// cells qm1, q0 | q1, q2 (field f of a cell at offset off[f]), in the
// reference's flux-line form (_muscl_hll_kernel!, muscl.jl:181-215): the left
// state is q0's right face, the right state is q1's left face taken as the
// right face of the reversed stencil.  off[] lists (rho, eint, u_normal, t1,
// t2); F comes back in that frame.
__device__ __forceinline__ void face_flux(const double *qm1, const double *q0, const double *q1,
                                          const double *q2, const int off[5], const MusclGeom &m,
                                          double F[5])
{
    double L[5], R[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        const double a = qm1[off[f]], b = q0[off[f]], c = q1[off[f]], d = q2[off[f]];
        L[f] = plm_pt(a, b, c, m.theta);
        R[f] = plm_pt(d, c, b, m.theta);
    }
    L[0] = jmax(L[0], m.small_rho);
    R[0] = jmax(R[0], m.small_rho);
    hll5(L, R, m.gamma, m.gamma - 1.0, F);
}

// cp.async one primitive plane p (with its halo) into a ring slot; cells
// outside the grid are left unwritten (no face that reads them is evaluated)
__device__ __forceinline__ void load_plane(const MusclGeom &m, const double *__restrict__ prim,
                                           double *slot, int64_t x0, int64_t y0, int64_t p)
{
    if (p < 0 || p >= m.n[2]) return;
    const int64_t nx = m.n[0], ny = m.n[1], N = m.N;
    const double *plane = prim + p * nx * ny;
    // window cell w = r * PW + c, its five fields at w + f * PF
    for (int w = threadIdx.x; w < PF; w += NT) {
        const int r = w / PW, c = w - r * PW;
        const int64_t x = x0 - 2 + c, y = y0 - 2 + r;
        if (x >= 0 && x < nx && y >= 0 && y < ny) {
            const double *src = plane + y * nx + x;
#pragma unroll
            for (int f = 0; f < 5; ++f) cp_async8(slot + f * PF + w, src + f * N);
        }
    }
}

// One RK stage over the cells of one 32 x 8 column, planes [k0, k0 + kz).
// STAGE 1: U = U0 + dU; STAGE 2: U = 0.5 (U0 + U + dU) (muscl_grid.jl:350-367).
template <int STAGE>
__global__ void __launch_bounds__(NT, 2) k_muscl_tile(MusclGeom m, const double *__restrict__ prim,
                                                      MusclFields U, const double *__restrict__ U0,
                                                      int kz)
{
    extern __shared__ __align__(16) double smem[];
    double *const ring = smem, *const fx = smem + NSLOT * PS, *const fy = fx + 5 * FXN;
    const int t = threadIdx.x, tx = t % TX, ty = t / TX;
    const int64_t nx = m.n[0], ny = m.n[1], nz = m.n[2], ng = m.ng, N = m.N;
    const int64_t x0 = (int64_t)blockIdx.x * TX, y0 = (int64_t)blockIdx.y * TY;
    const int64_t k0 = (int64_t)blockIdx.z * kz, k1 = k0 + kz < nz ? k0 + kz : nz;
    const int64_t x = x0 + tx, y = y0 + ty;
    const bool in = x < nx && y < ny;
    const bool act_x = x >= ng && x < nx - ng, act_y = y >= ng && y < ny - ng;
    // a face between cells c and c + 1 along an axis of n cells is needed iff
    // one of the two is active; its stencil c - 1 .. c + 2 is then in the grid
    auto face_ok = [&](int64_t c, int64_t n) { return c >= ng - 1 && c <= n - ng - 1; };
    auto slot = [&](int64_t p) { return ring + ((int)p + NSLOT) % NSLOT * PS; };  // p >= -2
    const int own = (ty + 2) * PW + tx + 2;  // this column's cell in a plane window
    const int zoff[5] = {0, PF, 4 * PF, 2 * PF, 3 * PF};  // rho, eint, vz | vx, vy

    for (int64_t p = k0 - 2; p <= k0 + 2; ++p) load_plane(m, prim, slot(p), x0, y0, p);
    cp_async_commit();
    cp_async_wait_group<0>();
    __syncthreads();
    double flo[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // z flux through this cell's lower face
    if (in && face_ok(k0 - 1, nz))
        face_flux(slot(k0 - 2) + own, slot(k0 - 1) + own, slot(k0) + own, slot(k0 + 1) + own, zoff,
                  m, flo);
    __syncthreads();  // slot of plane k0 - 2 is free
    if (k0 + 3 <= k1 + 1) load_plane(m, prim, slot(k0 + 3), x0, y0, k0 + 3);
    cp_async_commit();

    for (int64_t k = k0; k < k1; ++k) {
        cp_async_wait_group<1>();  // plane k + 2 has landed (k + 3 may be in flight)
        __syncthreads();
        const double *const pk = slot(k);
        double fhi[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (in && face_ok(k, nz))
            face_flux(slot(k - 1) + own, pk + own, slot(k + 1) + own, slot(k + 2) + own, zoff, m,
                      fhi);
        // the plane's x faces (33 per row) and y faces (9 per column), spread
        // over the CTA
        for (int it = t; it < FXN + FYN; it += NT) {
            const double *c0;
            double *out;
            int st, ostr;
            bool ok;
            int off[5] = {0, PF, 2 * PF, 3 * PF, 4 * PF};  // x: vx | vy, vz
            if (it < FXN) {
                const int r = it / (TX + 1), j = it - r * (TX + 1);  // face x0-1+j | x0+j
                ok = face_ok(x0 - 1 + j, nx) && y0 + r < ny;
                c0 = pk + (r + 2) * PW + j + 1;
                st = 1;
                out = fx + it;
                ostr = FXN;
            } else {
                const int i2 = it - FXN, r = i2 / TX, j = i2 - r * TX;  // face y0-1+r | y0+r
                ok = face_ok(y0 - 1 + r, ny) && x0 + j < nx;
                c0 = pk + (r + 1) * PW + j + 2;
                st = PW;
                out = fy + i2;
                ostr = FYN;
                off[2] = 3 * PF;  // y: vy | vz, vx
                off[3] = 4 * PF;
                off[4] = 2 * PF;
            }
            if (ok) {
                double F[5];
                face_flux(c0 - st, c0, c0 + st, c0 + 2 * st, off, m, F);
#pragma unroll
                for (int f = 0; f < 5; ++f) out[f * ostr] = F[f];
            }
        }
        __syncthreads();  // faces visible; slot of plane k - 1 is free
        if (k + 4 <= k1 + 1) load_plane(m, prim, slot(k + 4), x0, y0, k + 4);
        cp_async_commit();

        if (in) {
            const bool act_z = k >= ng && k < nz - ng;
            double dU[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            if (act_x) {  // x adds in place over active cells only; S1 is normal
                const double *lo = fx + ty * (TX + 1) + tx;
#pragma unroll
                for (int f = 0; f < 5; ++f)
                    dU[f] = dU[f] + -(lo[f * FXN + 1] - lo[f * FXN]) * m.dtdx;
            }
            {  // y: a zero-filled slab entry where inactive; (S2, S3, S1) rotated
                const double *lo = fy + ty * TX + tx;
                const int slot_y[5] = {0, 2, 3, 1, 4};
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    const double du = act_y ? -(lo[f * FYN + TX] - lo[f * FYN]) * m.dtdx : 0.0;
                    dU[slot_y[f]] = dU[slot_y[f]] + du;
                }
            }
            {  // z: (S3, S1, S2) rotated
                const int slot_z[5] = {0, 3, 1, 2, 4};
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    const double du = act_z ? -(fhi[f] - flo[f]) * m.dtdx : 0.0;
                    dU[slot_z[f]] = dU[slot_z[f]] + du;
                }
            }
            const int64_t i = (k * ny + y) * nx + x;
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const double u0 = U0[f * N + i];
                if constexpr (STAGE == 1) U.f[f][i] = u0 + dU[f];
                else U.f[f][i] = 0.5 * (u0 + U.f[f][i] + dU[f]);
            }
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) flo[f] = fhi[f];
    }
    cp_async_wait_group<0>();  // nothing in flight when the CTA retires
}

}  // namespace
}  // namespace vb

using vb::detail::fail;
using vb::detail::use;

struct vb_muscl {
    vb_ctx *ctx = nullptr;
    vb::MusclGeom m{};
    double *U = nullptr;     // owned state, 5 x N
    double *U0 = nullptr;    // step-start copy
    double *prim = nullptr;  // primitives of the stage input
    int kz = 1;              // z-planes per CTA of the tile pass (fixed by dims)
};

namespace {

int check_params(const vb_muscl_params *p, const vb_muscl *mu)
{
    if (!p) return fail(VB_EINVAL, "null parameters");
    if (p->flags != 0) return fail(VB_EINVAL, "flags must be 0");
    if (p->bc != VB_MUSCL_BC_NONE && p->bc != VB_MUSCL_BC_PERIODIC)
        return fail(VB_EINVAL, "unknown ghost-zone mode");
    if (p->bc == VB_MUSCL_BC_PERIODIC)  // every ghost's periodic source is an active cell
        for (int a = 0; a < 3; ++a)
            if (mu->m.n[a] < 3 * (int64_t)mu->m.ng)
                return fail(VB_EINVAL, "periodic ghost fill needs each dim >= 3 ng");
    if (!std::isfinite(p->dt) || !(p->gamma > 1.0) || !std::isfinite(p->theta) ||
        !(p->dx > 0.0) || !std::isfinite(p->small_rho))
        return fail(VB_EINVAL, "dt, theta and small_rho must be finite, gamma > 1, dx > 0");
    return VB_OK;
}

// z-planes per CTA: the fewest waves of 2 CTAs per SM, each wave's length
// the chunk plus the three-plane prologue (ring fill and the first lower face)
int choose_kz(int64_t tiles, int64_t nz)
{
    int64_t best_kz = nz, best = INT64_MAX;
    for (int64_t nch = 1; nch <= nz && nch <= 65535; ++nch) {
        const int64_t kz = (nz + nch - 1) / nch;
        if ((nz + kz - 1) / kz != nch) continue;
        const int64_t waves = (tiles * nch + 2 * 148 - 1) / (2 * 148);
        const int64_t cost = waves * (kz + 3);
        if (cost < best) {
            best = cost;
            best_kz = kz;
        }
    }
    return (int)best_kz;
}

// one muscl_step_3d! on the five fields
int queue_step(vb_muscl *mu, const vb::MusclFields &F, const vb_muscl_params *p)
{
    cudaStream_t s = mu->ctx->stream;
    vb::MusclGeom m = mu->m;
    m.gamma = p->gamma;
    m.theta = p->theta;
    m.dtdx = p->dt / p->dx;
    m.small_rho = p->small_rho;
    const dim3 pgrid((unsigned)((m.n[0] + 31) / 32), (unsigned)((m.n[1] + 7) / 8), (unsigned)m.n[2]);
    const int64_t gx = (m.n[0] + vb::TX - 1) / vb::TX, gy = (m.n[1] + vb::TY - 1) / vb::TY;
    const int kz = mu->kz;
    const dim3 tgrid((unsigned)gx, (unsigned)gy, (unsigned)((m.n[2] + kz - 1) / kz));
    if (p->bc == VB_MUSCL_BC_PERIODIC)
        vb::k_muscl_prep<true, true><<<pgrid, vb::MB, 0, s>>>(m, F, mu->U0, mu->prim);
    else
        vb::k_muscl_prep<true, false><<<pgrid, vb::MB, 0, s>>>(m, F, mu->U0, mu->prim);
    vb::k_muscl_tile<1><<<tgrid, vb::NT, vb::TILE_SMEM, s>>>(m, mu->prim, F, mu->U0, kz);
    VB_CHECK_LAUNCH(mu->ctx, 2);
    if (p->bc == VB_MUSCL_BC_PERIODIC)
        vb::k_muscl_prep<false, true><<<pgrid, vb::MB, 0, s>>>(m, F, mu->U0, mu->prim);
    else
        vb::k_muscl_prep<false, false><<<pgrid, vb::MB, 0, s>>>(m, F, mu->U0, mu->prim);
    vb::k_muscl_tile<2><<<tgrid, vb::NT, vb::TILE_SMEM, s>>>(m, mu->prim, F, mu->U0, kz);
    VB_CHECK_LAUNCH(mu->ctx, 2);
    return VB_OK;
}

vb::MusclFields owned(vb_muscl *mu)
{
    vb::MusclFields F;
    for (int f = 0; f < 5; ++f) F.f[f] = mu->U + f * mu->m.N;
    return F;
}

}  // namespace

extern "C" {

int vb_muscl_create(vb_ctx *ctx, const int64_t dims[3], int32_t ng, vb_muscl **out)
{
    if (!ctx || !dims || !out) return fail(VB_EINVAL, "null argument");
    *out = nullptr;
    if (ng < 2) return fail(VB_EINVAL, "ng must be at least 2 (the stencil reaches two cells)");
    int64_t N = 1;
    for (int a = 0; a < 3; ++a) {
        if (dims[a] < 2 * (int64_t)ng + 1) return fail(VB_EINVAL, "each dim needs 2 ng + 1 cells");
        if (N > INT64_MAX / dims[a]) return fail(VB_EINVAL, "cell count overflows");
        if (dims[a] > (a == 0 ? INT32_MAX : a == 1 ? 8 * 65535 : 65535))
            return fail(VB_EINVAL, "dims exceed the launch grid (ny <= 524280, nz <= 65535)");
        N *= dims[a];
    }
    int rc = use(ctx);
    if (rc) return rc;
    for (cudaError_t e : {cudaFuncSetAttribute(vb::k_muscl_tile<1>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)vb::TILE_SMEM),
                          cudaFuncSetAttribute(vb::k_muscl_tile<2>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)vb::TILE_SMEM)})
        if (e != cudaSuccess)
            return fail(VB_ECUDA, std::string("muscl shared memory: ") + cudaGetErrorString(e));
    vb_muscl *mu = new vb_muscl;
    mu->ctx = ctx;
    mu->m.N = N;
    mu->m.ng = ng;
    int64_t st = 1;
    for (int a = 0; a < 3; ++a) {
        mu->m.n[a] = dims[a];
        mu->m.stride[a] = st;
        st *= dims[a];
    }
    mu->kz = choose_kz(((dims[0] + vb::TX - 1) / vb::TX) * ((dims[1] + vb::TY - 1) / vb::TY), dims[2]);
    const size_t bytes = sizeof(double) * 5 * (size_t)N;
    cudaError_t e = cudaMalloc(&mu->U, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&mu->U0, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&mu->prim, bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(mu->U, 0, bytes, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(mu->U);
        cudaFree(mu->U0);
        cudaFree(mu->prim);
        delete mu;
        return fail(e == cudaErrorMemoryAllocation ? VB_ENOMEM : VB_ECUDA,
                    std::string("muscl allocation: ") + cudaGetErrorString(e));
    }
    *out = mu;
    return VB_OK;
}

int vb_muscl_destroy(vb_muscl *mu)
{
    if (!mu) return VB_OK;
    cudaSetDevice(mu->ctx->device);
    cudaStreamSynchronize(mu->ctx->stream);
    cudaFree(mu->U);
    cudaFree(mu->U0);
    cudaFree(mu->prim);
    delete mu;
    return VB_OK;
}

int vb_muscl_upload(vb_muscl *mu, const double *U)
{
    if (!mu || !U) return fail(VB_EINVAL, "null argument");
    int rc = use(mu->ctx);
    if (rc) return rc;
    VB_CUDA(cudaMemcpyAsync(mu->U, U, sizeof(double) * 5 * mu->m.N, cudaMemcpyHostToDevice,
                            mu->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(mu->ctx->stream));
    return VB_OK;
}

int vb_muscl_download(vb_muscl *mu, double *U)
{
    if (!mu || !U) return fail(VB_EINVAL, "null argument");
    int rc = use(mu->ctx);
    if (rc) return rc;
    VB_CUDA(cudaMemcpyAsync(U, mu->U, sizeof(double) * 5 * mu->m.N, cudaMemcpyDeviceToHost,
                            mu->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(mu->ctx->stream));
    return VB_OK;
}

int vb_muscl_state(vb_muscl *mu, double **dU)
{
    if (!mu || !dU) return fail(VB_EINVAL, "null argument");
    *dU = mu->U;
    return VB_OK;
}

int vb_muscl_step(vb_muscl *mu, const vb_muscl_params *p)
{
    VB_RANGE("vb_muscl_step");
    if (!mu) return fail(VB_EINVAL, "null handle");
    int rc = check_params(p, mu);
    if (!rc) rc = use(mu->ctx);
    if (!rc) rc = queue_step(mu, owned(mu), p);
    if (rc) return rc;
    VB_CUDA(cudaStreamSynchronize(mu->ctx->stream));
    return VB_OK;
}

int vb_muscl_run_async(vb_muscl *mu, const vb_muscl_params *p, int64_t nsteps)
{
    VB_RANGE("vb_muscl_run_async");
    if (!mu) return fail(VB_EINVAL, "null handle");
    if (nsteps < 0) return fail(VB_EINVAL, "nsteps < 0");
    int rc = check_params(p, mu);
    if (!rc) rc = use(mu->ctx);
    for (int64_t k = 0; k < nsteps && !rc; ++k) rc = queue_step(mu, owned(mu), p);
    return rc;
}

int vb_muscl_step_fields(vb_muscl *mu, double *D, double *S1, double *S2, double *S3, double *Tau,
                         const vb_muscl_params *p)
{
    VB_RANGE("vb_muscl_step_fields");
    if (!mu || !D || !S1 || !S2 || !S3 || !Tau) return fail(VB_EINVAL, "null argument");
    int rc = check_params(p, mu);
    if (!rc) rc = use(mu->ctx);
    if (rc) return rc;
    vb::MusclFields F;
    F.f[0] = D;
    F.f[1] = S1;
    F.f[2] = S2;
    F.f[3] = S3;
    F.f[4] = Tau;
    rc = queue_step(mu, F, p);
    if (rc) return rc;
    VB_CUDA(cudaStreamSynchronize(mu->ctx->stream));
    return VB_OK;
}

}  // extern "C"
