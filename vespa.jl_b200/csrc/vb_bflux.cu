// vb_bflux.cu -- bflux_plane (src/reflux.jl:148-191) on the device: one
// (dim, side) face plane of the boundary-flux register rasterised into the
// flat array a coupled code stores a coarse-fine face flux in (Enzo's
// Left/RightFluxes[field][dim]), in that code's units (value / Vcell).
//
// Plane offsets are column-major over the plane's extent (dim 0 fastest).  An
// offset maps to global index g = start + offset per axis and to Vespa's
// active index a = g - g0 + 1 on the axes across the face; along the flux
// axis the active index is the caller's flux_off.  The register entry of that
// cell (the lookup of the reference) is:
//   - source lo / hi: the outer face (dim+1, :lo / :hi, cell), present when
//     the cell is the boundary cell on that side of a non-periodic axis;
//   - source interior: the interior face (dim+1, cell), keyed by the face's
//     lo cell, present when the cell's hi neighbour along dim+1 is a cell
//     (periodic wrap included);
// anything else (outside the grid, not recorded, comp <= 0) rasterises to 0.
#include "../../include/vespa_b200.h"
#include "vb_launch.h"

namespace vb {

namespace {

__global__ void k_bflux_plane(Geom g, const double *__restrict__ bf, int64_t outer_n, PlaneSpec ps,
                              double *__restrict__ out, int64_t n)
{
    for (int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; lin < n;
         lin += (int64_t)gridDim.x * blockDim.x) {
        int64_t rem = lin, a[3] = {1, 1, 1};
        for (int d = 0; d < ps.R; ++d) {
            const int64_t od = rem % ps.dims[d];
            rem /= ps.dims[d];
            a[d] = d == ps.dim ? ps.flux_off : (ps.start[d] + od - ps.g0[d] + 1);
        }
        double v = 0.0;
        bool inside = ps.comp > 0;
        for (int d = 0; d < ps.R; ++d) inside = inside && a[d] >= 1 && a[d] <= g.n[d];
        if (inside) {
            const int d = ps.dim;
            const int k = ps.comp - 1;
            if (ps.source == VB_BFLUX_PLANE_INTERIOR) {
                if (a[d] < g.n[d] || g.bc_hi[d] == BC_PERIODIC) {
                    int64_t cell = 0, mul = 1;
                    for (int e = 0; e < ps.R; ++e) {
                        cell += (a[e] - 1) * mul;
                        mul *= g.n[e];
                    }
                    v = bf[outer_n + ((int64_t)d * 5 + k) * g.ncell + cell] / ps.vcell;
                }
            } else {
                const int side = ps.source == VB_BFLUX_PLANE_HI ? 1 : 0;
                const int bc = side ? g.bc_hi[d] : g.bc_lo[d];
                if (bc != BC_PERIODIC && a[d] == (side ? g.n[d] : 1)) {
                    int64_t off = 0;
                    for (int e = 0; e < d; ++e) off += 2 * 5 * (g.ncell / g.n[e]);
                    const int64_t P = g.ncell / g.n[d];
                    int64_t idx = 0, mul = 1;
                    for (int e = 0; e < ps.R; ++e) {
                        if (e == d) continue;
                        idx += (a[e] - 1) * mul;
                        mul *= g.n[e];
                    }
                    v = bf[off + (int64_t)side * 5 * P + (int64_t)k * P + idx] / ps.vcell;
                }
            }
        }
        out[lin] = v;
    }
}

}  // namespace

int launch_bflux_plane(const Geom &g, const double *bflux, int64_t outer_n, const PlaneSpec &ps,
                       double *d_out, int64_t n, cudaStream_t s)
{
    if (n <= 0 || !bflux || !d_out || ps.R != g.nd) return -1;
    const int bs = 256;
    const int64_t nb = (n + bs - 1) / bs;
    k_bflux_plane<<<(unsigned)(nb < 1184 ? nb : 1184), bs, 0, s>>>(g, bflux, outer_n, ps, d_out, n);
    return 1;
}

}  // namespace vb
