// vb_kern_mixed.cu -- VB_MIXED stage kernels: float64 state, cons2prim
// (including the E - kinetic pressure recovery), flux-difference
// accumulation and CFL reduction; float32 reconstruction and HLLC.
#include "vb_launch.h"
#include "vb_stage_generic.cuh"
#include "vb_stage_tiled3d_mixed.cuh"
#include "vb_stage_tiled2d.cuh"

namespace vb {

namespace {

template <int ND, int STAGE>
int launch_generic(const Geom &g, const double *Uin, const double *U0, double *Uout, Ctrl *ctrl,
                   double *bflux, double *bflux_int, cudaStream_t s)
{
    const int bs = 256;
    const int64_t nb = (g.ncell + bs - 1) / bs;
    if (nb <= 0 || nb > 0x7fffffffLL) return -1;
    k_stage_generic<float, ND, STAGE><<<(unsigned)nb, bs, 0, s>>>(g, Uin, U0, Uout, ctrl, bflux,
                                                                   bflux_int);
    return 1;
}

}  // namespace

int launch_stage_tiled3d_mixed(const BoxDesc *hbox, const BoxDesc *boxes, const int *item_box,
                               int nitems, unsigned int *work, int stage, cudaStream_t s, bool grav,
                               bool bf)
{
    return launch_tiled3d_mixed<2>(hbox, boxes, item_box, nitems, work, stage, s, grav, bf);
}

int launch_stage_tiled2d_mixed(const BoxDesc *hbox, int nitems, unsigned int *work, int stage,
                               cudaStream_t s, bool bf)
{
    return launch_tiled2d<true, 2>(hbox, nitems, work, stage, s, bf);
}

int launch_stage_mixed(const Geom &g, int stage, const double *Uin, const double *U0,
                       double *Uout, Ctrl *ctrl, double *bflux, cudaStream_t s, double *bflux_int)
{
    switch (g.nd * 10 + stage) {
    case 11: return launch_generic<1, 1>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 12: return launch_generic<1, 2>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 21: return launch_generic<2, 1>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 22: return launch_generic<2, 2>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 31: return launch_generic<3, 1>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    case 32: return launch_generic<3, 2>(g, Uin, U0, Uout, ctrl, bflux, bflux_int, s);
    default: return -1;
    }
}

}  // namespace vb
