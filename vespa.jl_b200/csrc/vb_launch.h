// vb_launch.h -- host-side launchers exported by the kernel translation units.
// Each returns the number of kernels it queued (for the launch counter) or a
// negative value when the launch configuration is invalid.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "vb_common.cuh"

namespace vb {

// TMA tensor maps of one stage input buffer (4-D: x, y, z, field) with the
// three box shapes the tiled 3D kernel loads: tile interior, x strip, y strip.
struct TiledMaps {
    CUtensorMap in_int, in_xs, in_ys;
};

// Tiled 3D path applicability: 16 x 16 column tiles, at least two planes,
// periodic axes periodic on both sides (checked at grid creation).
inline bool tiled3d_supported(const Geom &g)
{
    return g.nd == 3 && g.n[0] % 16 == 0 && g.n[1] % 16 == 0 && g.n[2] >= 2 &&
           g.n[0] <= (1 << 30) && g.n[1] <= (1 << 30) && g.n[2] <= (1 << 30);
}

// vb_kern_fp64.cu (compiled with -fmad=false)
int launch_stage_fp64(const Geom &g, int stage, const double *Uin, const double *U0,
                      double *Uout, Ctrl *ctrl, double *bflux, cudaStream_t s);
int launch_cfl(const Geom &g, const double *U, Ctrl *ctrl, cudaStream_t s);
int launch_finalize_cfl(const Geom &g, Ctrl *ctrl, cudaStream_t s);
int launch_set_dt(const Geom &g, Ctrl *ctrl, double dt, cudaStream_t s);
int launch_totals(const Geom &g, const double *U, double *partials, int npart, double *out,
                  cudaStream_t s);
int launch_hllc_faces(int64_t nf, const double *WL, const double *WR, const int32_t *axis,
                      double gamma, double *F, cudaStream_t s);

int launch_stage_tiled3d_fp64(const TiledMaps &m, const Geom &g, int kz, int stage,
                              const double *Uin, const double *U0, double *Uout, Ctrl *ctrl,
                              cudaStream_t s);

// vb_kern_mixed.cu
int launch_stage_tiled3d_mixed(const TiledMaps &m, const Geom &g, int kz, int stage,
                               const double *Uin, const double *U0, double *Uout, Ctrl *ctrl,
                               cudaStream_t s);
int launch_stage_mixed(const Geom &g, int stage, const double *Uin, const double *U0,
                       double *Uout, Ctrl *ctrl, double *bflux, cudaStream_t s);

constexpr int TOTALS_PARTS = 1024;  // fixed partial count: deterministic sum order

// vb_api.cu: record the calling thread's message for vb_last_error.
void set_last_error(const char *msg);

}  // namespace vb
