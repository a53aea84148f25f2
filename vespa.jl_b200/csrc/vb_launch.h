// vb_launch.h -- host-side launchers exported by the kernel translation units.
// Each returns the number of kernels it queued (for the launch counter) or a
// negative value when the launch configuration is invalid.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "vb_common.cuh"

namespace vb {

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

// vb_kern_mixed.cu
int launch_stage_mixed(const Geom &g, int stage, const double *Uin, const double *U0,
                       double *Uout, Ctrl *ctrl, double *bflux, cudaStream_t s);

constexpr int TOTALS_PARTS = 1024;  // fixed partial count: deterministic sum order

}  // namespace vb
