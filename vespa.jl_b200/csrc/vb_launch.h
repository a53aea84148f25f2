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

// One box of a tiled launch, in device memory: the tensor maps of its two
// stage inputs, its geometry, state buffers and control block, and where its
// work items start in the launch's global item numbering.  A single grid is a
// one-box table; a batch of independent problems is a table of many.
struct alignas(64) BoxDesc {
    CUtensorMap map[2][3];  // [stage-1 input U, stage-2 input U1][interior, x strip, y strip]
    Geom g;
    double *U, *U1;
    Ctrl *ctrl;
    double *bflux;  // boundary-flux planes being recorded, or null
    int kz;       // z planes per work item (3D: of the leading chunks, see chunk_span)
    int nchu;     // 3D: chunks of kz planes
    int nch;      // 3D: z chunks in all
    int ntx;      // column tiles along x
    int ntiles;   // column tiles per plane
    int item0;    // first global work item of this box
};

// z chunks of a 3D box, in queue order: nchu chunks of kz planes (the last
// one cut at nz), then, in the tapered form, the remaining planes (between kz
// and 2 kz of them, or all nz when nz <= 2 kz) in halving pieces of at most kz
// planes: a remainder of 16 planes or more gives up half of itself (rounded
// down), a smaller one is taken whole.  With kz >= 16 every piece then has 8
// to kz planes and the last one fewer than 16, so that the work queue ends on
// short items and the blocks finish together.  Single grids take the form the
// autotuner timed faster (the tapered one at 256^3 in both precisions; a
// VB_MIXED grid defaults to it); batches keep the uniform chunks.
__host__ __device__ inline int chunk_tail_piece(int r, int kz)
{
    const int p = r >= 16 ? r / 2 : r;
    return p < kz ? p : kz;
}
__host__ __device__ inline void chunk_span(int nz, int kz, int nchu, int c, int &k0, int &k1)
{
    if (c < nchu) {
        k0 = c * kz;
        k1 = k0 + kz < nz ? k0 + kz : nz;
        return;
    }
    int r = nz - nchu * kz;
    for (int j = nchu; j < c; ++j) r -= chunk_tail_piece(r, kz);
    k0 = nz - r;
    k1 = k0 + chunk_tail_piece(r, kz);
}
inline int chunk_count(int nz, int kz, bool taper, int *nchu)
{
    if (!taper) {
        *nchu = (nz + kz - 1) / kz;
        return *nchu;
    }
    const int u = nz > 2 * kz ? (nz + kz - 1) / kz - 2 : 0;
    int n = u;
    for (int r = nz - u * kz; r > 0; r -= chunk_tail_piece(r, kz)) ++n;
    *nchu = u;
    return n;
}

// Tiled 3D path applicability: 16 x 16 column tiles, at least two planes,
// periodic axes periodic on both sides (checked at grid creation).
inline bool tiled3d_supported(const Geom &g)
{
    return g.nd == 3 && g.n[0] % 16 == 0 && g.n[1] % 16 == 0 && g.n[2] >= 2 &&
           g.n[0] <= (1 << 30) && g.n[1] <= (1 << 30) && g.n[2] <= (1 << 30);
}

// Tiled 2D path applicability: 256-cell row segments marching y.
inline bool tiled2d_supported(const Geom &g)
{
    return g.nd == 2 && g.n[0] % 256 == 0 && g.n[1] >= 2 && g.n[0] <= (1 << 30) &&
           g.n[1] <= (1 << 30);
}
inline bool tiled_supported(const Geom &g) { return tiled3d_supported(g) || tiled2d_supported(g); }
// cells along the marching axis (z in 3D, y in 2D)
inline int64_t march_extent(const Geom &g) { return g.nd == 3 ? g.n[2] : g.n[1]; }

// vb_kern_fp64.cu (compiled with -fmad=false)
// bflux: the outer boundary-flux planes being recorded (or null); bflux_int:
// the interior face register [axis][5][ncell] (or null).
int launch_stage_fp64(const Geom &g, int stage, const double *Uin, const double *U0,
                      double *Uout, Ctrl *ctrl, double *bflux, cudaStream_t s,
                      double *bflux_int = nullptr);
int launch_cfl(const Geom &g, const double *U, Ctrl *ctrl, cudaStream_t s);
int launch_finalize_cfl(const Geom &g, Ctrl *ctrl, cudaStream_t s);
int launch_set_dt(const Geom &g, Ctrl *ctrl, double dt, cudaStream_t s);
int launch_totals(const Geom &g, const double *U, double *partials, int npart, double *out,
                  cudaStream_t s);
// fold `npart` five-component partial sums in index order (one block)
int launch_totals_final(const double *partials, int npart, double *out, cudaStream_t s);
int launch_hllc_faces(int64_t nf, const double *WL, const double *WR, const int32_t *axis,
                      double gamma, double *F, cudaStream_t s);

// Tiled stage.  hbox (host pointer) set: a single box passed by value; else a
// device box table `boxes` with `item_box` mapping each global work item to
// its box.  `work` holds the two stage cursors (reset by the dt kernels).
// grav: the self-gravity source and free-fall dt term (single boxes only).
// bf: also record the domain-boundary face fluxes into hbox->bflux (single
// boxes without gravity).
int launch_stage_tiled3d_fp64(const BoxDesc *hbox, const BoxDesc *boxes, const int *item_box,
                              int nitems, unsigned int *work, int stage, cudaStream_t s,
                              bool grav = false, bool bf = false);
// Tiled 2D stage (single box by value); bf: also record the domain-boundary
// face fluxes into hbox->bflux.
int launch_stage_tiled2d_fp64(const BoxDesc *hbox, int nitems, unsigned int *work, int stage,
                              cudaStream_t s, bool bf = false);
int launch_stage_tiled2d_mixed(const BoxDesc *hbox, int nitems, unsigned int *work, int stage,
                               cudaStream_t s, bool bf = false);
// Per-box dt finalisation (evolve!'s loop head) and clock advance for a table.
int launch_finalize_boxes(const BoxDesc *boxes, int nbox, unsigned int *work, cudaStream_t s);
int launch_advance_boxes(const BoxDesc *boxes, int nbox, cudaStream_t s);
// Clock advance of a single control block (t += dt, step += 1 while active).
int launch_advance(Ctrl *ctrl, cudaStream_t s);
// Copy the running CFL maximum of ctrl out to (put = 0) or in from (put = 1)
// the device word dev.
int launch_cfl_bits(Ctrl *ctrl, unsigned long long *dev, int put, cudaStream_t s);
// A bounded mbarrier wait that must run out after limit_ns, then the stage
// kernels' abandon path (CTRL_F_TIMEOUT in ctrl).
int launch_wait_selftest(Ctrl *ctrl, uint64_t limit_ns, cudaStream_t s);

// vb_kern_mixed.cu
int launch_stage_tiled3d_mixed(const BoxDesc *hbox, const BoxDesc *boxes, const int *item_box,
                               int nitems, unsigned int *work, int stage, cudaStream_t s,
                               bool grav = false, bool bf = false);
int launch_stage_mixed(const Geom &g, int stage, const double *Uin, const double *U0,
                       double *Uout, Ctrl *ctrl, double *bflux, cudaStream_t s,
                       double *bflux_int = nullptr);

// vb_adjoint_kern.cu (periodic meshes, float64): one adjoint RK2 stage,
//   out = 0.5*lam + (M ? M : 0) - invV * (dD/dU)^T mu,  mu = M ? M : 0.5*lam,
// at the state U; gL/gR (2*nd*5*ncell doubles) and code (nd*ncell) are scratch.
int launch_adj_stage(const Geom &g, const double *U, const double *lam, const double *M,
                     double invV, double *gL, double *gR, uint16_t *code, double *out,
                     cudaStream_t s);
// dts[ctrl->step - step0] = ctrl->dt while the step in flight is active
int launch_record_dt(const Ctrl *ctrl, double *dts, int64_t step0, int64_t cap, cudaStream_t s);

// bflux_plane raster request (src/reflux.jl:171-191): the plane [start,
// start + dims) in global indices, the grid's first active cell g0, the
// active index used along the flux axis, the 1-based component and the cell
// volume; source picks the lo or hi outer planes or the interior register.
struct PlaneSpec {
    int R, dim, source, comp;
    int64_t start[3], dims[3], g0[3];
    int64_t flux_off;
    double vcell;
};
// vb_bflux.cu: rasterise one plane from the register (outer planes of
// `outer_n` doubles, then the interior block) into n doubles at d_out.
int launch_bflux_plane(const Geom &g, const double *bflux, int64_t outer_n, const PlaneSpec &ps,
                       double *d_out, int64_t n, cudaStream_t s);

constexpr int TOTALS_PARTS = 1024;  // fixed partial count: deterministic sum order

// vb_api.cu: record the calling thread's message for vb_last_error.
void set_last_error(const char *msg);

}  // namespace vb
