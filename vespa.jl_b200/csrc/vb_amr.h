// vb_amr.h -- device view of the composite AMR mesh and the launchers of
// vb_amr_kern.cu.  Not part of the public ABI.
#pragma once

#include "vb_launch.h"

namespace vb {

constexpr int AMR_MAX_LEVEL = 15;  // levels above the base grid

// The mesh tables the kernels read (device pointers), by value per launch.
struct AmrDev {
    int nd;
    int bc_lo[3], bc_hi[3];
    double gamma, aexp;
    int64_t cap;     // leaf capacity: field stride of U, reg, rep
    int64_t fcap;    // face capacity: field stride of F
    int nleaf, nface, nent;  // leaves, faces, CSR entries
    const int *lev;       // level of each leaf
    const int *rep;       // [2*axis+side][cap]: representative neighbour, -1 boundary
    const int *fL, *fR;   // face sides (-1: boundary ghost)
    const int8_t *fax;    // face axis (0-based)
    const double *farea;  // face area
    const int *off;       // CSR offsets, nleaf+1
    const int *ent;       // CSR entries: face*2 + (1 if the leaf is the face's right side)
    double *reg;          // flux registers, [5][cap]
    double vol[AMR_MAX_LEVEL + 1];
    double w[AMR_MAX_LEVEL + 1][3];
};

// Per-stage parameters: dt, which level is updated (-1: all), active flux
// registers (coarse level and signed scale), and whether the stage-2
// epilogue folds the CFL maximum of every leaf.
struct AmrStageArgs {
    double dt;
    int level;
    int nreg;
    int reg_level[2];
    double reg_scale[2];
    int cfl_all;
    // set: dt is read from here (a subcycled level's substep dt, computed on
    // the device) and reg_scale holds the register signs (+1 / -1), the scale
    // being sign * (0.5 * dt) as evolve_level! forms it
    const double *dt_dev;
};

// Device state of one level of a subcycled root step (evolve_level!,
// src/driver.jl:553-578), for the graph that runs the recursion on the
// device: the dt target handed down (the parent's substep dt; the root step's
// dt at level 0), the substep dt and count, the level's CFL maximum.
struct AmrSubLevel {
    double dt_target;
    double dt_sub;
    unsigned long long invdt_bits;
    long long left;   // substeps still to run
    long long iters;  // substeps run so far
};
// A level runs at most this many substeps per parent substep; beyond it the
// root step stops with VB_ENONFINITE-like error bits (a non-finite or
// vanishing dt, never a sound run).
constexpr long long AMR_MAX_SUBSTEPS = 1ll << 20;
enum { AMR_SUB_NONFINITE = 1, AMR_SUB_TOO_MANY = 2 };

// Topology view for the regrid kernels (vb_amr_regrid.cu).
struct AmrTopo {
    int nd;
    int64_t base[3];
    int bc_lo[3], bc_hi[3];
    int n;          // leaves
    int64_t cap;    // leaf stride of cx and the per-side tables
    const int *lev;
    const int *cx;  // [3][cap] integer coordinates at the leaf's level
    const uint64_t *hkey;
    const int *hval;
    uint64_t hmask;  // hash capacity - 1 (a power of two minus one)
};

// face area per level and axis
struct AmrAreas {
    double area[AMR_MAX_LEVEL + 1][3];
};

int amr_scan(const int *in, int n, int *out, int *bsum, int *total, cudaStream_t s);
int launch_amr_hash_build(const AmrTopo &t, uint64_t *keys, int *vals, int *err, cudaStream_t s);
int launch_amr_balance(const AmrTopo &t, uint8_t *mark, int *changed, const int *gate,
                       cudaStream_t s);
int launch_amr_count_children(const AmrTopo &t, const uint8_t *mark, int *cnt, int *maxlev,
                              cudaStream_t s);
int launch_amr_emit(const AmrTopo &t, const uint8_t *mark, const int *off, int *lev_new,
                    int *cx_new, int64_t cap_new, const double *Uold, double *Unew, cudaStream_t s);
int launch_amr_kinds(const AmrTopo &t, int8_t *kind, int *rep, int *fcnt, cudaStream_t s);
int launch_amr_faces(const AmrTopo &t, const int8_t *kind, const int *rep, const int *fbase,
                     const AmrAreas &ar, int *fL, int *fR, int8_t *fax, double *farea, int *faceid,
                     cudaStream_t s);
int launch_amr_csr_count(const AmrTopo &t, const int8_t *kind, const int *fcnt, int *ecnt,
                         cudaStream_t s);
int launch_amr_csr_fill(const AmrTopo &t, const int8_t *kind, const int *rep, const int *faceid,
                        const int *off, int *ent, int *err, cudaStream_t s);

int launch_amr_stage(const AmrDev &m, int stage, const double *Uin, const double *U0,
                     double *Uout, double *F, const AmrStageArgs &a, Ctrl *ctrl, cudaStream_t s);
int launch_amr_cfl(const AmrDev &m, const double *U, int level, Ctrl *ctrl, cudaStream_t s);
// The same maximum into the word `bits` (not reset here).
int launch_amr_cfl_bits(const AmrDev &m, const double *U, int level, unsigned long long *bits,
                        cudaStream_t s);
// Device-driven subcycling (graph nodes, one thread each).  plan: from the
// level's CFL maximum and its dt target (the parent's substep dt when
// `target_src` is set) the substep count and dt, and the WHILE condition
// `h` of the level's substep loop; next: one substep done, condition for
// the next.  Error bits go to *err.
int launch_amr_sub_plan(AmrSubLevel *sub, int level, double cfl, const double *target_src,
                        cudaGraphConditionalHandle h, int *err, cudaStream_t s);
int launch_amr_sub_next(AmrSubLevel *sub, int level, cudaGraphConditionalHandle h, int *err,
                        cudaStream_t s);
int launch_amr_sub_target(AmrSubLevel *sub, double dt, cudaStream_t s);
int launch_amr_tag(const AmrDev &m, const double *U, double above, int max_level, uint8_t *tag,
                   double *ind, int *ntag, cudaStream_t s);
int launch_amr_reflux(const AmrDev &m, double *U, int level, cudaStream_t s);
int launch_amr_zero_reg(const AmrDev &m, int level, cudaStream_t s);
int launch_amr_totals(const AmrDev &m, const double *U, double *partials, int npart, double *out,
                      cudaStream_t s);

}  // namespace vb
