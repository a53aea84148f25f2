// vb_api.cu -- the extern "C" entry points of libvespa_b200 (include/vespa_b200.h).
//
// Host-side runtime: contexts (device + stream + scratch), device-resident
// uniform grids with their control block, the stepping loop that keeps dt on
// the device, and error reporting.  No C++ exception crosses the ABI.
#include <cudaTypedefs.h>

#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "vb_internal.h"

using vb::detail::fail;
using vb::detail::use;

#ifdef VB_CHECK
namespace vb {
namespace {
std::vector<unsigned (*)()> &check_readers()
{
    static std::vector<unsigned (*)()> v;
    return v;
}
std::mutex &check_mu()
{
    static std::mutex m;
    return m;
}
}  // namespace
// each translation unit's reader of its VB_DCHECK record (vb_common.cuh)
void check_register(unsigned (*read_and_clear)())
{
    std::lock_guard<std::mutex> lk(check_mu());
    check_readers().push_back(read_and_clear);
}
}  // namespace vb
#endif

namespace {
thread_local std::string g_err;
}  // namespace

namespace vb {
namespace detail {

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

int use(vb_ctx *ctx)
{
    if (!ctx) return fail(VB_EINVAL, "null context");
    VB_CUDA(cudaSetDevice(ctx->device));
    return VB_OK;
}

int ctx_scratch(vb_ctx *ctx, size_t bytes, void **out)
{
    if (bytes > ctx->scratch_bytes) {
        // the previous buffer may still be read by queued work
        VB_CUDA(cudaStreamSynchronize(ctx->stream));
        if (ctx->scratch) cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
        VB_CUDA(cudaMalloc(&ctx->scratch, bytes));
        ctx->scratch_bytes = bytes;
    }
    *out = ctx->scratch;
    return VB_OK;
}

}  // namespace detail
}  // namespace vb

namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry-point lookup (no
// link-time dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// 4-D (x, y, z, field) float64 tensor map over a state buffer with box
// (bx, by, 1, 5).  Out-of-range coordinates read zeros.
int encode_state_map(CUtensorMap *m, const double *base, const vb::Geom &g, uint32_t bx,
                     uint32_t by)
{
    auto enc = tensor_map_encoder();
    if (!enc) return fail(VB_ENOTSUP, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[4] = {(cuuint64_t)g.n[0], (cuuint64_t)g.n[1], (cuuint64_t)g.n[2], 5};
    cuuint64_t strides[3] = {(cuuint64_t)g.n[0] * 8, (cuuint64_t)(g.n[0] * g.n[1]) * 8,
                             (cuuint64_t)g.ncell * 8};
    cuuint32_t box[4] = {bx, by, 1, 5};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(VB_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return VB_OK;
}

// Autotuned z-chunk per (GPU model, dims, boundaries, precision),
// process-wide, and in the file named by VB_AUTOTUNE_CACHE when that is set:
// one "key kz taper" line per tuning, appended by vb_grid_autotune and read
// when a grid is created (the last line of a key wins).
std::mutex g_tune_mu;
std::map<std::string, std::pair<int, int>> g_tune_kz;  // (kz, tapered queue: 0 / 1 / -1 untuned)

// (call with g_tune_mu held) "model/SMs" of a device, looked up once
const std::string &device_model(int device)
{
    static std::map<int, std::string> names;
    auto it = names.find(device);
    if (it != names.end()) return it->second;
    cudaDeviceProp p{};
    std::string k = cudaGetDeviceProperties(&p, device) == cudaSuccess
                        ? std::string(p.name) + "/" + std::to_string(p.multiProcessorCount)
                        : "device" + std::to_string(device);
    for (char &c : k)
        if (c == ' ') c = '_';
    return names[device] = k;
}

// (call with g_tune_mu held)
std::string tune_key(int device, const vb::Geom &g, int precision)
{
    std::string k = device_model(device);
    k += ":" + std::to_string(precision);
    for (int a = 0; a < 3; ++a)
        k += ":" + std::to_string(g.n[a]) + "/" + std::to_string(g.bc_lo[a]) +
             std::to_string(g.bc_hi[a]);
    return k;
}

// (call with g_tune_mu held) the cache file's entry for `key`, if any
bool tune_file_lookup(const std::string &key, std::pair<int, int> *v)
{
    const char *path = std::getenv("VB_AUTOTUNE_CACHE");
    if (!path || !*path) return false;
    FILE *f = std::fopen(path, "r");
    if (!f) return false;
    char kbuf[512];
    int kz = 0, taper = 0;
    bool found = false;
    while (std::fscanf(f, "%511s %d %d", kbuf, &kz, &taper) == 3)
        if (key == kbuf && kz > 0 && taper >= -1 && taper <= 1) {
            *v = {kz, taper};
            found = true;
        }
    std::fclose(f);
    return found;
}

// (call with g_tune_mu held) append a tuning to the cache file, if one is named
void tune_file_append(const std::string &key, int kz, int taper)
{
    const char *path = std::getenv("VB_AUTOTUNE_CACHE");
    if (!path || !*path) return;
    FILE *f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s %d %d\n", key.c_str(), kz, taper);
    std::fclose(f);
}

}  // namespace

namespace vb {
namespace detail {

int encode_maps(vb::TiledMaps *m, const double *base, const vb::Geom &g)
{
    if (g.nd == 2) {  // 256-cell row segments and their 2-cell x halos
        int rc = encode_state_map(&m->in_int, base, g, 256, 1);
        if (!rc) rc = encode_state_map(&m->in_xs, base, g, 2, 1);
        if (!rc) m->in_ys = m->in_xs;
        return rc;
    }
    int rc = encode_state_map(&m->in_int, base, g, 16, 16);
    if (!rc) rc = encode_state_map(&m->in_xs, base, g, 2, 16);
    if (!rc) rc = encode_state_map(&m->in_ys, base, g, 16, 2);
    return rc;
}

int default_kz(const vb::Geom &g)
{
    const int64_t n = vb::march_extent(g);
    return n >= 64 ? 32 : (int)((n + 1) / 2);
}

// Column tiles (3D) or row segments (2D) per chunk of the marching axis.
int64_t tiles_per_chunk(const vb::Geom &g)
{
    return g.nd == 2 ? g.n[0] / 256 : (g.n[0] / 16) * (g.n[1] / 16);
}

// The automatic kernel choice takes a tiled kernel only when it yields enough
// work items for the persistent grid (two blocks per SM on 148 SMs, with a
// chunk of at least 8 planes/rows); small grids keep the cell-centric kernel.
bool tiled_auto(const vb::Geom &g)
{
    if (!vb::tiled_supported(g)) return false;
    const int64_t ext = vb::march_extent(g);
    return tiles_per_chunk(g) * ((ext + 7) / 8) >= 296;
}

// Default chunk of a single grid.  3D: the largest of 48, 40, 32, 24, 16 that
// gives two work items per persistent block (long chunks amortise the 4-plane
// prologue of an item), else the largest giving one (measured on B200, 128^3
// to 384^3: within 2 % of the best chunk); 2D: the largest of 32, 16 giving
// two.  Otherwise 8.
int grid_default_kz(const vb::Geom &g)
{
    const int64_t ext = vb::march_extent(g);
    const int64_t tiles = tiles_per_chunk(g);
    auto items = [&](int kz) { return tiles * ((ext + kz - 1) / kz); };
    if (g.nd == 3) {
        for (int64_t need : {592, 296})
            for (int kz : {48, 40, 32, 24, 16})
                if (kz <= ext && items(kz) >= need) return kz;
    } else {
        for (int kz : {32, 16})
            if (kz <= ext && items(kz) >= 592) return kz;
    }
    return (int)(ext >= 8 ? 8 : ext);
}

// Geometry of a descriptor, validated as Problem is (src/problem.jl:39-46),
// and RefMesh's derived widths, areas and volume (lib/RefMesh/src/RefMesh.jl:
// 122-142).
int make_geom(const vb_problem_desc *d, vb::Geom *out)
{
    if (!d) return fail(VB_EINVAL, "null problem descriptor");
    if (d->ndim < 1 || d->ndim > 3) return fail(VB_EINVAL, "ndim must be 1, 2 or 3");
    if (!(d->gamma > 1.0)) return fail(VB_EINVAL, "gamma must exceed 1");
    if (!(d->cfl > 0.0 && d->cfl <= 1.0)) return fail(VB_EINVAL, "cfl must be in (0, 1]");
    if (!(d->aexp > 0.0)) return fail(VB_EINVAL, "aexp must be positive");
    if (d->flags != 0) return fail(VB_EINVAL, "flags must be 0");
    vb::Geom g{};
    g.nd = d->ndim;
    int64_t s = 1;
    for (int a = 0; a < 3; ++a) {
        if (a < d->ndim) {
            if (d->dims[a] < 1) return fail(VB_EINVAL, "all dims must be positive");
            if (!(d->hi[a] > d->lo[a])) return fail(VB_EINVAL, "domain must have hi > lo");
            for (int side = 0; side < 2; ++side) {
                int bc = side ? d->bc_hi[a] : d->bc_lo[a];
                if (bc < VB_BC_OUTFLOW || bc > VB_BC_REFLECTING)
                    return fail(VB_EINVAL, "unknown boundary condition");
            }
            if ((d->bc_lo[a] == VB_BC_PERIODIC) != (d->bc_hi[a] == VB_BC_PERIODIC))
                return fail(VB_EINVAL, "a periodic axis must be periodic on both sides");
            g.n[a] = d->dims[a];
            g.bc_lo[a] = d->bc_lo[a];
            g.bc_hi[a] = d->bc_hi[a];
        } else {
            g.n[a] = 1;
            g.bc_lo[a] = g.bc_hi[a] = VB_BC_PERIODIC;
        }
        g.stride[a] = s;
        if (s > INT64_MAX / g.n[a]) return fail(VB_EINVAL, "cell count overflows");
        s *= g.n[a];
    }
    g.ncell = s;
    for (int a = 0; a < g.nd; ++a) g.w[a] = (d->hi[a] - d->lo[a]) / (double)d->dims[a];
    for (int a = 0; a < 3; ++a) g.invw[a] = a < g.nd ? 1.0 / g.w[a] : 0.0;
    for (int a = 0; a < g.nd; ++a) {
        double ar = 1.0;
        for (int e = 0; e < g.nd; ++e)
            if (e != a) ar *= g.w[e];
        g.area[a] = ar;
    }
    double v = g.w[0];
    for (int a = 1; a < g.nd; ++a) v = v * g.w[a];
    g.vol = v;
    g.gamma = d->gamma;
    g.cfl = d->cfl;
    g.aexp = d->aexp;
    g.zw0 = 0;
    g.zw1 = (int)g.n[2];
    g.zcls0 = -1;
    g.act0 = 0;
    g.act1 = g.ncell;
    *out = g;
    return VB_OK;
}

// Box-table entry of a tiled grid (host side).
vb::BoxDesc make_box(const vb::TiledMaps &mU, const vb::TiledMaps &mU1, const vb::Geom &g,
                     double *U, double *U1, vb::Ctrl *ctrl, int kz, int item0, bool taper)
{
    vb::BoxDesc b;
    std::memset(&b, 0, sizeof b);
    b.map[0][0] = mU.in_int;
    b.map[0][1] = mU.in_xs;
    b.map[0][2] = mU.in_ys;
    b.map[1][0] = mU1.in_int;
    b.map[1][1] = mU1.in_xs;
    b.map[1][2] = mU1.in_ys;
    b.g = g;
    b.U = U;
    b.U1 = U1;
    b.ctrl = ctrl;
    b.kz = kz;
    if (g.nd == 2) {
        b.ntx = (int)(g.n[0] / 256);
        b.ntiles = b.ntx;
    } else {
        b.ntx = (int)(g.n[0] / 16);
        b.ntiles = (int)((g.n[0] / 16) * (g.n[1] / 16));
        b.nch = vb::chunk_count((int)g.n[2], kz, taper, &b.nchu);
    }
    b.item0 = item0;
    return b;
}

int64_t box_items(const vb::Geom &g, int kz, bool taper)
{
    if (g.nd == 2) return (g.n[0] / 256) * ((g.n[1] + kz - 1) / kz);
    int nchu = 0;
    return (g.n[0] / 16) * (g.n[1] / 16) * vb::chunk_count((int)g.n[2], kz, taper, &nchu);
}

}  // namespace detail
}  // namespace vb

namespace {

using vb::detail::box_items;
using vb::detail::encode_maps;
using vb::detail::make_box;

// Whether the grid's 3D work queue uses tapered z chunks (VB_OPT_TILE_TAPER;
// by default single VB_MIXED grids do).
bool grid_taper(const vb_grid *gr)
{
    if (gr->taper >= 0) return gr->taper != 0;
    if (gr->taper_tuned >= 0) return gr->taper_tuned != 0;
    return gr->precision == VB_MIXED;
}

// Refresh the grid's box descriptor after kz, the taper (or the maps) changed.
int sync_box(vb_grid *gr)
{
    const int tp = grid_taper(gr) ? 1 : 0;
    if (gr->box_kz == gr->kz && gr->box_taper == tp) return VB_OK;
    gr->box = make_box(gr->maps_U, gr->maps_U1, gr->g, gr->U, gr->U1, gr->ctrl, gr->kz, 0, tp != 0);
    gr->box_kz = gr->kz;
    gr->box_taper = tp;
    return VB_OK;
}

int stage(vb_grid *gr, int st, const double *Uin, const double *U0, double *Uout)
{
    double *bf = gr->bflux_on ? gr->bflux : nullptr;
    double *bfi = bf && gr->bflux_interior ? gr->bflux + gr->bflux_outer_n : nullptr;
    const bool grav = gr->grav != nullptr;  // self-gravity: 3D tiled kernels carry the source
    // the tiled kernels record outer boundary fluxes themselves; interior
    // faces, and boundary fluxes together with gravity, take the cell kernel
    const bool use_tiled = gr->tiled && !bfi && !(bf && grav) && (!grav || gr->g.nd == 3);
    if (gr->slab && !use_tiled)
        return fail(VB_ENOTSUP, "a z-window (slab) grid steps with the tiled 3D kernels only");
    if (use_tiled) {
        int rc = sync_box(gr);
        if (rc) return rc;
        gr->box.bflux = bf;
        const int64_t items = box_items(gr->g, gr->kz, grid_taper(gr));
        if (items > 0x7fffffff) return fail(VB_ENOTSUP, "too many tiled work items");
        unsigned int *work = gr->ctrl->work;  // device address of the cursors
        if (gr->g.nd == 2) {
            int n2 = gr->precision == VB_MIXED
                         ? vb::launch_stage_tiled2d_mixed(&gr->box, (int)items, work, st,
                                                          gr->ctx->stream, bf != nullptr)
                         : vb::launch_stage_tiled2d_fp64(&gr->box, (int)items, work, st,
                                                         gr->ctx->stream, bf != nullptr);
            VB_CHECK_LAUNCH(gr->ctx, n2);
            return VB_OK;
        }
        int n = gr->precision == VB_MIXED
                    ? vb::launch_stage_tiled3d_mixed(&gr->box, nullptr, nullptr, (int)items, work,
                                                     st, gr->ctx->stream, grav, bf != nullptr)
                    : vb::launch_stage_tiled3d_fp64(&gr->box, nullptr, nullptr, (int)items, work,
                                                    st, gr->ctx->stream, grav, bf != nullptr);
        VB_CHECK_LAUNCH(gr->ctx, n);
        return VB_OK;
    }
    int n = gr->precision == VB_MIXED
                ? vb::launch_stage_mixed(gr->g, st, Uin, U0, Uout, gr->ctrl, bf, gr->ctx->stream, bfi)
                : vb::launch_stage_fp64(gr->g, st, Uin, U0, Uout, gr->ctrl, bf, gr->ctx->stream, bfi);
    VB_CHECK_LAUNCH(gr->ctx, n);
    return VB_OK;
}

// One RK2 step whose dt is already in the control block.
int rk2(vb_grid *gr)
{
    int rc = stage(gr, 1, gr->U, gr->U, gr->U1);
    if (rc) return rc;
    rc = stage(gr, 2, gr->U1, gr->U, gr->U);
    if (rc) return rc;
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_advance(gr->ctrl, gr->ctx->stream));
    gr->invdt_valid = true;
    return VB_OK;
}

int pull_ctrl(vb_grid *gr)
{
    VB_CUDA(cudaMemcpyAsync(gr->hctrl, gr->ctrl, sizeof(vb::Ctrl), cudaMemcpyDeviceToHost,
                            gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    return VB_OK;
}

int ensure_cfl(vb_grid *gr)
{
    if (gr->invdt_valid) return VB_OK;
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_cfl(gr->g, gr->U, gr->ctrl, gr->ctx->stream));
    gr->invdt_valid = true;
    return VB_OK;
}

// Queue `count` CFL-limited steps (each: finalize dt, stage 1, stage 2).  With
// self-gravity each active step first solves the Poisson problem for its
// starting density (evolve!, src/driver.jl:498; dt does not depend on phi,
// so finalising first is the same); that solve synchronises with the host.
int queue_direct(vb_grid *gr, int64_t count)
{
    for (int64_t i = 0; i < count; ++i) {
        VB_CHECK_LAUNCH(gr->ctx, vb::launch_finalize_cfl(gr->g, gr->ctrl, gr->ctx->stream));
        if (gr->grav) {
            int rc = pull_ctrl(gr);
            if (rc) return rc;
            if (!gr->hctrl->active) return VB_OK;
            rc = vb::detail::gravity_solve(gr, nullptr, nullptr);
            if (rc) return rc;
        }
        int rc = rk2(gr);
        if (rc) return rc;
    }
    return VB_OK;
}

constexpr int64_t GRAPH_STEPS = 8;

uint64_t graph_key(const vb_grid *gr)
{
    return (gr->tiled ? 1u : 0u) | (gr->bflux_on ? 2u : 0u) | (grid_taper(gr) ? 4u : 0u) |
           (gr->bflux_interior ? 8u : 0u) | ((uint64_t)gr->kz << 4);
}

// Capture GRAPH_STEPS steps into the grid's graph for its current configuration.
int capture_steps(vb_grid *gr)
{
    if (gr->gexec) {
        cudaGraphExecDestroy(gr->gexec);
        gr->gexec = nullptr;
    }
    cudaStream_t s = gr->ctx->stream;
    VB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int64_t before = gr->ctx->launches;
    int rc = queue_direct(gr, GRAPH_STEPS);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    const int64_t n = gr->ctx->launches - before;
    gr->ctx->launches = before;  // counted per replay
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(VB_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&gr->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        gr->gexec = nullptr;
        return fail(VB_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    gr->gkey = graph_key(gr);
    gr->glaunches = n;
    return VB_OK;
}

// Queue `count` CFL-limited steps (each: finalize dt, stage 1, stage 2,
// advance): whole groups of GRAPH_STEPS replay one captured graph, the rest
// launch directly.
int queue_steps(vb_grid *gr, int64_t count)
{
    while (gr->warmed && count >= GRAPH_STEPS && !gr->grav) {
        if (!gr->gexec || gr->gkey != graph_key(gr)) {
            int rc = capture_steps(gr);
            if (rc) return rc;
        }
        VB_CUDA(cudaGraphLaunch(gr->gexec, gr->ctx->stream));
        gr->ctx->launches += gr->glaunches;
        count -= GRAPH_STEPS;
    }
    if (count > 0) {
        int rc = queue_direct(gr, count);
        if (rc) return rc;
        gr->warmed = true;
    }
    return VB_OK;
}

// Host-side write of control fields (stream-ordered through a tiny copy).
int push_ctrl(vb_grid *gr)
{
    VB_CUDA(cudaMemcpyAsync(gr->ctrl, gr->hctrl, sizeof(vb::Ctrl), cudaMemcpyHostToDevice,
                            gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    return VB_OK;
}

}  // namespace

int vb::detail::grid_ensure_cfl(vb_grid *gr) { return ensure_cfl(gr); }
int vb::detail::grid_rk2(vb_grid *gr) { return rk2(gr); }
int vb::detail::grid_pull_ctrl(vb_grid *gr) { return pull_ctrl(gr); }
int vb::detail::grid_push_ctrl(vb_grid *gr) { return push_ctrl(gr); }

void vb::set_last_error(const char *msg) { g_err = msg; }

extern "C" {

int vb_abi_version(void) { return VB_ABI_VERSION; }

int vb_last_error(char *buf, size_t len)
{
    if (buf && len) {
        size_t n = g_err.size() < len - 1 ? g_err.size() : len - 1;
        std::memcpy(buf, g_err.data(), n);
        buf[n] = '\0';
    }
    return (int)g_err.size();
}

int vb_ctx_create(int device, vb_ctx **out)
{
    if (!out) return fail(VB_EINVAL, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(VB_ECUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return fail(VB_EINVAL, "device index out of range");
    VB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    VB_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10 || prop.minor != 0)
        return fail(VB_ENOTSUP, std::string("libvespa_b200 is built for sm_100a; device is ") +
                                    prop.name + " (sm_" + std::to_string(prop.major) +
                                    std::to_string(prop.minor) + ")");
    vb_ctx *ctx = new (std::nothrow) vb_ctx();
    if (!ctx) return fail(VB_ENOMEM, "host allocation failed");
    ctx->device = device;
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        return fail(VB_ECUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    {
        // scratch that comes and goes (autotuner copies, the AMR tables as
        // they grow) is allocated stream-ordered from the device's default
        // memory pool of this process; let the pool keep freed memory for
        // reuse instead of returning it at every synchronisation (a
        // cudaFree synchronises the whole device and at times took hundreds
        // of milliseconds)
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    }
    *out = ctx;
    return VB_OK;
}

int vb_ctx_destroy(vb_ctx *ctx)
{
    if (!ctx) return VB_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    for (cudaEvent_t &e : ctx->marks)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return VB_OK;
}

int vb_ctx_synchronize(vb_ctx *ctx)
{
    int rc = use(ctx);
    if (rc) return rc;
    VB_CUDA(cudaStreamSynchronize(ctx->stream));
    return VB_OK;
}

int vb_ctx_stream(vb_ctx *ctx, void **stream)
{
    if (!ctx || !stream) return fail(VB_EINVAL, "null argument");
    *stream = (void *)ctx->stream;
    return VB_OK;
}

int vb_ctx_launch_count(vb_ctx *ctx, int64_t *count)
{
    if (!ctx || !count) return fail(VB_EINVAL, "null argument");
    *count = ctx->launches;
    return VB_OK;
}

int vb_check_read(vb_ctx *ctx, int64_t *line)
{
    if (!ctx || !line) return fail(VB_EINVAL, "null argument");
#ifdef VB_CHECK
    int rc = use(ctx);
    if (rc) return rc;
    VB_CUDA(cudaStreamSynchronize(ctx->stream));
    unsigned int w = 0;
    std::lock_guard<std::mutex> lk(vb::check_mu());
    for (auto fn : vb::check_readers()) {
        const unsigned x = fn();
        if (!w) w = x;
    }
    *line = (int64_t)w;
#else
    *line = -1;  // a build without device bounds checks
#endif
    return VB_OK;
}

int vb_ctx_mark(vb_ctx *ctx, int slot)
{
    int rc = use(ctx);
    if (rc) return rc;
    if (slot < 0 || slot >= 16) return fail(VB_EINVAL, "slot must be in 0..15");
    if (!ctx->marks[slot]) VB_CUDA(cudaEventCreate(&ctx->marks[slot]));
    VB_CUDA(cudaEventRecord(ctx->marks[slot], ctx->stream));
    return VB_OK;
}

int vb_ctx_elapsed_ms(vb_ctx *ctx, int a, int b, float *ms)
{
    int rc = use(ctx);
    if (rc) return rc;
    if (!ms || a < 0 || a >= 16 || b < 0 || b >= 16 || !ctx->marks[a] || !ctx->marks[b])
        return fail(VB_EINVAL, "unrecorded mark or null output");
    VB_CUDA(cudaEventSynchronize(ctx->marks[b]));
    VB_CUDA(cudaEventElapsedTime(ms, ctx->marks[a], ctx->marks[b]));
    return VB_OK;
}

int vb_hllc_faces_device_async(vb_ctx *ctx, int64_t nf, const double *dWL, const double *dWR,
                               const int32_t *daxis, double gamma, double *dF)
{
    int rc = use(ctx);
    if (rc) return rc;
    if (nf < 0) return fail(VB_EINVAL, "nf < 0");
    if (nf == 0) return VB_OK;
    if (!dWL || !dWR || !daxis || !dF) return fail(VB_EINVAL, "null buffer");
    if (!(gamma > 1.0)) return fail(VB_EINVAL, "gamma must exceed 1");
    VB_CHECK_LAUNCH(ctx, vb::launch_hllc_faces(nf, dWL, dWR, daxis, gamma, dF, ctx->stream));
    return VB_OK;
}

int vb_hllc_faces(vb_ctx *ctx, int64_t nf, const double *WL, const double *WR,
                  const int32_t *axis, double gamma, double *F)
{
    VB_RANGE("vb_hllc_faces");
    int rc = use(ctx);
    if (rc) return rc;
    if (nf < 0) return fail(VB_EINVAL, "nf < 0");
    if (nf == 0) return VB_OK;  // the reference returns F untouched for nf == 0
    if (!WL || !WR || !axis || !F) return fail(VB_EINVAL, "null buffer");
    for (int64_t f = 0; f < nf; ++f)
        if (axis[f] < 1 || axis[f] > 3) return fail(VB_EINVAL, "axis entries must be 1, 2 or 3");
    const size_t bw = sizeof(double) * 5 * (size_t)nf;
    const size_t ba = sizeof(int32_t) * (size_t)nf;
    const size_t need = 3 * bw + ((ba + 255) & ~(size_t)255);
    void *scratch = nullptr;
    rc = vb::detail::ctx_scratch(ctx, need, &scratch);
    if (rc) return rc;
    char *base = (char *)scratch;
    double *dWL = (double *)base;
    double *dWR = (double *)(base + bw);
    double *dF = (double *)(base + 2 * bw);
    int32_t *dax = (int32_t *)(base + 3 * bw);
    VB_CUDA(cudaMemcpyAsync(dWL, WL, bw, cudaMemcpyHostToDevice, ctx->stream));
    VB_CUDA(cudaMemcpyAsync(dWR, WR, bw, cudaMemcpyHostToDevice, ctx->stream));
    VB_CUDA(cudaMemcpyAsync(dax, axis, ba, cudaMemcpyHostToDevice, ctx->stream));
    VB_CHECK_LAUNCH(ctx, vb::launch_hllc_faces(nf, dWL, dWR, dax, gamma, dF, ctx->stream));
    VB_CUDA(cudaMemcpyAsync(F, dF, bw, cudaMemcpyDeviceToHost, ctx->stream));
    VB_CUDA(cudaStreamSynchronize(ctx->stream));
    return VB_OK;
}

int vb_grid_create(vb_ctx *ctx, const vb_problem_desc *d, int precision, vb_grid **out)
{
    if (!out) return fail(VB_EINVAL, "null output pointer");
    *out = nullptr;
    int rc = use(ctx);
    if (rc) return rc;
    if (precision != VB_FP64 && precision != VB_MIXED) return fail(VB_EINVAL, "unknown precision");
    vb::Geom g{};
    rc = vb::detail::make_geom(d, &g);
    if (rc) return rc;

    vb_grid *gr = new (std::nothrow) vb_grid();
    if (!gr) return fail(VB_ENOMEM, "host allocation failed");
    gr->ctx = ctx;
    gr->g = g;
    gr->precision = precision;
    const size_t bytes = sizeof(double) * 5 * (size_t)g.ncell;
    auto cleanup = [&](int code, const std::string &msg) {
        vb_grid_destroy(gr);
        return fail(code, msg);
    };
    cudaError_t e;
    if ((e = cudaMalloc(&gr->U, bytes)) != cudaSuccess ||
        (e = cudaMalloc(&gr->U1, bytes)) != cudaSuccess ||
        (e = cudaMalloc(&gr->ctrl, sizeof(vb::Ctrl))) != cudaSuccess ||
        (e = cudaMalloc(&gr->partials, sizeof(double) * 5 * vb::TOTALS_PARTS)) != cudaSuccess ||
        (e = cudaMalloc(&gr->totals, sizeof(double) * 5)) != cudaSuccess ||
        (e = cudaMallocHost(&gr->hctrl, sizeof(vb::Ctrl))) != cudaSuccess ||
        (e = cudaMallocHost(&gr->htot, sizeof(double) * 5)) != cudaSuccess)
        return cleanup(VB_ENOMEM, std::string("grid allocation: ") + cudaGetErrorString(e));
    std::memset(gr->hctrl, 0, sizeof(vb::Ctrl));
    gr->hctrl->tfinal = INFINITY;
    gr->hctrl->step_limit = LLONG_MAX;
    if ((e = cudaMemsetAsync(gr->U, 0, bytes, ctx->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(gr->U1, 0, bytes, ctx->stream)) != cudaSuccess)
        return cleanup(VB_ECUDA, cudaGetErrorString(e));
    rc = push_ctrl(gr);
    if (rc) {
        std::string m = g_err;
        return cleanup(rc, m);
    }
    if (vb::tiled_supported(g)) {
        rc = encode_maps(&gr->maps_U, gr->U, g);
        if (!rc) rc = encode_maps(&gr->maps_U1, gr->U1, g);
        if (rc) {
            std::string m = g_err;
            return cleanup(rc, m);
        }
        gr->tiled = vb::detail::tiled_auto(g);
        gr->kz = vb::detail::grid_default_kz(g);
        std::lock_guard<std::mutex> lk(g_tune_mu);
        const std::string key = tune_key(ctx->device, g, precision);
        auto it = g_tune_kz.find(key);
        std::pair<int, int> v;
        if (it != g_tune_kz.end()) {
            gr->kz = it->second.first;
            gr->taper_tuned = it->second.second;
        } else if (tune_file_lookup(key, &v) && v.first <= vb::march_extent(g)) {
            gr->kz = v.first;
            gr->taper_tuned = v.second;
            g_tune_kz[key] = v;
        }
    }
    *out = gr;
    return VB_OK;
}

int vb_grid_autotune(vb_grid *gr, int nsteps, int64_t *best_kz, double *best_ms)
{
    VB_RANGE("vb_grid_autotune");
    if (!gr || nsteps < 1) return fail(VB_EINVAL, "bad argument");
    int rc = use(gr->ctx);
    if (rc) return rc;
    if (!gr->tiled || gr->bflux_on || gr->grav) {
        if (best_kz) *best_kz = gr->kz;
        if (best_ms) *best_ms = 0.0;
        return VB_OK;
    }
    const size_t bytes = sizeof(double) * 5 * (size_t)gr->g.ncell;
    double *save = nullptr;
    VB_CUDA(cudaMallocAsync(&save, bytes, gr->ctx->stream));
    cudaStream_t s = gr->ctx->stream;
    rc = pull_ctrl(gr);
    vb::Ctrl ctrl0 = *gr->hctrl;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int best = gr->kz, best_taper = gr->taper_tuned;
    float best_t = INFINITY;
    if (!rc && (cudaMemcpyAsync(save, gr->U, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
                cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = fail(VB_ECUDA, "autotune setup failed");
    // candidates: z chunk (3D planes / 2D rows) and, in 3D when the caller
    // left VB_OPT_TILE_TAPER at its default, uniform or tapered work queues
    const int cand[] = {16, 24, 32, 40, 48, 64, 96, 128};
    const int ntaper = (gr->g.nd == 3 && gr->taper < 0) ? 2 : 1;
    for (int ci = 0; ci < 8 * ntaper; ++ci) {
        const int kz = cand[ci % 8];
        if (rc) break;
        if (kz > vb::march_extent(gr->g)) continue;
        gr->kz = kz;
        if (ntaper == 2) gr->taper_tuned = ci / 8;
        rc = ensure_cfl(gr);
        if (!rc) rc = queue_steps(gr, 1);  // warm-up
        // capture this chunk's step graph before the timed region, so that
        // only graph replays are timed (capture and instantiation are host
        // work that would leave the stream idle between the events)
        if (!rc && nsteps >= GRAPH_STEPS && !gr->grav &&
            (!gr->gexec || gr->gkey != graph_key(gr)))
            rc = capture_steps(gr);
        if (rc) break;
        cudaEventRecord(e0, s);
        rc = queue_steps(gr, nsteps);
        cudaEventRecord(e1, s);
        if (rc) break;
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = fail(VB_ECUDA, "autotune timing failed");
            break;
        }
        if (ms < best_t) {
            best_t = ms;
            best = kz;
            best_taper = gr->taper_tuned;
        }
    }
    // restore the state and the clock whatever happened
    cudaMemcpyAsync(gr->U, save, bytes, cudaMemcpyDeviceToDevice, s);
    *gr->hctrl = ctrl0;
    int rc2 = push_ctrl(gr);
    cudaFreeAsync(save, s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    gr->invdt_valid = false;
    gr->kz = best;
    gr->taper_tuned = best_taper;
    if (rc) return rc;
    if (rc2) return rc2;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        const std::string key = tune_key(gr->ctx->device, gr->g, gr->precision);
        g_tune_kz[key] = {best, best_taper};
        tune_file_append(key, best, best_taper);
    }
    if (best_kz) *best_kz = best;
    if (best_ms) *best_ms = best_t / nsteps;
    return VB_OK;
}

int vb_grid_set_option(vb_grid *gr, int option, int64_t value)
{
    if (!gr) return fail(VB_EINVAL, "null grid");
    switch (option) {
    case VB_OPT_KERNEL:
        if (value == VB_KERNEL_CELL) {
            gr->tiled = false;
        } else if (value == VB_KERNEL_AUTO || value == VB_KERNEL_TILED) {
            if (!vb::tiled_supported(gr->g)) {
                if (value == VB_KERNEL_TILED)
                    return fail(VB_ENOTSUP, "tiled kernels need a 3D grid with nx, ny multiples of "
                                            "16 or a 2D grid with nx a multiple of 256");
                gr->tiled = false;
                return VB_OK;
            }
            if (!gr->maps_U.in_int.opaque[0] && !gr->maps_U.in_int.opaque[1]) {
                int rc = encode_maps(&gr->maps_U, gr->U, gr->g);
                if (!rc) rc = encode_maps(&gr->maps_U1, gr->U1, gr->g);
                if (rc) return rc;
            }
            gr->tiled = value == VB_KERNEL_TILED || vb::detail::tiled_auto(gr->g);
        } else {
            return fail(VB_EINVAL, "unknown kernel selector");
        }
        return VB_OK;
    case VB_OPT_TILE_KZ:
        if (value < 1 || value > vb::march_extent(gr->g))
            return fail(VB_EINVAL, "the chunk must be in 1..nz (3D) or 1..ny (2D)");
        gr->kz = (int)value;
        return VB_OK;
    case VB_OPT_TILE_TAPER:
        if (value < -1 || value > 1) return fail(VB_EINVAL, "taper must be -1 (auto), 0 or 1");
        gr->taper = (int)value;
        return VB_OK;
    default:
        return fail(VB_EINVAL, "unknown option");
    }
}

int vb_grid_get_option(const vb_grid *gr, int option, int64_t *value)
{
    if (!gr || !value) return fail(VB_EINVAL, "null argument");
    switch (option) {
    case VB_OPT_KERNEL: *value = gr->tiled ? VB_KERNEL_TILED : VB_KERNEL_CELL; return VB_OK;
    case VB_OPT_TILE_KZ: *value = gr->kz; return VB_OK;
    case VB_OPT_TILE_TAPER: *value = grid_taper(gr) ? 1 : 0; return VB_OK;
    default: return fail(VB_EINVAL, "unknown option");
    }
}

int vb_grid_destroy(vb_grid *gr)
{
    if (!gr) return VB_OK;
    if (gr->ctx) {
        cudaSetDevice(gr->ctx->device);
        cudaStreamSynchronize(gr->ctx->stream);
    }
    if (gr->gexec) cudaGraphExecDestroy(gr->gexec);
    vb::detail::gravity_free(gr->grav);
    cudaFree(gr->U);
    cudaFree(gr->U1);
    cudaFree(gr->ctrl);
    cudaFree(gr->partials);
    cudaFree(gr->totals);
    cudaFree(gr->bflux);
    cudaFreeHost(gr->hctrl);
    cudaFreeHost(gr->htot);
    delete gr;
    return VB_OK;
}

int vb_grid_ncell(const vb_grid *gr, int64_t *n)
{
    if (!gr || !n) return fail(VB_EINVAL, "null argument");
    *n = gr->g.ncell;
    return VB_OK;
}

int vb_grid_upload(vb_grid *gr, const double *U)
{
    VB_RANGE("vb_grid_upload");
    if (!gr || !U) return fail(VB_EINVAL, "null argument");
    int rc = use(gr->ctx);
    if (rc) return rc;
    VB_CUDA(cudaMemcpyAsync(gr->U, U, sizeof(double) * 5 * (size_t)gr->g.ncell,
                            cudaMemcpyHostToDevice, gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    gr->invdt_valid = false;
    return VB_OK;
}

int vb_grid_download(vb_grid *gr, double *U)
{
    VB_RANGE("vb_grid_download");
    if (!gr || !U) return fail(VB_EINVAL, "null argument");
    int rc = use(gr->ctx);
    if (rc) return rc;
    VB_CUDA(cudaMemcpyAsync(U, gr->U, sizeof(double) * 5 * (size_t)gr->g.ncell,
                            cudaMemcpyDeviceToHost, gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    return VB_OK;
}

int vb_grid_device_state(vb_grid *gr, double **dU)
{
    if (!gr || !dU) return fail(VB_EINVAL, "null argument");
    *dU = gr->U;
    gr->invdt_valid = false;  // the caller may write through the pointer
    return VB_OK;
}

int vb_grid_set_time(vb_grid *gr, double t, int64_t step)
{
    if (!gr) return fail(VB_EINVAL, "null grid");
    int rc = use(gr->ctx);
    if (rc) return rc;
    rc = pull_ctrl(gr);
    if (rc) return rc;
    gr->hctrl->t = t;
    gr->hctrl->step = step;
    return push_ctrl(gr);
}

int vb_grid_get_time(vb_grid *gr, double *t, int64_t *step)
{
    if (!gr) return fail(VB_EINVAL, "null grid");
    int rc = use(gr->ctx);
    if (rc) return rc;
    rc = pull_ctrl(gr);
    if (rc) return rc;
    if (t) *t = gr->hctrl->t;
    if (step) *step = gr->hctrl->step;
    return VB_OK;
}

int vb_compute_dt(vb_grid *gr, double *dt)
{
    VB_RANGE("vb_compute_dt");
    if (!gr || !dt) return fail(VB_EINVAL, "null argument");
    int rc = use(gr->ctx);
    if (rc) return rc;
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_cfl(gr->g, gr->U, gr->ctrl, gr->ctx->stream));
    gr->invdt_valid = true;
    rc = pull_ctrl(gr);
    if (rc) return rc;
    unsigned long long bits = gr->hctrl->invdt_bits;
    double invdt;
    std::memcpy(&invdt, &bits, sizeof invdt);
    if (std::isnan(invdt)) {
        *dt = NAN;
        return fail(VB_ENONFINITE, "non-finite or negative density/pressure in the state");
    }
    *dt = invdt == 0.0 ? INFINITY : gr->g.cfl / invdt;
    return VB_OK;
}

int vb_grid_set_zwindow(vb_grid *gr, int64_t zw0, int64_t zw1, int zcls0, double wz)
{
    if (!gr) return fail(VB_EINVAL, "null grid");
    vb::Geom &g = gr->g;
    if (g.nd != 3 || !gr->tiled)
        return fail(VB_ENOTSUP, "z windows need a 3D grid on the tiled kernel");
    if (!(zw0 >= 0 && zw0 < zw1 && zw1 <= g.n[2])) return fail(VB_EINVAL, "need 0 <= zw0 < zw1 <= nz");
    if (zcls0 < -1 || zcls0 > 2) return fail(VB_EINVAL, "zcls0 must be -1, 0, 1 or 2");
    if (!(wz > 0.0) || !std::isfinite(wz)) return fail(VB_EINVAL, "wz must be positive");
    if (gr->grav || gr->bflux_on)
        return fail(VB_ENOTSUP, "z windows exclude self-gravity and boundary-flux recording");
    // the z width of the whole domain, and the areas and volume derived from
    // it as the grid's own geometry derives them (product in axis order)
    g.w[2] = wz;
    g.invw[2] = 1.0 / wz;
    for (int a = 0; a < 3; ++a) {
        double ar = 1.0;
        for (int e = 0; e < 3; ++e)
            if (e != a) ar *= g.w[e];
        g.area[a] = ar;
    }
    g.vol = (g.w[0] * g.w[1]) * g.w[2];
    g.zw0 = (int)zw0;
    g.zw1 = (int)zw1;
    g.zcls0 = zcls0;
    g.act0 = zw0 * g.n[0] * g.n[1];
    g.act1 = zw1 * g.n[0] * g.n[1];
    gr->slab = true;
    gr->box_kz = -1;        // the box descriptor carries the geometry
    gr->invdt_valid = false;
    if (gr->gexec) {        // captured launches hold the old geometry
        cudaGraphExecDestroy(gr->gexec);
        gr->gexec = nullptr;
    }
    return VB_OK;
}

int vb_grid_step_phase(vb_grid *gr, int phase)
{
    VB_RANGE("vb_grid_step_phase");
    if (!gr) return fail(VB_EINVAL, "null grid");
    int rc = use(gr->ctx);
    if (rc) return rc;
    cudaStream_t s = gr->ctx->stream;
    switch (phase) {
    case VB_PHASE_CFL: return ensure_cfl(gr);
    case VB_PHASE_FINALIZE:
        VB_CHECK_LAUNCH(gr->ctx, vb::launch_finalize_cfl(gr->g, gr->ctrl, s));
        return VB_OK;
    case VB_PHASE_STAGE1: return stage(gr, 1, gr->U, gr->U, gr->U1);
    case VB_PHASE_STAGE2: return stage(gr, 2, gr->U1, gr->U, gr->U);
    case VB_PHASE_ADVANCE:
        VB_CHECK_LAUNCH(gr->ctx, vb::launch_advance(gr->ctrl, s));
        gr->invdt_valid = true;  // stage 2 folded the new state's CFL maximum
        return VB_OK;
    default: return fail(VB_EINVAL, "unknown phase");
    }
}

int vb_grid_planes(vb_grid *gr, int which, int64_t z0, int64_t n, void *dev, int put)
{
    VB_RANGE("vb_grid_planes");
    if (!gr || !dev) return fail(VB_EINVAL, "null argument");
    if (which != 0 && which != 1) return fail(VB_EINVAL, "which must be 0 (state) or 1 (stage-1 state)");
    const vb::Geom &g = gr->g;
    if (g.nd != 3 || z0 < 0 || n < 1 || z0 + n > g.n[2]) return fail(VB_EINVAL, "planes out of range");
    int rc = use(gr->ctx);
    if (rc) return rc;
    double *buf = (which ? gr->U1 : gr->U) + z0 * g.n[0] * g.n[1];
    const size_t width = sizeof(double) * (size_t)(n * g.n[0] * g.n[1]);
    const size_t pitch = sizeof(double) * (size_t)g.ncell;
    if (put)
        VB_CUDA(cudaMemcpy2DAsync(buf, pitch, dev, width, width, 5, cudaMemcpyDeviceToDevice,
                                  gr->ctx->stream));
    else
        VB_CUDA(cudaMemcpy2DAsync(dev, width, buf, pitch, width, 5, cudaMemcpyDeviceToDevice,
                                  gr->ctx->stream));
    return VB_OK;
}

int vb_grid_cfl_bits(vb_grid *gr, void *dev, int put)
{
    if (!gr || !dev) return fail(VB_EINVAL, "null argument");
    int rc = use(gr->ctx);
    if (rc) return rc;
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_cfl_bits(gr->ctrl, (unsigned long long *)dev, put ? 1 : 0,
                                                 gr->ctx->stream));
    return VB_OK;
}

int vb_grid_selftest_wait(vb_grid *gr, int64_t limit_ns)
{
    if (!gr) return fail(VB_EINVAL, "null grid");
    if (limit_ns < 1000 || limit_ns > 10000000000LL)
        return fail(VB_EINVAL, "limit_ns must be in [1e3, 1e10]");
    int rc = use(gr->ctx);
    if (rc) return rc;
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_wait_selftest(gr->ctrl, (uint64_t)limit_ns, gr->ctx->stream));
    rc = pull_ctrl(gr);
    if (rc) return rc;
    if (!(gr->hctrl->flags & vb::CTRL_F_TIMEOUT)) return fail(VB_ECUDA, "the self-test wait did not give up");
    // report as a stage would, and leave the grid usable
    gr->hctrl->flags &= ~vb::CTRL_F_TIMEOUT;
    rc = push_ctrl(gr);
    if (rc) return rc;
    return fail(VB_ETIMEOUT, "a bounded device wait (TMA stage load) gave up");
}

int vb_step(vb_grid *gr, double dt)
{
    VB_RANGE("vb_step");
    if (!gr) return fail(VB_EINVAL, "null grid");
    int rc = use(gr->ctx);
    if (rc) return rc;
    if (!std::isfinite(dt)) return fail(VB_EINVAL, "dt must be finite");
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_set_dt(gr->g, gr->ctrl, dt, gr->ctx->stream));
    rc = rk2(gr);
    if (rc) return rc;
    rc = pull_ctrl(gr);
    if (rc) return rc;
    if (gr->hctrl->flags & vb::CTRL_F_TIMEOUT)
        return fail(VB_ETIMEOUT, "a bounded device wait (TMA stage load) gave up");
    return VB_OK;
}

int vb_run_steps_async(vb_grid *gr, int64_t nsteps)
{
    VB_RANGE("vb_run_steps_async");
    if (!gr) return fail(VB_EINVAL, "null grid");
    if (nsteps < 0) return fail(VB_EINVAL, "nsteps < 0");
    int rc = use(gr->ctx);
    if (rc) return rc;
    rc = ensure_cfl(gr);
    if (rc) return rc;
    return queue_steps(gr, nsteps);
}

int vb_evolve(vb_grid *gr, double tfinal, int64_t max_steps, double *t, int64_t *nsteps)
{
    VB_RANGE("vb_evolve");
    if (!gr) return fail(VB_EINVAL, "null grid");
    int rc = use(gr->ctx);
    if (rc) return rc;
    rc = pull_ctrl(gr);
    if (rc) return rc;
    const long long step0 = gr->hctrl->step;
    gr->hctrl->tfinal = tfinal;
    gr->hctrl->step_limit = max_steps < 0 ? LLONG_MAX : step0 + max_steps;
    gr->hctrl->flags = 0;
    gr->hctrl->active = 1;
    rc = push_ctrl(gr);
    if (rc) return rc;
    rc = ensure_cfl(gr);
    if (rc) return rc;
    // chunks of steps between host checks of the control block
    int64_t chunk = 8;
    int status = VB_OK;
    for (;;) {
        rc = queue_steps(gr, chunk);
        if (rc) return rc;
        rc = pull_ctrl(gr);
        if (rc) return rc;
        if (gr->hctrl->flags & vb::CTRL_F_NONFINITE) {
            status = fail(VB_ENONFINITE, "non-finite dt: NaN or negative density/pressure");
            break;
        }
        if (gr->hctrl->flags & vb::CTRL_F_TIMEOUT) {
            status = fail(VB_ETIMEOUT, "a bounded device wait (TMA stage load) gave up");
            break;
        }
        if (!gr->hctrl->active) break;
        if (chunk < 64) chunk *= 2;
    }
    if (t) *t = gr->hctrl->t;
    if (nsteps) *nsteps = gr->hctrl->step - step0;
    gr->hctrl->tfinal = INFINITY;
    gr->hctrl->step_limit = LLONG_MAX;
    gr->hctrl->active = 0;
    rc = push_ctrl(gr);
    return status ? status : rc;
}

int vb_conserved_totals(vb_grid *gr, double out[5])
{
    VB_RANGE("vb_conserved_totals");
    if (!gr || !out) return fail(VB_EINVAL, "null argument");
    int rc = use(gr->ctx);
    if (rc) return rc;
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_totals(gr->g, gr->U, gr->partials, vb::TOTALS_PARTS,
                                               gr->totals, gr->ctx->stream));
    VB_CUDA(cudaMemcpyAsync(gr->htot, gr->totals, sizeof(double) * 5, cudaMemcpyDeviceToHost,
                            gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    std::memcpy(out, gr->htot, sizeof(double) * 5);
    return VB_OK;
}

int vb_grid_profile_step(vb_grid *gr, int nsteps, double *ms_fin, double *ms_s1, double *ms_s2)
{
    if (!gr || nsteps <= 0) return fail(VB_EINVAL, "bad argument");
    int rc = use(gr->ctx);
    if (rc) return rc;
    rc = ensure_cfl(gr);
    if (rc) return rc;
    cudaEvent_t ev[4];
    for (auto &e : ev) VB_CUDA(cudaEventCreate(&e));
    double acc[3] = {0, 0, 0};
    cudaStream_t s = gr->ctx->stream;
    for (int i = 0; i < nsteps && rc == VB_OK; ++i) {
        cudaEventRecord(ev[0], s);
        VB_CHECK_LAUNCH(gr->ctx, vb::launch_finalize_cfl(gr->g, gr->ctrl, s));
        cudaEventRecord(ev[1], s);
        rc = stage(gr, 1, gr->U, gr->U, gr->U1);
        cudaEventRecord(ev[2], s);
        if (rc == VB_OK) rc = stage(gr, 2, gr->U1, gr->U, gr->U);
        cudaEventRecord(ev[3], s);
        cudaEventSynchronize(ev[3]);
        float m;
        for (int k = 0; k < 3; ++k) {
            cudaEventElapsedTime(&m, ev[k], ev[k + 1]);
            acc[k] += m;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    if (ms_fin) *ms_fin = acc[0] / nsteps;
    if (ms_s1) *ms_s1 = acc[1] / nsteps;
    if (ms_s2) *ms_s2 = acc[2] / nsteps;
    return VB_OK;
}

namespace {
int64_t bflux_outer_size(const vb::Geom &g)
{
    int64_t s = 0;
    for (int a = 0; a < g.nd; ++a) s += 2 * 5 * (g.ncell / g.n[a]);
    return s;
}
}  // namespace

int vb_bflux_size(const vb_grid *gr, int64_t *n)
{
    if (!gr || !n) return fail(VB_EINVAL, "null argument");
    *n = gr->bflux ? gr->bflux_n : bflux_outer_size(gr->g);
    return VB_OK;
}

int vb_bflux_enable(vb_grid *gr, int enable)
{
    if (!gr) return fail(VB_EINVAL, "null grid");
    if (enable < VB_BFLUX_OFF || enable > VB_BFLUX_INTERIOR)
        return fail(VB_EINVAL, "enable must be VB_BFLUX_OFF, VB_BFLUX_OUTER or VB_BFLUX_INTERIOR");
    int rc = use(gr->ctx);
    if (rc) return rc;
    const bool interior = enable == VB_BFLUX_INTERIOR;
    if (enable != VB_BFLUX_OFF && (!gr->bflux || interior != gr->bflux_interior)) {
        // (re)allocate the register for this layout, zeroed
        const int64_t outer = bflux_outer_size(gr->g);
        const int64_t n = outer + (interior ? (int64_t)gr->g.nd * 5 * gr->g.ncell : 0);
        double *p = nullptr;
        VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
        VB_CUDA(cudaMalloc(&p, sizeof(double) * (size_t)n));
        cudaFree(gr->bflux);
        gr->bflux = p;
        gr->bflux_n = n;
        gr->bflux_outer_n = outer;
        gr->bflux_interior = interior;
        VB_CUDA(cudaMemsetAsync(gr->bflux, 0, sizeof(double) * (size_t)n, gr->ctx->stream));
        VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    }
    gr->bflux_on = enable != VB_BFLUX_OFF;
    return VB_OK;
}

int vb_bflux_plane(vb_grid *gr, int dim, int source, const int64_t *start, const int64_t *stop,
                   const int64_t *g0, int64_t flux_off, int comp, double vcell, double *out,
                   int64_t n)
{
    VB_RANGE("vb_bflux_plane");
    if (!gr || !start || !stop || !g0 || (!out && n > 0)) return fail(VB_EINVAL, "null argument");
    if (!gr->bflux) return fail(VB_EINVAL, "boundary-flux register not enabled");
    const int R = gr->g.nd;
    if (dim < 0 || dim >= R) return fail(VB_EINVAL, "dim must be in 0..ndim-1");
    if (source < VB_BFLUX_PLANE_LO || source > VB_BFLUX_PLANE_INTERIOR)
        return fail(VB_EINVAL, "unknown plane source");
    if (source == VB_BFLUX_PLANE_INTERIOR && !gr->bflux_interior)
        return fail(VB_EINVAL, "the register does not record interior faces (VB_BFLUX_INTERIOR)");
    if (comp > 5) return fail(VB_EINVAL, "comp must be at most 5 (comp <= 0 gives zeros)");
    int64_t cnt = 1;
    for (int d = 0; d < R; ++d) {
        if (stop[d] < start[d]) return fail(VB_EINVAL, "stop must not be below start");
        cnt *= stop[d] - start[d] + 1;
    }
    if (n != cnt) return fail(VB_EINVAL, "n must equal the plane's cell count");
    if (n == 0) return VB_OK;
    int rc = use(gr->ctx);
    if (rc) return rc;
    double *d_out = nullptr;
    rc = vb::detail::ctx_scratch(gr->ctx, sizeof(double) * (size_t)n, (void **)&d_out);
    if (rc) return rc;
    vb::PlaneSpec ps{};
    ps.R = R;
    ps.dim = dim;
    ps.source = source;
    for (int d = 0; d < R; ++d) {
        ps.start[d] = start[d];
        ps.dims[d] = stop[d] - start[d] + 1;
        ps.g0[d] = g0[d];
    }
    ps.flux_off = flux_off;
    ps.comp = comp;
    ps.vcell = vcell;
    VB_CHECK_LAUNCH(gr->ctx, vb::launch_bflux_plane(gr->g, gr->bflux, gr->bflux_outer_n, ps, d_out, n,
                                                    gr->ctx->stream));
    VB_CUDA(cudaMemcpyAsync(out, d_out, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost,
                            gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    return VB_OK;
}

int vb_bflux_read(vb_grid *gr, double *out, int64_t n)
{
    if (!gr || !out) return fail(VB_EINVAL, "null argument");
    if (!gr->bflux) return fail(VB_EINVAL, "boundary-flux register not enabled");
    if (n != gr->bflux_n) return fail(VB_EINVAL, "size mismatch (see vb_bflux_size)");
    int rc = use(gr->ctx);
    if (rc) return rc;
    VB_CUDA(cudaMemcpyAsync(out, gr->bflux, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost,
                            gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    return VB_OK;
}

int vb_bflux_clear(vb_grid *gr)
{
    if (!gr) return fail(VB_EINVAL, "null grid");
    if (!gr->bflux) return VB_OK;
    int rc = use(gr->ctx);
    if (rc) return rc;
    VB_CUDA(cudaMemsetAsync(gr->bflux, 0, sizeof(double) * (size_t)gr->bflux_n, gr->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(gr->ctx->stream));
    return VB_OK;
}

}  // extern "C"
