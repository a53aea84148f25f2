// vb_amr.cu -- the extern "C" AMR API: a composite leaf-only mesh over a base
// grid (lib/HGBackend/src/HGBackend.jl), its regrid (src/driver.jl:400-462)
// and the single-rate and subcycled drivers (src/driver.jl:483-605,
// src/reflux.jl:51-103), with the stepping on the device.
//
// Host side: the cell tree (leaves keyed by level and integer coordinates),
// 2:1 face balance on refinement, depth-first leaf order, and the tables the
// kernels read (representative neighbours, faces in emission order, per-leaf
// CSR of face contributions).  The tables are rebuilt after each regrid;
// between regrids every step runs on the device.
//
// Choices where the reference defers to HierarchicalGrids.jl (absent here):
// the base grid is a forest of roots in column-major order, children are
// ordered x fastest (x + 2y + 4z), the representative of a face with finer
// leaves is the first of them in that order, and balance is across faces.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <unordered_map>
#include <vector>

#include "vb_amr.h"
#include "vb_internal.h"

using vb::detail::fail;
using vb::detail::use;

namespace {

constexpr int CBITS = 20;  // bits per integer coordinate in a leaf key

struct Tree {
    int nd = 1;
    int64_t base[3] = {1, 1, 1};
    int bc_lo[3] = {0, 0, 0}, bc_hi[3] = {0, 0, 0};
    std::vector<int> lev;
    std::vector<int64_t> cx;  // 3 per leaf
    std::unordered_map<uint64_t, int> index;

    static uint64_t key(int l, const int64_t *c)
    {
        return ((uint64_t)l << 60) | ((uint64_t)c[0] << 40) | ((uint64_t)c[1] << 20) | (uint64_t)c[2];
    }
    int find(int l, const int64_t *c) const
    {
        auto it = index.find(key(l, c));
        return it == index.end() ? -1 : it->second;
    }
    int64_t n() const { return (int64_t)lev.size(); }

    uint64_t dfs_key(int l, const int64_t *c) const
    {
        uint64_t root = 0, mul = 1;
        for (int d = 0; d < nd; ++d) {
            root += (uint64_t)(c[d] >> l) * mul;
            mul *= (uint64_t)base[d];
        }
        uint64_t path = 0;
        for (int k = vb::AMR_MAX_LEVEL - 1; k >= 0; --k) {
            uint64_t digit = 0;
            for (int d = 0; d < nd; ++d) {
                const uint64_t s = (uint64_t)(c[d] & ((1LL << l) - 1)) << (vb::AMR_MAX_LEVEL - l);
                digit |= ((s >> k) & 1u) << d;
            }
            path = (path << nd) | digit;
        }
        return (root << (nd * vb::AMR_MAX_LEVEL)) | path;
    }

    // adjacent same-level coordinates across (d, hi); false at a non-periodic edge
    bool adjacent(int l, const int64_t *c, int d, bool hi, int64_t *cc) const
    {
        cc[0] = c[0];
        cc[1] = c[1];
        cc[2] = c[2];
        const int64_t nmax = base[d] << l;
        cc[d] += hi ? 1 : -1;
        if (cc[d] < 0 || cc[d] >= nmax) {
            if ((hi ? bc_hi[d] : bc_lo[d]) != vb::BC_PERIODIC) return false;
            cc[d] = (cc[d] + nmax) % nmax;
        }
        return true;
    }

    // 0 boundary, 1 same level, 2 coarser, 3 finer; *rep representative
    int neighbor(int i, int d, bool hi, int *rep) const
    {
        const int l = lev[i];
        int64_t cc[3];
        if (!adjacent(l, &cx[3 * i], d, hi, cc)) return 0;
        int j = find(l, cc);
        if (j >= 0) { *rep = j; return 1; }
        if (l > 0) {
            const int64_t cp[3] = {cc[0] >> 1, cc[1] >> 1, cc[2] >> 1};
            j = find(l - 1, cp);
            if (j >= 0) { *rep = j; return 2; }
        }
        int64_t cf[3] = {2 * cc[0], 2 * cc[1], 2 * cc[2]};
        if (!hi) cf[d] += 1;
        *rep = find(l + 1, cf);
        return 3;
    }
};

// One refinement batch: live cells keyed by coordinates, each remembering the
// pre-batch leaf whose cell mean it inherits.
struct Batch {
    const Tree &t;
    std::unordered_map<uint64_t, int> live;  // key -> slot
    std::vector<int> lev;
    std::vector<int64_t> cx;
    std::vector<int> src;
    std::vector<char> dead;
    int err = 0;

    explicit Batch(const Tree &tree) : t(tree)
    {
        const int64_t n = t.n();
        lev = t.lev;
        cx = t.cx;
        src.resize(n);
        dead.assign(n, 0);
        for (int64_t i = 0; i < n; ++i) {
            src[i] = (int)i;
            live[Tree::key(lev[i], &cx[3 * i])] = (int)i;
        }
    }
    int get(int l, const int64_t *c) const
    {
        auto it = live.find(Tree::key(l, c));
        return it == live.end() ? -1 : it->second;
    }
    // refine (l, c) after refining coarser face neighbours (2:1 balance)
    void refine(int l, const int64_t *c)
    {
        if (get(l, c) < 0) return;
        for (int d = 0; d < t.nd; ++d)
            for (int hi = 0; hi < 2; ++hi) {
                int64_t cc[3];
                if (l == 0 || !t.adjacent(l, c, d, hi, cc)) continue;
                if (get(l, cc) >= 0) continue;
                const int64_t cp[3] = {cc[0] >> 1, cc[1] >> 1, cc[2] >> 1};
                if (get(l - 1, cp) >= 0) refine(l - 1, cp);
            }
        const int s = get(l, c);
        if (s < 0) return;
        for (int d = 0; d < t.nd; ++d)
            if ((t.base[d] << (l + 1)) >= (1LL << CBITS)) err = 1;
        if (l + 1 > vb::AMR_MAX_LEVEL) err = 1;
        if (err) return;
        live.erase(Tree::key(l, c));
        dead[s] = 1;
        const int nch = 1 << t.nd;
        for (int ch = 0; ch < nch; ++ch) {
            int64_t k[3] = {0, 0, 0};
            for (int d = 0; d < t.nd; ++d) k[d] = 2 * c[d] + ((ch >> d) & 1);
            const int slot = (int)lev.size();
            lev.push_back(l + 1);
            cx.insert(cx.end(), k, k + 3);
            src.push_back(src[s]);
            dead.push_back(0);
            live[Tree::key(l + 1, k)] = slot;
        }
    }
};

}  // namespace

struct vb_amr {
    vb_ctx *ctx = nullptr;
    vb::Geom g{};  // base geometry: nd, bcs, gamma, cfl, aexp (cells per axis = base)
    Tree tree;
    double w0[3] = {1, 1, 1};
    double t = 0.0;
    int64_t step = 0;
    // device buffers
    int64_t cap = 0, fcap = 0, ecap = 0;
    double *U = nullptr, *U1 = nullptr, *F = nullptr, *reg = nullptr;
    int *lev = nullptr, *rep = nullptr, *fL = nullptr, *fR = nullptr, *off = nullptr, *ent = nullptr;
    int8_t *fax = nullptr;
    double *farea = nullptr;
    uint8_t *tag = nullptr;
    vb::Ctrl *ctrl = nullptr, *hctrl = nullptr;
    double *partials = nullptr, *totals = nullptr, *htot = nullptr;
    int nface = 0;
    vb::AmrDev dev{};
    double ms_regrid = 0.0;  // host wall time of the last evolve's regrids
};

namespace {

double level_width(const vb_amr *a, int l, int d) { return a->w0[d] * std::ldexp(1.0, -l); }

void release(vb_amr *a)
{
    cudaFree(a->U);
    cudaFree(a->U1);
    cudaFree(a->F);
    cudaFree(a->reg);
    cudaFree(a->lev);
    cudaFree(a->rep);
    cudaFree(a->fL);
    cudaFree(a->fR);
    cudaFree(a->off);
    cudaFree(a->ent);
    cudaFree(a->fax);
    cudaFree(a->farea);
    cudaFree(a->tag);
    cudaFree(a->ctrl);
    cudaFree(a->partials);
    cudaFree(a->totals);
    cudaFreeHost(a->hctrl);
    cudaFreeHost(a->htot);
}

template <typename T>
int realloc_dev(T **p, int64_t count)
{
    cudaFree(*p);
    *p = nullptr;
    VB_CUDA(cudaMalloc((void **)p, sizeof(T) * (size_t)(count > 0 ? count : 1)));
    return VB_OK;
}

// Build the kernels' tables from the tree and upload them.
int build_tables(vb_amr *a)
{
    const Tree &t = a->tree;
    const int n = (int)t.n(), nd = t.nd;
    std::vector<int> rep((size_t)6 * a->cap, -1);
    std::vector<int> fL, fR;
    std::vector<int8_t> fax;
    std::vector<double> farea;
    std::vector<std::vector<int>> lists((size_t)n);
    auto emit = [&](int L, int R, int d, double area) {
        const int f = (int)fL.size();
        fL.push_back(L);
        fR.push_back(R);
        fax.push_back((int8_t)d);
        farea.push_back(area);
        if (L >= 0) lists[L].push_back(2 * f);
        if (R >= 0) lists[R].push_back(2 * f + 1);
    };
    for (int i = 0; i < n; ++i) {
        const int li = t.lev[i];
        for (int d = 0; d < nd; ++d) {
            for (int hi = 0; hi < 2; ++hi) {
                int j = -1;
                if (t.neighbor(i, d, hi, &j)) rep[(size_t)(2 * d + hi) * a->cap + i] = j;
            }
            double area = 1.0;
            for (int e = 0; e < nd; ++e)
                if (e != d) area = area * level_width(a, li, e);
            int j = -1;
            int kind = t.neighbor(i, d, true, &j);
            if (kind == 0) emit(i, -1, d, area);
            else if (kind != 3) emit(i, j, d, area);
            kind = t.neighbor(i, d, false, &j);
            if (kind == 0) emit(-1, i, d, area);
            else if (kind == 2) emit(j, i, d, area);
        }
    }
    std::vector<int> off((size_t)n + 1, 0), ent;
    for (int i = 0; i < n; ++i) {
        off[i + 1] = off[i] + (int)lists[i].size();
        ent.insert(ent.end(), lists[i].begin(), lists[i].end());
    }
    const int nf = (int)fL.size();
    if (nf > a->fcap) {
        int64_t c = a->fcap ? a->fcap : 1024;
        while (c < nf) c *= 2;
        int rc = realloc_dev(&a->fL, c);
        if (!rc) rc = realloc_dev(&a->fR, c);
        if (!rc) rc = realloc_dev(&a->fax, c);
        if (!rc) rc = realloc_dev(&a->farea, c);
        if (!rc) rc = realloc_dev(&a->F, 5 * c);
        if (rc) return rc;
        a->fcap = c;
    }
    if ((int64_t)ent.size() > a->ecap) {
        int64_t c = a->ecap ? a->ecap : 4096;
        while (c < (int64_t)ent.size()) c *= 2;
        int rc = realloc_dev(&a->ent, c);
        if (rc) return rc;
        a->ecap = c;
    }
    cudaStream_t s = a->ctx->stream;
    VB_CUDA(cudaMemcpyAsync(a->lev, t.lev.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
    VB_CUDA(cudaMemcpyAsync(a->rep, rep.data(), sizeof(int) * rep.size(), cudaMemcpyHostToDevice, s));
    if (nf) {
        VB_CUDA(cudaMemcpyAsync(a->fL, fL.data(), sizeof(int) * nf, cudaMemcpyHostToDevice, s));
        VB_CUDA(cudaMemcpyAsync(a->fR, fR.data(), sizeof(int) * nf, cudaMemcpyHostToDevice, s));
        VB_CUDA(cudaMemcpyAsync(a->fax, fax.data(), sizeof(int8_t) * nf, cudaMemcpyHostToDevice, s));
        VB_CUDA(cudaMemcpyAsync(a->farea, farea.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, s));
    }
    VB_CUDA(cudaMemcpyAsync(a->off, off.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
    if (!ent.empty())
        VB_CUDA(cudaMemcpyAsync(a->ent, ent.data(), sizeof(int) * ent.size(), cudaMemcpyHostToDevice, s));
    VB_CUDA(cudaStreamSynchronize(s));  // the host vectors die here
    a->nface = nf;
    vb::AmrDev &m = a->dev;
    m.nd = nd;
    for (int d = 0; d < 3; ++d) {
        m.bc_lo[d] = a->g.bc_lo[d];
        m.bc_hi[d] = a->g.bc_hi[d];
    }
    m.gamma = a->g.gamma;
    m.aexp = a->g.aexp;
    m.cap = a->cap;
    m.fcap = a->fcap;
    m.nleaf = n;
    m.nface = nf;
    m.lev = a->lev;
    m.rep = a->rep;
    m.fL = a->fL;
    m.fR = a->fR;
    m.fax = a->fax;
    m.farea = a->farea;
    m.off = a->off;
    m.ent = a->ent;
    m.reg = a->reg;
    for (int l = 0; l <= vb::AMR_MAX_LEVEL; ++l) {
        double v = 1.0;
        for (int d = 0; d < 3; ++d) m.w[l][d] = d < nd ? level_width(a, l, d) : 1.0;
        for (int d = 0; d < nd; ++d) v = v * m.w[l][d];
        m.vol[l] = v;
    }
    return VB_OK;
}

// (Re)allocate the leaf-indexed buffers other than the state for `c` leaves.
int alloc_leaf_buffers(vb_amr *a, int64_t c)
{
    int rc = realloc_dev(&a->U1, 5 * c);
    if (!rc) rc = realloc_dev(&a->reg, 5 * c);
    if (!rc) rc = realloc_dev(&a->lev, c);
    if (!rc) rc = realloc_dev(&a->rep, 6 * c);
    if (!rc) rc = realloc_dev(&a->off, c + 1);
    if (!rc) rc = realloc_dev(&a->tag, c);
    if (rc) return rc;
    VB_CUDA(cudaMemsetAsync(a->reg, 0, sizeof(double) * 5 * c, a->ctx->stream));
    a->cap = c;
    return VB_OK;
}

int pull_ctrl(vb_amr *a)
{
    VB_CUDA(cudaMemcpyAsync(a->hctrl, a->ctrl, sizeof(vb::Ctrl), cudaMemcpyDeviceToHost,
                            a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

int push_ctrl(vb_amr *a)
{
    VB_CUDA(cudaMemcpyAsync(a->ctrl, a->hctrl, sizeof(vb::Ctrl), cudaMemcpyHostToDevice,
                            a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

// Refine the given leaves (with balance), remap the state and rebuild tables.
int refine_leaves(vb_amr *a, const std::vector<int> &which)
{
    if (which.empty()) return VB_OK;
    Tree &t = a->tree;
    Batch b(t);
    for (int i : which) {
        const int l = t.lev[i];
        const int64_t c[3] = {t.cx[3 * i], t.cx[3 * i + 1], t.cx[3 * i + 2]};
        b.refine(l, c);
        if (b.err) return fail(VB_ENOTSUP, "refinement beyond the supported depth");
    }
    // depth-first order of the live cells
    std::vector<std::pair<uint64_t, int>> order;
    order.reserve(b.live.size());
    for (size_t s = 0; s < b.lev.size(); ++s)
        if (!b.dead[s]) order.emplace_back(t.dfs_key(b.lev[s], &b.cx[3 * s]), (int)s);
    std::sort(order.begin(), order.end());
    const int64_t n = (int64_t)order.size();
    std::vector<int> lev(n), src(n);
    std::vector<int64_t> cx(3 * n);
    for (int64_t k = 0; k < n; ++k) {
        const int s = order[k].second;
        lev[k] = b.lev[s];
        std::memcpy(&cx[3 * k], &b.cx[3 * s], 3 * sizeof(int64_t));
        src[k] = b.src[s];
    }
    cudaStream_t st = a->ctx->stream;
    // remap the cell means into a buffer of the new capacity
    int64_t cap_new = a->cap;
    while (cap_new < n) cap_new *= 2;
    double *Unew = nullptr;
    int *dsrc = nullptr;
    VB_CUDA(cudaMalloc(&Unew, sizeof(double) * 5 * cap_new));
    cudaError_t e = cudaMalloc(&dsrc, sizeof(int) * n);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dsrc, src.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        cudaFree(Unew);
        cudaFree(dsrc);
        return fail(VB_ECUDA, std::string("regrid remap: ") + cudaGetErrorString(e));
    }
    int nl = vb::launch_amr_prolong((int)n, a->cap, cap_new, dsrc, a->U, Unew, st);
    a->ctx->launches += nl;
    e = cudaStreamSynchronize(st);
    cudaFree(dsrc);
    if (e != cudaSuccess) {
        cudaFree(Unew);
        return fail(VB_ECUDA, std::string("regrid remap: ") + cudaGetErrorString(e));
    }
    cudaFree(a->U);
    a->U = Unew;
    if (cap_new > a->cap) {
        int rc = alloc_leaf_buffers(a, cap_new);
        if (rc) return rc;
    }
    t.lev.swap(lev);
    t.cx.swap(cx);
    t.index.clear();
    for (int64_t i = 0; i < n; ++i) t.index[Tree::key(t.lev[i], &t.cx[3 * i])] = (int)i;
    return build_tables(a);
}

int compute_dt_level(vb_amr *a, int level, double *dt)
{
    cudaStream_t s = a->ctx->stream;
    VB_CUDA(cudaMemsetAsync(&a->ctrl->invdt_bits, 0, sizeof(unsigned long long), s));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_cfl(a->dev, a->U, level, a->ctrl, s));
    int rc = pull_ctrl(a);
    if (rc) return rc;
    double invdt;
    std::memcpy(&invdt, &a->hctrl->invdt_bits, sizeof invdt);
    if (std::isnan(invdt)) return fail(VB_ENONFINITE, "non-finite or negative density/pressure");
    *dt = invdt == 0.0 ? INFINITY : a->g.cfl / invdt;
    return VB_OK;
}

// step!(sim, dt; level) / step_level! with the given registers (host dt)
int step_level(vb_amr *a, double dt, int level, int nreg, const int *rl, const double *rsc)
{
    vb::AmrStageArgs s{};
    s.dt = dt;
    s.level = level;
    s.nreg = nreg;
    for (int r = 0; r < nreg; ++r) {
        s.reg_level[r] = rl[r];
        s.reg_scale[r] = rsc[r];
    }
    s.cfl_all = 0;
    cudaStream_t st = a->ctx->stream;
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 1, a->U, a->U, a->U1, a->F, s, a->ctrl, st));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 2, a->U1, a->U, a->U, a->F, s, a->ctrl, st));
    return VB_OK;
}

int max_level(const vb_amr *a)
{
    int m = 0;
    for (int l : a->tree.lev) m = l > m ? l : m;
    return m;
}

inline double jmin(double x, double y)
{
    if (x != x || y != y) return x + y;
    return y < x ? y : x;
}

// evolve_level! (src/driver.jl:553-578)
int evolve_level(vb_amr *a, int level, double dt_target, bool has_parent)
{
    double dt_stable;
    int rc = compute_dt_level(a, level, &dt_stable);
    if (rc) return rc;
    if (!std::isfinite(dt_stable)) return VB_OK;
    const double q = std::ceil(dt_target / dt_stable * (1 - 1e-12));
    const int64_t n = q < 1.0 ? 1 : (int64_t)q;
    const double dt_sub = dt_target / (double)n;
    const bool has_finer = level < max_level(a);
    cudaStream_t st = a->ctx->stream;
    for (int64_t k = 0; k < n; ++k) {
        if (has_finer) VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_zero_reg(a->dev, level, st));
        int rl[2] = {0, 0};
        double rsc[2] = {0.0, 0.0};
        int nr = 0;
        if (has_parent) { rl[nr] = level - 1; rsc[nr] = 1.0 * (0.5 * dt_sub); ++nr; }
        if (has_finer) { rl[nr] = level; rsc[nr] = -1.0 * (0.5 * dt_sub); ++nr; }
        rc = step_level(a, dt_sub, level, nr, rl, rsc);
        if (rc) return rc;
        if (has_finer) {
            rc = evolve_level(a, level + 1, dt_sub, true);
            if (rc) return rc;
            VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_reflux(a->dev, a->U, level, st));
        }
    }
    return VB_OK;
}

int regrid(vb_amr *a, double above, int maxl, int64_t *ntag)
{
    const int n = (int)a->tree.n();
    cudaStream_t st = a->ctx->stream;
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_tag(a->dev, a->U, above, maxl, a->tag, nullptr, st));
    std::vector<uint8_t> h((size_t)n);
    VB_CUDA(cudaMemcpyAsync(h.data(), a->tag, n, cudaMemcpyDeviceToHost, st));
    VB_CUDA(cudaStreamSynchronize(st));
    std::vector<int> which;
    for (int i = 0; i < n; ++i)
        if (h[i]) which.push_back(i);
    if (ntag) *ntag = (int64_t)which.size();
    return refine_leaves(a, which);
}

}  // namespace

extern "C" {

int vb_amr_create(vb_ctx *ctx, const vb_problem_desc *d, vb_amr **out)
{
    if (!ctx || !d || !out) return fail(VB_EINVAL, "null argument");
    *out = nullptr;
    vb::Geom g{};
    int rc = vb::detail::make_geom(d, &g);
    if (rc) return rc;
    for (int k = 0; k < g.nd; ++k)
        if (g.n[k] >= (1LL << CBITS)) return fail(VB_EINVAL, "base grid too large for AMR keys");
    rc = use(ctx);
    if (rc) return rc;
    vb_amr *a = new (std::nothrow) vb_amr;
    if (!a) return fail(VB_ENOMEM, "host allocation failed");
    a->ctx = ctx;
    a->g = g;
    Tree &t = a->tree;
    t.nd = g.nd;
    for (int k = 0; k < 3; ++k) {
        t.base[k] = k < g.nd ? g.n[k] : 1;
        t.bc_lo[k] = g.bc_lo[k];
        t.bc_hi[k] = g.bc_hi[k];
        a->w0[k] = k < g.nd ? g.w[k] : 1.0;
    }
    const int64_t n = t.base[0] * t.base[1] * t.base[2];
    if (n > INT_MAX / 8) {
        delete a;
        return fail(VB_EINVAL, "base grid too large");
    }
    t.lev.assign(n, 0);
    t.cx.resize(3 * n);
    for (int64_t i = 0; i < n; ++i) {
        t.cx[3 * i] = i % t.base[0];
        t.cx[3 * i + 1] = (i / t.base[0]) % t.base[1];
        t.cx[3 * i + 2] = i / (t.base[0] * t.base[1]);
        t.index[Tree::key(0, &t.cx[3 * i])] = (int)i;
    }
    cudaError_t e = cudaMalloc(&a->ctrl, sizeof(vb::Ctrl));
    if (e == cudaSuccess) e = cudaMallocHost(&a->hctrl, sizeof(vb::Ctrl));
    if (e == cudaSuccess) e = cudaMalloc(&a->partials, sizeof(double) * 5 * vb::TOTALS_PARTS);
    if (e == cudaSuccess) e = cudaMalloc(&a->totals, sizeof(double) * 5);
    if (e == cudaSuccess) e = cudaMallocHost(&a->htot, sizeof(double) * 5);
    if (e != cudaSuccess) {
        release(a);
        delete a;
        return fail(VB_ENOMEM, std::string("AMR buffers: ") + cudaGetErrorString(e));
    }
    std::memset(a->hctrl, 0, sizeof(vb::Ctrl));
    a->hctrl->tfinal = INFINITY;
    a->hctrl->step_limit = LLONG_MAX;
    int64_t cap = 1024;
    while (cap < n) cap *= 2;
    rc = realloc_dev(&a->U, 5 * cap);
    if (!rc) rc = alloc_leaf_buffers(a, cap);
    if (!rc) rc = push_ctrl(a);
    if (!rc) rc = build_tables(a);
    if (!rc) {
        VB_CUDA(cudaMemsetAsync(a->U, 0, sizeof(double) * 5 * a->cap, ctx->stream));
        VB_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    if (rc) {
        release(a);
        delete a;
        return rc;
    }
    *out = a;
    return VB_OK;
}

int vb_amr_destroy(vb_amr *a)
{
    if (!a) return VB_OK;
    cudaSetDevice(a->ctx->device);
    cudaStreamSynchronize(a->ctx->stream);
    release(a);
    delete a;
    return VB_OK;
}

int vb_amr_nleaf(const vb_amr *a, int64_t *n)
{
    if (!a || !n) return fail(VB_EINVAL, "null argument");
    *n = a->tree.n();
    return VB_OK;
}

int vb_amr_leaves(const vb_amr *a, int32_t *level, int64_t *coords)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    const int64_t n = a->tree.n();
    for (int64_t i = 0; i < n; ++i) {
        if (level) level[i] = a->tree.lev[i];
        if (coords) std::memcpy(coords + 3 * i, &a->tree.cx[3 * i], 3 * sizeof(int64_t));
    }
    return VB_OK;
}

int vb_amr_nface(const vb_amr *a, int64_t *n)
{
    if (!a || !n) return fail(VB_EINVAL, "null argument");
    *n = a->nface;
    return VB_OK;
}

int vb_amr_max_level(const vb_amr *a, int32_t *level)
{
    if (!a || !level) return fail(VB_EINVAL, "null argument");
    *level = max_level(a);
    return VB_OK;
}

int vb_amr_upload(vb_amr *a, const double *U)
{
    if (!a || !U) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    const int64_t n = a->tree.n();
    VB_CUDA(cudaMemcpy2DAsync(a->U, sizeof(double) * a->cap, U, sizeof(double) * n,
                              sizeof(double) * n, 5, cudaMemcpyHostToDevice, a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

int vb_amr_download(vb_amr *a, double *U)
{
    if (!a || !U) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    const int64_t n = a->tree.n();
    VB_CUDA(cudaMemcpy2DAsync(U, sizeof(double) * n, a->U, sizeof(double) * a->cap,
                              sizeof(double) * n, 5, cudaMemcpyDeviceToHost, a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

int vb_amr_set_time(vb_amr *a, double t, int64_t step)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    a->t = t;
    a->step = step;
    return VB_OK;
}

int vb_amr_get_time(const vb_amr *a, double *t, int64_t *step)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    if (t) *t = a->t;
    if (step) *step = a->step;
    return VB_OK;
}

int vb_amr_refine(vb_amr *a, const int64_t *leaves, int64_t n)
{
    if (!a || (n > 0 && !leaves)) return fail(VB_EINVAL, "null argument");
    const int64_t nl = a->tree.n();
    std::vector<int> which;
    for (int64_t k = 0; k < n; ++k) {
        if (leaves[k] < 0 || leaves[k] >= nl) return fail(VB_EINVAL, "leaf index out of range");
        which.push_back((int)leaves[k]);
    }
    int rc = use(a->ctx);
    if (rc) return rc;
    return refine_leaves(a, which);
}

int vb_amr_indicator(vb_amr *a, double *out)
{
    if (!a || !out) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    const int64_t n = a->tree.n();
    double *d = nullptr;
    VB_CUDA(cudaMalloc(&d, sizeof(double) * (n > 0 ? n : 1)));
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_tag(a->dev, a->U, INFINITY, 0, a->tag, d, a->ctx->stream));
    cudaError_t e = cudaMemcpyAsync(out, d, sizeof(double) * n, cudaMemcpyDeviceToHost, a->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(a->ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(VB_ECUDA, cudaGetErrorString(e));
    return VB_OK;
}

int vb_amr_regrid(vb_amr *a, double refine_above, int max_level_, int64_t *ntagged)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    return regrid(a, refine_above, max_level_, ntagged);
}

int vb_amr_compute_dt(vb_amr *a, int level, double *dt)
{
    if (!a || !dt) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    return compute_dt_level(a, level, dt);
}

int vb_amr_step(vb_amr *a, double dt)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    if (!std::isfinite(dt)) return fail(VB_EINVAL, "dt must be finite");
    int rc = use(a->ctx);
    if (rc) return rc;
    rc = step_level(a, dt, -1, 0, nullptr, nullptr);
    if (rc) return rc;
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    a->t += dt;
    a->step += 1;
    return VB_OK;
}

int vb_amr_step_level(vb_amr *a, double dt, int level)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    if (!std::isfinite(dt)) return fail(VB_EINVAL, "dt must be finite");
    int rc = use(a->ctx);
    if (rc) return rc;
    rc = step_level(a, dt, level, 0, nullptr, nullptr);
    if (rc) return rc;
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    return VB_OK;
}

int vb_amr_evolve(vb_amr *a, double tfinal, int64_t max_steps, double refine_above,
                  int max_level_, int every, int subcycle, double *t_out, int64_t *nsteps)
{
    if (!a) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    cudaStream_t st = a->ctx->stream;
    int64_t done = 0;
    a->ms_regrid = 0.0;
    auto do_regrid = [&]() -> int {
        if (every > 0 && a->step % every == 0) {
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, st);
            int r = regrid(a, refine_above, max_level_, nullptr);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            a->ms_regrid += ms;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return r;
        }
        return VB_OK;
    };
    if (subcycle) {
        while (a->t < tfinal * (1 - 1e-12)) {
            if (max_steps >= 0 && done >= max_steps) break;
            rc = do_regrid();
            if (rc) return rc;
            double dt0;
            rc = compute_dt_level(a, 0, &dt0);
            if (rc) return rc;
            const double dt_root = jmin(dt0, tfinal - a->t);
            rc = evolve_level(a, 0, dt_root, false);
            if (rc) return rc;
            a->t += dt_root;
            a->step += 1;
            ++done;
        }
    } else {
        // single rate: dt, stages and clock on the device between regrids
        vb::Geom gq = a->g;  // finalize kernel reads cfl (its invV is unused here)
        while (a->t < tfinal * (1 - 1e-12)) {
            if (max_steps >= 0 && done >= max_steps) break;
            rc = do_regrid();
            if (rc) return rc;
            int64_t chunk = every > 0 ? every - a->step % every : 64;
            if (max_steps >= 0 && chunk > max_steps - done) chunk = max_steps - done;
            a->hctrl->t = a->t;
            a->hctrl->step = a->step;
            a->hctrl->tfinal = tfinal;
            a->hctrl->step_limit = a->step + chunk;
            a->hctrl->active = 1;
            a->hctrl->flags = 0;
            rc = push_ctrl(a);
            if (rc) return rc;
            VB_CUDA(cudaMemsetAsync(&a->ctrl->invdt_bits, 0, sizeof(unsigned long long), st));
            VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_cfl(a->dev, a->U, -1, a->ctrl, st));
            vb::AmrStageArgs s{};
            s.level = -1;
            s.cfl_all = 1;
            s.dt = -1.0;  // read from the control block
            for (int64_t k = 0; k < chunk; ++k) {
                VB_CHECK_LAUNCH(a->ctx, vb::launch_finalize_cfl(gq, a->ctrl, st));
                VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 1, a->U, a->U, a->U1, a->F, s, a->ctrl, st));
                VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_stage(a->dev, 2, a->U1, a->U, a->U, a->F, s, a->ctrl, st));
                VB_CHECK_LAUNCH(a->ctx, vb::launch_advance(a->ctrl, st));
            }
            rc = pull_ctrl(a);
            if (rc) return rc;
            if (a->hctrl->flags & vb::CTRL_F_NONFINITE)
                return fail(VB_ENONFINITE, "non-finite dt: NaN or negative density/pressure");
            done += a->hctrl->step - a->step;
            a->t = a->hctrl->t;
            a->step = a->hctrl->step;
            if (!a->hctrl->active && a->step < a->hctrl->step_limit) break;  // reached tfinal
        }
    }
    if (t_out) *t_out = a->t;
    if (nsteps) *nsteps = done;
    return VB_OK;
}

int vb_amr_regrid_ms(const vb_amr *a, double *ms)
{
    if (!a || !ms) return fail(VB_EINVAL, "null argument");
    *ms = a->ms_regrid;
    return VB_OK;
}

int vb_amr_conserved_totals(vb_amr *a, double out[5])
{
    if (!a || !out) return fail(VB_EINVAL, "null argument");
    int rc = use(a->ctx);
    if (rc) return rc;
    VB_CHECK_LAUNCH(a->ctx, vb::launch_amr_totals(a->dev, a->U, a->partials, vb::TOTALS_PARTS,
                                                  a->totals, a->ctx->stream));
    VB_CUDA(cudaMemcpyAsync(a->htot, a->totals, sizeof(double) * 5, cudaMemcpyDeviceToHost,
                            a->ctx->stream));
    VB_CUDA(cudaStreamSynchronize(a->ctx->stream));
    std::memcpy(out, a->htot, sizeof(double) * 5);
    return VB_OK;
}

}  // extern "C"
