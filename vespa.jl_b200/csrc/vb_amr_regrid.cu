// vb_amr_regrid.cu -- the composite AMR mesh's topology work on the device:
// refinement with 2:1 face balance, the depth-first leaf order, and the
// tables the stage kernels read (representative neighbours, faces in the
// reference's emission order, per-leaf CSR of face contributions).
//
// Semantics (lib/HGBackend/src/HGBackend.jl:182-276, src/driver.jl:443-462):
//   - a leaf is (level, integer coordinates at that level); the base grid is
//     a forest of roots; leaves are ordered by root (column-major), then depth
//     first with children x fastest (child index x + 2y + 4z);
//   - refining a leaf first refines any face neighbour one level coarser
//     (closure computed by repeated marking);
//   - a refined leaf is replaced in place by its children, which keeps the
//     depth-first order without a sort; children inherit the cell mean;
//   - conforming faces are emitted from the hi side, coarse<->fine faces
//     from the fine side with the fine area, boundary faces by their cell;
//     per leaf the order is axis 0 hi, axis 0 lo, axis 1 hi, ...;
//   - across a face with finer leaves the representative neighbour is the
//     first of them in leaf order (lowest coordinates).
// All lookups go through an open-addressing hash of (level, coordinates) ->
// leaf index with bounded probing; an overflow sets an error flag instead of
// looping.
#include "vb_amr.h"

namespace vb {

namespace {

constexpr uint64_t EMPTY = ~0ull;

__device__ __forceinline__ uint64_t akey(int l, int c0, int c1, int c2)
{
    return ((uint64_t)l << 60) | ((uint64_t)c0 << 40) | ((uint64_t)c1 << 20) | (uint64_t)c2;
}

__device__ __forceinline__ uint64_t hmix(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

__device__ int hfind(const AmrTopo &t, uint64_t k)
{
    uint64_t h = hmix(k) & t.hmask;
    for (uint64_t probe = 0; probe <= t.hmask; ++probe) {
        const uint64_t v = t.hkey[h];
        if (v == k) return t.hval[h];
        if (v == EMPTY) return -1;
        h = (h + 1) & t.hmask;
    }
    return -1;
}

// same-level coordinates across (d, hi); false at a non-periodic edge
__device__ __forceinline__ bool adjacent(const AmrTopo &t, int l, const int *c, int d, bool hi,
                                         int *cc)
{
    cc[0] = c[0];
    cc[1] = c[1];
    cc[2] = c[2];
    const int nmax = (int)(t.base[d] << l);
    cc[d] += hi ? 1 : -1;
    if (cc[d] < 0 || cc[d] >= nmax) {
        if ((hi ? t.bc_hi[d] : t.bc_lo[d]) != BC_PERIODIC) return false;
        cc[d] = (cc[d] + nmax) % nmax;
    }
    return true;
}

__device__ __forceinline__ void coords(const AmrTopo &t, int i, int *c)
{
    c[0] = t.cx[i];
    c[1] = t.cx[t.cap + i];
    c[2] = t.cx[2 * t.cap + i];
}

// 0 boundary, 1 same level, 2 coarser, 3 finer; *rep representative
__device__ int neighbor(const AmrTopo &t, int i, int d, bool hi, int *rep)
{
    const int l = t.lev[i];
    int c[3], cc[3];
    coords(t, i, c);
    if (!adjacent(t, l, c, d, hi, cc)) return 0;
    int j = hfind(t, akey(l, cc[0], cc[1], cc[2]));
    if (j >= 0) { *rep = j; return 1; }
    if (l > 0) {
        j = hfind(t, akey(l - 1, cc[0] >> 1, cc[1] >> 1, cc[2] >> 1));
        if (j >= 0) { *rep = j; return 2; }
    }
    int cf[3] = {2 * cc[0], 2 * cc[1], 2 * cc[2]};
    if (!hi) cf[d] += 1;
    *rep = hfind(t, akey(l + 1, cf[0], cf[1], cf[2]));
    return 3;
}

__global__ void k_hash_clear(uint64_t *keys, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = EMPTY;
}

__global__ void k_hash_insert(AmrTopo t, uint64_t *keys, int *vals, int *err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    int c[3];
    coords(t, i, c);
    const uint64_t k = akey(t.lev[i], c[0], c[1], c[2]);
    uint64_t h = hmix(k) & t.hmask;
    for (uint64_t probe = 0; probe <= t.hmask; ++probe) {
        const unsigned long long prev =
            atomicCAS((unsigned long long *)&keys[h], (unsigned long long)EMPTY, (unsigned long long)k);
        if (prev == EMPTY || prev == k) {
            vals[h] = i;
            return;
        }
        h = (h + 1) & t.hmask;
    }
    atomicOr(err, 1);
}

// refine marks of coarser face neighbours of marked leaves (one pass); the
// pass does nothing when `gate` is set and zero (the previous pass changed no
// mark, or nothing was tagged), so passes queue without a host check between
// them.  The closure reached is the same whatever the order of the marks.
__global__ void k_balance(AmrTopo t, uint8_t *mark, int *changed, const int *gate)
{
    if (gate && *gate == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n || !mark[i]) return;
    const int l = t.lev[i];
    if (l == 0) return;
    int c[3], cc[3];
    coords(t, i, c);
    for (int d = 0; d < t.nd; ++d)
        for (int hi = 0; hi < 2; ++hi) {
            if (!adjacent(t, l, c, d, hi, cc)) continue;
            if (hfind(t, akey(l, cc[0], cc[1], cc[2])) >= 0) continue;
            const int j = hfind(t, akey(l - 1, cc[0] >> 1, cc[1] >> 1, cc[2] >> 1));
            if (j >= 0 && !mark[j]) {
                mark[j] = 1;
                *changed = 1;
            }
        }
}

__global__ void k_count_children(AmrTopo t, const uint8_t *mark, int *cnt, int *maxlev)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    const int m = mark ? mark[i] : 0;
    cnt[i] = m ? (1 << t.nd) : 1;
    atomicMax(maxlev, t.lev[i] + m);
}

// new leaves in place of the old ones; each copies its source's cell mean
__global__ void k_emit(AmrTopo t, const uint8_t *mark, const int *off, int *lev_new, int *cx_new,
                       int64_t cap_new, const double *__restrict__ Uold, double *__restrict__ Unew)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    int c[3];
    coords(t, i, c);
    const int l = t.lev[i];
    const int o = off[i];
    double u[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) u[k] = Uold[(int64_t)k * t.cap + i];
    const int nch = (mark && mark[i]) ? (1 << t.nd) : 0;
    if (nch == 0) {
        lev_new[o] = l;
        for (int d = 0; d < 3; ++d) cx_new[d * cap_new + o] = c[d];
#pragma unroll
        for (int k = 0; k < 5; ++k) Unew[(int64_t)k * cap_new + o] = u[k];
        return;
    }
    for (int ch = 0; ch < nch; ++ch) {
        lev_new[o + ch] = l + 1;
        for (int d = 0; d < 3; ++d)
            cx_new[d * cap_new + o + ch] = d < t.nd ? 2 * c[d] + ((ch >> d) & 1) : 0;
#pragma unroll
        for (int k = 0; k < 5; ++k) Unew[(int64_t)k * cap_new + o + ch] = u[k];
    }
}

// neighbour kinds and representatives per (axis, side); emitted-face count
__global__ void k_kinds(AmrTopo t, int8_t *kind, int *rep, int *fcnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    int nf = 0;
    for (int s = 0; s < 6; ++s) {
        const int d = s >> 1;
        const bool hi = s & 1;
        int r = -1, k = 0;
        if (d < t.nd) k = neighbor(t, i, d, hi, &r);
        kind[s * t.cap + i] = (int8_t)k;
        rep[s * t.cap + i] = k ? r : -1;
        if (d < t.nd) {
            if (hi) nf += (k != 3);
            else nf += (k == 0 || k == 2);
        }
    }
    fcnt[i] = nf;
}

__global__ void k_faces(AmrTopo t, const int8_t *kind, const int *rep, const int *fbase,
                        AmrAreas ar, int *fL, int *fR, int8_t *fax, double *farea, int *faceid)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    const int l = t.lev[i];
    int f = fbase[i];
    for (int s = 0; s < 6; ++s) faceid[s * t.cap + i] = -1;
    for (int d = 0; d < t.nd; ++d) {
        // hi face (left = i)
        const int kh = kind[(2 * d + 1) * t.cap + i];
        if (kh != 3) {
            fL[f] = i;
            fR[f] = kh == 0 ? -1 : rep[(2 * d + 1) * t.cap + i];
            fax[f] = (int8_t)d;
            farea[f] = ar.area[l][d];
            faceid[(2 * d + 1) * t.cap + i] = f;
            ++f;
        }
        // lo face (right = i): boundary, or i is the fine side
        const int kl = kind[(2 * d) * t.cap + i];
        if (kl == 0 || kl == 2) {
            fL[f] = kl == 0 ? -1 : rep[(2 * d) * t.cap + i];
            fR[f] = i;
            fax[f] = (int8_t)d;
            farea[f] = ar.area[l][d];
            faceid[(2 * d) * t.cap + i] = f;
            ++f;
        }
    }
}

// the finer leaves across (d, side) of leaf i (2^(nd-1) of them)
__device__ int fine_neighbors(const AmrTopo &t, int i, int d, bool hi, int *out)
{
    const int l = t.lev[i];
    int c[3], cc[3];
    coords(t, i, c);
    if (!adjacent(t, l, c, d, hi, cc)) return 0;
    int m = 0;
    const int nfree = t.nd - 1;
    for (int b = 0; b < (1 << nfree); ++b) {
        int cf[3] = {2 * cc[0], 2 * cc[1], 2 * cc[2]};
        cf[d] += hi ? 0 : 1;
        int bit = 0;
        for (int e = 0; e < t.nd; ++e) {
            if (e == d) continue;
            cf[e] += (b >> bit) & 1;
            ++bit;
        }
        const int j = hfind(t, akey(l + 1, cf[0], cf[1], cf[2]));
        if (j >= 0) out[m++] = j;
    }
    return m;
}

__global__ void k_csr_count(AmrTopo t, const int8_t *kind, const int *fcnt, int *ecnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    int e = fcnt[i];
    const int nfine = 1 << (t.nd - 1);
    for (int d = 0; d < t.nd; ++d) {
        const int kl = kind[(2 * d) * t.cap + i], kh = kind[(2 * d + 1) * t.cap + i];
        if (kl == 1) e += 1;
        if (kl == 3) e += nfine;
        if (kh == 3) e += nfine;
    }
    ecnt[i] = e;
}

__global__ void k_csr_fill(AmrTopo t, const int8_t *kind, const int *rep, const int *faceid,
                           const int *off, int *ent, int *err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    int code[32];
    int m = 0;
    auto push = [&](int f, int right) {
        if (f < 0 || m >= 32) {
            atomicOr(err, 2);
            return;
        }
        code[m++] = 2 * f + right;
    };
    for (int d = 0; d < t.nd; ++d) {
        const int fh = faceid[(2 * d + 1) * t.cap + i], fl = faceid[(2 * d) * t.cap + i];
        if (fh >= 0) push(fh, 0);
        if (fl >= 0) push(fl, 1);
        const int kl = kind[(2 * d) * t.cap + i], kh = kind[(2 * d + 1) * t.cap + i];
        if (kl == 1) push(faceid[(2 * d + 1) * t.cap + rep[(2 * d) * t.cap + i]], 1);
        int fn[4];
        if (kl == 3) {
            const int nn = fine_neighbors(t, i, d, false, fn);
            for (int k = 0; k < nn; ++k) push(faceid[(2 * d + 1) * t.cap + fn[k]], 1);
        }
        if (kh == 3) {
            const int nn = fine_neighbors(t, i, d, true, fn);
            for (int k = 0; k < nn; ++k) push(faceid[(2 * d) * t.cap + fn[k]], 0);
        }
    }
    // emission order: ascending face id (and left before right for one face)
    for (int a = 1; a < m; ++a) {
        const int v = code[a];
        int b = a - 1;
        while (b >= 0 && code[b] > v) {
            code[b + 1] = code[b];
            --b;
        }
        code[b + 1] = v;
    }
    const int o = off[i];
    if (m != off[i + 1] - o) atomicOr(err, 4);
    for (int k = 0; k < m && k < off[i + 1] - o; ++k) ent[o + k] = code[k];
}

// ---- exclusive scan of n ints (out has n + 1 entries; out[n] = total) ----
constexpr int SCAN_B = 1024;

__device__ __forceinline__ int block_excl_scan(int v, int *total)
{
    __shared__ int ws[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < (blockDim.x >> 5) ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        ws[lane] = s;
    }
    __syncthreads();
    const int incl = x + (w > 0 ? ws[w - 1] : 0);
    *total = ws[(blockDim.x >> 5) - 1];
    __syncthreads();
    return incl - v;
}

__global__ void __launch_bounds__(SCAN_B) k_scan_blocks(const int *in, int n, int *out, int *bsum)
{
    const int i = blockIdx.x * SCAN_B + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    int tot;
    const int ex = block_excl_scan(v, &tot);
    if (i < n) out[i] = ex;
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// one block: exclusive scan of the block sums, in chunks of SCAN_B
__global__ void __launch_bounds__(SCAN_B) k_scan_sums(int *bsum, int nb, int *total)
{
    int carry = 0;
    for (int base = 0; base < nb; base += SCAN_B) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? bsum[i] : 0;
        int tot;
        const int ex = block_excl_scan(v, &tot);
        if (i < nb) bsum[i] = ex + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(int *out, int n, const int *bsum, const int *total)
{
    const int i = blockIdx.x * SCAN_B + threadIdx.x;
    if (i < n) out[i] += bsum[blockIdx.x];
    if (i == 0) out[n] = *total;
}

unsigned nblk(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs > 0 ? (n + bs - 1) / bs : 1); }

}  // namespace

int amr_scan(const int *in, int n, int *out, int *bsum, int *total, cudaStream_t s)
{
    const int nb = (n + SCAN_B - 1) / SCAN_B;
    k_scan_blocks<<<nb > 0 ? nb : 1, SCAN_B, 0, s>>>(in, n, out, bsum);
    k_scan_sums<<<1, SCAN_B, 0, s>>>(bsum, nb > 0 ? nb : 1, total);
    k_scan_add<<<nb > 0 ? nb : 1, SCAN_B, 0, s>>>(out, n, bsum, total);
    return 3;
}

int launch_amr_hash_build(const AmrTopo &t, uint64_t *keys, int *vals, int *err, cudaStream_t s)
{
    k_hash_clear<<<nblk((int64_t)t.hmask + 1, 256), 256, 0, s>>>(keys, t.hmask + 1);
    k_hash_insert<<<nblk(t.n, 256), 256, 0, s>>>(t, keys, vals, err);
    return 2;
}

int launch_amr_balance(const AmrTopo &t, uint8_t *mark, int *changed, const int *gate,
                       cudaStream_t s)
{
    k_balance<<<nblk(t.n, 256), 256, 0, s>>>(t, mark, changed, gate);
    return 1;
}

int launch_amr_count_children(const AmrTopo &t, const uint8_t *mark, int *cnt, int *maxlev,
                              cudaStream_t s)
{
    k_count_children<<<nblk(t.n, 256), 256, 0, s>>>(t, mark, cnt, maxlev);
    return 1;
}

int launch_amr_emit(const AmrTopo &t, const uint8_t *mark, const int *off, int *lev_new,
                    int *cx_new, int64_t cap_new, const double *Uold, double *Unew, cudaStream_t s)
{
    k_emit<<<nblk(t.n, 256), 256, 0, s>>>(t, mark, off, lev_new, cx_new, cap_new, Uold, Unew);
    return 1;
}

int launch_amr_kinds(const AmrTopo &t, int8_t *kind, int *rep, int *fcnt, cudaStream_t s)
{
    k_kinds<<<nblk(t.n, 128), 128, 0, s>>>(t, kind, rep, fcnt);
    return 1;
}

int launch_amr_faces(const AmrTopo &t, const int8_t *kind, const int *rep, const int *fbase,
                     const AmrAreas &ar, int *fL, int *fR, int8_t *fax, double *farea, int *faceid,
                     cudaStream_t s)
{
    k_faces<<<nblk(t.n, 256), 256, 0, s>>>(t, kind, rep, fbase, ar, fL, fR, fax, farea, faceid);
    return 1;
}

int launch_amr_csr_count(const AmrTopo &t, const int8_t *kind, const int *fcnt, int *ecnt,
                         cudaStream_t s)
{
    k_csr_count<<<nblk(t.n, 256), 256, 0, s>>>(t, kind, fcnt, ecnt);
    return 1;
}

int launch_amr_csr_fill(const AmrTopo &t, const int8_t *kind, const int *rep, const int *faceid,
                        const int *off, int *ent, int *err, cudaStream_t s)
{
    k_csr_fill<<<nblk(t.n, 128), 128, 0, s>>>(t, kind, rep, faceid, off, ent, err);
    return 1;
}

}  // namespace vb
