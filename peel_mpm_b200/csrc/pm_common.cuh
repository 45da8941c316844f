// Shared device code of the AnisoMPM substep: control block, workspace
// layout, 3x3 algebra, the cyclic Jacobi eigensolver and the B-spline
// weights.  Reference: anisompm_py/src/anisompm.py.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "peelmpm.h"

namespace pm {

constexpr int kBlockEdge = 4;          // grid block = 4^3 nodes (active-block granularity)
constexpr int kSortBlock = 8;          // sort block = 8^3 cells (P2G work unit)
constexpr int kSortBlockBits = 9;      // log2(8^3)
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;   // keys per radix tile
// Radix digits: 8 bits per pass; the last pass takes 9 when exactly 9 bits
// remain, which saves a pass (25-bit keys: 8 + 8 + 9).
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kRadixBitsTop = 9;
constexpr int kRadixTop = 1 << kRadixBitsTop;
__host__ __device__ constexpr int radix_digit_bits(int remaining) {
    return remaining == kRadixBitsTop ? kRadixBitsTop : kRadixBits;
}
__host__ __device__ inline int radix_passes(int key_bits) {
    int p = 0;
    for (int rem = key_bits < 1 ? 1 : key_bits; rem > 0; rem -= radix_digit_bits(rem)) ++p;
    return p;
}
constexpr int kG2PThreads = 256;     // G2P particles per CTA

// Device control block: per-substep inputs and status counters.  The three
// bounds are float bit patterns (non-negative floats order like their bits):
// the largest magnitude of a particle's momentum contribution to one node, of
// a particle mass and of a particle damage; they fix the units of the grid's
// fixed-point accumulators for the substep (see fix_scale).  The constitutive
// kernel raises them with atomicMax into kBoundSlots slots per quantity (warps
// spread over the slots, so the atomics do not queue on one address) and a
// one-block kernel folds the slots into the bounds.  n_work / work_next: the
// P2G work list of non-empty 4^3-cell sub-blocks and its dynamic cursor
// (control block 0 of a batch serves all scenes).
constexpr int kBoundSlots = 128;
struct Ctrl {
    double time;
    long long step;
    int any_allow;
    unsigned n_active;
    unsigned nonfinite;
    unsigned dense_subblocks;   // sub-blocks beyond the fixed-point headroom (status error)
    unsigned mom_bound, mass_bound, dmg_bound;
    unsigned n_work, work_next;
    unsigned pad_;
    float col_origin[PM_MAX_COLLIDERS][3];
    float col_vel[PM_MAX_COLLIDERS][3];
    unsigned bound_slots[3][kBoundSlots];   // zero between substeps
};

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

__host__ __device__ inline int sort_bits(int n_grid) {
    unsigned long long cells = (unsigned long long)n_grid * n_grid * n_grid;
    int b = 1;
    while ((1ull << b) < cells) ++b;
    return b;
}

__host__ __device__ inline int sort_blocks_per_axis(int ng) { return (ng + kSortBlock - 1) / kSortBlock; }
__host__ __device__ inline int blocked_key_bits(int ng) {
    const unsigned long long nb = (unsigned long long)sort_blocks_per_axis(ng);
    const unsigned long long blocks = nb * nb * nb;
    int b = 0;
    while ((1ull << b) < blocks) ++b;
    return b + kSortBlockBits;
}

struct Layout {
    size_t ctrl, keys_a, keys_b, vals_a, vals_b, hist, block_mask, block_list;
    size_t g_mom, g_dmg, g_vel, g_gd, payload, inv_perm, work, tables, total;
    int passes, key_bits, n_tiles, nbs;
    long long n_blocks, n_nodes;
};

// n particles, n_nodes grid nodes, n_blocks 4^3 grid blocks, sort keys of
// key_bits bits, n_ctrl control blocks and table_bytes of scene tables.
__host__ __device__ inline Layout make_layout_sized(long long n, long long n_nodes, long long n_blocks, int key_bits,
                                                    int n_ctrl, size_t table_bytes) {
    Layout L;
    const size_t A = 256;
    L.n_tiles = (int)((n + kSortTile - 1) / kSortTile);
    if (L.n_tiles < 1) L.n_tiles = 1;
    L.key_bits = key_bits < 1 ? 1 : key_bits;
    L.passes = radix_passes(L.key_bits);
    L.nbs = 0;
    L.n_blocks = n_blocks;
    L.n_nodes = n_nodes;
    size_t nn = (size_t)(n > 0 ? n : 1);
    size_t o = 0;
    L.ctrl = o;       o = align_up(o + sizeof(Ctrl) * (size_t)(n_ctrl > 0 ? n_ctrl : 1), A);
    L.keys_a = o;     o = align_up(o + 4 * nn, A);
    L.keys_b = o;     o = align_up(o + 4 * nn, A);
    L.vals_a = o;     o = align_up(o + 4 * nn, A);
    L.vals_b = o;     o = align_up(o + 4 * nn, A);
    L.hist = o;       o = align_up(o + 4 * ((size_t)kRadixTop * L.n_tiles + kRadixTop), A);
    L.block_mask = o; o = align_up(o + (size_t)L.n_blocks, A);
    L.block_list = o; o = align_up(o + 4 * (size_t)L.n_blocks, A);
    L.g_mom = o;      o = align_up(o + 32 * (size_t)L.n_nodes, A);   // 4 x int64 fixed point per node
    L.g_dmg = o;      o = align_up(o + 16 * (size_t)L.n_nodes, A);   // 2 x int64 fixed point per node
    L.g_vel = o;      o = align_up(o + 16 * (size_t)L.n_nodes, A);
    L.g_gd = o;       o = align_up(o + 4 * (size_t)L.n_nodes, A);
    L.payload = o;    o = align_up(o + 80 * nn, A);
    L.inv_perm = o;   o = align_up(o + 4 * nn, A);
    L.work = o;       o = align_up(o + 4 * nn, A);                    // starts of the non-empty sub-blocks
    L.tables = o;     o = align_up(o + table_bytes, A);
    L.total = o;
    return L;
}

// Single scene: the sort must also hold the reference (x-major) numbering of
// pm_bin_sort.
__host__ __device__ inline Layout make_layout(long long n, int ng) {
    const int nbs = (ng + kBlockEdge - 1) / kBlockEdge;
    const int kb = sort_bits(ng) > blocked_key_bits(ng) ? sort_bits(ng) : blocked_key_bits(ng);
    Layout L = make_layout_sized(n, (long long)ng * ng * ng, (long long)nbs * nbs * nbs, kb, 1, 0);
    L.nbs = nbs;
    return L;
}

// Raw views of the workspace for kernels.
struct WS {
    Ctrl *ctrl;
    unsigned *keys_a, *keys_b;
    int *vals_a, *vals_b;
    unsigned *hist;          // [digits][n_tiles] tile counts (up to kRadixTop digits)
    unsigned *dtot;          // [digits] digit totals of the current pass
    unsigned char *block_mask;
    int *block_list;
    long long *g_mom;   // {mv.x, mv.y, mv.z, m} per node, int64 fixed point, zero between substeps
    long long *g_dmg;   // {sum w d, sum w} per node, int64 fixed point, zero between substeps
    float4 *g_vel;      // {v.x, v.y, v.z, unused}
    float *g_gd;        // normalised damage field
    float *g_sw;        // cubic weight sums (recorded for the adjoint; NULL otherwise)
    float4 *g_vpre;     // grid velocity before the colliders (recorded for the adjoint; NULL otherwise)
    float *tape_aff;    // APIC affine term, 9 planes (recorded for the adjoint; NULL otherwise)
    float *tape_pol;    // polar R, V, S and phi, 22 planes (recorded for the adjoint; NULL otherwise)
    long long tape_aff_stride;
    float4 *payload;    // P2G payload, 5 float4 per particle in sorted order
    const unsigned *sorted_keys;
    const int *perm;
    int *inv_perm;      // particle -> sorted position, written by the last radix pass
    int *work;          // sorted index of the first particle of every non-empty 4^3-cell sub-block
    int passes, key_bits, n_tiles, nbs;
    long long n_blocks;
};

inline WS make_ws(void *base, const Layout &L) {
    char *b = (char *)base;
    WS w;
    w.ctrl = (Ctrl *)(b + L.ctrl);
    w.keys_a = (unsigned *)(b + L.keys_a);
    w.keys_b = (unsigned *)(b + L.keys_b);
    w.vals_a = (int *)(b + L.vals_a);
    w.vals_b = (int *)(b + L.vals_b);
    w.hist = (unsigned *)(b + L.hist);
    w.dtot = w.hist + (size_t)kRadixTop * L.n_tiles;
    w.block_mask = (unsigned char *)(b + L.block_mask);
    w.block_list = (int *)(b + L.block_list);
    w.g_mom = (long long *)(b + L.g_mom);
    w.g_dmg = (long long *)(b + L.g_dmg);
    w.g_vel = (float4 *)(b + L.g_vel);
    w.g_gd = (float *)(b + L.g_gd);
    w.g_sw = nullptr;
    w.g_vpre = nullptr;
    w.tape_aff = nullptr;
    w.tape_pol = nullptr;
    w.tape_aff_stride = 0;
    w.payload = (float4 *)(b + L.payload);
    w.passes = L.passes;
    w.key_bits = L.key_bits;
    w.n_tiles = L.n_tiles;
    w.nbs = L.nbs;
    w.n_blocks = L.n_blocks;
    // pass 0 reads keys_a and writes keys_b; the result of an odd pass count is in *_b
    w.sorted_keys = (L.passes & 1) ? w.keys_b : w.keys_a;
    w.perm = (L.passes & 1) ? w.vals_b : w.vals_a;
    w.inv_perm = (int *)(b + L.inv_perm);
    w.work = (int *)(b + L.work);
    return w;
}

// Particle pointers as kernels see them (plane stride folded in).
// Mutable state is read from x .. D_hist and written to xo .. Dho: the same
// planes for an in-place substep, another state's planes for an out-of-place
// one (a recorded substep writing the next state of its segment).
struct Parts {
    long long n, ps;
    float *x, *v, *F, *C, *d, *lap, *D_hist;
    float *xo, *vo, *Fo, *Co, *d_o, *lapo, *Dho;
    const float *vol0, *mass, *mu, *lam, *sigma_c, *eta, *zeta, *l0, *residual, *A0;
    const unsigned char *allow;
    const float *n_interface;
    const unsigned char *interface_mask;
    const signed char *grip_tag;
    float *phi, *phi_shear, *tau_last, *J_last;
};

inline Parts make_parts(const pm_particles *P) {
    Parts q;
    q.n = P->n; q.ps = P->plane_stride;
    q.x = P->x; q.v = P->v; q.F = P->F; q.C = P->C; q.d = P->d; q.lap = P->lap; q.D_hist = P->D_hist;
    q.vol0 = P->vol0; q.mass = P->mass; q.mu = P->mu; q.lam = P->lam; q.sigma_c = P->sigma_c;
    q.eta = P->eta; q.zeta = P->zeta; q.l0 = P->l0; q.residual = P->residual; q.A0 = P->A0;
    q.allow = P->allow; q.n_interface = P->n_interface; q.interface_mask = P->interface_mask;
    q.grip_tag = (const signed char *)P->grip_tag; q.phi = P->phi; q.phi_shear = P->phi_shear;
    q.tau_last = P->tau_last; q.J_last = P->J_last;
    q.xo = q.x; q.vo = q.v; q.Fo = q.F; q.Co = q.C; q.d_o = q.d; q.lapo = q.lap; q.Dho = q.D_hist;
    return q;
}
// The same particles writing their updated state to O's planes (O->plane_stride equals P's).
inline Parts make_parts_out(const pm_particles *P, const pm_particles *O) {
    Parts q = make_parts(P);
    q.xo = O->x; q.vo = O->v; q.Fo = O->F; q.Co = O->C; q.d_o = O->d; q.lapo = O->lap; q.Dho = O->D_hist;
    return q;
}

// ------------------------------------------------------------------ scenes
// Kernels are written once against a scene policy.  PlainScenes is the single
// scene of AnisoMPM.substep, its parameters passed by value; every lookup is a
// constant.  BatchScenes describes many independent scenes packed into one
// particle array, one grid buffer and one sort: scene s owns particles
// [p_begin[s], p_begin[s+1]), grid nodes from node_base[s], sort blocks from
// sblock_base[s], 4^3 grid blocks from gblock_base[s] and G2P CTAs from
// cta_base[s]; lookups are binary searches over these prefix tables.
__device__ __forceinline__ int upper_index(const long long *a, int n, long long v) {
    int lo = 0, hi = n - 1;   // largest i in [0, n) with a[i] <= v
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a[mid] <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

struct PlainScenes {
    pm_params prm;
    static constexpr bool batched = false;
    int count() const { return 1; }
    __device__ __forceinline__ int of_particle(long long) const { return 0; }
    __device__ __forceinline__ int of_sblock(unsigned) const { return 0; }
    __device__ __forceinline__ int of_gblock(long long) const { return 0; }
    __device__ __forceinline__ int of_cta(long long) const { return 0; }
    __device__ __forceinline__ const pm_params &params(int) const { return prm; }
    __device__ __forceinline__ long long p_begin(int) const { return 0; }
    __device__ __forceinline__ long long p_end(int, long long n) const { return n; }
    __device__ __forceinline__ long long node_base(int) const { return 0; }
    __device__ __forceinline__ unsigned sblock_base(int) const { return 0; }
    __device__ __forceinline__ long long gblock_base(int) const { return 0; }
    __device__ __forceinline__ long long cta_base(int) const { return 0; }
};

struct BatchScenes {
    const pm_params *prms;        // [n]
    const long long *pb;          // particle begin, [n + 1]
    const long long *nodeb;       // grid node base, [n]
    const long long *sblk;        // first sort block, [n + 1]
    const long long *gblk;        // first 4^3 grid block, [n + 1]
    const long long *ctab;        // first G2P CTA, [n + 1]
    int n;
    static constexpr bool batched = true;
    int count() const { return n; }
    __device__ __forceinline__ int of_particle(long long p) const { return upper_index(pb, n, p); }
    __device__ __forceinline__ int of_sblock(unsigned b) const { return upper_index(sblk, n, (long long)b); }
    __device__ __forceinline__ int of_gblock(long long b) const { return upper_index(gblk, n, b); }
    __device__ __forceinline__ int of_cta(long long c) const { return upper_index(ctab, n, c); }
    __device__ __forceinline__ const pm_params &params(int s) const { return prms[s]; }
    __device__ __forceinline__ long long p_begin(int s) const { return pb[s]; }
    __device__ __forceinline__ long long p_end(int s, long long) const { return pb[s + 1]; }
    __device__ __forceinline__ long long node_base(int s) const { return nodeb[s]; }
    __device__ __forceinline__ unsigned sblock_base(int s) const { return (unsigned)sblk[s]; }
    __device__ __forceinline__ long long gblock_base(int s) const { return gblk[s]; }
    __device__ __forceinline__ long long cta_base(int s) const { return ctab[s]; }
};

// Division of a small non-negative int by a runtime divisor through a float
// reciprocal (tile index -> coordinates in the staging loops): with
// y = (i + 0.5) / d the fraction of y is at least 0.5/d from an integer and
// the two float roundings move y by at most y * 2^-23, which stays below
// 0.5/d for i < 2^22, so the truncation is floor(i / d) exactly.
struct FastDiv {
    int d;
    float r;
};
__device__ __forceinline__ FastDiv make_fastdiv(int d) { return FastDiv{d, __frcp_rn((float)d)}; }
__device__ __forceinline__ int fdiv(int i, const FastDiv &f) { return __float2int_rz(((float)i + 0.5f) * f.r); }

// ------------------------------------------------------------------ cells
// floor(v).to(long) then clamp, as the reference forms base cells: NaN or a
// value outside int64 becomes INT64_MIN in torch and clamps to node 0; values
// far outside the grid clamp to the edge, so the base is saturated to
// [-8, ng+8] (every stencil node then clamps identically).
__device__ __forceinline__ int sat_base(float f, int ng) {
    if (!(f >= -9.2233720368547758e18f && f < 9.2233720368547758e18f)) return -8;
    return (int)fminf(fmaxf(f, -8.0f), (float)(ng + 8));
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Quadratic B-spline (anisompm.py:544-557): base = floor(X - 0.5), fx = X - base,
// w0 = 0.5(1.5-fx)^2, w1 = 0.75-(fx-1)^2, w2 = 0.5(fx-0.5)^2.  X = x * fp32(inv_dx)
// and X - 0.5 are rounded exactly as the reference's two tensor ops.
struct Quad {
    int b[3];
    float fx[3];
    float w[3][3];   // [node][axis]
};
__device__ __forceinline__ void quad_weights(const float x[3], float inv_dx, int ng, Quad &q) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float X = __fmul_rn(x[a], inv_dx);
        const float fb = floorf(__fsub_rn(X, 0.5f));
        q.b[a] = sat_base(fb, ng);
        const float f = __fsub_rn(X, fb);
        q.fx[a] = f;
        const float t0 = 1.5f - f, t1 = f - 1.0f, t2 = f - 0.5f;
        q.w[0][a] = 0.5f * (t0 * t0);
        q.w[1][a] = 0.75f - t1 * t1;
        q.w[2][a] = 0.5f * (t2 * t2);
    }
}

// Cubic B-spline with second derivatives (anisompm.py:559-584): base =
// floor(X) - 1, f = X - floor(X).
struct Cubic {
    int b[3];
    float w[4][3];
    float w2[4][3];
};
__device__ __forceinline__ void cubic_weights(const float x[3], float inv_dx, int ng, Cubic &c) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float X = __fmul_rn(x[a], inv_dx);
        const float fb = floorf(X);
        const int bb = sat_base(fb, ng);
        c.b[a] = bb - 1;
        const float f = __fsub_rn(X, fb);
        const float one = 1.0f - f;
        c.w[0][a] = (1.0f / 6.0f) * (one * one * one);
        c.w[1][a] = (2.0f / 3.0f - f * f) + 0.5f * (f * f * f);
        c.w[2][a] = (2.0f / 3.0f - one * one) + 0.5f * (one * one * one);
        c.w[3][a] = (1.0f / 6.0f) * (f * f * f);
        c.w2[0][a] = one;
        c.w2[1][a] = 3.0f * f - 2.0f;
        c.w2[2][a] = 1.0f - 3.0f * f;
        c.w2[3][a] = f;
    }
}

// _node_index of the base cell (anisompm.py:586-590): x-major, z fastest.
__device__ __forceinline__ unsigned cell_key(const int b[3], int ng) {
    const int x = clampi(b[0], 0, ng - 1), y = clampi(b[1], 0, ng - 1), z = clampi(b[2], 0, ng - 1);
    return ((unsigned)x * (unsigned)ng + (unsigned)y) * (unsigned)ng + (unsigned)z;
}

// Morton (z-order) number of a cell inside its 8^3 sort block, bits
// x2 y2 z2 x1 y1 z1 x0 y0 z0: every aligned run of 8^k numbers is a brick of
// edge 2^k, and the top three bits name the cell's 4^3-cell sub-block (the
// P2G work unit).
__host__ __device__ __forceinline__ unsigned morton9(unsigned x, unsigned y, unsigned z) {
    unsigned m = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b)
        m |= (((x >> b) & 1u) << (3 * b + 2)) | (((y >> b) & 1u) << (3 * b + 1)) | (((z >> b) & 1u) << (3 * b));
    return m;
}
// Cell of Morton number m (low 6 bits: inside the 4^3 sub-block; 9 bits: inside the 8^3 block).
__host__ __device__ __forceinline__ void morton_decode(unsigned m, int c[3]) {
    c[0] = (int)(((m >> 2) & 1u) | ((m >> 4) & 2u) | ((m >> 6) & 4u));
    c[1] = (int)(((m >> 1) & 1u) | ((m >> 3) & 2u) | ((m >> 5) & 4u));
    c[2] = (int)((m & 1u) | ((m >> 2) & 2u) | ((m >> 4) & 4u));
}

// Sort key of the substep: the same base cell, numbered block-major (8^3-cell
// blocks in x-major order, cells in Morton order inside a block) so that a
// run of the sorted order is a compact brick.  A bijection of cell_key.
__device__ __forceinline__ unsigned blocked_key(const int b[3], int ng) {
    const int x = clampi(b[0], 0, ng - 1), y = clampi(b[1], 0, ng - 1), z = clampi(b[2], 0, ng - 1);
    const unsigned nb = (unsigned)sort_blocks_per_axis(ng);
    const unsigned blk = ((unsigned)(x >> 3) * nb + (unsigned)(y >> 3)) * nb + (unsigned)(z >> 3);
    return (blk << kSortBlockBits) | morton9((unsigned)x & 7u, (unsigned)y & 7u, (unsigned)z & 7u);
}

// ------------------------------------------------------- fixed-point grid sums
// P2G accumulates into int64 fixed point, so the sums are exact and do not
// depend on the order of the atomic additions: a substep is bit-reproducible
// run to run, which the adjoint's checkpoint re-runs rely on.  The unit of a
// quantity is 2^(e - kFixBits) with 2^e above the substep's bound on one
// contribution; a node total then holds 2^(63 - kFixBits) = 131,072
// worst-case contributions before it could overflow (a node's contributions
// come from at most 8 of the 4^3-cell sub-blocks, so the P2G kernel counts
// sub-blocks of more than kDenseSubblock particles as a status error), and
// every contribution is resolved to 2^-kFixBits of the bound: a node whose
// sum is 1e-6 of the largest contribution still gets float32's precision.
constexpr int kFixBits = 46;
constexpr int kDenseSubblock = 16383;
// Scale (2^(kFixBits - e)) and unit (its inverse) from a bound's float bits;
// bounds below 2^-75 (including zero) or not finite use 2^-75 / 2^127.
struct FixScale {
    float scale, unit;
};
__device__ __forceinline__ FixScale fix_scale(unsigned bound_bits) {
    float b = __uint_as_float(bound_bits);
    if (!(b >= 2.6470e-23f)) b = 2.6470e-23f;           // 2^-75; also NaN
    if (!(b <= 1.0e38f)) b = 1.0e38f;
    const int e = (int)((__float_as_uint(b) >> 23) & 0xffu) - 126;   // 2^(e-1) <= b < 2^e
    FixScale f;
    f.scale = __uint_as_float((unsigned)(127 + kFixBits - e) << 23);
    f.unit = __uint_as_float((unsigned)(127 - kFixBits + e) << 23);
    return f;
}
__device__ __forceinline__ long long to_fix(float v, float scale) { return __float2ll_rn(v * scale); }
__device__ __forceinline__ float from_fix(long long q, float unit) { return __ll2float_rn(q) * unit; }
// Magnitude bound of a value for the control block's atomicMax (NaN counts as 0).
__device__ __forceinline__ unsigned bound_bits(float v) {
    const float a = fabsf(v);
    return a <= 3.4e38f ? __float_as_uint(a) : 0u;
}

// ------------------------------------------------------------ 3x3 algebra
// Row-major 3x3; products accumulate k = 0, 1, 2.
__device__ __forceinline__ void mm3(const float *A, const float *B, float *Cm) {
    float T[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            T[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
#pragma unroll
    for (int k = 0; k < 9; ++k) Cm[k] = T[k];
}
__device__ __forceinline__ void mmt3(const float *A, const float *B, float *Cm) {   // A B^T
    float T[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            T[3 * i + j] = A[3 * i] * B[3 * j] + A[3 * i + 1] * B[3 * j + 1] + A[3 * i + 2] * B[3 * j + 2];
#pragma unroll
    for (int k = 0; k < 9; ++k) Cm[k] = T[k];
}

// The same products with every multiply and add rounded separately, k = 0,
// 1, 2 in order, as the reference's float32 matrix products round them: for
// updates applied to every particle every substep (the f_clamp rebuild of F,
// whose near-identity factor V diag(Sc/S) V^T is I up to rounding) contraction
// into FMAs would let F drift from the reference's by a rounding-level random
// walk.
__device__ __forceinline__ float dot3_rn(float a0, float b0, float a1, float b1, float a2, float b2) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1)), __fmul_rn(a2, b2));
}
__device__ __forceinline__ void mm3_rn(const float *A, const float *B, float *Cm) {
    float T[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            T[3 * i + j] = dot3_rn(A[3 * i], B[j], A[3 * i + 1], B[3 + j], A[3 * i + 2], B[6 + j]);
#pragma unroll
    for (int k = 0; k < 9; ++k) Cm[k] = T[k];
}
__device__ __forceinline__ void mmt3_rn(const float *A, const float *B, float *Cm) {   // A B^T
    float T[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            T[3 * i + j] = dot3_rn(A[3 * i], B[3 * j], A[3 * i + 1], B[3 * j + 1], A[3 * i + 2], B[3 * j + 2]);
#pragma unroll
    for (int k = 0; k < 9; ++k) Cm[k] = T[k];
}

// Packed float32 pairs: sm_100's FFMA2 / FMUL2 / FADD2 issue two independent
// IEEE round-to-nearest operations as one instruction (each lane rounds as
// the scalar operation would), halving the issue slots of paired arithmetic.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }

__device__ __forceinline__ float nan_to_num(float a) {
    if (a != a) return 0.0f;
    if (a > 3.402823466e38f) return 3.402823466e38f;
    if (a < -3.402823466e38f) return -3.402823466e38f;
    return a;
}

// One Jacobi rotation on pair (p,q) with the third index r, for a symmetric
// matrix stored as app/aqq/apq/apr/aqr (anisompm.py:72-91).  The reference's
// tangent t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), zeta = (aqq-app)/(2apq),
// is evaluated as t = sign(zeta) |b| / (|a| + sqrt(a^2 + b^2)) with
// (a, b) = (aqq - app, 2 apq) / max(|aqq - app|, |2 apq|): the same value
// without its two divisions and square root, and without overflow for any
// finite input (the reference's zeta^2 overflows to t = 0 only where t is
// below 3e-20 anyway); the normalisation is an exact power of two taken from
// the exponent bits.  The skip rule |apq| <= 1e-30 and sign(0) = +1 are the
// reference's.  Three MUFU operations (rsqrt, rcp, rsqrt) per rotation.
#define PM_JACOBI_ROT(APP, AQQ, APQ, APR, AQR, P, Q)                                  \
    {                                                                                 \
        const float app = APP, aqq = AQQ, apq = APQ, apr = APR, aqr = AQR;            \
        float c = 1.0f, s = 0.0f;                                                     \
        if (fabsf(apq) > 1e-30f) {                                                    \
            const float dd = aqq - app, bb = 2.0f * apq;                              \
            const float mx = fmaxf(fabsf(dd), fabsf(bb));                             \
            const unsigned ex_ = min((__float_as_uint(mx) >> 23) & 0xffu, 253u);      \
            const float im = __uint_as_float((254u - ex_) << 23); /* 2^(127-ex_) */ \
            const float a_ = dd * im, b_ = bb * im;                                   \
            const float h2 = fmaf(a_, a_, b_ * b_);                                   \
            const float hh = h2 * rsqrtf(h2);                                         \
            const float sg = (dd == 0.0f || ((dd > 0.0f) == (apq > 0.0f))) ? 1.0f : -1.0f; \
            const float t = sg * __fdividef(fabsf(b_), fabsf(a_) + hh);               \
            c = rsqrtf(fmaf(t, t, 1.0f));                                             \
            s = c * t;                                                                \
        }                                                                             \
        APP = c * c * app - 2.0f * s * c * apq + s * s * aqq;                         \
        AQQ = s * s * app + 2.0f * s * c * apq + c * c * aqq;                         \
        APQ = 0.0f;                                                                   \
        APR = c * apr - s * aqr;                                                      \
        AQR = s * apr + c * aqr;                                                      \
        _Pragma("unroll") for (int i_ = 0; i_ < 3; ++i_) {                            \
            const float vp = V[3 * i_ + P], vq = V[3 * i_ + Q];                       \
            V[3 * i_ + P] = c * vp - s * vq;                                          \
            V[3 * i_ + Q] = s * vp + c * vq;                                          \
        }                                                                             \
    }

// sym_eig (anisompm.py:48-95): symmetrise + nan_to_num, 5 (or `sweeps`) cyclic
// sweeps over pairs (0,1),(0,2),(1,2), eigenvalues ascending (stable order),
// eigenvector columns in V (row-major).  SWEEPS > 0 fixes the sweep count at
// compile time (the substep's 5); SWEEPS == 0 takes it from `sweeps_rt`, any
// count >= 1, as the reference's `sweeps` argument (anisompm.py:48, 68).
template <int SWEEPS>
__device__ __forceinline__ void sym_eig3(const float *Ain, float ev[3], float V[9], int sweeps_rt = SWEEPS) {
    const int n_sweeps = SWEEPS > 0 ? SWEEPS : sweeps_rt;
    float a00 = nan_to_num(0.5f * (Ain[0] + Ain[0]));
    float a11 = nan_to_num(0.5f * (Ain[4] + Ain[4]));
    float a22 = nan_to_num(0.5f * (Ain[8] + Ain[8]));
    float a01 = nan_to_num(0.5f * (Ain[1] + Ain[3]));
    float a02 = nan_to_num(0.5f * (Ain[2] + Ain[6]));
    float a12 = nan_to_num(0.5f * (Ain[5] + Ain[7]));
#pragma unroll
    for (int k = 0; k < 9; ++k) V[k] = (k % 4 == 0) ? 1.0f : 0.0f;
#pragma unroll
    for (int sw = 0; sw < n_sweeps; ++sw) {
        // Once every lane's off-diagonal is below 1e-10 of its diagonal, the
        // remaining sweeps of the reference change nothing at float32
        // precision: a rotation with |t| ~ |apq|/gap <= 1e-10 leaves c = 1 and
        // moves entries by less than half an ulp, and where eigenvalues lie
        // closer than the off-diagonals it only turns the eigenvector pair
        // inside their (numerically) degenerate plane, which leaves R, S and
        // sigma+ unchanged.  The warp then stops early.
        if (sw >= 1) {
            const float off = fabsf(a01) + fabsf(a02) + fabsf(a12);
            const float dia = fabsf(a00) + fabsf(a11) + fabsf(a22);
            if (__all_sync(__activemask(), off <= 1e-10f * dia)) break;
        }
        PM_JACOBI_ROT(a00, a11, a01, a02, a12, 0, 1)
        PM_JACOBI_ROT(a00, a22, a02, a01, a12, 0, 2)
        PM_JACOBI_ROT(a11, a22, a12, a01, a02, 1, 2)
    }
    ev[0] = a00; ev[1] = a11; ev[2] = a22;
    // stable ascending sort of three, eigenvector columns follow
#define PM_SWAPCOL(I, J)                                                               \
    {                                                                                  \
        float te = ev[I]; ev[I] = ev[J]; ev[J] = te;                                   \
        _Pragma("unroll") for (int r_ = 0; r_ < 3; ++r_) {                             \
            float tv = V[3 * r_ + I]; V[3 * r_ + I] = V[3 * r_ + J]; V[3 * r_ + J] = tv; \
        }                                                                              \
    }
    if (ev[1] < ev[0]) PM_SWAPCOL(0, 1)
    if (ev[2] < ev[1]) PM_SWAPCOL(1, 2)
    if (ev[1] < ev[0]) PM_SWAPCOL(0, 1)
#undef PM_SWAPCOL
}

// Eigensystem of the Cauchy stress of the fixed-corotated model, sig =
// sym(2 mu (F - R) F^T + tv I) / J, from the polar decomposition instead of a
// second Jacobi solve: with F = U S V^T and R = U V^T, (F - R) F^T =
// U (S^2 - S) U^T, so sig is diagonal in the left singular vectors U (an
// f_clamp rescaling of S keeps U).  Columns of Ucols must be the unit vectors
// F v_j / |F v_j|; the eigenvalues are the Rayleigh quotients q_j^T sig q_j.
// polar_u_ok() says whether U is usable: not when the smallest |F v_j| is
// below 1e-3 of the largest (a nearly singular F, whose U is ill-defined);
// the caller then solves sig by Jacobi sweeps as the reference does.
// Elsewhere the result agrees with the 5-sweep Jacobi solve to float32
// rounding; the order of the eigenpairs differs, which sigma+ = Q relu(e) Q^T
// and phi do not see.
__device__ __forceinline__ bool polar_u_ok(const float nrm[3]) {
    const float mx = fmaxf(nrm[0], fmaxf(nrm[1], nrm[2]));
    const float mn = fminf(nrm[0], fminf(nrm[1], nrm[2]));
    return mn >= 1e-3f * mx;
}
__device__ __forceinline__ void stress_eig_polar(const float Ucols[9], const float sig[9], float ev[3], float Q[9]) {
#pragma unroll
    for (int k = 0; k < 9; ++k) Q[k] = Ucols[k];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float q0 = Q[j], q1 = Q[3 + j], q2 = Q[6 + j];
        const float s0 = sig[0] * q0 + sig[1] * q1 + sig[2] * q2;
        const float s1 = sig[3] * q0 + sig[4] * q1 + sig[5] * q2;
        const float s2 = sig[6] * q0 + sig[7] * q1 + sig[8] * q2;
        ev[j] = q0 * s0 + q1 * s1 + q2 * s2;
    }
}

// The strain limit f_clamp (anisompm.py:622-636): Sc = clamp(S, lo, hi) and
// F <- F V diag(Sc / max(S, 1e-12)) V^T, every product rounded as the
// reference's matmuls round it.  S is replaced by Sc.
__device__ __forceinline__ void f_clamp_F(const float F0[9], const float V[9], float S[3], float lo, float hi,
                                          float Fc[9]) {
    float D[9], corr[9];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float sc = S[i] < lo ? lo : S[i];
        sc = sc > hi ? hi : sc;
        const float ratio = sc / (S[i] < 1e-12f ? 1e-12f : S[i]);
#pragma unroll
        for (int r = 0; r < 3; ++r) D[3 * r + i] = V[3 * r + i] * ratio;
        S[i] = sc;
    }
    mmt3_rn(D, V, corr);   // V diag(Sc/S) V^T
    mm3_rn(F0, corr, Fc);
}

// _resolve (anisompm.py:811-825) for one node
__device__ __forceinline__ void resolve(float v[3], const float vc[3], const float nn[3], bool sticky, float fr) {
    if (sticky) {
        v[0] = vc[0]; v[1] = vc[1]; v[2] = vc[2];
        return;
    }
    // every op rounded separately, as the reference's tensor ops round them
    const float r0 = __fsub_rn(v[0], vc[0]), r1 = __fsub_rn(v[1], vc[1]), r2 = __fsub_rn(v[2], vc[2]);
    const float vn = dot3_rn(r0, nn[0], r1, nn[1], r2, nn[2]);
    const float inward = vn < 0.0f ? vn : 0.0f;
    float t0 = __fsub_rn(r0, __fmul_rn(vn, nn[0])), t1 = __fsub_rn(r1, __fmul_rn(vn, nn[1])),
          t2 = __fsub_rn(r2, __fmul_rn(vn, nn[2]));
    if (fr > 0.0f) {
        const float vtm = sqrtf(dot3_rn(t0, t0, t1, t1, t2, t2));
        float sc = __fadd_rn(1.0f, __fdiv_rn(__fmul_rn(fr, inward), __fadd_rn(vtm, 1e-9f)));
        sc = sc < 0.0f ? 0.0f : sc;
        t0 = __fmul_rn(t0, sc); t1 = __fmul_rn(t1, sc); t2 = __fmul_rn(t2, sc);
    }
    const float keep = __fsub_rn(vn, inward);
    v[0] = __fadd_rn(__fadd_rn(vc[0], t0), __fmul_rn(keep, nn[0]));
    v[1] = __fadd_rn(__fadd_rn(vc[1], t1), __fmul_rn(keep, nn[1]));
    v[2] = __fadd_rn(__fadd_rn(vc[2], t2), __fmul_rn(keep, nn[2]));
}

// Whether grid node position `pos` lies inside collider `col` (origin o at
// this substep), and its outward normal there: halfspace_collider
// (anisompm.py:847-867) tests (pos - o) . n < 0 with the normalised normal;
// sphere_collider (828-844) tests |pos - o| < radius, normal (pos - o) /
// (|pos - o| + 1e-9).  Each op rounded separately as the reference's tensor
// ops round them.
__device__ __forceinline__ bool collider_hit(const pm_collider &col, const float o[3], const float pos[3],
                                             float nn[3]) {
    if (col.kind == 0) {
        nn[0] = (float)col.normal[0]; nn[1] = (float)col.normal[1]; nn[2] = (float)col.normal[2];
        const float sd = dot3_rn(__fsub_rn(pos[0], o[0]), nn[0], __fsub_rn(pos[1], o[1]), nn[1],
                                 __fsub_rn(pos[2], o[2]), nn[2]);
        return sd < 0.0f;
    }
    const float r0 = pos[0] - o[0], r1 = pos[1] - o[1], r2 = pos[2] - o[2];
    const float dist = sqrtf(dot3_rn(r0, r0, r1, r1, r2, r2));
    if (!(dist < (float)col.radius)) return false;
    const float den = dist + 1e-9f;
    nn[0] = r0 / den; nn[1] = r1 / den; nn[2] = r2 / den;
    return true;
}

// ------------------------------------------------------- cell-aggregated scatter
// Quadratic weights of one axis from fx (anisompm.py:549-556).
__device__ __forceinline__ void qw(float f, float w[3]) {
    const float t0 = 1.5f - f, t1 = f - 1.0f, t2 = f - 0.5f;
    w[0] = 0.5f * (t0 * t0);
    w[1] = 0.75f - t1 * t1;
    w[2] = 0.5f * (t2 * t2);
}
// Cubic weights of one axis expanded onto the 5 nodes [qb-1, qb+3] of a
// quadratic cell: with s = (fx >= 1) the particle's cubic base is qb - 1 + s
// and its fraction f = fx - s (both exact), so node n takes weight w[n - s]
// (anisompm.py:575-583).  cw5_2 expands the second-derivative factors w''
// (anisompm.py:579-583) the same way.
__device__ __forceinline__ void cw5(float fx, float e[5]) {
    const bool s1 = fx >= 1.0f;
    const float f = s1 ? fx - 1.0f : fx;
    const float one = 1.0f - f;
    const float w0 = (1.0f / 6.0f) * (one * one * one);
    const float w1 = (2.0f / 3.0f - f * f) + 0.5f * (f * f * f);
    const float w2 = (2.0f / 3.0f - one * one) + 0.5f * (one * one * one);
    const float w3 = (1.0f / 6.0f) * (f * f * f);
    e[0] = s1 ? 0.0f : w0;
    e[1] = s1 ? w0 : w1;
    e[2] = s1 ? w1 : w2;
    e[3] = s1 ? w2 : w3;
    e[4] = s1 ? w3 : 0.0f;
}
__device__ __forceinline__ void cw5_2(float fx, float e[5]) {
    const bool s1 = fx >= 1.0f;
    const float f = s1 ? fx - 1.0f : fx;
    const float w0 = 1.0f - f, w1 = 3.0f * f - 2.0f, w2 = 1.0f - 3.0f * f, w3 = f;
    e[0] = s1 ? 0.0f : w0;
    e[1] = s1 ? w0 : w1;
    e[2] = s1 ? w1 : w2;
    e[3] = s1 ? w2 : w3;
    e[4] = s1 ? w3 : 0.0f;
}

// A node's fixed-point sum over one chunk of work, split over two 32-bit
// planes: `lo` sums the low kSplitBits bits of every contribution (unsigned,
// so at most 2^(32 - kSplitBits) = 256 contributions per node and chunk) and
// `hi` the rest (q >> kSplitBits, signed; a contribution is below 2^kFixBits
// per particle, so a chunk of 256 particles keeps |hi| under 2^31).  Both
// adds are fire-and-forget (no returned value, no carry chain) and
// unconditional (a branch per add costs more than adding a zero); the pair
// is folded into an int64 tile, exactly, before either plane can overflow:
// after every chunk in the adjoint scatter, after every fourth chunk in the
// forward P2G (whose adds per particle are below 0.42 of 2^kFixBits).
constexpr int kSplitBits = 24;
__device__ __forceinline__ void plane_add(unsigned *lo, int *hi, float v, float scale) {
    const long long q = to_fix(v, scale);
    atomicAdd(lo, (unsigned)q & ((1u << kSplitBits) - 1u));
    atomicAdd(hi, (int)(q >> kSplitBits));
}
__device__ __forceinline__ long long plane_value(unsigned lo, int hi) {
    return (long long)hi * (1LL << kSplitBits) + (long long)lo;
}
// The same for an entry in global memory: one 64-bit atomic.
__device__ __forceinline__ void red_fix(long long *addr, float v, float scale) {
    const long long q = to_fix(v, scale);
    if (q != 0) atomicAdd((unsigned long long *)addr, (unsigned long long)q);
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace pm
