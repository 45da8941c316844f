// Reverse-mode adjoint of one plain substep (anisompm.py:593-803) for the
// differentiable form: given the adjoints of the state after substep t
// (x', v', F', C', d', lap', D_hist'), produce the adjoints of the state
// before it and accumulate the gradients of the per-particle parameters mu,
// lam, sigma_c and A0.
//
// The forward substep t is first recorded (pm_substep_record) into a tape
// slot: grid velocity and mass {v, m}, the normalised damage field gd, the
// cubic weight sums, the active 4^3 block list and the step's clock.  The
// adjoint then runs four kernels:
//   k_adj_pre       per particle (particle order): the G2P tail adjoint and
//                   the G2P adjoint's scatter payload, written to the
//                   particle's slot of the forward substep's recorded sort,
//                   and the bounds that fix the fixed-point units;
//   k_adj_tiles     G2P adjoint as a scatter over the recorded sub-block work
//                   list (the forward P2G's cell-aggregated tiles): the adjoint
//                   of the grid velocity and damage field in int64 fixed
//                   point, so the sums do not depend on the atomics' order and
//                   a backward pass is reproducible bit for bit;
//   k_adj_grid      grid-update adjoint over the recorded active blocks
//                   (normalisation by mass and by the cubic weight sum);
//   k_adj_particle  P2G adjoint as a gather plus the constitutive adjoint
//                   (particle order): recomputes the particle's constitutive
//                   update, gathers the grid adjoints, and runs the polar,
//                   stress, damage and eigen-split adjoints.
// Non-smooth operations take the branch the forward took (relu, max and clamp
// pass the adjoint where the forward passed the value; base cells are
// piecewise constant).  The strain limit (f_clamp) is differentiated as a
// function of the singular values (f_clamp_adj), grid colliders from the
// recorded pre-collider grid velocity (resolve_adj), and the directional
// stress at interface particles by dir_adjoint.
#include "pm_kernels.cuh"

namespace pm {

namespace {

__device__ __forceinline__ float relu_f(float v) { return v > 0.0f ? v : 0.0f; }

// Tape header of one slot.
struct TapeHead {
    unsigned n_active;
    int any_allow;
    long long step;
    double time;
    unsigned n_work;    // non-empty sub-blocks of the substep's sort
    unsigned pad;
    float col_origin[PM_MAX_COLLIDERS][3];   // the substep's collider origins and velocities
    float col_vel[PM_MAX_COLLIDERS][3];
};

// Control block of one adjoint substep: the bounds of the scatter's
// contributions (float bits) and the dynamic work cursor.
struct AdjCtrl {
    unsigned mom_bound, lap_bound, work_next, pad;
    unsigned slots[2][kBoundSlots];   // per-warp-slot bounds, folded by k_adj_bounds
};

// Quadratic weights with their derivatives wrt the local coordinate fx.
struct QuadD {
    int b[3];
    float fx[3];
    float w[3][3], dw[3][3];
};
__device__ __forceinline__ void quad_weights_d(const float x[3], float inv_dx, int ng, QuadD &q) {
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
        q.dw[0][a] = -t0;
        q.dw[1][a] = -2.0f * t1;
        q.dw[2][a] = t2;
    }
}

// Cubic weights, second derivatives and the derivatives of both wrt f.
struct CubicD {
    int b[3];
    float w[4][3], w2[4][3], dw[4][3], dw2[4][3];
};
__device__ __forceinline__ void cubic_weights_d(const float x[3], float inv_dx, int ng, CubicD &c) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float X = __fmul_rn(x[a], inv_dx);
        const float fb = floorf(X);
        c.b[a] = sat_base(fb, ng) - 1;
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
        c.dw[0][a] = -0.5f * one * one;
        c.dw[1][a] = -2.0f * f + 1.5f * f * f;
        c.dw[2][a] = 2.0f * one - 1.5f * one * one;
        c.dw[3][a] = 0.5f * f * f;
        c.dw2[0][a] = -1.0f;
        c.dw2[1][a] = 3.0f;
        c.dw2[2][a] = -3.0f;
        c.dw2[3][a] = 1.0f;
    }
}

__device__ __forceinline__ int node_of(int x, int y, int z, int ng) {
    return (clampi(x, 0, ng - 1) * ng + clampi(y, 0, ng - 1)) * ng + clampi(z, 0, ng - 1);
}

struct AdjIn {
    float xb[3], vb[3], Cb[9], Fb[9], db, lapb, Dhb;
};
__device__ __forceinline__ void load_adj(const pm_state_adj &A, long long p, AdjIn &a) {
    const long long s = A.plane_stride;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a.xb[k] = A.x[k * s + p];
        a.vb[k] = A.v[k * s + p];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        a.Cb[k] = A.C[k * s + p];
        a.Fb[k] = A.F[k * s + p];
    }
    a.db = A.d[p];
    a.lapb = A.lap[p];
    a.Dhb = A.D_hist[p];
}

// Adjoint of the end of G2P: x' = clamp(x + dt v'), F' = (I + dt C') F.
// Returns the total adjoints of v' and C' and the pass-through mask of x.
__device__ __forceinline__ void g2p_tail_adj(const pm_params &prm, const float xp[3], const float vpost[3],
                                             const float Fpre[9], const AdjIn &a, float vt[3], float Ct[9],
                                             bool inside[3]) {
    const float dt = (float)prm.dt;
    const float pad = (float)(2.0 * prm.dx), hi = (float)(prm.grid_lim - 2.0 * prm.dx);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float t = xp[k] + dt * vpost[k];
        inside[k] = (t >= pad) && (t <= hi);
        vt[k] = a.vb[k] + (inside[k] ? dt * a.xb[k] : 0.0f);
    }
    // C' enters F' = (I + dt C') F: Cbar += dt Fbar' F^T
    float FbFt[9];
    mmt3(a.Fb, Fpre, FbFt);
#pragma unroll
    for (int k = 0; k < 9; ++k) Ct[k] = a.Cb[k] + dt * FbFt[k];
}

// The F that G2P updated: with the strain limit, the limited F rebuilt from
// the taped V and S as the forward built it.
__device__ __forceinline__ void g2p_input_F(const pm_params &prm, const float *__restrict__ tpol, long long rs,
                                            long long p, float F[9]) {
    if (!prm.use_f_clamp) return;
    float V[9], S[3];
#pragma unroll
    for (int k = 0; k < 9; ++k) V[k] = tpol[(9 + k) * rs + p];
#pragma unroll
    for (int k = 0; k < 3; ++k) S[k] = tpol[(18 + k) * rs + p];
    f_clamp_F(F, V, S, (float)prm.f_clamp_lo, (float)prm.f_clamp_hi, F);
}

// ---------------------------------------------------------------- k_adj_pre
// Adjoint of v' = sum w v_i, C' = K sum w v_i dpos^T and lap' = sum L gd_i has
// the form of a P2G scatter: node i receives w (vt + K Ct dpos) and
// lb (w''x wy wz + wx w''y wz + wx wy w''z) with lb = L lapbar.  This kernel
// forms each particle's {fx | x, lb}, vt and K Ct (the momentum scatter's
// {fx, mv, aff} slots) at its position in the forward substep's sort.
constexpr int kAdjCW = 30;   // expanded cubic w and w'' per particle (5 per axis each)

__global__ void __launch_bounds__(256) k_adj_pre(const pm_params prm, const Parts pre, const Parts post,
                                                 const pm_state_adj ain, const int *__restrict__ iperm,
                                                 float4 *__restrict__ pay, AdjCtrl *actl,
                                                 const float *__restrict__ tpol, long long rs) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pre.n) return;
    const long long ps = pre.ps;
    const int ng = prm.n_grid;
    const float inv_dx = (float)prm.inv_dx, dx = (float)prm.dx;
    const float K = (float)(4.0 * prm.inv_dx * prm.inv_dx);
    const float L2 = (float)(prm.inv_dx * prm.inv_dx);
    float xp[3], vpost[3], F[9];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        xp[k] = pre.x[k * ps + p];
        vpost[k] = post.v[k * ps + p];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = pre.F[k * ps + p];
    g2p_input_F(prm, tpol, rs, p, F);
    AdjIn a;
    load_adj(ain, p, a);
    float vt[3], Ct[9];
    bool inside[3];
    g2p_tail_adj(prm, xp, vpost, F, a, vt, Ct, inside);
    float kc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) kc[k] = K * Ct[k];
    const float lb = a.lapb * L2;
    float fx[3];
    bool reg = true;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const float X = __fmul_rn(xp[ax], inv_dx);
        const float fb = floorf(__fsub_rn(X, 0.5f));
        reg = reg && (fb >= 1.0f) && (fb <= (float)(ng - 4));
        fx[ax] = __fsub_rn(X, fb);
    }
    float4 *dst = pay + 5 * (long long)iperm[p];
    dst[0] = reg ? make_float4(fx[0], fx[1], fx[2], 0.0f) : make_float4(xp[0], xp[1], xp[2], 0.0f);
    dst[1] = make_float4(vt[0], vt[1], vt[2], lb);
    dst[2] = make_float4(kc[0], kc[1], kc[2], kc[3]);
    dst[3] = make_float4(kc[4], kc[5], kc[6], kc[7]);
    dst[4] = make_float4(kc[8], reg ? 1.0f : 0.0f, 0.0f, 0.0f);
    // bounds of one node contribution: |w (vt + K Ct dpos)| with w <= 1,
    // |dpos| <= 1.5 dx per axis (the cubic stencil's quadratic part), and
    // |lb W''| with |w''x wy wz + wx w''y wz + wx wy w''z| <= 3 (|w''| <= 2, w <= 2/3)
    const float hx = 1.5f * dx;
    float bm = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        bm = fmaxf(bm, fabsf(vt[c]) + hx * (fabsf(kc[3 * c]) + fabsf(kc[3 * c + 1]) + fabsf(kc[3 * c + 2])));
    unsigned bmom = bound_bits(bm), blap = bound_bits(3.0f * lb);
    const unsigned am = __activemask();
    bmom = __reduce_max_sync(am, bmom);
    blap = __reduce_max_sync(am, blap);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(am) - 1)) {
        const int slot = (int)(((blockIdx.x << 3) + (threadIdx.x >> 5)) & (kBoundSlots - 1));
        atomicMax(&actl->slots[0][slot], bmom);
        atomicMax(&actl->slots[1][slot], blap);
    }
}

__global__ void __launch_bounds__(kBoundSlots) k_adj_bounds(AdjCtrl *actl) {
    __shared__ unsigned s_m[2][kBoundSlots / 32];
    const int t = threadIdx.x;
#pragma unroll
    for (int v = 0; v < 2; ++v) {
        const unsigned m = __reduce_max_sync(0xffffffffu, actl->slots[v][t]);
        if ((t & 31) == 0) s_m[v][t >> 5] = m;
    }
    __syncthreads();
    if (t < 2) {
        unsigned m = 0u;
#pragma unroll
        for (int k = 0; k < kBoundSlots / 32; ++k) m = max(m, s_m[t][k]);
        if (t == 0) actl->mom_bound = m;
        else actl->lap_bound = m;
    }
}

// One particle whose stencil needs the reference's edge clamping, straight
// into the global adjoint grid (4 int64 per node: momentum adjoint, damage
// adjoint).
__device__ __noinline__ void adj_scatter_global(const float xp[3], const float vt[3], const float kc[9], float lb,
                                                float inv_dx, float dx, int ng, float smom, float slap,
                                                long long *acc) {
    Quad q;
    quad_weights(xp, inv_dx, ng, q);
    Cubic c;
    cubic_weights(xp, inv_dx, ng, c);
    float wq[3][4], U[3][4][3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const bool s1 = q.b[ax] != c.b[ax];   // quadratic base one node above the cubic one
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            float w = 0.0f, oq = 0.0f;
            if (s1) {
                if (o >= 1) { w = q.w[o - 1][ax]; oq = (float)(o - 1); }
            } else {
                if (o < 3) { w = q.w[o][ax]; oq = (float)o; }
            }
            wq[ax][o] = w;
            const float dp = (oq - q.fx[ax]) * dx;
#pragma unroll
            for (int i = 0; i < 3; ++i) U[ax][o][i] = kc[3 * i + ax] * dp;
        }
    }
#pragma unroll
    for (int ox = 0; ox < 4; ++ox)
#pragma unroll
        for (int oy = 0; oy < 4; ++oy) {
            const float ab = lb * (c.w2[ox][0] * c.w[oy][1] + c.w[ox][0] * c.w2[oy][1]);
            const float e = lb * (c.w[ox][0] * c.w[oy][1]);
            const float wxy = wq[0][ox] * wq[1][oy];
            const float b0 = vt[0] + U[0][ox][0] + U[1][oy][0];
            const float b1 = vt[1] + U[0][ox][1] + U[1][oy][1];
            const float b2 = vt[2] + U[0][ox][2] + U[1][oy][2];
            const long long row = ((long long)clampi(c.b[0] + ox, 0, ng - 1) * ng + clampi(c.b[1] + oy, 0, ng - 1)) * ng;
#pragma unroll
            for (int oz = 0; oz < 4; ++oz) {
                const float wk = wxy * wq[2][oz];
                long long *g = acc + 4 * (row + clampi(c.b[2] + oz, 0, ng - 1));
                red_fix(g, wk * (b0 + U[2][oz][0]), smom);
                red_fix(g + 1, wk * (b1 + U[2][oz][1]), smom);
                red_fix(g + 2, wk * (b2 + U[2][oz][2]), smom);
                red_fix(g + 3, ab * c.w[oz][2] + e * c.w2[oz][2], slap);
            }
        }
}

// ---------------------------------------------------------------- k_adj_tiles
// The G2P adjoint scatter over the forward substep's non-empty 4^3-cell
// sub-blocks, with the forward P2G's cell-aggregated (cell, x-slab) items:
// quadratic slabs sum w (vt + K Ct dpos) into the momentum-adjoint tile
// (nodes [4s, 4s+6)^3), cubic slabs sum lb W'' into the damage-adjoint tile
// (nodes [4s-1, 4s+7)^3), both int64 fixed point, flushed with one atomic per
// touched node and component.  The adjoint touches exactly the nodes the
// forward P2G touched, so no block marks are needed.
constexpr int kATh = 256;
constexpr int kAPayStride = kATh + kATh / 32;
constexpr int kASub = 4, kAQE = 6, kACE = 8, kAQN = 216, kACN = 512;
// chunk planes with the forward P2G's conflict-free strides (z 1, y 8, x 52 / 68)
constexpr int kAQSY = 8, kAQSX = 52, kAQPl = 312, kACSY = 8, kACSX = 68, kACPl = 544;
constexpr size_t kAdjTileSmem = sizeof(unsigned) * 2 * (3 * kAQPl + kACPl) +
                                sizeof(float) * (17 + kAdjCW) * kAPayStride + sizeof(int) * (kATh + 2) + 2 * kATh;

__global__ void __launch_bounds__(kATh, 3) k_adj_tiles(const pm_params prm, const unsigned *__restrict__ keys,
                                                       const int *__restrict__ work, const TapeHead *head,
                                                       const float4 *__restrict__ pay, AdjCtrl *actl,
                                                       long long *__restrict__ acc, long long n) {
    extern __shared__ long long s_adj[];
    unsigned (*qlo)[kAQPl] = (unsigned (*)[kAQPl])(s_adj);                // [3][kAQPl] chunk planes
    int (*qhi)[kAQPl] = (int (*)[kAQPl])(qlo[3]);                         // [3][kAQPl]
    unsigned *clo = (unsigned *)(qhi[3]);                                 // [kACPl]
    int *chi = (int *)(clo + kACPl);                                      // [kACPl]
    float (*sp)[kAPayStride] = (float (*)[kAPayStride])(chi + kACPl);    // [17][kAPayStride]
    float (*cw)[kAPayStride] = (float (*)[kAPayStride])(sp[17]);        // [kAdjCW][kAPayStride]
    int *runs = (int *)(cw[kAdjCW]);                                      // [kATh + 2]
    unsigned char *regular = (unsigned char *)(runs + kATh + 2);          // [kATh]
    unsigned char *lcell = regular + kATh;                                // [kATh]
    __shared__ int s_wcnt[kATh / 32];
    __shared__ unsigned s_item;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const unsigned n_work = min(head->n_work, (unsigned)min(n, (long long)0x7fffffff));
    const int ng = prm.n_grid;
    const int nb = sort_blocks_per_axis(ng);
    const float inv_dx = (float)prm.inv_dx, dx = (float)prm.dx;
    const float smom = fix_scale(actl->mom_bound).scale, slap = fix_scale(actl->lap_bound).scale;
    for (int i = tid; i < 2 * (3 * kAQPl + kACPl); i += kATh) qlo[0][i] = 0u;
    for (;;) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(&actl->work_next, 1u);
        __syncthreads();
        const unsigned item = s_item;
        if (item >= n_work) break;
        const long long a = work[item];
        const unsigned key0 = keys[a];
        const unsigned sbk = key0 >> 6;
        const unsigned blk = key0 >> kSortBlockBits;
        const int bz = (int)(blk % nb), by = (int)((blk / nb) % nb), bx = (int)(blk / ((unsigned)nb * nb));
        const unsigned oct = (key0 >> 6) & 7u;
        const int org[3] = {bx * kSortBlock + (int)((oct >> 2) & 1u) * kASub,
                            by * kSortBlock + (int)((oct >> 1) & 1u) * kASub,
                            bz * kSortBlock + (int)(oct & 1u) * kASub};
        int pending = 0;   // chunks with particles since the planes were last folded
        for (long long sub = a;; sub += kATh) {
            const long long i = sub + tid;
            const unsigned key = i < n ? keys[i] : 0xffffffffu;
            const bool valid = i < n && (key >> 6) == sbk;
            if (valid) {
                const float4 *src = pay + 5 * i;
                const float4 q0 = src[0], q1 = src[1], q2 = src[2], q3 = src[3], q4 = src[4];
                const int t = tid + (tid >> 5);
                sp[0][t] = q0.x; sp[1][t] = q0.y; sp[2][t] = q0.z;
                sp[3][t] = q1.x; sp[4][t] = q1.y; sp[5][t] = q1.z; sp[16][t] = q1.w;
                sp[6][t] = q2.x; sp[7][t] = q2.y; sp[8][t] = q2.z; sp[9][t] = q2.w;
                sp[10][t] = q3.x; sp[11][t] = q3.y; sp[12][t] = q3.z; sp[13][t] = q3.w;
                sp[14][t] = q4.x;
                regular[tid] = q4.y != 0.0f ? 1 : 0;
                lcell[tid] = (unsigned char)(key & 63u);
                if (q4.y != 0.0f) {
                    float e[5];
                    cw5(q0.x, e);
#pragma unroll
                    for (int k = 0; k < 5; ++k) cw[k][t] = e[k];
                    cw5(q0.y, e);
#pragma unroll
                    for (int k = 0; k < 5; ++k) cw[5 + k][t] = e[k];
                    cw5(q0.z, e);
#pragma unroll
                    for (int k = 0; k < 5; ++k) cw[10 + k][t] = e[k];
                    cw5_2(q0.x, e);
#pragma unroll
                    for (int k = 0; k < 5; ++k) cw[15 + k][t] = e[k];
                    cw5_2(q0.y, e);
#pragma unroll
                    for (int k = 0; k < 5; ++k) cw[20 + k][t] = e[k];
                    cw5_2(q0.z, e);
#pragma unroll
                    for (int k = 0; k < 5; ++k) cw[25 + k][t] = e[k];
                }
            }
            int nruns, cnt;
            {
                const unsigned prev = (tid > 0 && i <= n) ? keys[i - 1] : 0xffffffffu;
                const bool flag = valid && (tid == 0 || key != prev);
                const unsigned fb = __ballot_sync(0xffffffffu, flag), vb = __ballot_sync(0xffffffffu, valid);
                if (lane == 0) s_wcnt[wid] = (int)(__popc(fb) | (__popc(vb) << 16));
                __syncthreads();
                int pos = __popc(fb & lanemask_lt()), tot = 0, vt = 0;
#pragma unroll
                for (int w2 = 0; w2 < kATh / 32; ++w2) {
                    const int c = s_wcnt[w2];
                    pos += (w2 < wid) ? (c & 0xffff) : 0;
                    tot += c & 0xffff;
                    vt += c >> 16;
                }
                if (flag) runs[pos] = tid;
                if (tid == 0) runs[tot] = vt;
                nruns = tot;
                cnt = vt;
                __syncthreads();
            }
            if (valid && !regular[tid]) {
                const int t = tid + (tid >> 5);
                const float xp[3] = {sp[0][t], sp[1][t], sp[2][t]};
                const float vt[3] = {sp[3][t], sp[4][t], sp[5][t]};
                float kc[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) kc[k] = sp[6 + k][t];
                adj_scatter_global(xp, vt, kc, sp[16][t], inv_dx, dx, ng, smom, slap, acc);
            }
            for (int it = tid; it < nruns * 8; it += kATh) {   // slab-major, as the forward P2G
                const bool quad = it < 3 * nruns;
                const int k = quad ? it : it - 3 * nruns;
                const int s8 = k / nruns;
                const int r = k - s8 * nruns;
                const int sl = quad ? s8 : 3 + s8;
                const int ja = runs[r], jb = runs[r + 1];
                int cq[3];
                morton_decode(lcell[ja], cq);
                if (sl < 3) {
                    const int ox = sl;
                    // packed pairs: components (0, 1) of every node, component 2 alone
                    float2 acc01[3][3];
                    float acc2[3][3];
#pragma unroll
                    for (int i2 = 0; i2 < 3; ++i2)
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            acc01[i2][j] = make_float2(0.0f, 0.0f);
                            acc2[i2][j] = 0.0f;
                        }
                    // a cell's particles share their base cell: all regular or all not
                    const int jend = regular[ja] ? jb : ja;
                    for (int j = ja; j < jend; ++j) {
                        const int t = j + (j >> 5);
                        const float fx0 = sp[0][t], fx1 = sp[1][t], fx2 = sp[2][t];
                        float wx[3], wy[3], wz[3];
                        qw(fx0, wx); qw(fx1, wy); qw(fx2, wz);
                        const float dxo = ((float)ox - fx0) * dx;
                        const float2 base01 = fma2(make_float2(sp[6][t], sp[9][t]), bc2(dxo),
                                                   make_float2(sp[3][t], sp[4][t]));
                        const float base2 = sp[5][t] + sp[12][t] * dxo;
                        const float2 ay01 = make_float2(sp[7][t], sp[10][t]), az01 = make_float2(sp[8][t], sp[11][t]);
                        const float ay2 = sp[13][t], az2 = sp[14][t];
                        const float wxs = ox == 0 ? wx[0] : (ox == 1 ? wx[1] : wx[2]);
                        // w (base + a_y dy + a_z dz) = wxy [wz (base + a_z dz)] + [wxy a_y dy] wz
                        float2 bz01[3], wz2[3];
                        float bz2[3];
#pragma unroll
                        for (int oz = 0; oz < 3; ++oz) {
                            const float dz = ((float)oz - fx2) * dx;
                            wz2[oz] = bc2(wz[oz]);
                            bz01[oz] = mul2(wz2[oz], fma2(az01, bc2(dz), base01));
                            bz2[oz] = wz[oz] * (base2 + az2 * dz);
                        }
#pragma unroll
                        for (int oy = 0; oy < 3; ++oy) {
                            const float wxy = wxs * wy[oy];
                            const float wdy = wxy * (((float)oy - fx1) * dx);
                            const float2 w2 = bc2(wxy), ady01 = mul2(bc2(wdy), ay01);
                            const float ady2 = wdy * ay2;
#pragma unroll
                            for (int oz = 0; oz < 3; ++oz) {
                                acc01[oy][oz] = fma2(ady01, wz2[oz], fma2(w2, bz01[oz], acc01[oy][oz]));
                                acc2[oy][oz] = fmaf(ady2, wz[oz], fmaf(wxy, bz2[oz], acc2[oy][oz]));
                            }
                        }
                    }
                    const int nx = cq[0] + ox;
#pragma unroll
                    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                        for (int oz = 0; oz < 3; ++oz) {
                            const int sidx = nx * kAQSX + (cq[1] + oy) * kAQSY + cq[2] + oz;
                            plane_add(&qlo[0][sidx], &qhi[0][sidx], acc01[oy][oz].x, smom);
                            plane_add(&qlo[1][sidx], &qhi[1][sidx], acc01[oy][oz].y, smom);
                            plane_add(&qlo[2][sidx], &qhi[2][sidx], acc2[oy][oz], smom);
                        }
                } else {
                    const int nxs = sl - 3;
                    // packed pairs of z-neighbours: nodes (0, 1), (2, 3) of a row, node 4 alone
                    float2 al01[5], al23[5];
                    float al4[5];
#pragma unroll
                    for (int i2 = 0; i2 < 5; ++i2) {
                        al01[i2] = al23[i2] = make_float2(0.0f, 0.0f);
                        al4[i2] = 0.0f;
                    }
                    const int jend = regular[ja] ? jb : ja;
                    for (int j = ja; j < jend; ++j) {
                        const int t = j + (j >> 5);
                        const float lb = sp[16][t];
                        const float ax = lb * cw[15 + nxs][t], bx2 = lb * cw[nxs][t];   // lb w''x, lb wx
                        const float2 ez01 = make_float2(cw[10][t], cw[11][t]), ez23 = make_float2(cw[12][t], cw[13][t]);
                        const float2 e2z01 = make_float2(cw[25][t], cw[26][t]), e2z23 = make_float2(cw[27][t], cw[28][t]);
                        const float ez4 = cw[14][t], e2z4 = cw[29][t];
#pragma unroll
                        for (int ny = 0; ny < 5; ++ny) {
                            const float wy = cw[5 + ny][t], w2y = cw[20 + ny][t];
                            const float t1 = ax * wy + bx2 * w2y;   // (w''x wy + wx w''y) lb
                            const float t2 = bx2 * wy;              // wx wy lb
                            const float2 t12 = bc2(t1), t22 = bc2(t2);
                            al01[ny] = fma2(t22, e2z01, fma2(t12, ez01, al01[ny]));
                            al23[ny] = fma2(t22, e2z23, fma2(t12, ez23, al23[ny]));
                            al4[ny] = fmaf(t2, e2z4, fmaf(t1, ez4, al4[ny]));
                        }
                    }
                    const int nx = cq[0] + nxs;
#pragma unroll
                    for (int ny = 0; ny < 5; ++ny)
#pragma unroll
                        for (int nz = 0; nz < 5; ++nz)
                        {
                            const int sidx = nx * kACSX + (cq[1] + ny) * kACSY + cq[2] + nz;
                            const float a = nz == 0 ? al01[ny].x : nz == 1 ? al01[ny].y : nz == 2 ? al23[ny].x
                                          : nz == 3 ? al23[ny].y : al4[ny];
                            plane_add(&clo[sidx], &chi[sidx], a, slap);
                        }
                }
            }
            __syncthreads();
            const bool last = cnt < kATh;
            pending += cnt > 0 ? 1 : 0;
            // fold the chunk planes straight into the global grid, one int64
            // atomic per nonzero node component, after every second chunk with
            // particles and after the last: one add per particle and node is
            // below 0.89 of 2^46 units (|w''x wy wz + wx w''y wz + wx wy w''z|
            // <= 2.67 against the bound's 3), so two chunks keep the high
            // plane under 512 * 0.89 * 2^22 < 2^31
            if (pending > 0 && (last || pending == 2)) {
                pending = 0;
                for (int li = tid; li < kAQN; li += kATh) {
                    const int tx = li / (kAQE * kAQE), ty = (li / kAQE) % kAQE, tz = li % kAQE;
                    const int sidx = tx * kAQSX + ty * kAQSY + tz;
                    long long q[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const unsigned lo = qlo[c][sidx];
                        const int hi = qhi[c][sidx];
                        q[c] = 0;
                        if ((lo | (unsigned)hi) != 0u) {
                            qlo[c][sidx] = 0u;
                            qhi[c][sidx] = 0;
                            q[c] = plane_value(lo, hi);
                        }
                    }
                    if ((q[0] | q[1] | q[2]) != 0) {
                        long long *g = acc + 4 * (((long long)(org[0] + tx) * ng + (org[1] + ty)) * ng + (org[2] + tz));
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                            if (q[c]) atomicAdd((unsigned long long *)(g + c), (unsigned long long)q[c]);
                    }
                }
                for (int li = tid; li < kACN; li += kATh) {
                    const int tx = li >> 6, ty = (li >> 3) & 7, tz = li & 7;
                    const int sidx = tx * kACSX + ty * kACSY + tz;
                    const unsigned lo = clo[sidx];
                    const int hi = chi[sidx];
                    if ((lo | (unsigned)hi) != 0u) {
                        clo[sidx] = 0u;
                        chi[sidx] = 0;
                        const long long q3 = plane_value(lo, hi);
                        if (q3 != 0) {
                            long long *g = acc + 4 * (((long long)(org[0] - 1 + tx) * ng + (org[1] - 1 + ty)) * ng +
                                                      (org[2] - 1 + tz));
                            atomicAdd((unsigned long long *)(g + 3), (unsigned long long)q3);
                        }
                    }
                }
            }
            if (last) break;
            __syncthreads();
        }
    }
}

// Adjoint of resolve() (the reference's _resolve, anisompm.py:811-825) at
// input velocity v: vb holds the adjoint of the output on entry and of the
// input on return.  Sticky: the output is the collider velocity, a constant.
// Slip: torch's subgradient conventions, clamp passing where its input lies
// inside the bounds inclusive (vn <= 0 for the inward part, scale >= 0 for
// the friction factor) and the norm passing nothing at zero.
__device__ __forceinline__ void resolve_adj(const float v[3], const float vc[3], const float nn[3], bool sticky,
                                            float fr, float vb[3]) {
    if (sticky) {
        vb[0] = vb[1] = vb[2] = 0.0f;
        return;
    }
    const float r[3] = {v[0] - vc[0], v[1] - vc[1], v[2] - vc[2]};
    const float vn = r[0] * nn[0] + r[1] * nn[1] + r[2] * nn[2];
    const float inward = vn < 0.0f ? vn : 0.0f;
    const float t[3] = {r[0] - vn * nn[0], r[1] - vn * nn[1], r[2] - vn * nn[2]};
    const float keepb = vb[0] * nn[0] + vb[1] * nn[1] + vb[2] * nn[2];
    float tb[3] = {vb[0], vb[1], vb[2]};
    float inwardb = -keepb;
    if (fr > 0.0f) {
        const float vtm = sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        const float den = vtm + 1e-9f;
        const float sraw = 1.0f + fr * inward / den;
        const float sc = sraw < 0.0f ? 0.0f : sraw;
        const float scb = tb[0] * t[0] + tb[1] * t[1] + tb[2] * t[2];
#pragma unroll
        for (int a = 0; a < 3; ++a) tb[a] *= sc;
        if (sraw >= 0.0f) {
            inwardb += scb * fr / den;
            const float vtmb = -scb * fr * inward / (den * den);
            if (vtm > 0.0f) {
#pragma unroll
                for (int a = 0; a < 3; ++a) tb[a] += vtmb * t[a] / vtm;
            }
        }
    }
    float vnb = keepb - (tb[0] * nn[0] + tb[1] * nn[1] + tb[2] * nn[2]);
    if (vn <= 0.0f) vnb += inwardb;
#pragma unroll
    for (int a = 0; a < 3; ++a) vb[a] = tb[a] + vnb * nn[a];
}

// ---------------------------------------------------------------- k_adj_grid
// Grid-update adjoint over the recorded active blocks.  Forward (active node,
// m > 1e-12): v = (mv / m + dt g) * damp; gd = sum wd / sum w when sum w >
// 1e-12.  Writes A = {mvbar, mbar}, B = {sumwd bar, sumw bar, gd, 0} and
// clears acc.
__global__ void __launch_bounds__(256) k_adj_grid(const pm_params prm, const int *__restrict__ blocks,
                                                  const TapeHead *head, const float4 *__restrict__ gvel,
                                                  const float4 *__restrict__ vpre,
                                                  const float *__restrict__ ggd, const float *__restrict__ gsw,
                                                  long long *__restrict__ acc, const AdjCtrl *actl,
                                                  float4 *__restrict__ A, float4 *__restrict__ B,
                                                  long long n_blocks) {
    const float umom = fix_scale(actl->mom_bound).unit, ulap = fix_scale(actl->lap_bound).unit;
    const long long nact = min((long long)head->n_active, n_blocks);
    const long long items = nact * 64;
    const int ng = prm.n_grid, nbs = (ng + kBlockEdge - 1) / kBlockEdge;
    const float dt = (float)prm.dt, damp = (float)prm.grid_damp, dx = (float)prm.dx;
    const float dg[3] = {damp * dt * (float)prm.gravity[0], damp * dt * (float)prm.gravity[1],
                         damp * dt * (float)prm.gravity[2]};
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        const int b = blocks[it >> 6];
        const int l = (int)(it & 63);
        const int bx = b / (nbs * nbs), by = (b / nbs) % nbs, bz = b % nbs;
        const int ix = bx * kBlockEdge + (l >> 4), iy = by * kBlockEdge + ((l >> 2) & 3), iz = bz * kBlockEdge + (l & 3);
        if (ix >= ng || iy >= ng || iz >= ng) continue;
        const long long node = ((long long)ix * ng + iy) * ng + iz;
        longlong2 *an = (longlong2 *)(acc + 4 * node);
        const longlong2 a01 = an[0], a23 = an[1];
        an[0] = make_longlong2(0, 0);
        an[1] = make_longlong2(0, 0);
        const float4 ab = make_float4(from_fix(a01.x, umom), from_fix(a01.y, umom), from_fix(a23.x, umom),
                                      from_fix(a23.y, ulap));
        float4 gv = gvel[node];
        float4 ao = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (gv.w > 1e-12f) {
            float vb[3] = {ab.x, ab.y, ab.z};
            if (vpre && prm.n_colliders > 0) {
                // colliders (anisompm.py:737-746): rerun them from the recorded
                // pre-collider velocity, keeping each one's input, then walk
                // them back
                const float4 vp = vpre[node];
                const float pos[3] = {(float)ix * dx, (float)iy * dx, (float)iz * dx};
                float vs[PM_MAX_COLLIDERS][3], nrm[PM_MAX_COLLIDERS][3];
                unsigned hit = 0u;
                float v[3] = {vp.x, vp.y, vp.z};
                for (int c = 0; c < prm.n_colliders; ++c) {
                    vs[c][0] = v[0]; vs[c][1] = v[1]; vs[c][2] = v[2];
                    if (collider_hit(prm.colliders[c], head->col_origin[c], pos, nrm[c])) {
                        hit |= 1u << c;
                        resolve(v, head->col_vel[c], nrm[c], prm.colliders[c].mode == 1,
                                (float)prm.colliders[c].friction);
                    }
                }
                for (int c = prm.n_colliders - 1; c >= 0; --c)
                    if (hit & (1u << c))
                        resolve_adj(vs[c], head->col_vel[c], nrm[c], prm.colliders[c].mode == 1,
                                    (float)prm.colliders[c].friction, vb);
                gv.x = vp.x; gv.y = vp.y; gv.z = vp.z;   // the velocity the mass and momentum made
            }
            const float im = 1.0f / gv.w;
            const float u0 = damp * vb[0], u1 = damp * vb[1], u2 = damp * vb[2];
            ao.x = u0 * im; ao.y = u1 * im; ao.z = u2 * im;
            // mv / m = v / damp - dt g:  mbar = -damp vbar . (mv/m) / m
            ao.w = -(vb[0] * (gv.x - dg[0]) + vb[1] * (gv.y - dg[1]) + vb[2] * (gv.z - dg[2])) * im;
        }
        A[node] = ao;
        const float sw = gsw[node], gd = ggd[node];
        float4 bo = make_float4(0.0f, 0.0f, gd, 0.0f);
        if (sw > 1e-12f) {
            bo.x = ab.w / sw;
            bo.y = -ab.w * gd / sw;
        }
        B[node] = bo;
    }
}

// ---------------------------------------------------------------- constitutive
// What the adjoint keeps of the forward constitutive update.  The damage
// driving geometry (Cauchy stress eigensystem, sigma+, A, M) is not kept: it
// is needed only where the history drive is active, and is recomputed there.
struct Cons {
    float F[9], V[9], S[3], Sc[3], R[9], lamC[3];   // F: after the strain limit; S before it, Sc after
    bool fclamp, iface;
    float n0[3];   // interface normal (iface)
    float J, Jraw, tdev[9], tv;
    bool dmg;
    float phi, drive, Dh0, Dh1, d0, lap, arg, cc, u, dn, d1, g, vdeg, res, sc, zeta, l0;
    bool allow;
};

// Damage driving geometry (anisompm.py:650-664): sig = sym(tdev + tv I) / J,
// its eigensystem, sigma+ = Q relu(e) Q^T, A = R A0 R^T, M = A sigma+ and
// phi = tr(M M) / sigma_c^2.
struct DamageGeom {
    float sig[9], ev[3], Q[9], sp[9], A[9], M[9], A0[9];
    float phi;
};
__device__ __forceinline__ void damage_geom(const float R[9], const float V[9], const float S[3], const float tdev[9],
                                            float tv, float J, float sc, const Parts &P, long long p,
                                            DamageGeom &g) {
    const long long ps = P.ps;
    float sg[9];
    const float rJ = 1.0f / J;   // as the forward computes it
#pragma unroll
    for (int k = 0; k < 9; ++k) sg[k] = (tdev[k] + ((k % 4 == 0) ? tv : 0.0f)) * rJ;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) g.sig[3 * i + j] = 0.5f * (sg[3 * i + j] + sg[3 * j + i]);
    {   // eigensystem as the forward took it: U = R V from the taped polar decomposition
        float U[9];
        mm3(R, V, U);
        if (polar_u_ok(S))
            stress_eig_polar(U, g.sig, g.ev, g.Q);
        else
            sym_eig3<5>(g.sig, g.ev, g.Q);
    }
    {
        float ED[9];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float e = g.ev[j] < 0.0f ? 0.0f : g.ev[j];
#pragma unroll
            for (int i = 0; i < 3; ++i) ED[3 * i + j] = g.Q[3 * i + j] * e;
        }
        mmt3(ED, g.Q, g.sp);
    }
    {
        float RA[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) g.A0[k] = P.A0[k * ps + p];
        mm3(R, g.A0, RA);
        mmt3(RA, R, g.A);
    }
    mm3(g.A, g.sp, g.M);
    const float trMM = (g.M[0] * g.M[0] + g.M[1] * g.M[3] + g.M[2] * g.M[6]) +
                       (g.M[3] * g.M[1] + g.M[4] * g.M[4] + g.M[5] * g.M[7]) +
                       (g.M[6] * g.M[2] + g.M[7] * g.M[5] + g.M[8] * g.M[8]);
    g.phi = trMM / (sc * sc);
}


// Forward constitutive update without interface particles, as the forward
// kernel computes it (the strain limit included), keeping the intermediates.  The polar
// decomposition (R, V, S) and, on damage steps, phi come from the tape that
// the recorded forward wrote (pol[k * rs + p]: R 0..8, V 9..17, S 18..20,
// phi 21), so neither eigensolve is repeated here.
// EXT: the strain limit and interface particles are compiled in (a kernel
// without them keeps fewer registers live).
template <bool EXT>
__device__ __forceinline__ void cons_forward(const pm_params &prm, const Parts &P, long long p, bool do_damage,
                                             Cons &c, float tau[9], const float *__restrict__ pol, long long rs) {
    const long long ps = P.ps;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        c.F[k] = P.F[k * ps + p];
        c.R[k] = pol[k * rs + p];
        c.V[k] = pol[(9 + k) * rs + p];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        c.S[i] = pol[(18 + i) * rs + p];
        c.lamC[i] = c.S[i] > sqrtf(1e-12f) ? 1.0f : 0.0f;   // 0 where S = sqrt(max(lamC, 1e-12)) clamped
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) c.Sc[i] = c.S[i];
    c.fclamp = EXT && prm.use_f_clamp != 0;
    if (c.fclamp) f_clamp_F(c.F, c.V, c.Sc, (float)prm.f_clamp_lo, (float)prm.f_clamp_hi, c.F);
    c.Jraw = c.Sc[0] * c.Sc[1] * c.Sc[2];
    c.J = c.Jraw < 1e-6f ? 1e-6f : c.Jraw;
    const float mu = P.mu[p], lam = P.lam[p];
    {
        float FmR[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) FmR[k] = (2.0f * mu) * (c.F[k] - c.R[k]);
        mmt3(FmR, c.F, c.tdev);
    }
    c.tv = lam * (c.J - 1.0f) * c.J;
    c.dmg = do_damage;
    c.d0 = P.d[p];
    c.Dh0 = P.D_hist[p];
    c.d1 = c.d0;
    c.Dh1 = c.Dh0;
    c.allow = P.allow[p] != 0;
    if (do_damage) {
        c.sc = P.sigma_c[p];
        c.phi = pol[21 * rs + p];
        c.zeta = P.zeta[p];
        c.drive = c.zeta * relu_f(c.phi - 1.0f);
        c.Dh1 = c.drive > c.Dh0 ? c.drive : c.Dh0;
        c.l0 = P.l0[p];
        c.lap = P.lap[p];
        const float resist = c.d0 - (c.l0 * c.l0) * c.lap;
        c.arg = (1.0f - c.d0) * c.Dh1 - resist;
        const float ddot = relu_f(c.arg);
        const float dt_dmg = (float)(prm.dt * (double)prm.damage_every);
        c.cc = dt_dmg / P.eta[p];
        c.u = c.d0 + c.cc * ddot;
        c.dn = c.u < 0.0f ? 0.0f : (c.u > 1.0f ? 1.0f : c.u);
        if (c.allow) c.d1 = c.dn > c.d0 ? c.dn : c.d0;
    }
    c.res = P.residual[p];
    const float omd = 1.0f - c.d1;
    c.g = (omd * omd) * (1.0f - c.res) + c.res;
    c.vdeg = (c.J >= 1.0f) ? c.g : 1.0f;
#pragma unroll
    for (int k = 0; k < 9; ++k) tau[k] = c.g * c.tdev[k] + ((k % 4 == 0) ? c.vdeg * c.tv : 0.0f);
    c.iface = EXT && P.interface_mask && P.interface_mask[p];
    if (c.iface) {
        c.n0[0] = P.n_interface[p];
        c.n0[1] = P.n_interface[ps + p];
        c.n0[2] = P.n_interface[2 * ps + p];
    }
}

// Adjoint of the directional (delamination) stress at an interface particle
// (directional_kirchhoff, anisompm.py:190-227 via 697-703): tau = Q tc Q +
// gI P tc P + g (P tc Q + Q tc P) with tc = tdev + tv I, P = m m^T, Q = I - P,
// m = F n0 / (|F n0| + 1e-9) and gI = g where m^T tc m > 0, else 1.  Given
// taub: the adjoints of g (gb), tdev, tv and the direct part of F (Fb, added).
__device__ __forceinline__ void dir_adjoint(const Cons &c, const float taub[9], float &gb, float tdevb[9],
                                            float &tvb, float Fb[9]) {
    float tc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) tc[k] = c.tdev[k] + ((k % 4 == 0) ? c.tv : 0.0f);
    float u[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) u[i] = c.F[3 * i] * c.n0[0] + c.F[3 * i + 1] * c.n0[1] + c.F[3 * i + 2] * c.n0[2];
    const float un = sqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const float mn = un + 1e-9f;
    const float m[3] = {u[0] / mn, u[1] / mn, u[2] / mn};
    float Pm[9], Qm[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Pm[3 * i + j] = m[i] * m[j];
            Qm[3 * i + j] = ((i == j) ? 1.0f : 0.0f) - Pm[3 * i + j];
        }
    float snn = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) snn += m[i] * tc[3 * i + j] * m[j];
    const bool tens = snn > 0.0f;
    const float gI = tens ? c.g : 1.0f;
    // pieces of the forward, for the adjoint of g
    float T1[9], perp[9], shs[9], X[9];
    mm3(Pm, tc, T1);                        // P tc
    mm3(T1, Pm, perp);                      // P tc P
    mm3(T1, Qm, shs);                       // P tc Q
    mm3(Qm, tc, T1);                        // Q tc
    mm3(T1, Pm, X);                         // Q tc P
    gb = 0.0f;
#pragma unroll
    for (int k = 0; k < 9; ++k) gb += taub[k] * (shs[k] + X[k] + (tens ? perp[k] : 0.0f));
    // tcb = Q taub Q + gI P taub P + g (P taub Q + Q taub P)
    float PT[9], QT[9], A1[9], A2[9], A3[9], A4[9];
    mm3(Pm, taub, PT);
    mm3(Qm, taub, QT);
    mm3(QT, Qm, A1);
    mm3(PT, Pm, A2);
    mm3(PT, Qm, A3);
    mm3(QT, Pm, A4);
    float trc = 0.0f;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const float tcb = A1[k] + gI * A2[k] + c.g * (A3[k] + A4[k]);
        tdevb[k] = tcb;
        if (k % 4 == 0) trc += tcb;
    }
    tvb = trc;
    // Pbar, Qbar from the four products (P, Q symmetric; Xbar of each piece:
    // par taub, perp gI taub, both shears g taub)
    float Pb[9], Qb[9];
    {
        float tcP[9], tcQ[9], tcT[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) tcT[3 * i + j] = tc[3 * j + i];
        mm3(tcT, Pm, tcP);                  // tc^T P
        mm3(tcT, Qm, tcQ);                  // tc^T Q
        float PtcT[9], QtcT[9];
        mm3(Pm, tcT, PtcT);                 // P tc^T
        mm3(Qm, tcT, QtcT);                 // Q tc^T
        float B1[9], B2[9], B3[9], B4[9], B5[9], B6[9], B7[9], B8[9];
        mm3(taub, PtcT, B1);                // perp: Xb P tc^T
        mm3(tcP, taub, B2);                 //       tc^T P Xb
        mm3(taub, QtcT, B3);                // sh1 = P tc Q: Pb += Xb Q tc^T
        mm3(tcP, taub, B4);                 //               Qb += tc^T P Xb
        mm3(taub, PtcT, B5);                // sh2 = Q tc P: Qb += Xb P tc^T
        mm3(tcQ, taub, B6);                 //               Pb += tc^T Q Xb
        mm3(taub, QtcT, B7);                // par = Q tc Q: Qb += Xb Q tc^T
        mm3(tcQ, taub, B8);                 //               Qb += tc^T Q Xb
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            Pb[k] = gI * (B1[k] + B2[k]) + c.g * (B3[k] + B6[k]);
            Qb[k] = c.g * (B4[k] + B5[k]) + B7[k] + B8[k];
        }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) Pb[k] -= Qb[k];   // Q = I - P
    float mb[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        mb[i] = (Pb[3 * i] + Pb[i]) * m[0] + (Pb[3 * i + 1] + Pb[3 + i]) * m[1] + (Pb[3 * i + 2] + Pb[6 + i]) * m[2];
    const float mbu = mb[0] * u[0] + mb[1] * u[1] + mb[2] * u[2];
    const float cu = un > 0.0f ? mbu / (un * mn * mn) : 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float ub = mb[i] / mn - cu * u[i];
#pragma unroll
        for (int j = 0; j < 3; ++j) Fb[3 * i + j] += ub * c.n0[j];
    }
}

// Adjoint of the eigen split sp = Q diag(relu(e)) Q^T of the symmetric sig:
// sigbar = Q (Gam o (Q^T sym(spbar) Q)) Q^T with Gam_ii = [e_i > 0] and
// Gam_ij = (relu(e_i) - relu(e_j)) / (e_i - e_j), guarded for near-equal
// eigenvalues by the mean of the diagonal terms (Daleckii-Krein formula for
// the isotropic matrix function relu).
__device__ __forceinline__ void eigsplit_adj(const float ev[3], const float Q[9], const float spb[9], float sgb[9]) {
    float Sy[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Sy[3 * i + j] = 0.5f * (spb[3 * i + j] + spb[3 * j + i]);
    float T[9], Bq[9];
    mm3(Sy, Q, T);                       // Sy Q
    // Bq = Q^T (Sy Q)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Bq[3 * i + j] = Q[i] * T[j] + Q[3 + i] * T[3 + j] + Q[6 + i] * T[6 + j];
    float gd[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) gd[i] = ev[i] >= 0.0f ? 1.0f : 0.0f;   // clamp(min=0) passes at 0
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float gm;
            if (i == j) {
                gm = gd[i];
            } else {
                const float de = ev[i] - ev[j];
                const float scale = fabsf(ev[i]) + fabsf(ev[j]);
                if (fabsf(de) > 1e-6f * scale && fabsf(de) > 1e-30f)
                    gm = (relu_f(ev[i]) - relu_f(ev[j])) / de;
                else
                    gm = 0.5f * (gd[i] + gd[j]);
            }
            Bq[3 * i + j] *= gm;
        }
    // sgb = Q Bq Q^T
    mm3(Q, Bq, T);
    mmt3(T, Q, sgb);
}

// Fb: the adjoint of the pre-substep F; with the strain limit, the adjoint
// of the limited F (direct terms only) and, apart, the polar rotation's
// contribution to the pre-substep F (Fp) and the adjoint of the limited
// singular values (Scb), which f_clamp_adj combines.
struct ConsAdj {
    float Fb[9], Fp[9], Scb[3], mub, lamb, scb, A0b[9], d0b, lapb, Dh0b;
};

// Reverse of cons_forward given taubar, the adjoint of the updated damage d1
// and of the updated history D_hist1.
__device__ __forceinline__ void cons_adjoint(const Cons &c, const float mu, const float lam, const float taub[9],
                                             float d1b, float Dh1b, const Parts &P, long long p, ConsAdj &o) {
    float gb = 0.0f, tdevb[9], tvb, Fbd[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) Fbd[k] = 0.0f;
    if (c.iface) {
        dir_adjoint(c, taub, gb, tdevb, tvb, Fbd);
    } else {   // tau = g tdev + vdeg tv I
        const float trt = taub[0] + taub[4] + taub[8];
#pragma unroll
        for (int k = 0; k < 9; ++k) gb += taub[k] * c.tdev[k];
        if (c.J >= 1.0f) gb += c.tv * trt;
#pragma unroll
        for (int k = 0; k < 9; ++k) tdevb[k] = c.g * taub[k];
        tvb = c.vdeg * trt;
    }
    d1b += gb * (-2.0f * (1.0f - c.d1) * (1.0f - c.res));
    float Jb = 0.0f, Rb[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        Rb[k] = 0.0f;
        o.A0b[k] = 0.0f;
    }
    o.d0b = 0.0f;
    o.lapb = 0.0f;
    o.Dh0b = 0.0f;
    o.scb = 0.0f;
    if (c.dmg) {
        // torch.maximum sends half of the adjoint to each operand on a tie;
        // clamp passes it on [lo, hi] inclusive; relu only where the input > 0
        float dnb = 0.0f;
        if (!c.allow || c.dn < c.d0) {
            o.d0b += d1b;
        } else if (c.dn > c.d0) {
            dnb = d1b;
        } else {
            dnb = 0.5f * d1b;
            o.d0b += 0.5f * d1b;
        }
        float ddotb = 0.0f;
        if (c.u >= 0.0f && c.u <= 1.0f) {
            o.d0b += dnb;
            ddotb = c.cc * dnb;
        }
        float Dh1t = Dh1b;
        if (c.arg > 0.0f) {
            Dh1t += (1.0f - c.d0) * ddotb;
            o.d0b += -(c.Dh1 + 1.0f) * ddotb;
            o.lapb += (c.l0 * c.l0) * ddotb;
        }
        float driveb = 0.0f;
        if (c.drive > c.Dh0) {
            driveb = Dh1t;
        } else if (c.drive < c.Dh0) {
            o.Dh0b += Dh1t;
        } else {
            driveb = 0.5f * Dh1t;
            o.Dh0b += 0.5f * Dh1t;
        }
        const float phib = (c.phi > 1.0f) ? c.zeta * driveb : 0.0f;
        if (phib != 0.0f) {
            DamageGeom dg;
            damage_geom(c.R, c.V, c.S, c.tdev, c.tv, c.J, c.sc, P, p, dg);
            const float isc2 = 1.0f / (c.sc * c.sc);
            o.scb += -2.0f * c.phi / c.sc * phib;
            float Mb[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) Mb[3 * i + j] = 2.0f * phib * isc2 * dg.M[3 * j + i];
            float Ab[9], spb[9];
            mmt3(Mb, dg.sp, Ab);                    // Mb sp^T
            // spb = A^T Mb
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    spb[3 * i + j] = dg.A[i] * Mb[j] + dg.A[3 + i] * Mb[3 + j] + dg.A[6 + i] * Mb[6 + j];
            // A = R A0 R^T:  Rb += Ab R A0^T + Ab^T R A0;  A0b += R^T Ab R
            {
                float T1[9], T2[9], RA0t[9], RA0[9];
                mmt3(c.R, dg.A0, RA0t);             // R A0^T
                mm3(c.R, dg.A0, RA0);               // R A0
                mm3(Ab, RA0t, T1);
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        T2[3 * i + j] = Ab[i] * RA0[j] + Ab[3 + i] * RA0[3 + j] + Ab[6 + i] * RA0[6 + j];   // Ab^T RA0
#pragma unroll
                for (int k = 0; k < 9; ++k) Rb[k] += T1[k] + T2[k];
                float AbR[9];
                mm3(Ab, c.R, AbR);
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        o.A0b[3 * i + j] = c.R[i] * AbR[j] + c.R[3 + i] * AbR[3 + j] + c.R[6 + i] * AbR[6 + j];
            }
            float sgb[9];
            eigsplit_adj(dg.ev, dg.Q, spb, sgb);
            // sig = sym(tdev + tv I) / J
            const float iJ = 1.0f / c.J;
            float dots = 0.0f;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                tdevb[k] += sgb[k] * iJ;
                dots += sgb[k] * dg.sig[k];
            }
            tvb += (sgb[0] + sgb[4] + sgb[8]) * iJ;
            Jb += -dots * iJ;
        }
    } else {
        o.d0b += d1b;
        o.Dh0b += Dh1b;
    }
    // tv = lam (J - 1) J
    o.lamb = tvb * (c.J - 1.0f) * c.J;
    Jb += tvb * lam * (2.0f * c.J - 1.0f);
    // tdev = 2 mu (F - R) F^T
    float FmR[9], FmRFt[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) FmR[k] = c.F[k] - c.R[k];
    mmt3(FmR, c.F, FmRFt);
    float mub = 0.0f;
#pragma unroll
    for (int k = 0; k < 9; ++k) mub += tdevb[k] * FmRFt[k];
    o.mub = 2.0f * mub;
    float TF[9], TtFmR[9];
    mm3(tdevb, c.F, TF);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            TtFmR[3 * i + j] = tdevb[i] * FmR[j] + tdevb[3 + i] * FmR[3 + j] + tdevb[6 + i] * FmR[6 + j];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        o.Fb[k] = (2.0f * mu) * (TF[k] + TtFmR[k]) + Fbd[k];
        Rb[k] += -(2.0f * mu) * TF[k];
    }
    // J = max(S0 S1 S2, 1e-6); S = sqrt(max(lamC, 1e-12))
    float Sb[3] = {0.0f, 0.0f, 0.0f};
    if (c.Jraw > 1e-6f) {
        Sb[0] = Jb * c.Sc[1] * c.Sc[2];
        Sb[1] = Jb * c.Sc[0] * c.Sc[2];
        Sb[2] = Jb * c.Sc[0] * c.Sc[1];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (c.lamC[i] == 0.0f) Sb[i] = 0.0f;
        o.Scb[i] = Sb[i];
        if (c.fclamp) Sb[i] = 0.0f;   // through the limited values: f_clamp_adj
    }
    // polar F = R U: Fbar += R V (G + diag(Sbar)) V^T with
    // G_ij = (B_ij - B_ji) / (S_i + S_j), B = V^T R^T Rbar V
    float RtRb[9], T[9], Bm[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            RtRb[3 * i + j] = c.R[i] * Rb[j] + c.R[3 + i] * Rb[3 + j] + c.R[6 + i] * Rb[6 + j];
    mm3(RtRb, c.V, T);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Bm[3 * i + j] = c.V[i] * T[j] + c.V[3 + i] * T[3 + j] + c.V[6 + i] * T[6 + j];
    float G[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (i == j) {
                G[3 * i + j] = Sb[i];
            } else {
                float den = c.S[i] + c.S[j];
                den = den < 1e-6f ? 1e-6f : den;
                G[3 * i + j] = (Bm[3 * i + j] - Bm[3 * j + i]) / den;
            }
        }
    float RV[9], RVG[9], Fp[9];
    mm3(c.R, c.V, RV);
    mm3(RV, G, RVG);
    mmt3(RVG, c.V, Fp);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        o.Fp[k] = Fp[k];
        if (!c.fclamp) o.Fb[k] += Fp[k];
    }
}

// Adjoint of the strain limit F -> Fc = U g(S) V^T (anisompm.py:622-636 with
// U = R V, S the singular values before the limit, g = clamp(., lo, hi)),
// given Fcb (the adjoint of Fc) and Scb (of g(S)): returns U G V^T with
// X = U^T Fcb V, G_ii = g'(S_i) (X_ii + Scb_i) and, off the diagonal, the
// divided differences of a singular-value function:
// G_ij = a (X_ij + X_ji)/2 + b (X_ij - X_ji)/2, a = (g_i - g_j)/(S_i - S_j)
// (the mean of g' at equal values), b = (g_i + g_j)/(S_i + S_j).  g' passes
// on [lo, hi] inclusive, as torch's clamp does.
__device__ __forceinline__ void f_clamp_adj(const Cons &c, float lo, float hi, const float Fcb[9],
                                            const float Scb[3], float out[9]) {
    float U[9], T[9], X[9], G[9], g[3], gp[3];
    mm3(c.R, c.V, U);
    mm3(Fcb, c.V, T);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) X[3 * i + j] = U[i] * T[j] + U[3 + i] * T[3 + j] + U[6 + i] * T[6 + j];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        g[i] = c.Sc[i];
        gp[i] = (c.S[i] >= lo && c.S[i] <= hi) ? 1.0f : 0.0f;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (i == j) {
                G[3 * i + i] = c.lamC[i] != 0.0f ? gp[i] * (X[3 * i + i] + Scb[i]) : 0.0f;
            } else {
                const float ds = c.S[i] - c.S[j];
                const float a = fabsf(ds) > 1e-6f * fmaxf(c.S[i], c.S[j]) ? (g[i] - g[j]) / ds : 0.5f * (gp[i] + gp[j]);
                const float den = fmaxf(c.S[i] + c.S[j], 1e-6f);
                const float b = (g[i] + g[j]) / den;
                const float xs = 0.5f * (X[3 * i + j] + X[3 * j + i]), xa = 0.5f * (X[3 * i + j] - X[3 * j + i]);
                G[3 * i + j] = a * xs + b * xa;
            }
        }
    float UG[9];
    mm3(U, G, UG);
    mmt3(UG, c.V, out);
}

constexpr int kAQ = 512;    // staged quadratic nodes per CTA ({v, m} and {mvbar, mbar}: 32 B each)
constexpr int kAC = 1024;   // staged cubic nodes per CTA (16 B each)

// Gathers of k_adj_particle for one particle, from the CTA's shared-memory
// tile (TILE) or from global memory with the reference's clamped indices.
template <bool TILE>
__device__ __forceinline__ void adj_gather(const float xp[3], float inv_dx, float dx, float K, int ng,
                                           const float vt[3], const float Ct[9], const float mv[3], float m,
                                           const float aff[9], float d1, float lb, const float4 *sv,
                                           const float4 *sa, const float4 *sb, const int lo[3], const int qd[3],
                                           const int cd[3], const float4 *__restrict__ gvel,
                                           const float4 *__restrict__ A, const float4 *__restrict__ B,
                                           float xb[3], float vsum[3], float mvb[3], float affb[9], float &d1b) {
    {
        // Per node o: wbar = g . u + an . c + an.w m with u = vt + K Ct dpos and
        // c = mv + aff dpos; the sums over the 27 nodes are contracted over z
        // first (Z0 = sum_z wz wbar, Z1 = sum_z w'z wbar, Gz = sum_z wz g,
        // Az = sum_z wz an, Azd = sum_z wz dpos_z an), then folded with the x
        // and y weights per (x, y) row.
        QuadD q;
        quad_weights_d(xp, inv_dx, ng, q);
        float DX[3], DY[3], DZ[3];
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            DX[o] = ((float)o - q.fx[0]) * dx;
            DY[o] = ((float)o - q.fx[1]) * dx;
            DZ[o] = ((float)o - q.fx[2]) * dx;
        }
        float z0[3] = {0.0f, 0.0f, 0.0f}, z1[3] = {0.0f, 0.0f, 0.0f};   // per axis of xbar
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            float ux[3], cx[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                ux[i] = vt[i] + K * Ct[3 * i] * DX[ox];
                cx[i] = mv[i] + aff[3 * i] * DX[ox];
            }
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
                float uxy[3], cxy[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    uxy[i] = ux[i] + K * Ct[3 * i + 1] * DY[oy];
                    cxy[i] = cx[i] + aff[3 * i + 1] * DY[oy];
                }
                float Z0 = 0.0f, Z1 = 0.0f, Gz[3] = {0.0f, 0.0f, 0.0f}, Az[3] = {0.0f, 0.0f, 0.0f},
                      Azd[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int oz = 0; oz < 3; ++oz) {
                    float4 g, an;
                    if (TILE) {
                        const int t = ((q.b[0] + ox - lo[0]) * qd[1] + (q.b[1] + oy - lo[1])) * qd[2] + q.b[2] + oz - lo[2];
                        g = sv[t];
                        an = sa[t];
                    } else {
                        const int node = node_of(q.b[0] + ox, q.b[1] + oy, q.b[2] + oz, ng);
                        g = __ldg(&gvel[node]);
                        an = __ldg(&A[node]);
                    }
                    const float u0 = uxy[0] + K * Ct[2] * DZ[oz], u1 = uxy[1] + K * Ct[5] * DZ[oz],
                                u2 = uxy[2] + K * Ct[8] * DZ[oz];
                    const float c0 = cxy[0] + aff[2] * DZ[oz], c1 = cxy[1] + aff[5] * DZ[oz],
                                c2 = cxy[2] + aff[8] * DZ[oz];
                    const float wbar = (g.x * u0 + g.y * u1 + g.z * u2) + (an.x * c0 + an.y * c1 + an.z * c2) + an.w * m;
                    const float wz = q.w[oz][2], wzd = wz * DZ[oz];
                    Z0 += wz * wbar;
                    Z1 += q.dw[oz][2] * wbar;
                    Gz[0] += wz * g.x; Gz[1] += wz * g.y; Gz[2] += wz * g.z;
                    Az[0] += wz * an.x; Az[1] += wz * an.y; Az[2] += wz * an.z;
                    Azd[0] += wzd * an.x; Azd[1] += wzd * an.y; Azd[2] += wzd * an.z;
                }
                const float wx = q.w[ox][0], wy = q.w[oy][1], wxy = wx * wy;
                z0[0] += q.dw[ox][0] * wy * Z0;
                z0[1] += wx * q.dw[oy][1] * Z0;
                z1[2] += wxy * Z1;
                const float wxyx = wxy * DX[ox], wxyy = wxy * DY[oy];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    vsum[i] += wxy * Gz[i];
                    mvb[i] += wxy * Az[i];
                    affb[3 * i] += wxyx * Az[i];
                    affb[3 * i + 1] += wxyy * Az[i];
                    affb[3 * i + 2] += wxy * Azd[i];
                }
            }
        }
        xb[0] += inv_dx * z0[0];
        xb[1] += inv_dx * z0[1];
        xb[2] += inv_dx * z1[2];
    }
    {
        CubicD cw;
        cubic_weights_d(xp, inv_dx, ng, cw);
        float dsum = 0.0f;
#pragma unroll
        for (int ox = 0; ox < 4; ++ox)
#pragma unroll
            for (int oy = 0; oy < 4; ++oy) {
                const int row = TILE ? ((cw.b[0] + ox - lo[0] + 1) * cd[1] + (cw.b[1] + oy - lo[1] + 1)) * cd[2]
                                     : (clampi(cw.b[0] + ox, 0, ng - 1) * ng + clampi(cw.b[1] + oy, 0, ng - 1)) * ng;
                float swd = 0.0f, swb = 0.0f, sdwb = 0.0f, g0 = 0.0f, g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
#pragma unroll
                for (int oz = 0; oz < 4; ++oz) {
                    const float4 bn = TILE ? sb[row + cw.b[2] + oz - lo[2] + 1] : __ldg(&B[row + clampi(cw.b[2] + oz, 0, ng - 1)]);
                    const float wz = cw.w[oz][2], dwz = cw.dw[oz][2];
                    const float wbar = bn.x * d1 + bn.y;
                    swd += wz * bn.x;
                    swb += wz * wbar;
                    sdwb += dwz * wbar;
                    g0 += wz * bn.z;
                    g1 += cw.w2[oz][2] * bn.z;
                    g2 += dwz * bn.z;
                    g3 += cw.dw2[oz][2] * bn.z;
                }
                const float wx = cw.w[ox][0], wy = cw.w[oy][1], dwx = cw.dw[ox][0], dwy = cw.dw[oy][1];
                const float sx = cw.w2[ox][0], sy = cw.w2[oy][1], tx = cw.dw2[ox][0], ty = cw.dw2[oy][1];
                dsum += wx * wy * swd;
                xb[0] += inv_dx * dwx * wy * swb + lb * ((tx * wy + dwx * sy) * g0 + dwx * wy * g1);
                xb[1] += inv_dx * wx * dwy * swb + lb * ((sx * dwy + wx * ty) * g0 + wx * dwy * g1);
                xb[2] += inv_dx * wx * wy * sdwb + lb * ((sx * wy + wx * sy) * g2 + wx * wy * g3);
            }
        d1b += dsum;
    }
}

// ---------------------------------------------------------------- k_adj_particle
// The gathers come first, with the forward's APIC affine term read from the
// tape, so the constitutive recompute and its adjoint run last with none of
// the gather state live.  The output adjoint of F is written in two parts:
// (I + dt C')^T Fbar' before the gathers, the constitutive part added at the
// end (same thread, same address).
template <bool EXT>
__global__ void __launch_bounds__(128, 4) k_adj_particle(const pm_params prm, const Parts pre, const Parts post,
                                                         const pm_state_adj ain, const pm_state_adj aout,
                                                         const pm_param_adj grads, const TapeHead *head,
                                                         const float4 *__restrict__ gvel,
                                                         const float4 *__restrict__ A, const float4 *__restrict__ B,
                                                         const float *__restrict__ taff, const float *__restrict__ tpol,
                                                         long long taff_stride) {
    __shared__ float4 sv[kAQ], sa[kAQ], sb[kAC];
    __shared__ int s_box[6];
    const int tid = threadIdx.x;
    const long long p = (long long)blockIdx.x * blockDim.x + tid;
    const bool valid = p < pre.n;
    const long long ps = pre.ps, as = ain.plane_stride, os = aout.plane_stride;
    const int ng = prm.n_grid;
    const float inv_dx = (float)prm.inv_dx, dx = (float)prm.dx, dt = (float)prm.dt;
    const float K = (float)(4.0 * prm.inv_dx * prm.inv_dx);
    const float L2 = (float)(prm.inv_dx * prm.inv_dx);
    float xp[3] = {0.0f, 0.0f, 0.0f};
    // ---- stage the CTA's grid footprint (as k_g2p does): {v, m} and the
    // momentum adjoints of the quadratic nodes of the regular particles' base
    // cells' bounding box, the damage adjoints of its cubic nodes
    bool reg = valid;
    int qb[3] = {0, 0, 0};
    if (valid) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            xp[k] = pre.x[k * ps + p];
            const float fb = floorf(__fsub_rn(__fmul_rn(xp[k], inv_dx), 0.5f));
            reg = reg && (fb >= 1.0f) && (fb <= (float)(ng - 4));
            qb[k] = reg ? (int)fb : 0;
        }
    }
    if (tid < 6) s_box[tid] = tid < 3 ? 0x7fffffff : -0x7fffffff;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int mn = __reduce_min_sync(0xffffffffu, reg ? qb[k] : 0x7fffffff);
        const int mx = __reduce_max_sync(0xffffffffu, reg ? qb[k] : -0x7fffffff);
        if ((tid & 31) == 0) {
            atomicMin(&s_box[k], mn);
            atomicMax(&s_box[3 + k], mx);
        }
    }
    __syncthreads();
    const int lo[3] = {s_box[0], s_box[1], s_box[2]};
    const bool any = s_box[3] >= lo[0];
    const int qd[3] = {s_box[3] - lo[0] + 3, s_box[4] - lo[1] + 3, s_box[5] - lo[2] + 3};
    const int cd[3] = {qd[0] + 2, qd[1] + 2, qd[2] + 2};
    const int qn = any ? qd[0] * qd[1] * qd[2] : 0, cn = any ? cd[0] * cd[1] * cd[2] : 0;
    const bool tile = any && qn <= kAQ && cn <= kAC;
    if (tile) {   // regular nodes lie inside the grid
        const FastDiv qyz = make_fastdiv(qd[1] * qd[2]), qz = make_fastdiv(qd[2]);
        for (int i = tid; i < qn; i += blockDim.x) {
            const int ix = fdiv(i, qyz), r = i - ix * qyz.d, iy = fdiv(r, qz);
            const int gx = lo[0] + ix, gy = lo[1] + iy, gz = lo[2] + r - iy * qz.d;
            const long long node = ((long long)gx * ng + gy) * ng + gz;
            sv[i] = gvel[node];
            sa[i] = A[node];
        }
        const FastDiv cyz = make_fastdiv(cd[1] * cd[2]), cz = make_fastdiv(cd[2]);
        for (int i = tid; i < cn; i += blockDim.x) {
            const int ix = fdiv(i, cyz), r = i - ix * cyz.d, iy = fdiv(r, cz);
            const int gx = lo[0] - 1 + ix, gy = lo[1] - 1 + iy, gz = lo[2] - 1 + r - iy * cz.d;
            sb[i] = B[((long long)gx * ng + gy) * ng + gz];
        }
    }
    __syncthreads();
    if (!valid) return;
    const TapeHead h = *head;
    float xb[3] = {0.0f, 0.0f, 0.0f};
    float vt[3], Ct[9];
    {
        float vpost[3], F[9];
#pragma unroll
        for (int k = 0; k < 3; ++k) vpost[k] = post.v[k * ps + p];
#pragma unroll
        for (int k = 0; k < 9; ++k) F[k] = pre.F[k * ps + p];
        if (EXT) g2p_input_F(prm, tpol, taff_stride, p, F);
        AdjIn a;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            a.xb[k] = ain.x[k * as + p];
            a.vb[k] = ain.v[k * as + p];
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            a.Cb[k] = ain.C[k * as + p];
            a.Fb[k] = ain.F[k * as + p];
        }
        bool inside[3];
        g2p_tail_adj(prm, xp, vpost, F, a, vt, Ct, inside);
#pragma unroll
        for (int k = 0; k < 3; ++k) xb[k] = inside[k] ? a.xb[k] : 0.0f;   // x' = clamp(x + dt v')
        // F' = (I + dt C') F:  Fbar = (I + dt C')^T Fbar' (+ the constitutive part below)
        float Cp[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) Cp[k] = post.C[k * ps + p];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                aout.F[(3 * i + j) * os + p] =
                    a.Fb[3 * i + j] + dt * (Cp[i] * a.Fb[j] + Cp[3 + i] * a.Fb[3 + j] + Cp[6 + i] * a.Fb[6 + j]);
    }
    // ---- P2G inputs of the forward: velocity after the grips, mass, affine term
    float v[3] = {pre.v[p], pre.v[ps + p], pre.v[2 * ps + p]};
    bool gripped = false;
    if (pre.grip_tag) {
        const int gi = pre.grip_tag[p];
        if (gi >= 0 && gi < prm.n_grips) {
            gripped = true;
            const double f = prm.grips[gi].ramp > 0.0 ? fmin(h.time / prm.grips[gi].ramp, 1.0) : 1.0;
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) v[ax] = (float)(prm.grips[gi].vel[ax] * f);
        }
    }
    const float m = pre.mass[p];
    const float mv[3] = {m * v[0], m * v[1], m * v[2]};
    float aff[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) aff[k] = taff[k * taff_stride + p];
    // ---- gathers (quadratic: G2P adjoint position part and P2G adjoint;
    // cubic: damage scatter adjoint and the Laplacian's position part)
    float vsum[3] = {0.0f, 0.0f, 0.0f}, mvb[3] = {0.0f, 0.0f, 0.0f}, affb[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) affb[k] = 0.0f;
    float d1b = ain.d[p];
    {
        const float d1 = post.d[p];
        const float lb = ain.lap[p] * L2 * inv_dx;
        if (reg && tile)
            adj_gather<true>(xp, inv_dx, dx, K, ng, vt, Ct, mv, m, aff, d1, lb, sv, sa, sb, lo, qd, cd, gvel, A, B,
                             xb, vsum, mvb, affb, d1b);
        else
            adj_gather<false>(xp, inv_dx, dx, K, ng, vt, Ct, mv, m, aff, d1, lb, sv, sa, sb, lo, qd, cd, gvel, A, B,
                              xb, vsum, mvb, affb, d1b);
    }
    // dpos = node - x:  xbar -= K Cbar^T sum(w v_i) + aff^T sum(w mvbar_i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
        xb[j] -= K * (Ct[j] * vsum[0] + Ct[3 + j] * vsum[1] + Ct[6 + j] * vsum[2]) +
                 (aff[j] * mvb[0] + aff[3 + j] * mvb[1] + aff[6 + j] * mvb[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        aout.x[k * os + p] = xb[k];
        aout.v[k * os + p] = gripped ? 0.0f : m * mvb[k];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) aout.C[k * os + p] = m * affb[k];
    // ---- constitutive recompute and adjoint
    const bool do_damage = h.any_allow != 0 && (h.step % (long long)prm.damage_every) == 0;
    const float coeff =
        __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn((float)(-prm.dt), pre.vol0[p]), 4.0f), inv_dx), inv_dx);
    float taub[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) taub[k] = coeff * affb[k];
    Cons c;
    float tau[9];
    cons_forward<EXT>(prm, pre, p, do_damage, c, tau, tpol, taff_stride);
    ConsAdj o;
    cons_adjoint(c, pre.mu[p], pre.lam[p], taub, d1b, ain.D_hist[p], pre, p, o);
    if (c.fclamp) {
        // the G2P part above and the stress's direct part are adjoints of the
        // limited F: through the limit to the pre-substep F, plus the polar
        // rotation's part
        float Fcb[9], F0b[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) Fcb[k] = aout.F[k * os + p] + o.Fb[k];
        f_clamp_adj(c, (float)prm.f_clamp_lo, (float)prm.f_clamp_hi, Fcb, o.Scb, F0b);
#pragma unroll
        for (int k = 0; k < 9; ++k) aout.F[k * os + p] = F0b[k] + o.Fp[k];
    } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) aout.F[k * os + p] += o.Fb[k];
    }
    aout.d[p] = o.d0b;
    aout.lap[p] = o.lapb;
    aout.D_hist[p] = o.Dh0b;
    const long long gs = grads.plane_stride;
    if (grads.mu) grads.mu[p] += o.mub;
    if (grads.lam) grads.lam[p] += o.lamb;
    // sigma_c and A0 enter only through an active damage drive: most
    // particles add zero, so skip their read-modify-write
    if (grads.sigma_c && o.scb != 0.0f) grads.sigma_c[p] += o.scb;
    if (grads.A0) {
        bool nz = false;
#pragma unroll
        for (int k = 0; k < 9; ++k) nz = nz || o.A0b[k] != 0.0f;
        if (nz) {
#pragma unroll
            for (int k = 0; k < 9; ++k) grads.A0[k * gs + p] += o.A0b[k];
        }
    }
}

__global__ void k_tape_head(const Ctrl *ctrl, TapeHead *head, long long n) {
    if (threadIdx.x == 0) {
        head->n_active = ctrl->n_active;
        head->any_allow = ctrl->any_allow;
        head->step = ctrl->step;
        head->time = ctrl->time;
        head->n_work = (unsigned)min((long long)ctrl->n_work, n);
    }
    if (threadIdx.x < PM_MAX_COLLIDERS) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            head->col_origin[threadIdx.x][a] = ctrl->col_origin[threadIdx.x][a];
            head->col_vel[threadIdx.x][a] = ctrl->col_vel[threadIdx.x][a];
        }
    }
}

}  // namespace

// One-time kernel attribute set-up for the current device (not a stream
// operation; pm_prepare runs it before any capture).
void prepare_adjoint() {
    static int done[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(k_adj_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAdjTileSmem);
        done[dev] = 1;
    }
}

// ------------------------------------------------------------------ tape layout
TapeLayout make_tape_layout(long long n, int ng, int slots, int flags) {
    TapeLayout T;
    const size_t A = 256;
    const long long G = (long long)ng * ng * ng;
    const int nbs = (ng + kBlockEdge - 1) / kBlockEdge;
    const long long nb = (long long)nbs * nbs * nbs;
    const long long np = (n + 63) / 64 * 64 > 0 ? (n + 63) / 64 * 64 : 64;
    size_t o = 0;
    T.head = o;    o = align_up(o + sizeof(TapeHead) * (size_t)(slots > 0 ? slots : 1), A);
    T.actl = o;    o = align_up(o + sizeof(AdjCtrl), A);
    T.acc = o;     o = align_up(o + 32 * (size_t)G, A);     // 4 x int64 per node
    T.adj_q = o;   o = align_up(o + 16 * (size_t)G, A);
    T.adj_c = o;   o = align_up(o + 16 * (size_t)G, A);
    T.apay = o;    o = align_up(o + 80 * (size_t)np, A);
    T.slot0 = o;
    size_t s = 0;
    T.vel = s;     s = align_up(s + 16 * (size_t)G, A);
    T.gd = s;      s = align_up(s + 4 * (size_t)G, A);
    T.sw = s;      s = align_up(s + 4 * (size_t)G, A);
    T.vpre = s;    s = align_up(s + ((flags & PM_TAPE_COLLIDERS) ? 16 * (size_t)G : 0), A);   // pre-collider v
    T.blocks = s;  s = align_up(s + 4 * (size_t)nb, A);
    T.keys = s;    s = align_up(s + 4 * (size_t)np, A);
    T.iperm = s;   s = align_up(s + 4 * (size_t)np, A);
    T.work = s;    s = align_up(s + 4 * (size_t)np, A);
    T.aff = s;     s = align_up(s + 36 * (size_t)np, A);
    T.pol = s;     s = align_up(s + 88 * (size_t)np, A);
    T.aff_stride = np;
    T.slot_bytes = s;
    T.total = o + s * (size_t)(slots > 0 ? slots : 1);
    T.n_blocks = nb;
    T.slots = slots;
    T.flags = flags;
    return T;
}

void record_redirect(const TapeLayout &T, void *tape, int slot, WS &w) {
    char *b = (char *)tape + T.slot0 + T.slot_bytes * (size_t)slot;
    w.g_vel = (float4 *)(b + T.vel);
    w.g_gd = (float *)(b + T.gd);
    w.g_sw = (float *)(b + T.sw);
    w.g_vpre = (T.flags & PM_TAPE_COLLIDERS) ? (float4 *)(b + T.vpre) : nullptr;
    w.block_list = (int *)(b + T.blocks);
    w.inv_perm = (int *)(b + T.iperm);   // the substep's sort stays on the tape for the adjoint
    w.work = (int *)(b + T.work);
    w.tape_aff = (float *)(b + T.aff);
    w.tape_pol = (float *)(b + T.pol);
    w.tape_aff_stride = T.aff_stride;
}

void launch_tape_head(const TapeLayout &T, void *tape, int slot, const WS &w, long long n, cudaStream_t s) {
    TapeHead *h = (TapeHead *)((char *)tape + T.head) + slot;
    k_tape_head<<<1, 32, 0, s>>>(w.ctrl, h, n);
    if (n > 0) {
        char *b = (char *)tape + T.slot0 + T.slot_bytes * (size_t)slot;
        cudaMemcpyAsync(b + T.keys, w.sorted_keys, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s);
    }
}

void launch_adjoint(const pm_params &prm, const Parts &pre, const Parts &post, const pm_state_adj &ain,
                    const pm_state_adj &aout, const pm_param_adj &grads, const TapeLayout &T, void *tape, int slot,
                    cudaStream_t s) {
    char *base = (char *)tape;
    char *b = base + T.slot0 + T.slot_bytes * (size_t)slot;
    const TapeHead *h = (const TapeHead *)(base + T.head) + slot;
    AdjCtrl *actl = (AdjCtrl *)(base + T.actl);
    long long *acc = (long long *)(base + T.acc);
    float4 *apay = (float4 *)(base + T.apay);
    float4 *Aq = (float4 *)(base + T.adj_q);
    float4 *Bc = (float4 *)(base + T.adj_c);
    const float4 *gvel = (const float4 *)(b + T.vel);
    const float *ggd = (const float *)(b + T.gd);
    const float *gsw = (const float *)(b + T.sw);
    const int *blocks = (const int *)(b + T.blocks);
    const long long n = pre.n;
    if (n <= 0) return;
    prepare_adjoint();
    cudaMemsetAsync(actl, 0, sizeof(AdjCtrl), s);
    k_adj_pre<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(prm, pre, post, ain, (const int *)(b + T.iperm), apay, actl,
                                                          (const float *)(b + T.pol), T.aff_stride);
    k_adj_bounds<<<1, kBoundSlots, 0, s>>>(actl);
    {
        static int slots_dev[64] = {0};
        int dev = 0;
        cudaGetDevice(&dev);
        int slots = (dev >= 0 && dev < 64) ? slots_dev[dev] : 0;
        if (slots <= 0) {
            slots = resident_slots((const void *)k_adj_tiles, kATh, kAdjTileSmem);
            if (dev >= 0 && dev < 64) slots_dev[dev] = slots;
        }
        const long long blocks_t = std::max<long long>(1, std::min<long long>(slots, (n + 63) / 64));
        k_adj_tiles<<<(unsigned)blocks_t, kATh, kAdjTileSmem, s>>>(prm, (const unsigned *)(b + T.keys),
                                                                  (const int *)(b + T.work), h, apay, actl, acc, n);
    }
    const long long max_items = T.n_blocks * 64;
    const int gb = (int)std::max<long long>(1, std::min<long long>((max_items + 255) / 256, 148LL * 8));
    const float4 *vpre = (T.flags & PM_TAPE_COLLIDERS) ? (const float4 *)(b + T.vpre) : nullptr;
    k_adj_grid<<<gb, 256, 0, s>>>(prm, blocks, h, gvel, vpre, ggd, gsw, acc, actl, Aq, Bc, T.n_blocks);
    const float *taff = (const float *)(b + T.aff);
    const float *tpol = (const float *)(b + T.pol);
    const unsigned pb = (unsigned)((n + 127) / 128);
    if (prm.use_f_clamp || pre.interface_mask)
        k_adj_particle<true><<<pb, 128, 0, s>>>(prm, pre, post, ain, aout, grads, h, gvel, Aq, Bc, taff, tpol,
                                                T.aff_stride);
    else
        k_adj_particle<false><<<pb, 128, 0, s>>>(prm, pre, post, ain, aout, grads, h, gvel, Aq, Bc, taff, tpol,
                                                 T.aff_stride);
}

}  // namespace pm
