// Constitutive update + P2G, cell-aggregated, in two kernels.
//
// k_stress, one thread per particle in particle order (coalesced state
// reads): particle BC, polar decomposition (Jacobi eigensolve of F^T F),
// fixed-corotated Kirchhoff stress, anisotropic phase-field damage (the
// Cauchy stress's eigensystem taken from the polar decomposition, a Jacobi
// solve only for nearly singular F), degradation and the APIC affine term;
// the P2G payload (5 float4) goes to the particle's slot in the sorted order,
// and the substep's bounds on one node contribution (momentum, mass, damage)
// are raised in the control block.
//
// k_p2g_tiles, persistent CTAs taking work items from a list of the
// non-empty 4^3-cell sub-blocks of the sort (the cells of a sub-block are a
// contiguous run of the Morton-ordered sort).  A work item covers the
// quadratic nodes [4s, 4s+6)^3 ({mv, m}) and the cubic nodes [4s-1, 4s+7)^3
// ({sum w d, sum w}).  Chunks of 256 particles stage their payload in shared
// memory, then one work item per (cell, x-slab): all particles of a cell
// share their quadratic base, so an item sums the cell's contributions to 9
// quadratic nodes (3 slabs) or 25 cubic nodes (5 slabs; a cell's cubic
// stencils span 5^3 nodes) in float registers (packed pairs: sm_100's FFMA2
// issues two FMAs per instruction), in the sorted order, and adds each node
// once as exact fixed point (units from the control block's bounds) into two
// 32-bit shared planes per component.  Every fourth chunk and after the last
// one the planes go to the global int64 grid, one atomic per nonzero node
// and component; integer addition is associative, so the grid sums, and with
// them the whole substep, are the same bits whatever order the atomics run
// in.  The touched 4^3 grid blocks are marked.  Particles whose stencil needs
// the reference's edge clamping (base cell outside [1, n_grid-4]) scatter
// directly to the global grid instead.
//
// Reference: anisompm.py:601-724 (constitutive, damage, P2G) and 768-776
// (cubic damage scatter).
#include "pm_kernels.cuh"

namespace pm {

constexpr int kP2GThreads = 256;
constexpr int kPay = 17;         // payload floats: x(3) mv(3) affine(9) m d
// Payload rows are padded by one word per 32 particles: the lanes of an item
// warp read particle j of 32 different cells, whose sorted positions are
// close to multiples of the cell occupancy (8): unpadded, those fall on 4
// banks; padded, on distinct ones.
constexpr int kPayStride = kP2GThreads + kP2GThreads / 32;
__device__ __forceinline__ int pay_col(int j) { return j + (j >> 5); }

__device__ __forceinline__ float clamp_min(float v, float lo) { return v < lo ? lo : v; }   // torch.clamp(min=)
__device__ __forceinline__ float relu(float v) { return v > 0.0f ? v : (v != v ? v : 0.0f); }
// torch.maximum: NaN if either operand is NaN
__device__ __forceinline__ float tmax(float a, float b) { return (a != a || b != b) ? a + b : (a > b ? a : b); }

// Constitutive update of particle p (anisompm.py:614-706).  Writes tau and
// updates F (f_clamp), d, D_hist and the diagnostics in place.
// When `rec` is set (recording a substep for the adjoint) the polar
// decomposition (R, V, S) and, on damage steps, phi are written to its planes:
// rec[k * rs + p] for R (k 0..8), V (9..17), S (18..20), phi (21).
// Per-particle inputs of the constitutive update, all loaded before any
// store (the state planes share one buffer, so a store would otherwise keep
// later loads from being issued early).  The inputs of the affine term and
// the payload (C, v, x, vol0, mass, grip) are loaded after it: they are not
// needed earlier, and holding them across the eigensolve costs registers.
struct StressIn {
    float F[9], A0[9];
    float d, lap, Dh, mu, lam, sc, eta, zeta, l0, res;
    bool allow;
};

__device__ __forceinline__ void constitutive(const pm_params &prm, const Parts &P, long long p, bool do_damage,
                                             const StressIn &in, float tau[9], float &d_out, float *rec = nullptr,
                                             long long rs = 0) {
    const long long ps = P.ps;
    float F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = in.F[k];
    float Cg[9];   // C = F^T F (615)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Cg[3 * i + j] = F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j];
    float lamC[3], V[9];
    sym_eig3<5>(Cg, lamC, V);                                        // (616)
    float S[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) S[i] = sqrtf(clamp_min(lamC[i], 1e-12f));   // (617)
    float W[9], R[9];
    bool u_ok;
    mm3(F, V, W);                                                    // (619)
    {
        float wn[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            wn[j] = sqrtf(W[j] * W[j] + W[3 + j] * W[3 + j] + W[6 + j] * W[6 + j]);
            const float rn = 1.0f / (wn[j] + 1e-12f);                 // one division per column
#pragma unroll
            for (int i = 0; i < 3; ++i) W[3 * i + j] *= rn;          // (620)
        }
        u_ok = polar_u_ok(wn);
    }
    mmt3(W, V, R);                                                   // R = What V^T (621)
    if (rec) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            rec[k * rs + p] = R[k];
            rec[(9 + k) * rs + p] = V[k];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) rec[(18 + k) * rs + p] = S[k];
    }
    if (prm.use_f_clamp) {                                           // (622-636)
        f_clamp_F(F, V, S, (float)prm.f_clamp_lo, (float)prm.f_clamp_hi, F);
#pragma unroll
        for (int k = 0; k < 9; ++k) P.Fo[k * ps + p] = F[k];
    }
    const float J = clamp_min(S[0] * S[1] * S[2], 1e-6f);            // (637)
    const float mu = in.mu, lam = in.lam;
    float tdev[9];
    {
        float FmR[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) FmR[k] = (2.0f * mu) * (F[k] - R[k]);
        mmt3(FmR, F, tdev);                                          // 2mu (F-R) F^T (643)
    }
    const float tv = lam * (J - 1.0f) * J;                           // (644)

    if (do_damage) {                                                 // (647-685)
        float sg[9];
        const float rJ = 1.0f / J;
#pragma unroll
        for (int k = 0; k < 9; ++k) sg[k] = (tdev[k] + ((k % 4 == 0) ? tv : 0.0f)) * rJ;
        float sgs[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) sgs[3 * i + j] = 0.5f * (sg[3 * i + j] + sg[3 * j + i]);
        float ev[3], EV[9];
        if (u_ok)   // (652: sym_eig of sig)
            stress_eig_polar(W, sgs, ev, EV);
        else
            sym_eig3<5>(sgs, ev, EV);
        float sp[9];
        {
            float ED[9];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const float e = ev[j] < 0.0f ? 0.0f : ev[j];
#pragma unroll
                for (int i = 0; i < 3; ++i) ED[3 * i + j] = EV[3 * i + j] * e;
            }
            mmt3(ED, EV, sp);                                        // sigma+ (654-655)
        }
        float A[9];
        {
            float A0[9], RA[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) A0[k] = in.A0[k];
            mm3(R, A0, RA);
            mmt3(RA, R, A);                                          // A = R A0 R^T (661)
        }
        float M[9];
        mm3(A, sp, M);
        const float trMM = (M[0] * M[0] + M[1] * M[3] + M[2] * M[6]) + (M[3] * M[1] + M[4] * M[4] + M[5] * M[7]) +
                           (M[6] * M[2] + M[7] * M[5] + M[8] * M[8]);
        const float sc = in.sc;
        const float phi = trMM / (sc * sc);                          // (663-664)
        if (rec) rec[21 * rs + p] = phi;
        if (P.phi) P.phi[p] = phi;
        if (P.phi_shear) {                                           // (670-673)
            float phs = 0.0f;
            if (P.n_interface) {
                const float n0 = P.n_interface[p], n1 = P.n_interface[ps + p], n2 = P.n_interface[2 * ps + p];
                const float s0 = sp[0] * n0 + sp[1] * n1 + sp[2] * n2;
                const float s1 = sp[3] * n0 + sp[4] * n1 + sp[5] * n2;
                const float s2 = sp[6] * n0 + sp[7] * n1 + sp[8] * n2;
                const float tn = s0 * n0 + s1 * n1 + s2 * n2;
                const float t0 = s0 - tn * n0, t1 = s1 - tn * n1, t2 = s2 - tn * n2;
                const float q = sqrtf(t0 * t0 + t1 * t1 + t2 * t2) / sc;
                phs = q * q;
            }
            P.phi_shear[p] = phs;
        }
        const float drive = in.zeta * relu(phi - 1.0f);
        const float dh0 = in.Dh;
        const float Dh = tmax(dh0, drive);
        P.Dho[p] = Dh;                                               // history max (679)
        const float d = in.d;
        const float l0 = in.l0;
        const float resist = d - (l0 * l0) * in.lap;
        const float ddot = relu((1.0f - d) * Dh - resist);           // (681-682)
        const float dt_dmg = (float)(prm.dt * (double)prm.damage_every);
        float dn = d + (dt_dmg / in.eta) * ddot;
        dn = dn < 0.0f ? 0.0f : dn;
        dn = dn > 1.0f ? 1.0f : dn;                                  // (683-684)
        if (in.allow) {                                              // monotone, where allowed (685)
            d_out = tmax(dn, d);
            P.d_o[p] = d_out;
        }
    }
    const float d = d_out;
    const float res = in.res;
    const float omd = 1.0f - d;
    const float g = (omd * omd) * (1.0f - res) + res;                // (688)
    const float vdeg = (J >= 1.0f) ? g : 1.0f;                       // (690)
#pragma unroll
    for (int k = 0; k < 9; ++k) tau[k] = g * tdev[k] + ((k % 4 == 0) ? vdeg * tv : 0.0f);
    if (P.interface_mask && P.interface_mask[p]) {
        // directional_kirchhoff(tau_dev + tau_vol, F, d, n, g, g, tension_gate=True)
        // (anisompm.py:190-227 via 697-703)
        float tc[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) tc[k] = tdev[k] + ((k % 4 == 0) ? tv : 0.0f);
        const float n0 = P.n_interface[p], n1 = P.n_interface[ps + p], n2 = P.n_interface[2 * ps + p];
        float m[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) m[i] = F[3 * i] * n0 + F[3 * i + 1] * n1 + F[3 * i + 2] * n2;
        const float mn = sqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) + 1e-9f;
#pragma unroll
        for (int i = 0; i < 3; ++i) m[i] = m[i] / mn;
        float Pm[9], Qm[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                Pm[3 * i + j] = m[i] * m[j];
                Qm[3 * i + j] = ((i == j) ? 1.0f : 0.0f) - Pm[3 * i + j];
            }
        float T1[9], perp[9], sh1[9], sh2[9], par[9];
        mm3(Pm, tc, T1);
        mm3(T1, Pm, perp);
        mm3(T1, Qm, sh1);
        mm3(Qm, tc, T1);
        mm3(T1, Pm, sh2);
        mm3(T1, Qm, par);
        float tm0 = m[0] * tc[0] + m[1] * tc[3] + m[2] * tc[6];
        float tm1 = m[0] * tc[1] + m[1] * tc[4] + m[2] * tc[7];
        float tm2 = m[0] * tc[2] + m[1] * tc[5] + m[2] * tc[8];
        const float snn = tm0 * m[0] + tm1 * m[1] + tm2 * m[2];
        const float gI = (snn > 0.0f) ? g : 1.0f;
#pragma unroll
        for (int k = 0; k < 9; ++k) tau[k] = par[k] + gI * perp[k] + g * (sh1[k] + sh2[k]);
    }
    if (prm.record_stress) {
        if (P.tau_last) {
#pragma unroll
            for (int k = 0; k < 9; ++k) P.tau_last[k * ps + p] = tau[k];
        }
        if (P.J_last) P.J_last[p] = J;
    }
}

// One thread per particle in particle order: particle BC, constitutive update,
// damage update, degradation and the APIC affine term (anisompm.py:601-713);
// the P2G payload goes to w.payload[s] (5 float4, coalesced):
//   {fx | x, m} {m v, d} {affine 0..3} {affine 4..7} {affine 8, regular, 0, 0}
// with fx = X - floor(X - 0.5) per axis for particles whose stencil needs no
// clamping (regular, base cell in [1, n_grid-4]) and the position x otherwise.
// MINB: resident CTAs per SM the registers are budgeted for (3: 80 registers;
// 4: 64 registers with a few spills), a tunable.
template <class SC, int MINB>
__global__ void __launch_bounds__(256, MINB) k_stress(const SC sc, const Parts P, const WS w) {
    // particle order: the state reads and writes are coalesced; the payload
    // goes to the particle's sorted position
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.n) return;
    const int sid = sc.of_particle(p);
    const pm_params &prm = sc.params(sid);
    const long long s = w.inv_perm[p];
    const long long ps = P.ps;
    const int ng = prm.n_grid;
    const float inv_dx = (float)prm.inv_dx;
    const Ctrl *ctrl = w.ctrl + sid;
    const bool do_damage = ctrl->any_allow != 0 && (ctrl->step % (long long)prm.damage_every) == 0;
    StressIn in;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        in.F[k] = P.F[k * ps + p];
        in.A0[k] = do_damage ? P.A0[k * ps + p] : 0.0f;
    }
    in.d = P.d[p];
    in.lap = P.lap[p];
    in.Dh = P.D_hist[p];
    in.mu = P.mu[p];
    in.lam = P.lam[p];
    in.sc = P.sigma_c[p];
    in.eta = P.eta[p];
    in.zeta = P.zeta[p];
    in.l0 = P.l0[p];
    in.res = P.residual[p];
    in.allow = P.allow[p] != 0;
    float tau[9];
    float d_new = in.d;
    constitutive(prm, P, p, do_damage, in, tau, d_new, w.tape_pol, w.tape_aff_stride);
    if (P.d_o != P.d) {   // out of place: every particle's d and D_hist go to the output state
        P.d_o[p] = d_new;
        if (!do_damage) P.Dho[p] = in.Dh;
    }
    float Cp[9], v[3], xp[3];
#pragma unroll
    for (int k = 0; k < 9; ++k) Cp[k] = P.C[k * ps + p];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = P.v[k * ps + p];
        xp[k] = P.x[k * ps + p];
    }
    const float vol0 = P.vol0[p], m = P.mass[p];
    {                                                                // particle BCs (601-602)
        const int g = P.grip_tag ? P.grip_tag[p] : -1;
        if (g >= 0 && g < prm.n_grips) {
            const double f = prm.grips[g].ramp > 0.0 ? fmin(ctrl->time / prm.grips[g].ramp, 1.0) : 1.0;
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) v[ax] = (float)(prm.grips[g].vel[ax] * f);
        }
    }
    // stress_coeff = -dt*vol0*4*inv_dx*inv_dx; affine = coeff*tau + m*C (711-713)
    const float coeff =
        __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn((float)(-prm.dt), vol0), 4.0f), inv_dx), inv_dx);
    float aff[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) aff[k] = coeff * tau[k] + m * Cp[k];
    float fx[3];
    bool reg = true;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const float X = __fmul_rn(xp[ax], inv_dx);
        const float fb = floorf(__fsub_rn(X, 0.5f));
        reg = reg && (fb >= 1.0f) && (fb <= (float)(ng - 4));
        fx[ax] = __fsub_rn(X, fb);                                   // in [0.5, 1.5)
    }
    float4 *dst = w.payload + 5 * s;
    dst[0] = reg ? make_float4(fx[0], fx[1], fx[2], m) : make_float4(xp[0], xp[1], xp[2], m);
    dst[1] = make_float4(m * v[0], m * v[1], m * v[2], d_new);
    dst[2] = make_float4(aff[0], aff[1], aff[2], aff[3]);
    dst[3] = make_float4(aff[4], aff[5], aff[6], aff[7]);
    dst[4] = make_float4(aff[8], reg ? 1.0f : 0.0f, 0.0f, 0.0f);
    {   // bounds of one node contribution: |w (m v + aff dpos)| with w <= 1 and |dpos| <= 1.5 dx per axis
        const float hx = 1.5f * (float)prm.dx;
        float bm = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            bm = fmaxf(bm, fabsf(m * v[c]) + hx * (fabsf(aff[3 * c]) + fabsf(aff[3 * c + 1]) + fabsf(aff[3 * c + 2])));
        unsigned bmom = bound_bits(bm), bmass = bound_bits(m), bdmg = bound_bits(d_new);
        Ctrl *cw = w.ctrl + sid;
        // any partition of the warp is correct here: each group raises the
        // bounds to its own maximum, in the slot of its warp
        const unsigned am = __activemask();
        const int slot = (int)(((blockIdx.x << 3) + (threadIdx.x >> 5)) & (kBoundSlots - 1));
        if (!SC::batched || __all_sync(am, sid == __shfl_sync(am, sid, __ffs(am) - 1))) {
            bmom = __reduce_max_sync(am, bmom);
            bmass = __reduce_max_sync(am, bmass);
            bdmg = __reduce_max_sync(am, bdmg);
            if ((threadIdx.x & 31) == (unsigned)(__ffs(am) - 1)) {
                atomicMax(&cw->bound_slots[0][slot], bmom);
                atomicMax(&cw->bound_slots[1][slot], bmass);
                atomicMax(&cw->bound_slots[2][slot], bdmg);
            }
        } else {
            atomicMax(&cw->bound_slots[0][slot], bmom);
            atomicMax(&cw->bound_slots[1][slot], bmass);
            atomicMax(&cw->bound_slots[2][slot], bdmg);
        }
    }
    if (w.tape_aff) {
#pragma unroll
        for (int k = 0; k < 9; ++k) w.tape_aff[k * w.tape_aff_stride + p] = aff[k];
    }
}

// Scatter one particle straight into the global grid with the reference's
// clamped node indices (anisompm.py:716-724, 771-776): the path for particles
// whose stencil leaves the grid.  `sc` holds the fixed-point scales of
// {momentum, mass, w d, w}.
__device__ __forceinline__ void mark_node_block(unsigned char *mask, int nbs, int x, int y, int z) {
    unsigned char *m = &mask[((long long)(x >> 2) * nbs + (y >> 2)) * nbs + (z >> 2)];
    if (*m == 0) *m = 1;
}

__device__ __noinline__ void scatter_particle_global(const float xp[3], const float mv[3], const float aff[9],
                                                     float m, float d, float inv_dx, float dx, int ng,
                                                     const float sc[4], long long *g_mom, long long *g_dmg,
                                                     unsigned char *mask, int nbs) {
    {
        Quad q;
        quad_weights(xp, inv_dx, ng, q);
        int NX[3], NY[3], NZ[3];
        float DX[3], DY[3], DZ[3];
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            NX[o] = clampi(q.b[0] + o, 0, ng - 1);
            NY[o] = clampi(q.b[1] + o, 0, ng - 1);
            NZ[o] = clampi(q.b[2] + o, 0, ng - 1);
            DX[o] = ((float)o - q.fx[0]) * dx;
            DY[o] = ((float)o - q.fx[1]) * dx;
            DZ[o] = ((float)o - q.fx[2]) * dx;
        }
#pragma unroll
        for (int ox = 0; ox < 3; ++ox)
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
                const float wxy = q.w[ox][0] * q.w[oy][1];
#pragma unroll
                for (int oz = 0; oz < 3; ++oz) {
                    const float wk = wxy * q.w[oz][2];
                    const float a0 = aff[0] * DX[ox] + aff[1] * DY[oy] + aff[2] * DZ[oz];
                    const float a1 = aff[3] * DX[ox] + aff[4] * DY[oy] + aff[5] * DZ[oz];
                    const float a2 = aff[6] * DX[ox] + aff[7] * DY[oy] + aff[8] * DZ[oz];
                    long long *g = g_mom + 4 * (((long long)NX[ox] * ng + NY[oy]) * ng + NZ[oz]);
                    red_fix(g, wk * (mv[0] + a0), sc[0]);
                    red_fix(g + 1, wk * (mv[1] + a1), sc[0]);
                    red_fix(g + 2, wk * (mv[2] + a2), sc[0]);
                    red_fix(g + 3, wk * m, sc[1]);
                    mark_node_block(mask, nbs, NX[ox], NY[oy], NZ[oz]);
                }
            }
    }
    {
        Cubic c;
        cubic_weights(xp, inv_dx, ng, c);
        int NX[4], NY[4], NZ[4];
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            NX[o] = clampi(c.b[0] + o, 0, ng - 1);
            NY[o] = clampi(c.b[1] + o, 0, ng - 1);
            NZ[o] = clampi(c.b[2] + o, 0, ng - 1);
        }
#pragma unroll
        for (int ox = 0; ox < 4; ++ox)
#pragma unroll
            for (int oy = 0; oy < 4; ++oy) {
                const float wxy = c.w[ox][0] * c.w[oy][1];
#pragma unroll
                for (int oz = 0; oz < 4; ++oz) {
                    const float wk = wxy * c.w[oz][2];
                    long long *g = g_dmg + 2 * (((long long)NX[ox] * ng + NY[oy]) * ng + NZ[oz]);
                    red_fix(g, wk * d, sc[2]);
                    red_fix(g + 1, wk, sc[3]);
                    mark_node_block(mask, nbs, NX[ox], NY[oy], NZ[oz]);
                }
            }
    }
}

constexpr int kSubEdge = 4;                    // sub-block edge in cells (the P2G work unit)
constexpr int kQE = kSubEdge + 2;              // 6: quadratic tile edge, nodes [4s, 4s+6)
constexpr int kCE = kSubEdge + 4;              // 8: cubic tile edge, nodes [4s-1, 4s+7)
constexpr int kQN = kQE * kQE * kQE;           // 216
constexpr int kCN = kCE * kCE * kCE;           // 512
constexpr int kSub = kP2GThreads;              // particles per chunk
constexpr int kCW = 15;                        // expanded cubic weights per particle (5 per axis)
// Chunk planes (32-bit words, one node per word) are laid out with z stride
// 1, y stride 8 and x stride 52 (quadratic) / 68 (cubic): the 32 cells of a
// chunk of a sub-block (x in one half, all y and z) then land on 32 distinct
// banks for every node offset, so a warp of items over distinct cells adds
// without bank conflicts.
constexpr int kQSY = 8, kQSX = 52, kQPl = 312;   // 5*52 + 5*8 + 6 = 306 <= 312
constexpr int kCSY = 8, kCSX = 68, kCPl = 544;   // 7*68 + 7*8 + 8 = 540 <= 544
constexpr size_t kP2GSmem = sizeof(unsigned) * 2 * (4 * kQPl + 2 * kCPl) +
                            sizeof(float) * (kPay + kCW) * kPayStride + sizeof(int) * (kSub + 2) + 2 * kSub;

// Folds control block blockIdx.x's bound slots into its three bounds and
// clears the slots for the next substep.
__global__ void __launch_bounds__(kBoundSlots) k_bounds(Ctrl *ctrl) {
    Ctrl *c = ctrl + blockIdx.x;
    __shared__ unsigned s_m[3][kBoundSlots / 32];
    const int t = threadIdx.x;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const unsigned m = __reduce_max_sync(0xffffffffu, c->bound_slots[v][t]);
        c->bound_slots[v][t] = 0u;
        if ((t & 31) == 0) s_m[v][t >> 5] = m;
    }
    __syncthreads();
    if (t < 3) {
        unsigned m = 0u;
#pragma unroll
        for (int k = 0; k < kBoundSlots / 32; ++k) m = max(m, s_m[t][k]);
        if (t == 0) c->mom_bound = m;
        if (t == 1) c->mass_bound = m;
        if (t == 2) c->dmg_bound = m;
    }
}

// Sorted index of the first particle of every non-empty 4^3-cell sub-block
// (where key >> 6 changes), appended in any order: the accumulation is exact,
// so the order in which work items run does not change the result.
__global__ void __launch_bounds__(256) k_subblocks(const unsigned *__restrict__ keys, long long n,
                                                   int *__restrict__ work, Ctrl *ctrl) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += stride) {
        const long long i = base + threadIdx.x;
        const bool st = i < n && (i == 0 || (keys[i] >> 6) != (keys[i - 1] >> 6));
        const unsigned ball = __ballot_sync(0xffffffffu, st);
        unsigned slot0 = 0;
        if ((threadIdx.x & 31) == 0 && ball) slot0 = atomicAdd(&ctrl->n_work, (unsigned)__popc(ball));
        slot0 = __shfl_sync(0xffffffffu, slot0, 0);
        const unsigned slot = slot0 + __popc(ball & lanemask_lt());
        if (st && slot < (unsigned long long)n) work[slot] = (int)i;   // bounded even without a clock reset
    }
}

// MINB: resident CTAs per SM the registers are budgeted for (3: 80
// registers; 4: 64 registers with a few spills), a tunable.
template <class SC, int MINB>
__global__ void __launch_bounds__(kP2GThreads, MINB) k_p2g_tiles(const SC sc, const WS w, long long n) {
    extern __shared__ long long s_raw[];
    unsigned (*qlo)[kQPl] = (unsigned (*)[kQPl])(s_raw);                 // [4][kQPl] chunk planes
    int (*qhi)[kQPl] = (int (*)[kQPl])(qlo[4]);                         // [4][kQPl]
    unsigned (*clo)[kCPl] = (unsigned (*)[kCPl])(qhi[4]);                // [2][kCPl]
    int (*chi)[kCPl] = (int (*)[kCPl])(clo[2]);                         // [2][kCPl]
    float (*pay)[kPayStride] = (float (*)[kPayStride])(chi[2]);         // [kPay][kPayStride]
    float (*cwt)[kPayStride] = (float (*)[kPayStride])(pay[kPay]);     // [kCW][kPayStride]
    int *runs = (int *)(cwt[kCW]);                                      // [kSub + 2]
    unsigned char *regular = (unsigned char *)(runs + kSub + 2);        // [kSub]
    unsigned char *lcell = regular + kSub;                              // [kSub] cell inside the sub-block
    __shared__ int s_wcnt[kP2GThreads / 32];
    __shared__ unsigned char s_bmark[27];
    __shared__ unsigned s_item;

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const unsigned *keys = w.sorted_keys;
    Ctrl *ctrl0 = w.ctrl;
    const unsigned n_work = min(ctrl0->n_work, (unsigned)min(n, (long long)0x7fffffff));

    // the planes start zero; every fold clears what it visits
    for (int i = tid; i < 2 * (4 * kQPl + 2 * kCPl); i += kP2GThreads) qlo[0][i] = 0u;
    if (tid < 27) s_bmark[tid] = 0;
    for (;;) {
        __syncthreads();                  // the previous item's tiles, marks and shared state are done
        if (tid == 0) s_item = atomicAdd(&ctrl0->work_next, 1u);
        __syncthreads();
        const unsigned item = s_item;
        if (item >= n_work) break;
        const long long a = w.work[item];
        const unsigned key0 = keys[a];
        const unsigned sbk = key0 >> 6;                      // sub-block id
        const unsigned gblk = key0 >> kSortBlockBits;        // sub-blocks never span scenes
        const int sid = sc.of_sblock(gblk);
        const pm_params &prm = sc.params(sid);
        const Ctrl *cs = w.ctrl + sid;
        const int ng = prm.n_grid;
        const int nb = sort_blocks_per_axis(ng);
        const int nbs = (ng + kBlockEdge - 1) / kBlockEdge;
        const float inv_dx = (float)prm.inv_dx, dx = (float)prm.dx;
        const FixScale fm = fix_scale(cs->mom_bound), fma_ = fix_scale(cs->mass_bound),
                       fd = fix_scale(cs->dmg_bound), fw = fix_scale(__float_as_uint(1.0f));
        const float scl[4] = {fm.scale, fma_.scale, fd.scale, fw.scale};
        long long *g_mom = w.g_mom + 4 * sc.node_base(sid);
        long long *g_dmg = w.g_dmg + 2 * sc.node_base(sid);
        unsigned char *bmask = w.block_mask + sc.gblock_base(sid);
        const unsigned blk = gblk - sc.sblock_base(sid);
        const int bz = (int)(blk % nb), by = (int)((blk / nb) % nb), bx = (int)(blk / ((unsigned)nb * nb));
        const unsigned oct = (key0 >> 6) & 7u;               // Morton: the sub-block inside its 8^3 block
        const int org[3] = {bx * kSortBlock + (int)((oct >> 2) & 1u) * kSubEdge,
                            by * kSortBlock + (int)((oct >> 1) & 1u) * kSubEdge,
                            bz * kSortBlock + (int)(oct & 1u) * kSubEdge};   // first cell of the sub-block

        long long item_n = 0;                               // particles of the sub-block
        int chunk = 0;
        for (long long sub = a;; sub += kSub, ++chunk) {
            // ---------------- the chunk's payload (written by k_stress in sorted
            // order) into shared memory: coalesced float4 loads
            const long long i = sub + tid;
            const unsigned key = i < n ? keys[i] : 0xffffffffu;
            const bool valid = i < n && (key >> 6) == sbk;
            if (valid) {
                const float4 *src = w.payload + 5 * i;
                const float4 q0 = src[0], q1 = src[1], q2 = src[2], q3 = src[3], q4 = src[4];
                const int t = pay_col(tid);
                pay[0][t] = q0.x; pay[1][t] = q0.y; pay[2][t] = q0.z; pay[15][t] = q0.w;
                pay[3][t] = q1.x; pay[4][t] = q1.y; pay[5][t] = q1.z; pay[16][t] = q1.w;
                pay[6][t] = q2.x; pay[7][t] = q2.y; pay[8][t] = q2.z; pay[9][t] = q2.w;
                pay[10][t] = q3.x; pay[11][t] = q3.y; pay[12][t] = q3.z; pay[13][t] = q3.w;
                pay[14][t] = q4.x;
                regular[tid] = q4.y != 0.0f ? 1 : 0;
                lcell[tid] = (unsigned char)(key & 63u);
                if (q4.y != 0.0f) {   // the cubic weights of the cell's 5 node layers, once per particle
                    float e[5];
                    cw5(q0.x, e);
#pragma unroll
                    for (int k = 0; k < 5; ++k) cwt[k][t] = e[k];
                    cw5(q0.y, e);
#pragma unroll
                    for (int k = 0; k < 5; ++k) cwt[5 + k][t] = e[k];
                    cw5(q0.z, e);
#pragma unroll
                    for (int k = 0; k < 5; ++k) cwt[10 + k][t] = e[k];
                }
            }
            // runs of equal cell key inside the chunk (ordered compaction), and
            // the chunk's particle count (the valid lanes are a prefix)
            int nruns, cnt;
            {
                const unsigned prev = (tid > 0 && i <= n) ? keys[i - 1] : 0xffffffffu;
                const bool flag = valid && (tid == 0 || key != prev);
                const unsigned fb = __ballot_sync(0xffffffffu, flag), vb = __ballot_sync(0xffffffffu, valid);
                if (lane == 0) s_wcnt[wid] = (int)(__popc(fb) | (__popc(vb) << 16));
                __syncthreads();
                int pos = __popc(fb & lanemask_lt()), tot = 0, vt = 0;
#pragma unroll
                for (int w2 = 0; w2 < kP2GThreads / 32; ++w2) {
                    const int c = s_wcnt[w2];
                    pos += (w2 < wid) ? (c & 0xffff) : 0;
                    tot += c & 0xffff;
                    vt += c >> 16;
                }
                if (flag) runs[pos] = tid;
                if (tid == 0) runs[tot] = vt;
                nruns = tot;
                cnt = vt;
                item_n += vt;
                __syncthreads();
            }
            // ---------------- particles that need clamped nodes
            if (valid && !regular[tid]) {
                const int t = pay_col(tid);
                const float xp[3] = {pay[0][t], pay[1][t], pay[2][t]};   // positions for these particles
                const float mv[3] = {pay[3][t], pay[4][t], pay[5][t]};
                float aff[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) aff[k] = pay[6 + k][t];
                scatter_particle_global(xp, mv, aff, pay[15][t], pay[16][t], inv_dx, dx, ng, scl, g_mom, g_dmg,
                                        bmask, nbs);
            }
            // ---------------- (cell, slab) items into the chunk planes: items
            // 0 .. 3*nruns-1 are quadratic x-slabs, then 5*nruns cubic x-slabs,
            // slab-major, so the lanes of a warp mostly run one kind and one
            // slab over distinct cells (distinct nodes at every step)
            for (int it = tid; it < nruns * 8; it += kP2GThreads) {
                const bool quad = it < 3 * nruns;
                const int k = quad ? it : it - 3 * nruns;
                const int s8 = k / nruns;
                const int r = k - s8 * nruns;
                const int sl = quad ? s8 : 3 + s8;
                const int ja = runs[r], jb = runs[r + 1];
                int cq[3];
                morton_decode(lcell[ja], cq);                    // cell inside the sub-block
                if (sl == 0) {
                    // the cell's stencils (quadratic nodes c..c+2, cubic c-1..c+3 per
                    // axis) span grid blocks s-1+b .. s+b with b = (c > 0): marked
                    // whatever the sums, so that the grid update writes every node a
                    // gather reads (a node whose contributions all round to zero
                    // still gets its zero velocity and damage)
                    const int b0 = cq[0] > 0, b1 = cq[1] > 0, b2 = cq[2] > 0;
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        s_bmark[((b0 + (k >> 2)) * 3 + b1 + ((k >> 1) & 1)) * 3 + b2 + (k & 1)] = 1;
                }
                if (sl < 3) {
                    const int ox = sl;
                    // packed pairs: components (0, 1) and (2, mass) of every node
                    float2 acc[3][3][2];
#pragma unroll
                    for (int i2 = 0; i2 < 3; ++i2)
#pragma unroll
                        for (int j = 0; j < 3; ++j) acc[i2][j][0] = acc[i2][j][1] = make_float2(0.0f, 0.0f);
                    const int jend = regular[ja] ? jb : ja;
                    for (int j = ja; j < jend; ++j) {
                        const int t = pay_col(j);
                        const float fx0 = pay[0][t], fx1 = pay[1][t], fx2 = pay[2][t];
                        float wx[3], wy[3], wz[3];
                        qw(fx0, wx); qw(fx1, wy); qw(fx2, wz);
                        const float dxo = ((float)ox - fx0) * dx;
                        const float m = pay[15][t];
                        const float2 base01 = fma2(make_float2(pay[6][t], pay[9][t]), bc2(dxo),
                                                   make_float2(pay[3][t], pay[4][t]));
                        const float base2 = pay[5][t] + pay[12][t] * dxo;
                        const float2 ay01 = make_float2(pay[7][t], pay[10][t]), az01 = make_float2(pay[8][t], pay[11][t]);
                        const float ay2 = pay[13][t], az2 = pay[14][t];
                        const float wxs = ox == 0 ? wx[0] : (ox == 1 ? wx[1] : wx[2]);
                        float2 bz[3][2], wz2[3];
#pragma unroll
                        for (int oz = 0; oz < 3; ++oz) {
                            const float dz = ((float)oz - fx2) * dx;
                            wz2[oz] = bc2(wz[oz]);
                            bz[oz][0] = mul2(wz2[oz], fma2(az01, bc2(dz), base01));
                            bz[oz][1] = mul2(wz2[oz], make_float2(base2 + az2 * dz, m));
                        }
#pragma unroll
                        for (int oy = 0; oy < 3; ++oy) {
                            const float wxy = wxs * wy[oy];
                            const float wdy = wxy * (((float)oy - fx1) * dx);
                            const float2 w2 = bc2(wxy);
                            const float2 ady01 = mul2(bc2(wdy), ay01), ady2 = make_float2(wdy * ay2, 0.0f);
#pragma unroll
                            for (int oz = 0; oz < 3; ++oz) {
                                acc[oy][oz][0] = fma2(ady01, wz2[oz], fma2(w2, bz[oz][0], acc[oy][oz][0]));
                                acc[oy][oz][1] = fma2(ady2, wz2[oz], fma2(w2, bz[oz][1], acc[oy][oz][1]));
                            }
                        }
                    }
                    const int nx = cq[0] + ox;
#pragma unroll
                    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                        for (int oz = 0; oz < 3; ++oz) {
                            const int sidx = nx * kQSX + (cq[1] + oy) * kQSY + cq[2] + oz;
                            plane_add(&qlo[0][sidx], &qhi[0][sidx], acc[oy][oz][0].x, scl[0]);
                            plane_add(&qlo[1][sidx], &qhi[1][sidx], acc[oy][oz][0].y, scl[0]);
                            plane_add(&qlo[2][sidx], &qhi[2][sidx], acc[oy][oz][1].x, scl[0]);
                            plane_add(&qlo[3][sidx], &qhi[3][sidx], acc[oy][oz][1].y, scl[1]);
                        }
                } else {
                    const int nxs = sl - 3;
                    float2 acw[5][5];   // packed pairs (sum w d, sum w) of every node
#pragma unroll
                    for (int i2 = 0; i2 < 5; ++i2)
#pragma unroll
                        for (int j = 0; j < 5; ++j) acw[i2][j] = make_float2(0.0f, 0.0f);
                    const int jend = regular[ja] ? jb : ja;
                    for (int j = ja; j < jend; ++j) {
                        const int t = pay_col(j);
                        const float wxs = cwt[nxs][t];
                        const float d = pay[16][t];
                        float2 ez2[5];
#pragma unroll
                        for (int k = 0; k < 5; ++k) {
                            const float ez = cwt[10 + k][t];
                            ez2[k] = make_float2(d * ez, ez);
                        }
#pragma unroll
                        for (int ny = 0; ny < 5; ++ny) {
                            const float2 w2 = bc2(wxs * cwt[5 + ny][t]);
#pragma unroll
                            for (int nz = 0; nz < 5; ++nz) acw[ny][nz] = fma2(w2, ez2[nz], acw[ny][nz]);
                        }
                    }
                    const int nx = cq[0] + nxs;
#pragma unroll
                    for (int ny = 0; ny < 5; ++ny)
#pragma unroll
                        for (int nz = 0; nz < 5; ++nz) {
                            const int sidx = nx * kCSX + (cq[1] + ny) * kCSY + cq[2] + nz;
                            plane_add(&clo[0][sidx], &chi[0][sidx], acw[ny][nz].x, scl[2]);
                            plane_add(&clo[1][sidx], &chi[1][sidx], acw[ny][nz].y, scl[3]);
                        }
                }
            }
            __syncthreads();
            const bool last = cnt < kSub;                       // uniform: the last chunk of the sub-block
            // the planes take up to four chunks (1,024 particles) before they
            // must be folded: one add per node is below 0.42 (the largest
            // quadratic weight) of 2^46 units per particle, so the high plane
            // stays under 1024 * 0.42 * 2^22 < 2^31; a node takes at most one
            // add per covering cell and chunk, fewer than 2^7 adds of 24 bits
            // into the unsigned low plane
            if (last || (chunk & 3) == 3) {
                // ---------------- fold the chunk planes straight into the global
                // grid, one int64 atomic per nonzero node component, clearing
                // them.  Integer addition is associative, so a sub-block of more
                // than four chunks, folded more than once, adds the same total.
                for (int li = tid; li < kQN; li += kP2GThreads) {
                    const int tx = li / (kQE * kQE), ty = (li / kQE) % kQE, tz = li % kQE;
                    const int sidx = tx * kQSX + ty * kQSY + tz;
                    long long q[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const unsigned lo = qlo[c][sidx];
                        const int hi = qhi[c][sidx];
                        q[c] = 0;
                        if ((lo | (unsigned)hi) != 0u) {
                            qlo[c][sidx] = 0u;
                            qhi[c][sidx] = 0;
                            q[c] = plane_value(lo, hi);
                        }
                    }
                    if ((q[0] | q[1] | q[2] | q[3]) != 0) {
                        long long *g = g_mom + 4 * (((long long)(org[0] + tx) * ng + (org[1] + ty)) * ng + (org[2] + tz));
#pragma unroll
                        for (int c = 0; c < 4; ++c)
                            if (q[c]) atomicAdd((unsigned long long *)(g + c), (unsigned long long)q[c]);
                    }
                }
                for (int li = tid; li < kCN; li += kP2GThreads) {
                    const int tx = li >> 6, ty = (li >> 3) & 7, tz = li & 7;
                    const int sidx = tx * kCSX + ty * kCSY + tz;
                    long long q[2];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const unsigned lo = clo[c][sidx];
                        const int hi = chi[c][sidx];
                        q[c] = 0;
                        if ((lo | (unsigned)hi) != 0u) {
                            clo[c][sidx] = 0u;
                            chi[c][sidx] = 0;
                            q[c] = plane_value(lo, hi);
                        }
                    }
                    if ((q[0] | q[1]) != 0) {
                        long long *g = g_dmg + 2 * (((long long)(org[0] - 1 + tx) * ng + (org[1] - 1 + ty)) * ng +
                                                    (org[2] - 1 + tz));
                        if (q[0]) atomicAdd((unsigned long long *)g, (unsigned long long)q[0]);
                        if (q[1]) atomicAdd((unsigned long long *)(g + 1), (unsigned long long)q[1]);
                    }
                }
            }
            if (last) break;
            __syncthreads();                                    // the planes are clear for the next chunk
        }
        // a sub-block denser than the fixed-point headroom allows: its nodes'
        // sums are not guaranteed exact; counted for the status
        if (tid == 0 && item_n > kDenseSubblock) atomicAdd(&w.ctrl[sid].dense_subblocks, 1u);
        __syncthreads();
        if (tid < 27 && s_bmark[tid]) {
            s_bmark[tid] = 0;
            const int sbx = org[0] >> 2, sby = org[1] >> 2, sbz = org[2] >> 2;   // the sub-block's grid block
            const int bxx = sbx - 1 + tid / 9, byy = sby - 1 + (tid / 3) % 3, bzz = sbz - 1 + tid % 3;
            if (bxx >= 0 && byy >= 0 && bzz >= 0 && bxx < nbs && byy < nbs && bzz < nbs)
                bmask[((long long)bxx * nbs + byy) * nbs + bzz] = 1;
        }
    }
}

// Particles per CTA: equal ranges that fill whole waves of the resident CTA
// slots, so no SM idles behind a partial last wave.
int balanced_range(long long n, int slots, int max_range) {
    if (slots < 1) slots = 1;
    const long long waves = (n + (long long)slots * max_range - 1) / ((long long)slots * max_range);
    long long r = (n + slots * waves - 1) / (slots * waves);
    r = (r + 31) / 32 * 32;
    return (int)std::max<long long>(32, std::min<long long>(r, max_range));
}

int resident_slots(const void *kernel, int threads, size_t smem) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
    return std::max(1, sms * std::max(per, 1));
}

// One-time kernel attribute set-up for the current device (not a stream
// operation, so it must not first happen inside a stream capture).
void prepare_p2g() {
    static int done[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(k_p2g_tiles<PlainScenes, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2GSmem);
        cudaFuncSetAttribute(k_p2g_tiles<BatchScenes, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2GSmem);
        cudaFuncSetAttribute(k_p2g_tiles<PlainScenes, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2GSmem);
        cudaFuncSetAttribute(k_p2g_tiles<BatchScenes, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2GSmem);
        done[dev] = 1;
    }
}

// Persistent P2G CTAs: every resident slot of the device (work items are
// taken from the list dynamically).  `ctas_per_sm`: 0 = the 80-register
// kernel with as many CTAs as fit (3 per SM); 4 = the 64-register kernel at 4
// per SM; 1..3 = the 80-register kernel capped at that many per SM.
template <class SC>
void launch_p2g(const SC &sc, const Parts &P, const WS &w, cudaStream_t s, int ctas_per_sm, int stress_ctas) {
    if (P.n <= 0) return;
    prepare_p2g();
    const int lb = (int)std::min<long long>((P.n + 255) / 256, 148LL * 8);
    k_subblocks<<<lb, 256, 0, s>>>(w.sorted_keys, P.n, w.work, w.ctrl);
    if (stress_ctas == 4)
        k_stress<SC, 4><<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(sc, P, w);
    else
        k_stress<SC, 3><<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(sc, P, w);
    k_bounds<<<sc.count(), kBoundSlots, 0, s>>>(w.ctrl);
    static int slots_dev[64][2] = {{0}};
    int dev = 0;
    cudaGetDevice(&dev);
    const bool wide = ctas_per_sm >= 4;
    int slots = (dev >= 0 && dev < 64) ? slots_dev[dev][wide] : 0;
    if (slots <= 0) {
        slots = wide ? resident_slots((const void *)k_p2g_tiles<SC, 4>, kP2GThreads, kP2GSmem)
                     : resident_slots((const void *)k_p2g_tiles<SC, 3>, kP2GThreads, kP2GSmem);
        if (dev >= 0 && dev < 64) slots_dev[dev][wide] = slots;
    }
    if (ctas_per_sm > 0 && !wide) {   // the cap
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        slots = std::min(slots, sms * ctas_per_sm);
    }
    const unsigned blocks = (unsigned)std::max<long long>(1, std::min<long long>(slots, (P.n + 63) / 64));
    if (wide)
        k_p2g_tiles<SC, 4><<<blocks, kP2GThreads, kP2GSmem, s>>>(sc, w, P.n);
    else
        k_p2g_tiles<SC, 3><<<blocks, kP2GThreads, kP2GSmem, s>>>(sc, w, P.n);
}
template void launch_p2g<PlainScenes>(const PlainScenes &, const Parts &, const WS &, cudaStream_t, int, int);
template void launch_p2g<BatchScenes>(const BatchScenes &, const Parts &, const WS &, cudaStream_t, int, int);

}  // namespace pm
