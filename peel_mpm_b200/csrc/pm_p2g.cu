// Fused constitutive update + P2G.
//
// One CTA takes 2048 consecutive particles of the block-sorted order and splits
// them into segments that share one 8^3-cell sort block.  For each segment a
// 12^3-node shared-memory tile (the block's stencil footprint) is zeroed, then
// in sub-chunks of 256:
//   phase 1 (one particle per thread): particle BC, polar decomposition by a
//   Jacobi eigensolve of F^T F, fixed-corotated Kirchhoff stress, anisotropic
//   phase-field damage (second Jacobi eigensolve, of the Cauchy stress),
//   degradation and the APIC affine term; the P2G payload goes to shared
//   memory;
//   phase 2: lane l of warp w scatters element 8*l + w of the sub-chunk, so
//   the lanes of a warp hold particles ~8 apart in cell order (mostly in
//   different cells) and their shared-memory atomics rarely hit one address.
// The tile is then flushed with one vector atomic per touched node.
//
// Reference: anisompm.py:601-724 (constitutive, damage, P2G) and 768-776
// (cubic damage scatter).
#include "pm_kernels.cuh"

namespace pm {

constexpr int kP2GThreads = 256;
constexpr int kPay = 17;         // payload floats: x(3) mv(3) affine(9) m d
constexpr int kPayStride = kP2GThreads + kP2GThreads / 32;

__device__ __forceinline__ float clamp_min(float v, float lo) { return v < lo ? lo : v; }   // torch.clamp(min=)
__device__ __forceinline__ float relu(float v) { return v > 0.0f ? v : (v != v ? v : 0.0f); }
// torch.maximum: NaN if either operand is NaN
__device__ __forceinline__ float tmax(float a, float b) { return (a != a || b != b) ? a + b : (a > b ? a : b); }

// Constitutive update of particle p (anisompm.py:614-706).  Writes tau and
// updates F (f_clamp), d, D_hist and the diagnostics in place.
__device__ __forceinline__ void constitutive(const pm_params &prm, const Parts &P, long long p, bool do_damage,
                                             float tau[9]) {
    const long long ps = P.ps;
    float F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = P.F[k * ps + p];
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
    mm3(F, V, W);                                                    // (619)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float nr = sqrtf(W[j] * W[j] + W[3 + j] * W[3 + j] + W[6 + j] * W[6 + j]) + 1e-12f;
#pragma unroll
        for (int i = 0; i < 3; ++i) W[3 * i + j] = W[3 * i + j] / nr;   // (620)
    }
    mmt3(W, V, R);                                                   // R = What V^T (621)
    if (prm.use_f_clamp) {                                           // (622-636)
        const float lo = (float)prm.f_clamp_lo, hi = (float)prm.f_clamp_hi;
        float D[9], corr[9];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            float sc = S[i] < lo ? lo : S[i];
            sc = sc > hi ? hi : sc;
            const float ratio = sc / clamp_min(S[i], 1e-12f);
#pragma unroll
            for (int r = 0; r < 3; ++r) D[3 * r + i] = V[3 * r + i] * ratio;
            S[i] = sc;
        }
        mmt3(D, V, corr);
        mm3(F, corr, F);
#pragma unroll
        for (int k = 0; k < 9; ++k) P.F[k * ps + p] = F[k];
    }
    const float J = clamp_min(S[0] * S[1] * S[2], 1e-6f);            // (637)
    const float mu = P.mu[p], lam = P.lam[p];
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
#pragma unroll
        for (int k = 0; k < 9; ++k) sg[k] = (tdev[k] + ((k % 4 == 0) ? tv : 0.0f)) / J;
        float sgs[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) sgs[3 * i + j] = 0.5f * (sg[3 * i + j] + sg[3 * j + i]);
        float ev[3], EV[9];
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
            for (int k = 0; k < 9; ++k) A0[k] = P.A0[k * ps + p];
            mm3(R, A0, RA);
            mmt3(RA, R, A);                                          // A = R A0 R^T (661)
        }
        float M[9];
        mm3(A, sp, M);
        const float trMM = (M[0] * M[0] + M[1] * M[3] + M[2] * M[6]) + (M[3] * M[1] + M[4] * M[4] + M[5] * M[7]) +
                           (M[6] * M[2] + M[7] * M[5] + M[8] * M[8]);
        const float sc = P.sigma_c[p];
        const float phi = trMM / (sc * sc);                          // (663-664)
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
        const float drive = P.zeta[p] * relu(phi - 1.0f);
        const float dh0 = P.D_hist[p];
        const float Dh = tmax(dh0, drive);
        P.D_hist[p] = Dh;                                            // history max (679)
        const float d = P.d[p];
        const float l0 = P.l0[p];
        const float resist = d - (l0 * l0) * P.lap[p];
        const float ddot = relu((1.0f - d) * Dh - resist);           // (681-682)
        const float dt_dmg = (float)(prm.dt * (double)prm.damage_every);
        float dn = d + (dt_dmg / P.eta[p]) * ddot;
        dn = dn < 0.0f ? 0.0f : dn;
        dn = dn > 1.0f ? 1.0f : dn;                                  // (683-684)
        if (P.allow[p]) P.d[p] = tmax(dn, d);                        // monotone, where allowed (685)
    }
    const float d = P.d[p];
    const float res = P.residual[p];
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

// Static shared tile of one sort block: nodes [8*blk - 1, 8*blk + 11) per axis
// hold every quadratic [qb, qb+2] and cubic [qb-1, qb+3] stencil node of the
// block's particles (clamped coordinates included).
constexpr int kTE = kSortBlock + 4;            // 12
constexpr int kTileNodes = kTE * kTE * kTE;    // 1728

// Scatter one particle's quadratic momentum (27 nodes) and cubic damage (64
// nodes) into the shared tile whose node origin is org.
__device__ __forceinline__ void scatter_particle(const float xp[3], const float mv[3], const float aff[9], float m,
                                                 float d, float inv_dx, float dx, int ng, const int org[3],
                                                 float *__restrict__ tile) {
    {
        Quad q;
        quad_weights(xp, inv_dx, ng, q);
        int NX[3], NY[3], NZ[3];
        float DX[3], DY[3], DZ[3];
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            NX[o] = (clampi(q.b[0] + o, 0, ng - 1) - org[0]) * (kTE * kTE);
            NY[o] = (clampi(q.b[1] + o, 0, ng - 1) - org[1]) * kTE;
            NZ[o] = clampi(q.b[2] + o, 0, ng - 1) - org[2];
            DX[o] = ((float)o - q.fx[0]) * dx;                       // dpos (718)
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
                    const int node = NX[ox] + NY[oy] + NZ[oz];
                    const float a0 = aff[0] * DX[ox] + aff[1] * DY[oy] + aff[2] * DZ[oz];
                    const float a1 = aff[3] * DX[ox] + aff[4] * DY[oy] + aff[5] * DZ[oz];
                    const float a2 = aff[6] * DX[ox] + aff[7] * DY[oy] + aff[8] * DZ[oz];
                    atomicAdd(&tile[0 * kTileNodes + node], wk * (mv[0] + a0));
                    atomicAdd(&tile[1 * kTileNodes + node], wk * (mv[1] + a1));
                    atomicAdd(&tile[2 * kTileNodes + node], wk * (mv[2] + a2));
                    atomicAdd(&tile[3 * kTileNodes + node], wk * m);
                }
            }
    }
    {
        Cubic c;
        cubic_weights(xp, inv_dx, ng, c);
        int NX[4], NY[4], NZ[4];
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            NX[o] = (clampi(c.b[0] + o, 0, ng - 1) - org[0]) * (kTE * kTE);
            NY[o] = (clampi(c.b[1] + o, 0, ng - 1) - org[1]) * kTE;
            NZ[o] = clampi(c.b[2] + o, 0, ng - 1) - org[2];
        }
#pragma unroll
        for (int ox = 0; ox < 4; ++ox)
#pragma unroll
            for (int oy = 0; oy < 4; ++oy) {
                const float wxy = c.w[ox][0] * c.w[oy][1];
#pragma unroll
                for (int oz = 0; oz < 4; ++oz) {
                    const float wk = wxy * c.w[oz][2];
                    const int node = NX[ox] + NY[oy] + NZ[oz];
                    atomicAdd(&tile[4 * kTileNodes + node], wk * d);
                    atomicAdd(&tile[5 * kTileNodes + node], wk);
                }
            }
    }
}

constexpr int kP2GRange = 2048;   // sorted particles per CTA
constexpr size_t kP2GSmem = sizeof(float) * (6 * kTileNodes + kPay * kPayStride) +
                            sizeof(unsigned) * kP2GRange + sizeof(int) * (kP2GRange + 2);

// One CTA per kP2GRange sorted particles, split into segments of one sort
// block each; a segment is accumulated in the block's tile and flushed.
template <int STRIDE>
__global__ void __launch_bounds__(kP2GThreads, 2) k_p2g(const pm_params prm, const Parts P, const WS w) {
    extern __shared__ float4 s_raw[];
    float *s_tile = (float *)s_raw;                                   // [6][kTileNodes]
    float (*s_pay)[kPayStride] = (float (*)[kPayStride])(s_tile + 6 * kTileNodes);
    unsigned *s_blk = (unsigned *)(s_tile + 6 * kTileNodes + kPay * kPayStride);
    int *s_seg = (int *)(s_blk + kP2GRange);                          // segment starts, then count
    __shared__ int s_wcnt[kP2GThreads / 32];

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const long long n = P.n;
    const long long r0 = (long long)blockIdx.x * kP2GRange;
    const int len = (int)min((long long)kP2GRange, n - r0);
    const int ng = prm.n_grid;
    const int nb = sort_blocks_per_axis(ng);
    const float inv_dx = (float)prm.inv_dx, dx = (float)prm.dx;
    const Ctrl *ctrl = w.ctrl;
    const bool do_damage = ctrl->any_allow != 0 && (ctrl->step % (long long)prm.damage_every) == 0;

    // ---- segment the range at sort-block boundaries (ordered compaction)
    for (int i = tid; i < len; i += kP2GThreads) s_blk[i] = w.sorted_keys[r0 + i] >> kSortBlockBits;
    __syncthreads();
    constexpr int PER = kP2GRange / kP2GThreads;
    int flags = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid * PER + k;
        if (i < len && (i == 0 || s_blk[i] != s_blk[i - 1])) flags |= 1 << k;
    }
    const int cnt = __popc(flags);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_wcnt[wid] = incl;
    __syncthreads();
    int pos = incl - cnt;
    for (int w2 = 0; w2 < wid; ++w2) pos += s_wcnt[w2];
#pragma unroll
    for (int k = 0; k < PER; ++k)
        if (flags & (1 << k)) s_seg[pos++] = tid * PER + k;
    if (tid == kP2GThreads - 1) {
        int total = 0;
        for (int w2 = 0; w2 < kP2GThreads / 32; ++w2) total += s_wcnt[w2];
        s_seg[kP2GRange + 1] = total;
    }
    __syncthreads();
    const int nseg = s_seg[kP2GRange + 1];

    for (int sg = 0; sg < nseg; ++sg) {
        const int a = s_seg[sg];
        const int b = (sg + 1 < nseg) ? s_seg[sg + 1] : len;
        const unsigned blk = s_blk[a];
        const int bz = (int)(blk % nb), by = (int)((blk / nb) % nb), bx = (int)(blk / ((unsigned)nb * nb));
        const int org[3] = {bx * kSortBlock - 1, by * kSortBlock - 1, bz * kSortBlock - 1};
        for (int i = tid; i < 6 * kTileNodes; i += kP2GThreads) s_tile[i] = 0.0f;

        for (int sub = a; sub < b; sub += kP2GThreads) {
            // phase 1: constitutive update of one particle per thread
            const int cnt_sub = min(kP2GThreads, b - sub);
            if (tid < cnt_sub) {
                const long long p = w.perm[r0 + sub + tid];
                const long long ps = P.ps;
                float tau[9];
                constitutive(prm, P, p, do_damage, tau);
                float v[3] = {P.v[p], P.v[ps + p], P.v[2 * ps + p]};
                if (P.grip_tag) {                                    // particle BCs (601-602)
                    const int g = P.grip_tag[p];
                    if (g >= 0 && g < prm.n_grips) {
                        const double f = prm.grips[g].ramp > 0.0 ? fmin(ctrl->time / prm.grips[g].ramp, 1.0) : 1.0;
#pragma unroll
                        for (int ax = 0; ax < 3; ++ax) v[ax] = (float)(prm.grips[g].vel[ax] * f);
                    }
                }
                const float m = P.mass[p];
                // stress_coeff = -dt*vol0*4*inv_dx*inv_dx; affine = coeff*tau + m*C (711-713)
                const float coeff = __fmul_rn(
                    __fmul_rn(__fmul_rn(__fmul_rn((float)(-prm.dt), P.vol0[p]), 4.0f), inv_dx), inv_dx);
                const int t = tid + (tid >> 5);
#pragma unroll
                for (int k = 0; k < 9; ++k) s_pay[6 + k][t] = coeff * tau[k] + m * P.C[k * ps + p];
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) {
                    s_pay[ax][t] = P.x[ax * ps + p];
                    s_pay[3 + ax][t] = m * v[ax];
                }
                s_pay[15][t] = m;
                s_pay[16][t] = P.d[p];
            }
            __syncthreads();
            // phase 2: scatter; lane l of warp w takes element STRIDE*l + w
            const int j = (STRIDE == 1) ? tid : (lane * STRIDE + wid);
            if (j < cnt_sub) {
                const int t = j + (j >> 5);
                const float xp[3] = {s_pay[0][t], s_pay[1][t], s_pay[2][t]};
                const float mv[3] = {s_pay[3][t], s_pay[4][t], s_pay[5][t]};
                float aff[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) aff[k] = s_pay[6 + k][t];
                scatter_particle(xp, mv, aff, s_pay[15][t], s_pay[16][t], inv_dx, dx, ng, org, s_tile);
            }
            __syncthreads();
        }
        // flush the tile: one vector atomic per touched node
        for (int i = tid; i < kTileNodes; i += kP2GThreads) {
            const int tx = i / (kTE * kTE), ty = (i / kTE) % kTE, tz = i % kTE;
            const int gx = org[0] + tx, gy = org[1] + ty, gz = org[2] + tz;
            if (gx < 0 || gy < 0 || gz < 0 || gx >= ng || gy >= ng || gz >= ng) continue;
            const float a0 = s_tile[i], a1 = s_tile[kTileNodes + i], a2 = s_tile[2 * kTileNodes + i],
                        a3 = s_tile[3 * kTileNodes + i], a4 = s_tile[4 * kTileNodes + i],
                        a5 = s_tile[5 * kTileNodes + i];
            const long long node = ((long long)gx * ng + gy) * ng + gz;
            if (a0 != 0.0f || a1 != 0.0f || a2 != 0.0f || a3 != 0.0f)
                atomicAdd(&w.g_mom[node], make_float4(a0, a1, a2, a3));
            if (a4 != 0.0f || a5 != 0.0f) atomicAdd(&w.g_dmg[node], make_float2(a4, a5));
        }
        __syncthreads();
    }
}

void launch_p2g(const pm_params &prm, const Parts &P, const WS &w, cudaStream_t s) {
    const long long blocks = (P.n + kP2GRange - 1) / kP2GRange;
    if (blocks <= 0) return;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_p2g<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2GSmem);
        configured = true;
    }
    k_p2g<8><<<(unsigned)blocks, kP2GThreads, kP2GSmem, s>>>(prm, P, w);
}

}  // namespace pm
