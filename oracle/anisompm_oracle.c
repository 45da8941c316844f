/*
 * CPU oracle for the AnisoMPM substep -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference solver's substep
 * (anisompm_py/src/anisompm.py, class AnisoMPM) used to check the CUDA path.
 * Nothing in the product links or calls this file; only tests/, the smoke
 * check and the CPU-baseline legs of bench.py load it.
 *
 * Compiled twice: -DORACLE_REAL=float (the reference's default dtype) and
 * -DORACLE_REAL=double (the FP64 comparison run).  Arithmetic mirrors the
 * reference's op-by-op rounding: Python scalars enter as `real` constants, each
 * tensor op rounds separately (build with -ffp-contract=off), reductions
 * accumulate in index order.
 *
 * Layout is the reference's own (array-of-structs): x (N,3), F (N,3,3) row
 * major, etc.
 *
 * Scatter order.  scatter_mode 0 follows the reference exactly: stencil offset
 * outermost, particles in index order (anisompm.py:716-724, 771-776), single
 * threaded.  scatter_mode 1 colours particles into x-slabs of 4 base cells and
 * scatters even slabs, then odd slabs, in parallel (slabs of one colour touch
 * disjoint nodes); it is deterministic for any thread count and differs from
 * mode 0 only in the summation order inside a node.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <tgmath.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;
#define R(c) ((real)(c))

#if defined(ORACLE_F64)
#define REAL_MAX DBL_MAX
#else
#define REAL_MAX FLT_MAX
#endif

typedef struct {
    int64_t n;
    int32_t n_grid;
    int32_t nthreads;
    int32_t scatter_mode;
    int32_t do_damage;          /* allow.any() && step % damage_every == 0 (anisompm.py:647) */
    double grid_lim, dx, inv_dx, dt, dt_dmg;
    double gravity[3];
    double grid_damp;
    int32_t use_f_clamp;
    double f_clamp_lo, f_clamp_hi;
    int32_t any_interface;
    int32_t n_colliders;
    /* per collider 16 doubles: kind(0 half,1 sphere), mode(0 slip,1 sticky), friction,
       radius, normal[3], origin(t)[3], origin(t+1e-4)[3], pad */
    const double *colliders;
    int32_t n_grips;
    const int32_t *grip_tag;    /* (N) group or -1 */
    const double *grip_vel;     /* (n_grips,3) velocity at this substep's time */
} oracle_params;

typedef struct {
    real *x, *v, *F, *C, *d, *lap, *D_hist;
    const real *vol0, *mass, *mu, *lam, *sigma_c, *eta, *zeta, *l0, *residual, *A0;
    const uint8_t *allow;
    const real *n_interface;
    const uint8_t *interface_mask;
    real *phi, *phi_shear, *tau_last, *J_last;   /* nullable diagnostics */
} oracle_state;

/* optional intermediate grids (nullable): dense ng^3 */
typedef struct {
    real *grid_mv;   /* (G,3) after P2G */
    real *grid_m;    /* (G) */
    real *grid_v;    /* (G,3) after grid update + colliders */
    real *grid_dc;   /* (G) cubic scatter of w*d */
    real *grid_dwc;  /* (G) cubic scatter of w */
    real *gd;        /* (G) normalised damage field */
} oracle_grids;

/* ------------------------------------------------------------------ small LA */
static inline real nan_to_num(real a) {
    if (a != a) return R(0);
    if (a > REAL_MAX) return REAL_MAX;
    if (a < -REAL_MAX) return -REAL_MAX;
    return a;
}

/* C = A @ B, 3x3 row-major, k-ordered accumulation */
static inline void mm3(const real *A, const real *B, real *C) {
    real T[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            real acc = A[3 * i + 0] * B[0 * 3 + j];
            acc = acc + A[3 * i + 1] * B[1 * 3 + j];
            acc = acc + A[3 * i + 2] * B[2 * 3 + j];
            T[3 * i + j] = acc;
        }
    memcpy(C, T, sizeof(T));
}
/* C = A @ B^T */
static inline void mmt3(const real *A, const real *B, real *C) {
    real T[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            real acc = A[3 * i + 0] * B[3 * j + 0];
            acc = acc + A[3 * i + 1] * B[3 * j + 1];
            acc = acc + A[3 * i + 2] * B[3 * j + 2];
            T[3 * i + j] = acc;
        }
    memcpy(C, T, sizeof(T));
}
/* C = A^T @ B */
static inline void mtm3(const real *A, const real *B, real *C) {
    real T[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            real acc = A[0 * 3 + i] * B[0 * 3 + j];
            acc = acc + A[1 * 3 + i] * B[1 * 3 + j];
            acc = acc + A[2 * 3 + i] * B[2 * 3 + j];
            T[3 * i + j] = acc;
        }
    memcpy(C, T, sizeof(T));
}

/* Batched cyclic Jacobi for one symmetric 3x3 (anisompm.py:48-95).  Pair order
 * (0,1),(0,2),(1,2); rotation skipped when |apq| <= 1e-30; sign(0) = +1;
 * eigenvalues sorted ascending (stable), eigenvector columns follow. */
static void sym_eig3(const real *Ain, int sweeps, real *evals, real *V) {
    real A[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            A[3 * i + j] = nan_to_num(R(0.5) * (Ain[3 * i + j] + Ain[3 * j + i]));
    real W[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    static const int PQ[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int sw = 0; sw < sweeps; ++sw) {
        for (int k = 0; k < 3; ++k) {
            const int p = PQ[k][0], q = PQ[k][1], r = 3 - p - q;
            const real app = A[3 * p + p], aqq = A[3 * q + q], apq = A[3 * p + q];
            const real apr = A[3 * p + r], aqr = A[3 * q + r];
            real t = R(0);
            if (fabs(apq) > R(1e-30)) {
                const real z = (aqq - app) / (R(2.0) * apq);
                const real sgn = (z >= R(0)) ? R(1) : R(-1);
                t = sgn / (fabs(z) + sqrt(R(1.0) + z * z));
            }
            const real c = R(1.0) / sqrt(R(1.0) + t * t);
            const real s = c * t;
            A[3 * p + p] = c * c * app - R(2.0) * s * c * apq + s * s * aqq;
            A[3 * q + q] = s * s * app + R(2.0) * s * c * apq + c * c * aqq;
            A[3 * p + q] = R(0); A[3 * q + p] = R(0);
            const real npr = c * apr - s * aqr, nqr = s * apr + c * aqr;
            A[3 * p + r] = npr; A[3 * r + p] = npr;
            A[3 * q + r] = nqr; A[3 * r + q] = nqr;
            for (int i = 0; i < 3; ++i) {
                const real vp = W[3 * i + p], vq = W[3 * i + q];
                W[3 * i + p] = c * vp - s * vq;
                W[3 * i + q] = s * vp + c * vq;
            }
        }
    }
    real e[3] = {A[0], A[4], A[8]};
    int idx[3] = {0, 1, 2};
    /* stable insertion sort ascending */
    for (int i = 1; i < 3; ++i) {
        int j = i;
        while (j > 0 && e[idx[j - 1]] > e[idx[j]]) { int tmp = idx[j]; idx[j] = idx[j - 1]; idx[j - 1] = tmp; --j; }
    }
    for (int j = 0; j < 3; ++j) {
        evals[j] = e[idx[j]];
        for (int i = 0; i < 3; ++i) V[3 * i + j] = W[3 * i + idx[j]];
    }
}

void oracle_sym_eig(const real *A, int64_t n, int32_t sweeps, real *evals, real *evecs) {
    for (int64_t p = 0; p < n; ++p) sym_eig3(A + 9 * p, sweeps, evals + 3 * p, evecs + 9 * p);
}

/* --------------------------------------------------------------- weights */
/* floor(v).to(long) as torch does it on x86: NaN / out of int64 range -> INT64_MIN */
static inline int64_t floor_to_long(real v) {
    real f = floor(v);
    if (!(f >= R(-9223372036854775808.0) && f < R(9223372036854775808.0))) return INT64_MIN;
    return (int64_t)f;
}
static inline int64_t clampl(int64_t v, int64_t lo, int64_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* _weights (anisompm.py:544-557): quadratic base, fx, per-axis weights w[node][axis] */
static inline void quad_weights(const real *xp, real inv_dx, int64_t base[3], real fx[3], real w[3][3]) {
    for (int a = 0; a < 3; ++a) {
        const real X = xp[a] * inv_dx;
        base[a] = floor_to_long(X - R(0.5));
        fx[a] = X - (real)base[a];
        const real t0 = R(1.5) - fx[a], t1 = fx[a] - R(1.0), t2 = fx[a] - R(0.5);
        w[0][a] = R(0.5) * (t0 * t0);
        w[1][a] = R(0.75) - t1 * t1;
        w[2][a] = R(0.5) * (t2 * t2);
    }
}

/* _cubic_weights (anisompm.py:559-584) */
static inline void cubic_weights(const real *xp, real inv_dx, int64_t base[3], real w[4][3], real w2[4][3]) {
    for (int a = 0; a < 3; ++a) {
        const real X = xp[a] * inv_dx;
        const int64_t fl = floor_to_long(X);
        base[a] = (fl == INT64_MIN) ? INT64_MIN : fl - 1;
        const real f = X - (real)(base[a] == INT64_MIN ? INT64_MIN : base[a] + 1);
        const real one = R(1.0) - f;
        w[0][a] = R(1.0 / 6.0) * (one * one * one);
        w[1][a] = R(2.0 / 3.0) - f * f + R(0.5) * (f * f * f);
        w[2][a] = R(2.0 / 3.0) - one * one + R(0.5) * (one * one * one);
        w[3][a] = R(1.0 / 6.0) * (f * f * f);
        w2[0][a] = one;
        w2[1][a] = R(3.0) * f - R(2.0);
        w2[2][a] = R(1.0) - R(3.0) * f;
        w2[3][a] = f;
    }
}

/* _node_index (anisompm.py:586-590) */
static inline int64_t node_index(const int64_t b[3], int ox, int oy, int oz, int64_t ng) {
    const int64_t nx = clampl(b[0] == INT64_MIN ? INT64_MIN : b[0] + ox, 0, ng - 1);
    const int64_t ny = clampl(b[1] == INT64_MIN ? INT64_MIN : b[1] + oy, 0, ng - 1);
    const int64_t nz = clampl(b[2] == INT64_MIN ? INT64_MIN : b[2] + oz, 0, ng - 1);
    return (nx * ng + ny) * ng + nz;
}

/* Binning keys: _node_index of the quadratic base cell (anisompm.py:546-548, 586-590). */
void oracle_bin_keys(const real *x, int64_t n, int32_t ng, double inv_dx, int64_t *keys) {
    const real ivd = (real)inv_dx;
    for (int64_t p = 0; p < n; ++p) {
        int64_t b[3]; real fx[3], w[3][3];
        quad_weights(x + 3 * p, ivd, b, fx, w);
        keys[p] = node_index(b, 0, 0, 0, ng);
    }
}

/* ------------------------------------------------------- constitutive part */
/* Per-particle constitutive + damage + degradation (anisompm.py:614-706).
 * Writes tau (9) and updates F (f_clamp), d, D_hist, diagnostics. */
static void constitutive(const oracle_params *P, oracle_state *S, int64_t p, real tau[9]) {
    real *F = S->F + 9 * p;
    real C[9], lamC[3], V[9];
    mtm3(F, F, C);                                        /* C = F^T F  (615) */
    sym_eig3(C, 5, lamC, V);                              /* (616) */
    real Sv[3];
    for (int i = 0; i < 3; ++i) Sv[i] = sqrt(lamC[i] > R(1e-12) ? lamC[i] : R(1e-12));   /* (617) */
    real W[9], What[9], Rm[9];
    mm3(F, V, W);                                         /* W = F V (619) */
    for (int j = 0; j < 3; ++j) {
        real nrm = sqrt(W[0 * 3 + j] * W[0 * 3 + j] + W[1 * 3 + j] * W[1 * 3 + j] + W[2 * 3 + j] * W[2 * 3 + j]);
        for (int i = 0; i < 3; ++i) What[3 * i + j] = W[3 * i + j] / (nrm + R(1e-12));
    }
    mmt3(What, V, Rm);                                    /* R = What V^T (621) */
    if (P->use_f_clamp) {                                 /* (622-636) */
        real Sc[3], D[9], corr[9];
        const real lo = (real)P->f_clamp_lo, hi = (real)P->f_clamp_hi;
        for (int i = 0; i < 3; ++i) {
            Sc[i] = Sv[i] < lo ? lo : (Sv[i] > hi ? hi : Sv[i]);
            const real sd = Sv[i] > R(1e-12) ? Sv[i] : R(1e-12);
            const real ratio = Sc[i] / sd;
            for (int r = 0; r < 3; ++r) D[3 * r + i] = V[3 * r + i] * ratio;   /* V diag(ratio) */
        }
        mmt3(D, V, corr);
        mm3(F, corr, F);
        for (int i = 0; i < 3; ++i) Sv[i] = Sc[i];
    }
    real J = Sv[0] * Sv[1] * Sv[2];
    if (J < R(1e-6)) J = R(1e-6);                        /* (637) */
    const real mu = S->mu[p], lam = S->lam[p];
    real FmR[9], tau_dev[9];
    for (int i = 0; i < 9; ++i) FmR[i] = (R(2.0) * mu) * (F[i] - Rm[i]);
    mmt3(FmR, F, tau_dev);                                /* 2mu (F-R) F^T (643) */
    const real tv = lam * (J - R(1.0)) * J;               /* (644) */

    if (P->do_damage) {                                   /* (647-685) */
        real sig[9], sigs[9];
        for (int i = 0; i < 9; ++i) sig[i] = (tau_dev[i] + ((i % 4 == 0) ? tv : R(0))) / J;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) sigs[3 * i + j] = R(0.5) * (sig[3 * i + j] + sig[3 * j + i]);
        real ev[3], EV[9], EVD[9], sp[9];
        sym_eig3(sigs, 5, ev, EV);
        for (int j = 0; j < 3; ++j) {
            const real e = ev[j] > R(0) ? ev[j] : R(0);
            for (int i = 0; i < 3; ++i) EVD[3 * i + j] = EV[3 * i + j] * e;
        }
        mmt3(EVD, EV, sp);                                /* sigma+ (654-655) */
        real RA[9], A[9], M[9], MM[9];
        mm3(Rm, S->A0 + 9 * p, RA);
        mmt3(RA, Rm, A);                                  /* A = R A0 R^T (661) */
        mm3(A, sp, M);
        mm3(M, M, MM);
        const real sc = S->sigma_c[p];
        const real phi = (MM[0] + MM[4] + MM[8]) / (sc * sc);   /* (663-664) */
        const real *nI = S->n_interface ? S->n_interface + 3 * p : NULL;
        real phs = R(0);
        if (nI) {                                          /* (670-673) */
            real Sn[3];
            for (int i = 0; i < 3; ++i) Sn[i] = sp[3 * i + 0] * nI[0] + sp[3 * i + 1] * nI[1] + sp[3 * i + 2] * nI[2];
            const real tn = Sn[0] * nI[0] + Sn[1] * nI[1] + Sn[2] * nI[2];
            real tt[3];
            for (int i = 0; i < 3; ++i) tt[i] = Sn[i] - tn * nI[i];
            const real ts = sqrt(tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2]);
            const real q = ts / sc;
            phs = q * q;
        }
        if (S->phi) S->phi[p] = phi;
        if (S->phi_shear) S->phi_shear[p] = phs;
        const real drive = S->zeta[p] * (phi - R(1.0) > R(0) ? phi - R(1.0) : R(0));
        const real Dh = S->D_hist[p] > drive ? S->D_hist[p] : drive;   /* (679) */
        S->D_hist[p] = Dh;
        const real d = S->d[p];
        const real l0 = S->l0[p];
        const real resist = d - (l0 * l0) * S->lap[p];
        real ddot = (R(1.0) - d) * Dh - resist;
        if (ddot < R(0)) ddot = R(0);
        real dn = d + ((real)P->dt_dmg / S->eta[p]) * ddot;
        dn = dn < R(0) ? R(0) : (dn > R(1) ? R(1) : dn);
        if (S->allow[p]) S->d[p] = dn > d ? dn : d;       /* (685) */
    }
    const real d = S->d[p];
    const real res = S->residual[p];
    const real omd = R(1.0) - d;
    const real g = (omd * omd) * (R(1.0) - res) + res;    /* (688) */
    const real vdeg = (J >= R(1.0)) ? g : R(1.0);         /* (690) */
    for (int i = 0; i < 9; ++i) tau[i] = g * tau_dev[i] + ((i % 4 == 0) ? vdeg * tv : R(0));
    if (P->any_interface && S->interface_mask && S->interface_mask[p]) {
        /* directional_kirchhoff(tau_dev+tau_vol, F, d, n, g_dir, g_dir, tension_gate) (190-227, 697-703) */
        const real *n0 = S->n_interface + 3 * p;
        real tc[9];
        for (int i = 0; i < 9; ++i) tc[i] = tau_dev[i] + ((i % 4 == 0) ? tv : R(0));
        real m[3];
        for (int i = 0; i < 3; ++i) m[i] = F[3 * i + 0] * n0[0] + F[3 * i + 1] * n0[1] + F[3 * i + 2] * n0[2];
        const real mn = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) + R(1e-9);
        for (int i = 0; i < 3; ++i) m[i] = m[i] / mn;
        real Pm[9], Qm[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                Pm[3 * i + j] = m[i] * m[j];
                Qm[3 * i + j] = ((i == j) ? R(1) : R(0)) - Pm[3 * i + j];
            }
        real T1[9], perp[9], sh1[9], sh2[9], par[9];
        mm3(Pm, tc, T1); mm3(T1, Pm, perp);
        mm3(T1, Qm, sh1);
        mm3(Qm, tc, T1); mm3(T1, Pm, sh2);
        mm3(T1, Qm, par);
        real gI = g, gII = g;
        real tm[3];
        for (int i = 0; i < 3; ++i) tm[i] = m[0] * tc[0 * 3 + i] + m[1] * tc[1 * 3 + i] + m[2] * tc[2 * 3 + i];
        const real snn = tm[0] * m[0] + tm[1] * m[1] + tm[2] * m[2];
        if (!(snn > R(0))) gI = R(1);
        for (int i = 0; i < 9; ++i) tau[i] = par[i] + gI * perp[i] + gII * (sh1[i] + sh2[i]);
    }
    if (S->tau_last) memcpy(S->tau_last + 9 * p, tau, 9 * sizeof(real));
    if (S->J_last) S->J_last[p] = J;
}

/* ---------------------------------------------------- per-particle scatter */
static inline void p2g_particle(const oracle_params *P, const oracle_state *S, int64_t p, const real *affine,
                                const real *vbc, real *gmv, real *gm, real *gdc, real *gdwc, int quad, int k_only) {
    const int64_t ng = P->n_grid;
    const real ivd = (real)P->inv_dx, dx = (real)P->dx;
    const real m = S->mass[p];
    if (quad) {
        int64_t b[3]; real fx[3], w[3][3];
        quad_weights(S->x + 3 * p, ivd, b, fx, w);
        real mv[3] = {m * vbc[0], m * vbc[1], m * vbc[2]};
        for (int k = 0; k < 27; ++k) {
            if (k_only >= 0 && k != k_only) continue;
            const int ox = k / 9, oy = (k / 3) % 3, oz = k % 3;
            const int64_t idx = node_index(b, ox, oy, oz, ng);
            const real wk = w[ox][0] * w[oy][1] * w[oz][2];
            real dpos[3] = {((real)ox - fx[0]) * dx, ((real)oy - fx[1]) * dx, ((real)oz - fx[2]) * dx};
            for (int i = 0; i < 3; ++i) {
                real ad = affine[3 * i + 0] * dpos[0];
                ad = ad + affine[3 * i + 1] * dpos[1];
                ad = ad + affine[3 * i + 2] * dpos[2];
                gmv[3 * idx + i] += wk * (mv[i] + ad);
            }
            gm[idx] += wk * m;
        }
    } else {
        int64_t b[3]; real w[4][3], w2[4][3];
        cubic_weights(S->x + 3 * p, ivd, b, w, w2);
        const real d = S->d[p];
        for (int k = 0; k < 64; ++k) {
            if (k_only >= 0 && k != k_only) continue;
            const int ox = k / 16, oy = (k / 4) % 4, oz = k % 4;
            const int64_t idx = node_index(b, ox, oy, oz, ng);
            const real wk = w[ox][0] * w[oy][1] * w[oz][2];
            gdc[idx] += wk * d;
            gdwc[idx] += wk;
        }
    }
}

/* ------------------------------------------------------------------ colliders */
/* _resolve (anisompm.py:811-825) applied to one node */
static void resolve(real v[3], const real vcol[3], const real n[3], int sticky, real friction) {
    if (sticky) { v[0] = vcol[0]; v[1] = vcol[1]; v[2] = vcol[2]; return; }
    real vrel[3] = {v[0] - vcol[0], v[1] - vcol[1], v[2] - vcol[2]};
    const real vn = vrel[0] * n[0] + vrel[1] * n[1] + vrel[2] * n[2];
    const real inward = vn < R(0) ? vn : R(0);
    real vt[3] = {vrel[0] - vn * n[0], vrel[1] - vn * n[1], vrel[2] - vn * n[2]};
    if (friction > R(0)) {
        const real vtm = sqrt(vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
        real scale = R(1.0) + friction * inward / (vtm + R(1e-9));
        if (scale < R(0)) scale = R(0);
        for (int i = 0; i < 3; ++i) vt[i] = vt[i] * scale;
    }
    for (int i = 0; i < 3; ++i) v[i] = vcol[i] + vt[i] + (vn - inward) * n[i];
}

static void apply_colliders(const oracle_params *P, int64_t node, real v[3]) {
    const int64_t ng = P->n_grid;
    const real dx = (real)P->dx;
    const real pos[3] = {(real)(node / (ng * ng)) * dx, (real)((node / ng) % ng) * dx, (real)(node % ng) * dx};
    for (int c = 0; c < P->n_colliders; ++c) {
        const double *cd = P->colliders + 16 * c;
        const int kind = (int)cd[0], sticky = (int)cd[1];
        const real fr = (real)cd[2], rad = (real)cd[3];
        const real o[3] = {(real)cd[7], (real)cd[8], (real)cd[9]};
        const real o2[3] = {(real)cd[10], (real)cd[11], (real)cd[12]};
        const real vcol[3] = {(o2[0] - o[0]) / R(1e-4), (o2[1] - o[1]) / R(1e-4), (o2[2] - o[2]) / R(1e-4)};
        if (kind == 0) {   /* halfspace_collider (847-867) */
            const real n[3] = {(real)cd[4], (real)cd[5], (real)cd[6]};
            real sd = (pos[0] - o[0]) * n[0];
            sd = sd + (pos[1] - o[1]) * n[1];
            sd = sd + (pos[2] - o[2]) * n[2];
            if (sd < R(0)) resolve(v, vcol, n, sticky, fr);
        } else {           /* sphere_collider (828-844) */
            const real rel[3] = {pos[0] - o[0], pos[1] - o[1], pos[2] - o[2]};
            const real dist = sqrt(rel[0] * rel[0] + rel[1] * rel[1] + rel[2] * rel[2]);
            if (dist < rad) {
                const real n[3] = {rel[0] / (dist + R(1e-9)), rel[1] / (dist + R(1e-9)), rel[2] / (dist + R(1e-9))};
                resolve(v, vcol, n, sticky, fr);
            }
        }
    }
}

/* -------------------------------------------------------------------- substep */
int oracle_substep(const oracle_params *P, oracle_state *S, oracle_grids *GO) {
    const int64_t n = P->n, ng = P->n_grid, G = ng * ng * ng;
    const real ivd = (real)P->inv_dx, dx = (real)P->dx, dt = (real)P->dt;
    int nth = P->nthreads > 0 ? P->nthreads : 1;
#ifdef _OPENMP
    omp_set_num_threads(nth);
#endif
    real *affine = (real *)malloc(sizeof(real) * 9 * (size_t)(n > 0 ? n : 1));
    real *vbc = (real *)malloc(sizeof(real) * 3 * (size_t)(n > 0 ? n : 1));
    real *gmv = (real *)calloc((size_t)G * 3, sizeof(real));
    real *gm = (real *)calloc((size_t)G, sizeof(real));
    real *gdc = (real *)calloc((size_t)G, sizeof(real));
    real *gdwc = (real *)calloc((size_t)G, sizeof(real));
    if (!affine || !vbc || !gmv || !gm || !gdc || !gdwc) return 1;

    /* particle BCs (601-602) -> velocity used by P2G; constitutive (614-706) */
    {
        const real sc0 = (real)(-P->dt);
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) {
            real tau[9];
            for (int i = 0; i < 3; ++i) vbc[3 * p + i] = S->v[3 * p + i];
            if (P->n_grips > 0 && P->grip_tag && P->grip_tag[p] >= 0) {
                const double *gv = P->grip_vel + 3 * P->grip_tag[p];
                for (int i = 0; i < 3; ++i) vbc[3 * p + i] = (real)gv[i];
            }
            constitutive(P, S, p, tau);
            /* stress_coeff = -dt*vol0*4*inv_dx*inv_dx, affine = coeff*tau + mass*C (711-713) */
            const real coeff = (((sc0 * S->vol0[p]) * R(4.0)) * ivd) * ivd;
            for (int i = 0; i < 9; ++i) affine[9 * p + i] = coeff * tau[i] + S->mass[p] * S->C[9 * p + i];
        }
    }
    /* P2G quadratic momentum (716-724) and cubic damage scatter (768-776) */
    if (P->scatter_mode == 0) {
        for (int k = 0; k < 27; ++k)
            for (int64_t p = 0; p < n; ++p) p2g_particle(P, S, p, affine + 9 * p, vbc + 3 * p, gmv, gm, gdc, gdwc, 1, k);
        for (int k = 0; k < 64; ++k)
            for (int64_t p = 0; p < n; ++p) p2g_particle(P, S, p, affine + 9 * p, vbc + 3 * p, gmv, gm, gdc, gdwc, 0, k);
    } else {
        const int64_t nslab = (ng + 2) / 4 + 1;
        int64_t *cnt = (int64_t *)calloc((size_t)nslab + 1, sizeof(int64_t));
        int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
        int64_t *slab = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
        for (int64_t p = 0; p < n; ++p) {
            int64_t b[3]; real fx[3], w[3][3];
            quad_weights(S->x + 3 * p, ivd, b, fx, w);
            const int64_t s = (clampl(b[0] == INT64_MIN ? -1 : b[0], -1, ng) + 1) / 4;
            slab[p] = s; cnt[s + 1]++;
        }
        for (int64_t s = 0; s < nslab; ++s) cnt[s + 1] += cnt[s];
        int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)nslab);
        memcpy(fill, cnt, sizeof(int64_t) * (size_t)nslab);
        for (int64_t p = 0; p < n; ++p) order[fill[slab[p]]++] = p;
        for (int colour = 0; colour < 2; ++colour) {
#pragma omp parallel for schedule(dynamic, 1)
            for (int64_t s = colour; s < nslab; s += 2)
                for (int64_t i = cnt[s]; i < cnt[s + 1]; ++i) {
                    const int64_t p = order[i];
                    p2g_particle(P, S, p, affine + 9 * p, vbc + 3 * p, gmv, gm, gdc, gdwc, 1, -1);
                    p2g_particle(P, S, p, affine + 9 * p, vbc + 3 * p, gmv, gm, gdc, gdwc, 0, -1);
                }
        }
        free(cnt); free(order); free(slab); free(fill);
    }
    if (GO && GO->grid_mv) memcpy(GO->grid_mv, gmv, sizeof(real) * 3 * (size_t)G);
    if (GO && GO->grid_m) memcpy(GO->grid_m, gm, sizeof(real) * (size_t)G);
    if (GO && GO->grid_dc) memcpy(GO->grid_dc, gdc, sizeof(real) * (size_t)G);
    if (GO && GO->grid_dwc) memcpy(GO->grid_dwc, gdwc, sizeof(real) * (size_t)G);

    /* grid update (727-746) in place: gmv -> grid_v;  damage normalise (777-779): gdc -> gd */
    {
        const real gdt[3] = {dt * (real)P->gravity[0], dt * (real)P->gravity[1], dt * (real)P->gravity[2]};
        const real damp = (real)P->grid_damp;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < G; ++i) {
            const int active = gm[i] > R(1e-12);
            const real inv_m = active ? R(1.0) / gm[i] : R(0);
            real v[3];
            for (int a = 0; a < 3; ++a) {
                v[a] = gmv[3 * i + a] * inv_m + gdt[a];
                if (P->grid_damp != 1.0) v[a] = v[a] * damp;
                if (!active) v[a] = R(0);
            }
            if (active && P->n_colliders > 0) apply_colliders(P, i, v);
            for (int a = 0; a < 3; ++a) gmv[3 * i + a] = v[a];
            gdc[i] = gdwc[i] > R(1e-12) ? gdc[i] / gdwc[i] : R(0);
        }
    }
    if (GO && GO->grid_v) memcpy(GO->grid_v, gmv, sizeof(real) * 3 * (size_t)G);
    if (GO && GO->gd) memcpy(GO->gd, gdc, sizeof(real) * (size_t)G);

    /* G2P (749-760), cubic Laplacian gather (781-791), advection (793-802) */
    {
        const real cfac = (real)(4.0 * P->inv_dx * P->inv_dx);
        const real lfac = (real)(P->inv_dx * P->inv_dx);
        const real pad = (real)(2.0 * P->dx), hi = (real)(P->grid_lim - 2.0 * P->dx);
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) {
            int64_t b[3]; real fx[3], w[3][3];
            real *xp = S->x + 3 * p;
            quad_weights(xp, ivd, b, fx, w);
            real nv[3] = {0, 0, 0}, nC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int k = 0; k < 27; ++k) {
                const int ox = k / 9, oy = (k / 3) % 3, oz = k % 3;
                const int64_t idx = node_index(b, ox, oy, oz, ng);
                const real wk = w[ox][0] * w[oy][1] * w[oz][2];
                const real *gv = gmv + 3 * idx;
                const real dpos[3] = {((real)ox - fx[0]) * dx, ((real)oy - fx[1]) * dx, ((real)oz - fx[2]) * dx};
                for (int i = 0; i < 3; ++i) nv[i] = nv[i] + wk * gv[i];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) nC[3 * i + j] = nC[3 * i + j] + wk * (gv[i] * dpos[j]);
            }
            for (int i = 0; i < 9; ++i) nC[i] = nC[i] * cfac;
            int64_t cb[3]; real cw[4][3], cw2[4][3];
            cubic_weights(xp, ivd, cb, cw, cw2);
            real lap = R(0);
            for (int k = 0; k < 64; ++k) {
                const int ox = k / 16, oy = (k / 4) % 4, oz = k % 4;
                const int64_t idx = node_index(cb, ox, oy, oz, ng);
                const real lw = lfac * (cw2[ox][0] * cw[oy][1] * cw[oz][2] + cw[ox][0] * cw2[oy][1] * cw[oz][2]
                                        + cw[ox][0] * cw[oy][1] * cw2[oz][2]);
                lap = lap + lw * gdc[idx];
            }
            for (int i = 0; i < 3; ++i) S->v[3 * p + i] = nv[i];
            memcpy(S->C + 9 * p, nC, sizeof(nC));
            S->lap[p] = lap;
            for (int i = 0; i < 3; ++i) {
                real xn = xp[i] + dt * nv[i];
                xn = xn < pad ? pad : (xn > hi ? hi : xn);
                xp[i] = xn;
            }
            real A[9];
            for (int i = 0; i < 9; ++i) A[i] = ((i % 4 == 0) ? R(1) : R(0)) + dt * nC[i];
            mm3(A, S->F + 9 * p, S->F + 9 * p);
        }
    }
    free(affine); free(vbc); free(gmv); free(gm); free(gdc); free(gdwc);
    return 0;
}

int oracle_real_bytes(void) { return (int)sizeof(real); }
