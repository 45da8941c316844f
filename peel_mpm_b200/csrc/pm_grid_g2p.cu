// Grid update (active 4^3 blocks only), G2P with the damage Laplacian and
// advection, the per-substep clock, and the standalone batched eigensolver.
#include "pm_kernels.cuh"

namespace pm {

// ------------------------------------------------------------------ clock
// Per-substep reset of a control block's counters and bounds.
__device__ __forceinline__ void reset_ctrl(Ctrl *c, bool shared_counters) {
    c->any_allow = 0;
    c->mom_bound = 0;
    c->mass_bound = 0;
    c->dmg_bound = 0;
    if (shared_counters) {
        c->n_active = 0;
        c->n_work = 0;
        c->work_next = 0;
    }
}

__global__ void k_set_clock(Ctrl *c, const pm_clock clk, int ncol) {
    const int t = threadIdx.x;
    if (t == 0) {
        c->time = clk.time;
        c->step = clk.step;
        reset_ctrl(c, true);
    }
    if (t < ncol) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float o = (float)clk.col_origin[t][a], o2 = (float)clk.col_origin_next[t][a];
            c->col_origin[t][a] = o;
            c->col_vel[t][a] = __fdiv_rn(__fsub_rn(o2, o), 1e-4f);   // (o2 - o) / dt_fd (anisompm.py:838, 862)
        }
    }
}

__global__ void k_set_clock_dev(Ctrl *c, const pm_clock *dev, int row, int ncol) {
    const pm_clock *clk = dev + row;
    const int t = threadIdx.x;
    if (t == 0) {
        c->time = clk->time;
        c->step = clk->step;
        reset_ctrl(c, true);
    }
    if (t < ncol) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float o = (float)clk->col_origin[t][a], o2 = (float)clk->col_origin_next[t][a];
            c->col_origin[t][a] = o;
            c->col_vel[t][a] = __fdiv_rn(__fsub_rn(o2, o), 1e-4f);
        }
    }
}

// Batched clock: block s loads scene s's clock from dev[s]; block 0 also
// resets the shared active-block counter.
__global__ void k_set_clock_b(Ctrl *c, const pm_params *prms, const pm_clock *dev) {
    const int sid = blockIdx.x, t = threadIdx.x;
    const pm_clock *clk = dev + sid;
    Ctrl *cs = c + sid;
    if (t == 0) {
        cs->time = clk->time;
        cs->step = clk->step;
        reset_ctrl(cs, sid == 0);
    }
    if (t < prms[sid].n_colliders) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float o = (float)clk->col_origin[t][a], o2 = (float)clk->col_origin_next[t][a];
            cs->col_origin[t][a] = o;
            cs->col_vel[t][a] = __fdiv_rn(__fsub_rn(o2, o), 1e-4f);
        }
    }
}

void launch_set_clock_batch(const BatchScenes &sc, const WS &w, const pm_clock *dev, cudaStream_t s) {
    k_set_clock_b<<<sc.n, 32, 0, s>>>(w.ctrl, sc.prms, dev);
}

void launch_set_clock(const pm_params &prm, const WS &w, const pm_clock &clk, cudaStream_t s) {
    k_set_clock<<<1, 32, 0, s>>>(w.ctrl, clk, prm.n_colliders);
}
void launch_set_clock_dev(const pm_params &prm, const WS &w, const pm_clock *dev, int row, cudaStream_t s) {
    k_set_clock_dev<<<1, 32, 0, s>>>(w.ctrl, dev, row, prm.n_colliders);
}

// ------------------------------------------------------------ grid update
// One thread per z-row of 4 nodes of an active 4^3 block: the row's scene,
// parameters and node address are resolved once and its 4 nodes' loads are
// independent.  Reads and clears the P2G accumulators, writes grid velocity
// and the normalised damage field (anisompm.py:727-746, 777-779).
template <class SC>
__global__ void __launch_bounds__(256) k_grid(const SC sc, const WS w) {
    const long long nact = min((long long)w.ctrl->n_active, w.n_blocks);
    const long long items = nact * 16;
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        const int gb = w.block_list[it >> 4];
        const int sid = sc.of_gblock(gb);
        const pm_params &prm = sc.params(sid);
        const Ctrl *ctrl = w.ctrl + sid;
        const int ng = prm.n_grid, nbs = (ng + kBlockEdge - 1) / kBlockEdge;
        const int b = (int)(gb - sc.gblock_base(sid));
        const int l = (int)(it & 15);
        const int bx = b / (nbs * nbs), by = (b / nbs) % nbs, bz = b % nbs;
        const int ix = bx * kBlockEdge + (l >> 2), iy = by * kBlockEdge + (l & 3), iz0 = bz * kBlockEdge;
        if (ix >= ng || iy >= ng) continue;
        const int nz = min(kBlockEdge, ng - iz0);
        const long long row = sc.node_base(sid) + ((long long)ix * ng + iy) * ng + iz0;
        // exact fixed-point sums -> float, each rounded once
        const FixScale fm = fix_scale(ctrl->mom_bound), fmm = fix_scale(ctrl->mass_bound),
                       fd = fix_scale(ctrl->dmg_bound), fw = fix_scale(__float_as_uint(1.0f));
        longlong2 qm[kBlockEdge][2], qd[kBlockEdge];
#pragma unroll
        for (int k = 0; k < kBlockEdge; ++k) {
            if (k < nz) {
                const longlong2 *gm = (const longlong2 *)(w.g_mom + 4 * (row + k));
                qm[k][0] = gm[0];
                qm[k][1] = gm[1];
                qd[k] = *(const longlong2 *)(w.g_dmg + 2 * (row + k));
            }
        }
        float4 mom[kBlockEdge];
        float2 dmg[kBlockEdge];
#pragma unroll
        for (int k = 0; k < kBlockEdge; ++k) {
            if (k < nz) {
                mom[k] = make_float4(from_fix(qm[k][0].x, fm.unit), from_fix(qm[k][0].y, fm.unit),
                                     from_fix(qm[k][1].x, fm.unit), from_fix(qm[k][1].y, fmm.unit));
                dmg[k] = make_float2(from_fix(qd[k].x, fd.unit), from_fix(qd[k].y, fw.unit));
            }
        }
        const float dt = (float)prm.dt;
        const float gdt[3] = {dt * (float)prm.gravity[0], dt * (float)prm.gravity[1], dt * (float)prm.gravity[2]};
        const float damp = (float)prm.grid_damp;
        const bool do_damp = prm.grid_damp != 1.0;
        const float dx = (float)prm.dx;
        const int ncol = prm.n_colliders;
#pragma unroll
        for (int k = 0; k < kBlockEdge; ++k) {
            if (k >= nz) continue;
            const long long node = row + k;
            longlong2 *gm = (longlong2 *)(w.g_mom + 4 * node);
            gm[0] = make_longlong2(0, 0);
            gm[1] = make_longlong2(0, 0);
            *(longlong2 *)(w.g_dmg + 2 * node) = make_longlong2(0, 0);
            const bool active = mom[k].w > 1e-12f;
            const float inv_m = active ? 1.0f / mom[k].w : 0.0f;
            // (mv * inv_m) + dt g, each op rounded as the reference's tensor ops (727-733)
            float v[3] = {__fadd_rn(__fmul_rn(mom[k].x, inv_m), gdt[0]), __fadd_rn(__fmul_rn(mom[k].y, inv_m), gdt[1]),
                          __fadd_rn(__fmul_rn(mom[k].z, inv_m), gdt[2])};
            if (do_damp) {
                v[0] *= damp; v[1] *= damp; v[2] *= damp;
            }
            if (!active) v[0] = v[1] = v[2] = 0.0f;
            if (w.g_vpre && ncol > 0) w.g_vpre[node] = make_float4(v[0], v[1], v[2], 0.0f);   // for the adjoint
            if (active && ncol > 0) {
                const float pos[3] = {(float)ix * dx, (float)iy * dx, (float)(iz0 + k) * dx};
                for (int c = 0; c < ncol; ++c) {
                    const pm_collider col = prm.colliders[c];
                    float nn[3];
                    if (collider_hit(col, ctrl->col_origin[c], pos, nn))
                        resolve(v, ctrl->col_vel[c], nn, col.mode == 1, (float)col.friction);
                }
            }
            w.g_vel[node] = make_float4(v[0], v[1], v[2], mom[k].w);   // .w: node mass (read by the adjoint)
            w.g_gd[node] = dmg[k].y > 1e-12f ? dmg[k].x / dmg[k].y : 0.0f;
            if (w.g_sw) w.g_sw[node] = dmg[k].y;
        }
    }
}

template <class SC>
void launch_grid(const SC &sc, const WS &w, cudaStream_t s, int ctas_per_sm) {
    const long long max_items = w.n_blocks * 16;
    // a batch has many more active nodes than one scene and every row starts
    // with a dependent chain of table loads (scene lookup, parameters): by
    // default give each row its own thread rather than a grid-stride loop;
    // ctas_per_sm (the tunable) sets the grid-stride cap instead
    const long long cap = ctas_per_sm > 0 ? 148LL * ctas_per_sm : (SC::batched ? 148LL * 64 : 148LL * 8);
    const int blocks = (int)std::max<long long>(1, std::min<long long>((max_items + 255) / 256, cap));
    k_grid<SC><<<blocks, 256, 0, s>>>(sc, w);
}
template void launch_grid<PlainScenes>(const PlainScenes &, const WS &, cudaStream_t, int);
template void launch_grid<BatchScenes>(const BatchScenes &, const WS &, cudaStream_t, int);

// Accumulators as floats {mv, m} and {sum w d, sum w} (inspection of a
// substep between P2G and the grid update; no effect on the state).
__global__ void k_grid_sums(const WS w, long long n_nodes, float4 *mom, float2 *dmg) {
    const Ctrl *ctrl = w.ctrl;
    const FixScale fm = fix_scale(ctrl->mom_bound), fmm = fix_scale(ctrl->mass_bound),
                   fd = fix_scale(ctrl->dmg_bound), fw = fix_scale(__float_as_uint(1.0f));
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes;
         i += (long long)gridDim.x * blockDim.x) {
        const long long *g = w.g_mom + 4 * i, *h = w.g_dmg + 2 * i;
        mom[i] = make_float4(from_fix(g[0], fm.unit), from_fix(g[1], fm.unit), from_fix(g[2], fm.unit),
                             from_fix(g[3], fmm.unit));
        dmg[i] = make_float2(from_fix(h[0], fd.unit), from_fix(h[1], fw.unit));
    }
}

void launch_grid_sums(const WS &w, long long n_nodes, float *mom, float *dmg, cudaStream_t s) {
    const int blocks = (int)std::max<long long>(1, std::min<long long>((n_nodes + 255) / 256, 148LL * 16));
    k_grid_sums<<<blocks, 256, 0, s>>>(w, n_nodes, (float4 *)mom, (float2 *)dmg);
}

// --------------------------------------------------------------------- G2P
// One CTA per 256 particles in particle order (coalesced state reads and
// writes; inputs built from lattices or meshes are spatially coherent in that
// order).  The CTA first stages its grid footprint in shared memory:
// velocities of the quadratic nodes [lo, hi+2] and the damage field of the
// cubic nodes [lo-1, hi+3] of its base cells' bounding box [lo, hi]
// (coalesced along z).  Then one thread per
// particle gathers from shared memory: quadratic gather of grid velocity (APIC
// v and C), cubic gather of the damage Laplacian at the start-of-step
// position, then x += dt v, F <- (I + dt C) F, x clamped to [2dx, lim-2dx]
// (anisompm.py:749-760, 781-803).  A footprint larger than the staging
// buffers (incoherent particle order), or a particle whose stencil needs the
// reference's edge clamping, gathers from global memory instead.
constexpr int kGTQ = 1200;   // staged quadratic nodes (float4)
constexpr int kGTC = 2400;   // staged cubic nodes (float)

template <bool TILE>
__device__ __forceinline__ void g2p_particle(const pm_params &prm, const Parts &P, const float4 *gvel,
                                             const float *ggd, unsigned *nonfinite, long long p, const float xp[3],
                                             const int lo[3], const int qd[3], const int cd[3],
                                             const float4 *sq, const float *sc) {
    const long long ps = P.ps;
    const int ng = prm.n_grid;
    const float inv_dx = (float)prm.inv_dx, dx = (float)prm.dx, dt = (float)prm.dt;
    // Cubic Laplacian gather first (anisompm.py:781-791; only lap stays live
    // across the quadratic gather): for each (x, y) column
    // A = sum_z wz gd and B = sum_z w''z gd; per x, SA = sum_y wy A,
    // SA2 = sum_y w''y A, SB = sum_y wy B; then
    // lap = sum_x w''x SA + wx (SA2 + SB).
    float lap = 0.0f;
    {
        Cubic c;
        cubic_weights(xp, inv_dx, ng, c);
        int NX[4], NY[4], NZ[4];
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            if (TILE) {
                NX[o] = (c.b[0] + o - lo[0] + 1) * cd[1] * cd[2];
                NY[o] = (c.b[1] + o - lo[1] + 1) * cd[2];
                NZ[o] = c.b[2] + o - lo[2] + 1;
            } else {
                NX[o] = clampi(c.b[0] + o, 0, ng - 1) * ng * ng;
                NY[o] = clampi(c.b[1] + o, 0, ng - 1) * ng;
                NZ[o] = clampi(c.b[2] + o, 0, ng - 1);
            }
        }
#pragma unroll
        for (int ox = 0; ox < 4; ++ox) {
            float SA = 0.0f, SA2 = 0.0f, SB = 0.0f;
#pragma unroll
            for (int oy = 0; oy < 4; ++oy) {
                float A = 0.0f, B = 0.0f;
#pragma unroll
                for (int oz = 0; oz < 4; ++oz) {
                    const int node = NX[ox] + NY[oy] + NZ[oz];
                    const float gd = TILE ? sc[node] : __ldg(&ggd[node]);
                    A += c.w[oz][2] * gd;
                    B += c.w2[oz][2] * gd;
                }
                SA += c.w[oy][1] * A;
                SA2 += c.w2[oy][1] * A;
                SB += c.w[oy][1] * B;
            }
            lap += c.w2[ox][0] * SA + c.w[ox][0] * (SA2 + SB);
        }
        lap *= (float)(prm.inv_dx * prm.inv_dx);
    }
    // Quadratic gather (anisompm.py:749-760) as a contraction over z, then y,
    // then x: with dpos_j = (o_j - fx_j) dx,
    //   Z0[x,y] = sum_z wz g,  Zd[x,y] = sum_z (wz DZ) g         (per column)
    //   T[x] = sum_y wy Z0,  Ty[x] = sum_y (wy DY) Z0,  Tz[x] = sum_y wy Zd
    //   v = sum_x wx T,  C_.x = sum_x (wx DX) T,  C_.y = sum_x wx Ty,  C_.z = sum_x wx Tz
    // so every node costs 6 FMAs and one float4 load, every column 9 more.
    float nv[3] = {0.0f, 0.0f, 0.0f}, nC[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) nC[k] = 0.0f;
    {
        Quad q;
        quad_weights(xp, inv_dx, ng, q);
        int NX[3], NY[3], NZ[3];
        float wzd[3], wyd[3], wxd[3];
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            if (TILE) {
                NX[o] = (q.b[0] + o - lo[0]) * qd[1] * qd[2];
                NY[o] = (q.b[1] + o - lo[1]) * qd[2];
                NZ[o] = q.b[2] + o - lo[2];
            } else {
                NX[o] = clampi(q.b[0] + o, 0, ng - 1) * ng * ng;
                NY[o] = clampi(q.b[1] + o, 0, ng - 1) * ng;
                NZ[o] = clampi(q.b[2] + o, 0, ng - 1);
            }
            wxd[o] = q.w[o][0] * (((float)o - q.fx[0]) * dx);
            wyd[o] = q.w[o][1] * (((float)o - q.fx[1]) * dx);
            wzd[o] = q.w[o][2] * (((float)o - q.fx[2]) * dx);
        }
#pragma unroll
        for (int ox = 0; ox < 3; ++ox) {
            float T[3] = {0.0f, 0.0f, 0.0f}, Ty[3] = {0.0f, 0.0f, 0.0f}, Tz[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
                float Z0[3] = {0.0f, 0.0f, 0.0f}, Zd[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int oz = 0; oz < 3; ++oz) {
                    const int node = NX[ox] + NY[oy] + NZ[oz];
                    const float4 g = TILE ? sq[node] : __ldg(&gvel[node]);
                    const float wz = q.w[oz][2], wd = wzd[oz];
                    Z0[0] += wz * g.x; Z0[1] += wz * g.y; Z0[2] += wz * g.z;
                    Zd[0] += wd * g.x; Zd[1] += wd * g.y; Zd[2] += wd * g.z;
                }
                const float wy = q.w[oy][1], wd = wyd[oy];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    T[i] += wy * Z0[i];
                    Ty[i] += wd * Z0[i];
                    Tz[i] += wy * Zd[i];
                }
            }
            const float wx = q.w[ox][0], wd = wxd[ox];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                nv[i] += wx * T[i];
                nC[3 * i] += wd * T[i];
                nC[3 * i + 1] += wx * Ty[i];
                nC[3 * i + 2] += wx * Tz[i];
            }
        }
        const float cfac = (float)(4.0 * prm.inv_dx * prm.inv_dx);
#pragma unroll
        for (int k = 0; k < 9; ++k) nC[k] *= cfac;
    }
    // advection, F update, domain clamp (793-802).  These accumulate over every
    // substep, so each multiply and add is rounded separately as in the
    // reference's tensor ops (x + dt v, (I + dt C) F), without FMA contraction.
    const float pad = (float)(2.0 * prm.dx), hi = (float)(prm.grid_lim - 2.0 * prm.dx);
    float xn[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float t = __fadd_rn(xp[a], __fmul_rn(dt, nv[a]));
        t = t < pad ? pad : t;
        xn[a] = t > hi ? hi : t;
    }
    float F[9], Fn[9], A[9];   // F is loaded after the gathers: fewer registers live across them
    const float *Fin = prm.use_f_clamp ? P.Fo : P.F;   // the constitutive update wrote the clamped F there
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = Fin[k * ps + p];
#pragma unroll
    for (int k = 0; k < 9; ++k) A[k] = __fadd_rn((k % 4 == 0) ? 1.0f : 0.0f, __fmul_rn(dt, nC[k]));
    mm3_rn(A, F, Fn);
    bool finite = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) finite = finite && isfinite(xn[a]);
#pragma unroll
    for (int k = 0; k < 9; ++k) finite = finite && isfinite(Fn[k]);
    if (!finite) atomicAdd(nonfinite, 1u);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        P.xo[a * ps + p] = xn[a];
        P.vo[a * ps + p] = nv[a];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        P.Fo[k * ps + p] = Fn[k];
        P.Co[k * ps + p] = nC[k];
    }
    P.lapo[p] = lap;
}

// MINB: resident CTAs per SM the registers are budgeted for (3: 80 registers;
// 4: 64 registers with a few spills), a tunable.
template <class SC, int MINB>
__global__ void __launch_bounds__(kG2PThreads, MINB) k_g2p(const SC scn, const Parts P, const WS w) {
    __shared__ float4 sq[kGTQ];
    __shared__ float sc[kGTC];
    __shared__ int s_box[6];
    const int tid = threadIdx.x;
    // particle order: state reads and writes are coalesced; a CTA never spans scenes
    const int sid = scn.of_cta(blockIdx.x);
    const pm_params &prm = scn.params(sid);
    const long long p = scn.p_begin(sid) + ((long long)blockIdx.x - scn.cta_base(sid)) * kG2PThreads + tid;
    const bool valid = p < scn.p_end(sid, P.n);
    const float4 *gvel = w.g_vel + scn.node_base(sid);
    const float *ggd = w.g_gd + scn.node_base(sid);
    const int ng = prm.n_grid;
    const long long ps = P.ps;
    const float inv_dx = (float)prm.inv_dx;
    float xp[3] = {0.0f, 0.0f, 0.0f};
    int qb[3] = {0, 0, 0};
    bool reg = valid;
    if (valid) {
#pragma unroll
        for (int a = 0; a < 3; ++a) xp[a] = P.x[a * ps + p];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float fb = floorf(__fsub_rn(__fmul_rn(xp[a], inv_dx), 0.5f));
            reg = reg && (fb >= 1.0f) && (fb <= (float)(ng - 4));
            qb[a] = reg ? (int)fb : 0;
        }
    }
    // bounding box of the regular particles' base cells
    int cl[3], ch[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        cl[a] = reg ? qb[a] : 0x7fffffff;
        ch[a] = reg ? qb[a] : -0x7fffffff;
    }
    if (tid < 6) s_box[tid] = tid < 3 ? 0x7fffffff : -0x7fffffff;
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int mn = __reduce_min_sync(0xffffffffu, cl[a]), mx = __reduce_max_sync(0xffffffffu, ch[a]);
        if ((tid & 31) == 0) {
            atomicMin(&s_box[a], mn);
            atomicMax(&s_box[3 + a], mx);
        }
    }
    __syncthreads();
    const int lo[3] = {s_box[0], s_box[1], s_box[2]};
    const bool any = s_box[3] >= lo[0];
    const int qd[3] = {s_box[3] - lo[0] + 3, s_box[4] - lo[1] + 3, s_box[5] - lo[2] + 3};
    const int cd[3] = {qd[0] + 2, qd[1] + 2, qd[2] + 2};
    const long long qn = any ? (long long)qd[0] * qd[1] * qd[2] : 0, cn = any ? (long long)cd[0] * cd[1] * cd[2] : 0;
    const bool tile = any && qn <= kGTQ && cn <= kGTC;
    if (tile) {   // regular nodes lie inside the grid, so no bounds test is needed
        const FastDiv qyz = make_fastdiv(qd[1] * qd[2]), qz = make_fastdiv(qd[2]);
        for (int i = tid; i < qn; i += kG2PThreads) {
            const int ix = fdiv(i, qyz), r = i - ix * qyz.d, iy = fdiv(r, qz);
            const int gx = lo[0] + ix, gy = lo[1] + iy, gz = lo[2] + r - iy * qz.d;
            sq[i] = gvel[((long long)gx * ng + gy) * ng + gz];
        }
        const FastDiv cyz = make_fastdiv(cd[1] * cd[2]), cz = make_fastdiv(cd[2]);
        for (int i = tid; i < cn; i += kG2PThreads) {
            const int ix = fdiv(i, cyz), r = i - ix * cyz.d, iy = fdiv(r, cz);
            const int gx = lo[0] - 1 + ix, gy = lo[1] - 1 + iy, gz = lo[2] - 1 + r - iy * cz.d;
            sc[i] = ggd[((long long)gx * ng + gy) * ng + gz];
        }
    }
    __syncthreads();
    if (!valid) return;
    if (reg && tile)
        g2p_particle<true>(prm, P, gvel, ggd, &w.ctrl[sid].nonfinite, p, xp, lo, qd, cd, sq, sc);
    else
        g2p_particle<false>(prm, P, gvel, ggd, &w.ctrl[sid].nonfinite, p, xp, lo, qd, cd, sq, sc);
}

// n_ctas: CTAs over all scenes (each scene's particles start a new CTA); the
// plain form derives it from P.n.
template <class SC>
void launch_g2p(const SC &sc, const Parts &P, const WS &w, cudaStream_t s, long long n_ctas, int ctas_per_sm) {
    const long long blocks = n_ctas >= 0 ? n_ctas : (P.n + kG2PThreads - 1) / kG2PThreads;
    if (blocks <= 0) return;
    // 0: the default build (4 per SM for one scene; 3 for a batch, whose scene
    // lookups need more registers)
    const int minb = ctas_per_sm > 0 ? ctas_per_sm : (SC::batched ? 3 : 4);
    if (minb >= 4)
        k_g2p<SC, 4><<<(unsigned)blocks, kG2PThreads, 0, s>>>(sc, P, w);
    else
        k_g2p<SC, 3><<<(unsigned)blocks, kG2PThreads, 0, s>>>(sc, P, w);
}
template void launch_g2p<PlainScenes>(const PlainScenes &, const Parts &, const WS &, cudaStream_t, long long, int);
template void launch_g2p<BatchScenes>(const BatchScenes &, const Parts &, const WS &, cudaStream_t, long long, int);

// ---------------------------------------------------------------- sym_eig
__global__ void __launch_bounds__(256) k_sym_eig(const float *__restrict__ A, long long n, int sweeps,
                                                 float *__restrict__ ev, float *__restrict__ V) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float a[9], e[3], vv[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = A[9 * p + k];
    if (sweeps == 5)
        sym_eig3<5>(a, e, vv);           // the substep's count, unrolled
    else
        sym_eig3<0>(a, e, vv, sweeps);   // any other count >= 0
#pragma unroll
    for (int k = 0; k < 3; ++k) ev[3 * p + k] = e[k];
#pragma unroll
    for (int k = 0; k < 9; ++k) V[9 * p + k] = vv[k];
}

void launch_sym_eig(const float *A, long long n, int sweeps, float *ev, float *V, cudaStream_t s) {
    if (n <= 0) return;
    k_sym_eig<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A, n, sweeps, ev, V);
}

}  // namespace pm
