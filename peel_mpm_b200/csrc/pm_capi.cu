// C ABI of the AnisoMPM substep (declarations in include/peelmpm.h).
// Validates arguments, carves the caller's workspace and enqueues kernels;
// never allocates and never synchronises (except pm_read_status).
#include <cstdio>
#include <cstring>
#include <string>

#include "pm_kernels.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const char *msg) {
    g_err = msg;
    return code;
}

int cuda_check(const char *where) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return PM_OK;
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s: %s", where, cudaGetErrorString(e));
    g_err = buf;
    return PM_ERR_CUDA;
}

// Device must be compute capability 10.x (the binary carries sm_100a code only).
int check_device() {
    static int ok_dev[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return fail(PM_ERR_CUDA, "no CUDA device");
    if (ok_dev[dev] == 1) return PM_OK;
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return fail(PM_ERR_UNSUPPORTED, "peelmpm kernels are built for sm_100a only");
    ok_dev[dev] = 1;
    return PM_OK;
}

int check_params(const pm_params *prm) {
    if (!prm) return fail(PM_ERR_ARG, "params is NULL");
    if (prm->n_grid < 4 || prm->n_grid > 1024) return fail(PM_ERR_ARG, "n_grid must be in [4, 1024]");
    if (prm->damage_every < 1) return fail(PM_ERR_ARG, "damage_every must be >= 1");
    if (prm->n_grips < 0 || prm->n_grips > PM_MAX_GRIPS) return fail(PM_ERR_ARG, "too many grips");
    if (prm->n_colliders < 0 || prm->n_colliders > PM_MAX_COLLIDERS) return fail(PM_ERR_ARG, "too many colliders");
    if (prm->p2g_ctas_per_sm < 0 || prm->p2g_ctas_per_sm > 8) return fail(PM_ERR_ARG, "p2g_ctas_per_sm must be in [0, 8]");
    if (prm->grid_ctas_per_sm < 0 || prm->grid_ctas_per_sm > 64)
        return fail(PM_ERR_ARG, "grid_ctas_per_sm must be in [0, 64]");
    if (prm->stress_ctas_per_sm != 0 && prm->stress_ctas_per_sm != 3 && prm->stress_ctas_per_sm != 4)
        return fail(PM_ERR_ARG, "stress_ctas_per_sm must be 0, 3 or 4");
    if (prm->g2p_ctas_per_sm != 0 && prm->g2p_ctas_per_sm != 3 && prm->g2p_ctas_per_sm != 4)
        return fail(PM_ERR_ARG, "g2p_ctas_per_sm must be 0, 3 or 4");
    if (!(prm->dx > 0.0) || !(prm->inv_dx > 0.0)) return fail(PM_ERR_ARG, "dx must be positive");
    return PM_OK;
}

int check_particles(const pm_particles *P, bool need_all) {
    if (!P) return fail(PM_ERR_ARG, "particles is NULL");
    if (P->n < 0 || P->n >= (1LL << 31)) return fail(PM_ERR_ARG, "particle count must be in [0, 2^31)");
    if (P->plane_stride < P->n) return fail(PM_ERR_ARG, "plane_stride < n");
    if (!P->x) return fail(PM_ERR_ARG, "x is NULL");
    if (need_all) {
        if (!P->v || !P->F || !P->C || !P->d || !P->lap || !P->D_hist || !P->vol0 || !P->mass || !P->mu ||
            !P->lam || !P->sigma_c || !P->eta || !P->zeta || !P->l0 || !P->residual || !P->A0 || !P->allow)
            return fail(PM_ERR_ARG, "a required particle array is NULL");
        if (P->interface_mask && !P->n_interface) return fail(PM_ERR_ARG, "interface_mask needs n_interface");
    }
    return PM_OK;
}

int get_ws(void *ws, size_t bytes, long long n, int ng, pm::WS *out) {
    if (!ws) return fail(PM_ERR_WORKSPACE, "workspace is NULL");
    if (((uintptr_t)ws & 255) != 0) return fail(PM_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    const pm::Layout L = pm::make_layout(n, ng);
    if (bytes < L.total) return fail(PM_ERR_WORKSPACE, "workspace too small for (n, n_grid)");
    *out = pm::make_ws(ws, L);
    return PM_OK;
}

}  // namespace

namespace pm {
// Lets other translation units of the library report through pm_last_error().
int report_error(int code, const char *msg) { return fail(code, msg); }
int api_check_device() { return check_device(); }
int api_check_params(const pm_params *prm) { return check_params(prm); }
int api_check_particles(const pm_particles *P, bool need_all) { return check_particles(P, need_all); }
int api_cuda_check(const char *where) { return cuda_check(where); }
}  // namespace pm

extern "C" {

int pm_abi_version(void) { return PM_ABI_VERSION; }

const char *pm_last_error(void) { return g_err.c_str(); }

size_t pm_struct_size(int32_t which) {
    switch (which) {
        case 0: return sizeof(pm_params);
        case 1: return sizeof(pm_particles);
        case 2: return sizeof(pm_clock);
        case 3: return sizeof(pm_status_info);
        case 4: return sizeof(pm_ws_layout);
        case 5: return sizeof(pm_grip);
        case 6: return sizeof(pm_collider);
        case 7: return sizeof(pm_batch_layout);
        case 8: return sizeof(pm_state_adj);
        case 9: return sizeof(pm_param_adj);
        case 10: return sizeof(pm_camera);
        case 11: return sizeof(pm_render_params);
        default: return 0;
    }
}

int pm_prepare(void) {
    int rc = check_device();
    if (rc) return rc;
    pm::prepare_p2g();
    pm::prepare_sort();
    pm::prepare_adjoint();
    return cuda_check("pm_prepare");
}

int pm_workspace_size(int64_t n, int32_t n_grid, size_t *bytes) {
    if (!bytes) return fail(PM_ERR_ARG, "bytes is NULL");
    if (n < 0 || n_grid < 4 || n_grid > 1024) return fail(PM_ERR_ARG, "bad n or n_grid");
    *bytes = pm::make_layout(n, n_grid).total;
    return PM_OK;
}

int pm_workspace_layout(int64_t n, int32_t n_grid, pm_ws_layout *out) {
    if (!out) return fail(PM_ERR_ARG, "out is NULL");
    if (n < 0 || n_grid < 4 || n_grid > 1024) return fail(PM_ERR_ARG, "bad n or n_grid");
    const pm::Layout L = pm::make_layout(n, n_grid);
    out->ctrl = L.ctrl; out->keys_a = L.keys_a; out->keys_b = L.keys_b; out->vals_a = L.vals_a;
    out->vals_b = L.vals_b; out->hist = L.hist; out->block_mask = L.block_mask; out->block_list = L.block_list;
    out->g_mom = L.g_mom; out->g_dmg = L.g_dmg; out->g_vel = L.g_vel; out->g_gd = L.g_gd;
    out->payload = L.payload; out->inv_perm = L.inv_perm; out->work = L.work; out->total = L.total;
    out->sort_passes = L.passes;
    out->n_tiles = L.n_tiles;
    return PM_OK;
}

int pm_grid_sums(const void *ws, size_t ws_bytes, int64_t n, int32_t n_grid, float *mom, float *dmg, void *stream) {
    int rc;
    if ((rc = check_device())) return rc;
    if (!mom || !dmg) return fail(PM_ERR_ARG, "mom or dmg is NULL");
    pm::WS w;
    if ((rc = get_ws(const_cast<void *>(ws), ws_bytes, n, n_grid, &w))) return rc;
    pm::launch_grid_sums(w, (long long)n_grid * n_grid * n_grid, mom, dmg, (cudaStream_t)stream);
    return cuda_check("pm_grid_sums");
}

int pm_workspace_init(void *ws, size_t ws_bytes, int64_t n, int32_t n_grid, void *stream) {
    int rc = check_device();
    if (rc) return rc;
    pm::WS w;
    if ((rc = get_ws(ws, ws_bytes, n, n_grid, &w))) return rc;
    const pm::Layout L = pm::make_layout(n, n_grid);
    if (cudaMemsetAsync(ws, 0, L.total, (cudaStream_t)stream) != cudaSuccess) return cuda_check("pm_workspace_init");
    return cuda_check("pm_workspace_init");
}

int pm_set_clock(const pm_params *prm, void *ws, size_t ws_bytes, int64_t n, const pm_clock *clk, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_params(prm))) return rc;
    if (!clk) return fail(PM_ERR_ARG, "clock is NULL");
    pm::WS w;
    if ((rc = get_ws(ws, ws_bytes, n, prm->n_grid, &w))) return rc;
    pm::launch_set_clock(*prm, w, *clk, (cudaStream_t)stream);
    return cuda_check("pm_set_clock");
}

int pm_bin(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_params(prm)) || (rc = check_particles(P, false))) return rc;
    pm::WS w;
    if ((rc = get_ws(ws, ws_bytes, P->n, prm->n_grid, &w))) return rc;
    const pm::Parts parts = pm::make_parts(P);
    cudaStream_t s = (cudaStream_t)stream;
    pm::launch_keys(pm::PlainScenes{*prm}, w, parts, s);
    pm::launch_sort(w, P->n, s, w.inv_perm, true);
    return cuda_check("pm_bin");
}

int pm_p2g(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_params(prm)) || (rc = check_particles(P, true))) return rc;
    pm::WS w;
    if ((rc = get_ws(ws, ws_bytes, P->n, prm->n_grid, &w))) return rc;
    pm::launch_p2g(pm::PlainScenes{*prm}, pm::make_parts(P), w, (cudaStream_t)stream, prm->p2g_ctas_per_sm, prm->stress_ctas_per_sm);
    pm::launch_compact(w, (cudaStream_t)stream);
    return cuda_check("pm_p2g");
}

int pm_grid_update(const pm_params *prm, void *ws, size_t ws_bytes, int64_t n, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_params(prm))) return rc;
    pm::WS w;
    if ((rc = get_ws(ws, ws_bytes, n, prm->n_grid, &w))) return rc;
    pm::launch_grid(pm::PlainScenes{*prm}, w, (cudaStream_t)stream, prm->grid_ctas_per_sm);
    return cuda_check("pm_grid_update");
}

int pm_g2p(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_params(prm)) || (rc = check_particles(P, true))) return rc;
    pm::WS w;
    if ((rc = get_ws(ws, ws_bytes, P->n, prm->n_grid, &w))) return rc;
    pm::launch_g2p(pm::PlainScenes{*prm}, pm::make_parts(P), w, (cudaStream_t)stream, -1, prm->g2p_ctas_per_sm);
    return cuda_check("pm_g2p");
}

static int substep_common(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes,
                          const pm_clock *clk, const pm_clock *dev_clocks, int32_t row, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_params(prm)) || (rc = check_particles(P, true))) return rc;
    pm::WS w;
    if ((rc = get_ws(ws, ws_bytes, P->n, prm->n_grid, &w))) return rc;
    const pm::Parts parts = pm::make_parts(P);
    cudaStream_t s = (cudaStream_t)stream;
    if (clk)
        pm::launch_set_clock(*prm, w, *clk, s);
    else
        pm::launch_set_clock_dev(*prm, w, dev_clocks, row, s);
    if (P->n > 0) {
        const pm::PlainScenes sc{*prm};
        pm::launch_keys(sc, w, parts, s);
        pm::launch_sort(w, P->n, s, w.inv_perm, true);
        pm::launch_p2g(sc, parts, w, s, prm->p2g_ctas_per_sm, prm->stress_ctas_per_sm);
        pm::launch_compact(w, s);
        pm::launch_grid(sc, w, s, prm->grid_ctas_per_sm);
        pm::launch_g2p(sc, parts, w, s, -1, prm->g2p_ctas_per_sm);
    }
    return cuda_check("pm_substep");
}

int pm_substep(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes, const pm_clock *clk,
               void *stream) {
    if (!clk) return fail(PM_ERR_ARG, "clock is NULL");
    return substep_common(prm, P, ws, ws_bytes, clk, nullptr, 0, stream);
}

int pm_substep_dev_clock(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes,
                         const pm_clock *dev_clocks, int32_t row, void *stream) {
    if (!dev_clocks || row < 0) return fail(PM_ERR_ARG, "bad device clock table");
    return substep_common(prm, P, ws, ws_bytes, nullptr, dev_clocks, row, stream);
}

// ------------------------------------------------------------------ adjoint
static int get_tape(void *tape, size_t bytes, long long n, int ng, int slots, int flags, int slot,
                    pm::TapeLayout *T) {
    if (!tape) return fail(PM_ERR_WORKSPACE, "tape is NULL");
    if (((uintptr_t)tape & 255) != 0) return fail(PM_ERR_WORKSPACE, "tape must be 256-byte aligned");
    if (slots < 1 || slot < 0 || slot >= slots) return fail(PM_ERR_ARG, "bad tape slot");
    *T = pm::make_tape_layout(n, ng, slots, flags);
    if (bytes < T->total) return fail(PM_ERR_WORKSPACE, "tape too small for (n, n_grid, slots, flags)");
    return PM_OK;
}

static int tape_flags(const pm_params *prm) { return prm->n_colliders > 0 ? PM_TAPE_COLLIDERS : 0; }

int pm_tape_size(int64_t n, int32_t n_grid, int32_t slots, int32_t flags, size_t *bytes) {
    if (!bytes) return fail(PM_ERR_ARG, "bytes is NULL");
    if (n < 0 || n_grid < 4 || n_grid > 1024 || slots < 1) return fail(PM_ERR_ARG, "bad n, n_grid or slots");
    if (flags & ~PM_TAPE_COLLIDERS) return fail(PM_ERR_ARG, "unknown tape flags");
    *bytes = pm::make_tape_layout(n, n_grid, slots, flags).total;
    return PM_OK;
}

int pm_tape_init(void *tape, size_t tape_bytes, int64_t n, int32_t n_grid, int32_t slots, int32_t flags,
                 void *stream) {
    int rc;
    if ((rc = check_device())) return rc;
    if (n < 0 || n_grid < 4 || n_grid > 1024) return fail(PM_ERR_ARG, "bad n or n_grid");
    if (flags & ~PM_TAPE_COLLIDERS) return fail(PM_ERR_ARG, "unknown tape flags");
    pm::TapeLayout T;
    if ((rc = get_tape(tape, tape_bytes, n, n_grid, slots, flags, 0, &T))) return rc;
    if (cudaMemsetAsync(tape, 0, T.total, (cudaStream_t)stream) != cudaSuccess) return cuda_check("pm_tape_init");
    return cuda_check("pm_tape_init");
}

int pm_substep_record(const pm_params *prm, const pm_particles *P, const pm_particles *out, void *ws, size_t ws_bytes,
                      const pm_clock *clk, void *tape, size_t tape_bytes, int32_t slots, int32_t slot, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_params(prm)) || (rc = check_particles(P, true))) return rc;
    if (!clk) return fail(PM_ERR_ARG, "clock is NULL");
    if (out) {
        if (out->n != P->n || out->plane_stride != P->plane_stride)
            return fail(PM_ERR_ARG, "out differs from P in n or plane_stride");
        if (!out->x || !out->v || !out->F || !out->C || !out->d || !out->lap || !out->D_hist)
            return fail(PM_ERR_ARG, "an out state plane is NULL");
        if (out->x == P->x || out->F == P->F || out->d == P->d)
            return fail(PM_ERR_ARG, "out must not alias P's state (pass NULL to advance in place)");
    }
    pm::WS w;
    if ((rc = get_ws(ws, ws_bytes, P->n, prm->n_grid, &w))) return rc;
    pm::TapeLayout T;
    if ((rc = get_tape(tape, tape_bytes, P->n, prm->n_grid, slots, tape_flags(prm), slot, &T))) return rc;
    pm::record_redirect(T, tape, slot, w);
    const pm::Parts parts = out ? pm::make_parts_out(P, out) : pm::make_parts(P);
    cudaStream_t s = (cudaStream_t)stream;
    pm::launch_set_clock(*prm, w, *clk, s);
    if (P->n > 0) {
        const pm::PlainScenes sc{*prm};
        pm::launch_keys(sc, w, parts, s);
        pm::launch_sort(w, P->n, s, w.inv_perm, true);
        pm::launch_p2g(sc, parts, w, s, prm->p2g_ctas_per_sm, prm->stress_ctas_per_sm);
        pm::launch_compact(w, s);
        pm::launch_grid(sc, w, s, prm->grid_ctas_per_sm);
        pm::launch_g2p(sc, parts, w, s, -1, prm->g2p_ctas_per_sm);
    }
    pm::launch_tape_head(T, tape, slot, w, P->n, s);
    return cuda_check("pm_substep_record");
}

static int check_adj(const pm_state_adj *a, long long n) {
    if (!a) return fail(PM_ERR_ARG, "adjoint state is NULL");
    if (a->plane_stride < n) return fail(PM_ERR_ARG, "adjoint plane_stride < n");
    if (!a->x || !a->v || !a->F || !a->C || !a->d || !a->lap || !a->D_hist)
        return fail(PM_ERR_ARG, "an adjoint state plane is NULL");
    return PM_OK;
}

int pm_substep_adjoint(const pm_params *prm, const pm_particles *pre, const pm_particles *post,
                       const pm_state_adj *adj_in, const pm_state_adj *adj_out, const pm_param_adj *grads,
                       void *tape, size_t tape_bytes, int32_t slots, int32_t slot, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_params(prm)) || (rc = check_particles(pre, true)) ||
        (rc = check_particles(post, true)))
        return rc;
    if (pre->n != post->n) return fail(PM_ERR_ARG, "pre and post differ in n");
    if ((rc = check_adj(adj_in, pre->n)) || (rc = check_adj(adj_out, pre->n))) return rc;
    if (adj_in->x == adj_out->x) return fail(PM_ERR_ARG, "adj_in and adj_out must be distinct");
    if (!grads || (grads->A0 && grads->plane_stride < pre->n)) return fail(PM_ERR_ARG, "bad parameter gradients");
    pm::TapeLayout T;
    if ((rc = get_tape(tape, tape_bytes, pre->n, prm->n_grid, slots, tape_flags(prm), slot, &T))) return rc;
    pm::launch_adjoint(*prm, pm::make_parts(pre), pm::make_parts(post), *adj_in, *adj_out, *grads, T, tape, slot,
                       (cudaStream_t)stream);
    return cuda_check("pm_substep_adjoint");
}

int pm_observe(const pm_particles *P, const int8_t *group, int32_t n_groups, float d_threshold, float *row,
               float *phi_peak, float *phi_shear_peak, int32_t *status, int32_t onset_group, float onset_fraction,
               int32_t frame, float *snap_d, float *snap_x, int64_t snap_stride, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_particles(P, false))) return rc;
    if (!P->d) return fail(PM_ERR_ARG, "d is NULL");
    if (n_groups < 1 || n_groups > PM_OBS_MAX_GROUPS) return fail(PM_ERR_ARG, "n_groups must be in [1, 8]");
    if (!row || !status) return fail(PM_ERR_ARG, "row or status is NULL");
    if (onset_group >= n_groups) return fail(PM_ERR_ARG, "onset_group out of range");
    if (snap_x && snap_stride < P->n) return fail(PM_ERR_ARG, "snap_stride < n");
    pm::launch_observe(pm::make_parts(P), group, n_groups, d_threshold, row, phi_peak, phi_shear_peak, status,
                       onset_group, onset_fraction, frame, snap_d, snap_x, snap_stride, (cudaStream_t)stream);
    return cuda_check("pm_observe");
}

// ------------------------------------------------------------------ renderer
int pm_render_workspace_size(int64_t n, int32_t width, int32_t height, int32_t r_max, size_t *bytes) {
    if (!bytes) return fail(PM_ERR_ARG, "bytes is NULL");
    if (n < 0 || n >= (1LL << 31) || width < 1 || height < 1 || (int64_t)width * height > (1LL << 30))
        return fail(PM_ERR_ARG, "bad n, width or height");
    if (r_max < 1 || r_max > 1024) return fail(PM_ERR_ARG, "r_max must be in [1, 1024]");
    *bytes = pm::render_workspace_bytes(n, width, height, r_max);
    return PM_OK;
}

int pm_render_gaussians(const pm_camera *cam, const pm_render_params *rp, const float *xyz, const float *cov3d,
                        const float *color, int64_t n, float *image, void *ws, size_t ws_bytes, void *stream) {
    int rc;
    if ((rc = check_device())) return rc;
    if (!cam || !rp || !image) return fail(PM_ERR_ARG, "camera, parameters or image is NULL");
    if (n > 0 && (!xyz || !cov3d || !color)) return fail(PM_ERR_ARG, "NULL gaussian array");
    size_t need = 0;
    if ((rc = pm_render_workspace_size(n, cam->width, cam->height, rp->r_max, &need))) return rc;
    if (!ws || ((uintptr_t)ws & 255) != 0 || ws_bytes < need)
        return fail(PM_ERR_WORKSPACE, "render workspace missing, misaligned or too small");
    pm::launch_render(*cam, *rp, xyz, cov3d, color, n, image, ws, (cudaStream_t)stream);
    return cuda_check("pm_render_gaussians");
}

int pm_carry_gaussians(const pm_particles *P, const int32_t *bind, const float *off0, const float *cov0,
                       const float *color0, int64_t g_n, const float *affine, float crack_tint, float *pos, float *cov,
                       float *color, void *stream) {
    int rc;
    if ((rc = check_device()) || (rc = check_particles(P, false))) return rc;
    if (!P->F || (crack_tint > 0.0f && !P->d)) return fail(PM_ERR_ARG, "F (and d for the crack tint) required");
    if (g_n < 0) return fail(PM_ERR_ARG, "g_n < 0");
    if (g_n > 0 && (!bind || !off0 || !cov0 || !color0 || !affine || !pos || !cov || !color))
        return fail(PM_ERR_ARG, "NULL array");
    pm::launch_carry(pm::make_parts(P), bind, off0, cov0, color0, g_n, affine, crack_tint, pos, cov, color,
                     (cudaStream_t)stream);
    return cuda_check("pm_carry_gaussians");
}

int pm_read_status(const void *ws, size_t ws_bytes, int64_t n, int32_t n_grid, pm_status_info *out, void *stream) {
    int rc;
    if ((rc = check_device())) return rc;
    if (!out) return fail(PM_ERR_ARG, "out is NULL");
    pm::WS w;
    if ((rc = get_ws(const_cast<void *>(ws), ws_bytes, n, n_grid, &w))) return rc;
    pm::Ctrl c;
    if (cudaMemcpyAsync(&c, w.ctrl, sizeof c, cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess ||
        cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
        return cuda_check("pm_read_status");
    out->nonfinite = c.nonfinite;
    out->dense_subblocks = c.dense_subblocks;
    out->n_active_blocks = c.n_active;
    out->any_allow = c.any_allow;
    return PM_OK;
}

int pm_sym_eig(const float *A, int64_t n, int32_t sweeps, float *evals, float *evecs, void *stream) {
    int rc;
    if ((rc = check_device())) return rc;
    if (n < 0) return fail(PM_ERR_ARG, "n < 0");
    if (n > 0 && (!A || !evals || !evecs)) return fail(PM_ERR_ARG, "NULL array");
    if (sweeps < 0) return fail(PM_ERR_ARG, "sweeps must be >= 0");
    pm::launch_sym_eig(A, n, sweeps, evals, evecs, (cudaStream_t)stream);
    return cuda_check("pm_sym_eig");
}

int pm_bin_workspace_size(int64_t n, int32_t n_grid, size_t *bytes) {
    if (!bytes) return fail(PM_ERR_ARG, "bytes is NULL");
    if (n < 0 || n_grid < 4 || n_grid > 1024) return fail(PM_ERR_ARG, "bad n or n_grid");
    *bytes = pm::make_layout(n, n_grid).block_mask;   // control block, keys, ids and histograms come first
    return PM_OK;
}

int pm_bin_sort(const float *x, int64_t n, int64_t plane_stride, int32_t n_grid, double inv_dx, uint32_t *keys_out,
                int32_t *perm_out, void *ws, size_t ws_bytes, void *stream) {
    int rc;
    if ((rc = check_device())) return rc;
    if (n < 0 || plane_stride < n || n_grid < 4 || n_grid > 1024 || !(inv_dx > 0.0))
        return fail(PM_ERR_ARG, "bad size argument");
    if (n > 0 && (!x || !keys_out || !perm_out)) return fail(PM_ERR_ARG, "NULL array");
    if (!ws) return fail(PM_ERR_WORKSPACE, "workspace is NULL");
    if (((uintptr_t)ws & 255) != 0) return fail(PM_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    const pm::Layout L = pm::make_layout(n, n_grid);
    if (ws_bytes < L.block_mask) return fail(PM_ERR_WORKSPACE, "workspace smaller than pm_bin_workspace_size");
    const pm::WS w = pm::make_ws(ws, L);   // only the sort buffers are touched
    if (n == 0) return PM_OK;
    cudaStream_t s = (cudaStream_t)stream;
    pm::launch_keys_only(x, n, plane_stride, n_grid, (float)inv_dx, false, w, s);
    pm::launch_sort(w, n, s);
    if (cudaMemcpyAsync(keys_out, w.sorted_keys, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(perm_out, w.perm, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return cuda_check("pm_bin_sort");
    return cuda_check("pm_bin_sort");
}

}  // extern "C"
