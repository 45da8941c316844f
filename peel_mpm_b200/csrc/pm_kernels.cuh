// Launchers shared between the kernel files and the C ABI layer.
#pragma once

#include <algorithm>

#include "pm_common.cuh"

namespace pm {

template <class SC> void launch_keys(const SC &sc, const WS &w, const Parts &P, cudaStream_t s);
// hist0_ready: the first pass's tile histogram was written by launch_keys
// (the substep path), so the sort starts at that pass's column scan.
void launch_sort(const WS &w, long long n, cudaStream_t s, int *inv = nullptr, bool hist0_ready = false);
void launch_compact(const WS &w, cudaStream_t s);
void prepare_p2g();
void prepare_sort();
void prepare_adjoint();
void launch_keys_only(const float *x, long long n, long long ps, int ng, float inv_dx, bool blocked, const WS &w,
                      cudaStream_t s);
template <class SC>
void launch_p2g(const SC &sc, const Parts &P, const WS &w, cudaStream_t s, int ctas_per_sm = 0, int stress_ctas = 0);
template <class SC> void launch_grid(const SC &sc, const WS &w, cudaStream_t s, int ctas_per_sm = 0);
void launch_grid_sums(const WS &w, long long n_nodes, float *mom, float *dmg, cudaStream_t s);
template <class SC>
void launch_g2p(const SC &sc, const Parts &P, const WS &w, cudaStream_t s, long long n_ctas = -1, int ctas_per_sm = 0);
void launch_set_clock(const pm_params &prm, const WS &w, const pm_clock &clk, cudaStream_t s);
void launch_set_clock_dev(const pm_params &prm, const WS &w, const pm_clock *dev, int row, cudaStream_t s);
void launch_set_clock_batch(const BatchScenes &sc, const WS &w, const pm_clock *dev, cudaStream_t s);
int balanced_range(long long n, int slots, int max_range);
int resident_slots(const void *kernel, int threads, size_t smem);
void launch_sym_eig(const float *A, long long n, int sweeps, float *ev, float *V, cudaStream_t s);

// Tape of recorded substeps for the adjoint: a header per slot, the
// adjoint's control block, its int64 fixed-point scatter grid, two float
// adjoint grids and its sorted-order payload, shared by all slots; then per
// slot {v, m} grid, gd, cubic weight sums, the active block list, the sort of
// the substep (sorted keys, each particle's sorted position, the sub-block
// work list), the particles' APIC affine term and their polar decomposition
// (R, V, S) and damage drive phi.
struct TapeLayout {
    size_t head, actl, acc, adj_q, adj_c, apay, slot0, vel, gd, sw, vpre, blocks, keys, iperm, work, aff, pol,
        slot_bytes, total;
    long long n_blocks, aff_stride;
    int slots, flags;
};
TapeLayout make_tape_layout(long long n, int ng, int slots, int flags);
void record_redirect(const TapeLayout &T, void *tape, int slot, WS &w);
void launch_tape_head(const TapeLayout &T, void *tape, int slot, const WS &w, long long n, cudaStream_t s);
void launch_adjoint(const pm_params &prm, const Parts &pre, const Parts &post, const pm_state_adj &ain,
                    const pm_state_adj &aout, const pm_param_adj &grads, const TapeLayout &T, void *tape, int slot,
                    cudaStream_t s);

// Per-frame observables (pm_observe.cu): values per group per frame row.
constexpr int kObsValues = 8;   // phi max, phi_shear max, d sum, d max, n(d > thr), count, y sum, unused
int launch_observe(const Parts &P, const int8_t *group, int n_groups, float thr, float *row, float *phi_pp,
                   float *psh_pp, int *status, int onset_group, float onset_frac, int frame, float *snap_d,
                   float *snap_x, long long snap_stride, cudaStream_t s);

// Gaussian-splat renderer (pm_render.cu).
size_t render_workspace_bytes(long long n, int width, int height, int r_max);
void launch_render(const pm_camera &cam, const pm_render_params &rp, const float *xyz, const float *cov,
                   const float *color, long long n, float *img, void *ws, cudaStream_t s);
void launch_carry(const Parts &P, const int *bind, const float *off0, const float *cov0, const float *color0,
                  long long g_n, const float *affine, float tint, float *pos, float *cov, float *color,
                  cudaStream_t s);

// Argument checks and error reporting of the C ABI (pm_capi.cu), shared with
// the other entry-point files.
int report_error(int code, const char *msg);
int api_check_device();
int api_check_params(const pm_params *prm);
int api_check_particles(const pm_particles *P, bool need_all);
int api_cuda_check(const char *where);

}  // namespace pm
