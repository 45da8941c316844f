/*
 * peelmpm.h -- C ABI of the B200 (sm_100a) AnisoMPM substep.
 *
 * Plain pointers and sizes only.  Every entry point:
 *   - returns PM_OK (0) or a pm_status code; pm_last_error() describes the
 *     last failure on the calling thread;
 *   - enqueues work on the given CUDA stream (a cudaStream_t passed as
 *     void*) and never allocates device memory: the caller provides every
 *     buffer, including the workspace; entry points not marked
 *     "synchronises" never synchronise and can be captured in a CUDA graph;
 *   - reads and writes particle state in place.
 *
 * Particle state is structure-of-arrays: a field with c components is c
 * planes of `plane_stride` floats, component k of particle p at
 * ptr[k * plane_stride + p].  Matrices (F, C, A0, tau_last) are 9 planes in
 * row-major component order (k = 3*i + j).  This is the layout a
 * reference-shaped (N,3) / (N,3,3) tensor view with strides (1, stride) /
 * (1, 3*stride, stride) aliases.
 *
 * Reference: anisompm_py/src/anisompm.py (class AnisoMPM).  The comment on
 * each function names the reference code it replaces.
 */
#ifndef PEELMPM_H
#define PEELMPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PM_ABI_VERSION 2
#define PM_MAX_GRIPS 32
#define PM_MAX_COLLIDERS 8

typedef enum pm_status {
    PM_OK = 0,
    PM_ERR_ARG = 1,          /* bad size, null required pointer, unsupported option */
    PM_ERR_CUDA = 2,         /* a launch failed (pm_last_error has cudaGetErrorString) */
    PM_ERR_WORKSPACE = 3,    /* workspace too small or not initialised for (n, n_grid) */
    PM_ERR_UNSUPPORTED = 4   /* device is not sm_100 */
} pm_status;

/* Particle grip: particles tagged g get v = vel * min(t / ramp, 1) before P2G
 * (ramp <= 0: no ramp).  Device form of the particle_bc hook
 * (anisompm.py:601-602; idiom of test_block.py:109-113, peel_test.py:233-236). */
typedef struct pm_grip {
    double vel[3];
    double ramp;
} pm_grip;

/* Grid collider (anisompm.py:811-867).  kind 0 = half-space (normal = unit
 * outward normal of the material side), 1 = sphere (radius).  mode 0 = slip,
 * 1 = sticky.  Origins are per-substep inputs (pm_clock). */
typedef struct pm_collider {
    int32_t kind;
    int32_t mode;
    double friction;
    double radius;
    double normal[3];
} pm_collider;

/* Static solver parameters (AnisoMPM.__init__, anisompm.py:304-347). */
typedef struct pm_params {
    int32_t n_grid;
    int32_t damage_every;
    double grid_lim;
    double dx;
    double inv_dx;
    double dt;
    double gravity[3];
    double grid_damp;
    int32_t use_f_clamp;
    int32_t record_stress;      /* write tau_last / J_last diagnostics */
    double f_clamp_lo;
    double f_clamp_hi;
    int32_t n_grips;
    int32_t n_colliders;
    int32_t p2g_ctas_per_sm;    /* resident P2G CTAs per SM (0: the 80-register build, as many as fit;
                                   4 or more: the 64-register build at 4 per SM; 1..3: a cap); a
                                   tuning knob with no effect on results (the grid sums are exact) */
    int32_t grid_ctas_per_sm;   /* grid-update CTAs per SM (0: the library default, else 1..64); a
                                   tuning knob with no effect on results */
    int32_t stress_ctas_per_sm; /* resident constitutive-update CTAs per SM: 0 or 3 (the 80-register
                                   build), 4 (the 64-register build); a tuning knob with no effect on
                                   results */
    int32_t g2p_ctas_per_sm;    /* resident G2P CTAs per SM: 0 (the library default: 4 for one scene,
                                   3 for a batch), 3 (the 80-register build) or 4 (the 64-register
                                   build); a tuning knob with no effect on results */
    pm_grip grips[PM_MAX_GRIPS];
    pm_collider colliders[PM_MAX_COLLIDERS];
} pm_params;

/* Per-substep inputs: time, step counter (_step) and collider origins at t and
 * t + 1e-4 (the collider velocity is their forward difference, as in
 * sphere_collider / halfspace_collider). */
typedef struct pm_clock {
    double time;
    int64_t step;
    double col_origin[PM_MAX_COLLIDERS][3];
    double col_origin_next[PM_MAX_COLLIDERS][3];
} pm_clock;

/* Particle arrays (device pointers), state of add_object/_append
 * (anisompm.py:374-463). */
typedef struct pm_particles {
    int64_t n;
    int64_t plane_stride;            /* >= n */
    /* mutable state */
    float *x, *v, *F, *C;            /* 3, 3, 9, 9 planes */
    float *d, *lap, *D_hist;
    /* material, read-only during a substep */
    const float *vol0, *mass, *mu, *lam, *sigma_c, *eta, *zeta, *l0, *residual;
    const float *A0;                 /* 9 planes */
    const uint8_t *allow;            /* damage allowed (bool) */
    /* optional (NULL = absent) */
    const float *n_interface;        /* 3 planes; needed for phi_shear */
    const uint8_t *interface_mask;   /* directional stress particles */
    const int8_t *grip_tag;          /* grip index or -1 */
    float *phi, *phi_shear;          /* written on damage steps */
    float *tau_last;                 /* 9 planes, written when record_stress */
    float *J_last;
} pm_particles;

/* Device-side status counters (a copy is read back by pm_read_status). */
typedef struct pm_status_info {
    uint32_t nonfinite;              /* particles whose new x or F is not finite (sticky) */
    uint32_t dense_subblocks;        /* 4^3-cell sub-blocks of more than 16,383 particles: their grid
                                        nodes may exceed the exact fixed-point sums' headroom */
    uint32_t n_active_blocks;        /* active 4^3 grid blocks in the last substep */
    int32_t any_allow;               /* allow.any() seen by the last substep */
} pm_status_info;

/* ---------------------------------------------------------------- queries */
int pm_abi_version(void);
const char *pm_last_error(void);

/* sizeof the ABI structs, for binding checks: 0 pm_params, 1 pm_particles,
 * 2 pm_clock, 3 pm_status_info, 4 pm_ws_layout, 5 pm_grip, 6 pm_collider,
 * 7 pm_batch_layout, 8 pm_state_adj, 9 pm_param_adj, 10 pm_camera, 11 pm_render_params. */
size_t pm_struct_size(int32_t which);

/* One-time set-up of the current device (kernel attributes).  Every entry
 * point does it on first use; call it before capturing pm_* calls into a CUDA
 * graph, since attribute changes are not stream operations. */
int pm_prepare(void);

/* Workspace for n particles on an n_grid^3 grid: grids, sort buffers, block
 * lists and the control block.  Must be zeroed once by pm_workspace_init. */
int pm_workspace_size(int64_t n, int32_t n_grid, size_t *bytes);
int pm_workspace_init(void *ws, size_t ws_bytes, int64_t n, int32_t n_grid, void *stream);

/* Byte offsets of the workspace's views (for inspection and tests).  g_mom
 * and g_dmg hold int64 fixed-point sums (4 and 2 per node) whose units are
 * fixed per substep from the particles' bounds; pm_grid_sums converts them. */
typedef struct pm_ws_layout {
    size_t ctrl, keys_a, keys_b, vals_a, vals_b, hist, block_mask, block_list;
    size_t g_mom, g_dmg, g_vel, g_gd, payload, inv_perm, work, total;
    int32_t sort_passes;             /* sorted keys/perm end in *_a if even, *_b if odd */
    int32_t n_tiles;
} pm_ws_layout;
int pm_workspace_layout(int64_t n, int32_t n_grid, pm_ws_layout *out);

/* The P2G accumulators of a plain workspace as floats, between pm_p2g and
 * pm_grid_update: mom (n_grid^3, 4) {m v, m} and dmg (n_grid^3, 2)
 * {sum w d, sum w} (anisompm.py:716-724, 771-776).  For inspection; the
 * substep itself never needs it. */
int pm_grid_sums(const void *ws, size_t ws_bytes, int64_t n, int32_t n_grid, float *mom, float *dmg, void *stream);

/* ------------------------------------------------------------ the substep */

/* Whole substep: clock, binning, P2G, grid update, G2P.
 * Replaces AnisoMPM.substep(time) (anisompm.py:593-803). */
int pm_substep(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes,
               const pm_clock *clk, void *stream);

/* Same, reading the clock from row `row` of a device array of pm_clock (so a
 * captured graph replays with new times).  Replaces one iteration of
 * AnisoMPM.run_frame (anisompm.py:805-807). */
int pm_substep_dev_clock(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes,
                         const pm_clock *dev_clocks, int32_t row, void *stream);

/* The pieces of pm_substep, in order.  Each needs the previous ones of the
 * same substep to have been enqueued. */
int pm_set_clock(const pm_params *prm, void *ws, size_t ws_bytes, int64_t n, const pm_clock *clk,
                 void *stream);
/* Binning of the substep: the quadratic base cell of every particle
 * (anisompm.py:544-548), numbered block-major (8^3-cell blocks, x-major;
 * a bijection of _node_index, anisompm.py:586-590), stable LSD radix sort of
 * (key, particle id), and the active 4^3 grid blocks.  No reference
 * counterpart: the reference scatters in particle order. */
int pm_bin(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes, void *stream);
/* Particle BCs, constitutive update, damage update, degradation, quadratic
 * P2G and cubic damage scatter (anisompm.py:601-724, 768-776). */
int pm_p2g(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes, void *stream);
/* Grid velocity update with gravity, damping, mask, colliders, and damage
 * field normalisation (anisompm.py:727-746, 777-779). */
int pm_grid_update(const pm_params *prm, void *ws, size_t ws_bytes, int64_t n, void *stream);
/* Quadratic G2P (APIC), cubic damage Laplacian gather, advection, F update,
 * domain clamp (anisompm.py:749-760, 781-803). */
int pm_g2p(const pm_params *prm, const pm_particles *P, void *ws, size_t ws_bytes, void *stream);

/* Copies the status counters to host memory (synchronises `stream`). */
int pm_read_status(const void *ws, size_t ws_bytes, int64_t n, int32_t n_grid, pm_status_info *out,
                   void *stream);

/* ---------------------------------------------------------------- adjoint */

/* Reverse mode of the plain substep for gradients of a loss on the final
 * state with respect to per-particle parameters and the initial state.  The
 * reference gets these from PyTorch autograd through substep()
 * (anisompm.py:593-803); here the caller records each forward substep of a
 * checkpoint segment into a tape slot and then runs pm_substep_adjoint from
 * the last slot to the first.  Every part of the substep is differentiated:
 * grips, gravity, grid damping, damage_every, f_clamp, grid colliders (the
 * tape then needs PM_TAPE_COLLIDERS) and interface particles. */

/* Adjoints of the mutable state, same plane layout as pm_particles. */
typedef struct pm_state_adj {
    int64_t plane_stride;
    float *x, *v, *F, *C;            /* 3, 3, 9, 9 planes */
    float *d, *lap, *D_hist;
} pm_state_adj;

/* Per-particle parameter gradients, accumulated (+=) by every adjoint
 * substep; a NULL plane is skipped. */
typedef struct pm_param_adj {
    int64_t plane_stride;
    float *mu, *lam, *sigma_c;
    float *A0;                       /* 9 planes */
} pm_param_adj;

/* Tape for `slots` recorded substeps of n particles on an n_grid^3 grid:
 * per slot 24 bytes per grid node and 124 bytes per particle, plus three
 * shared adjoint grids (48 bytes per node).  flags: PM_TAPE_COLLIDERS when the
 * recorded substeps have grid colliders (each slot then also keeps the grid
 * velocity before the colliders, 16 bytes per node); pm_substep_record and
 * pm_substep_adjoint derive the layout from their pm_params and reject a
 * tape sized without it.  Zeroed once by pm_tape_init. */
#define PM_TAPE_COLLIDERS 1
int pm_tape_size(int64_t n, int32_t n_grid, int32_t slots, int32_t flags, size_t *bytes);
int pm_tape_init(void *tape, size_t tape_bytes, int64_t n, int32_t n_grid, int32_t slots, int32_t flags,
                 void *stream);

/* pm_substep that also records the substep's grid state into tape slot
 * `slot`.  out == NULL: the particle state P advances in place as in
 * pm_substep.  Otherwise the updated state (x, v, F, C, d, lap, D_hist) is
 * written to out's planes (same n and plane_stride, planes disjoint from P's)
 * and P's state is left as it was: a recorded segment keeps every substep's
 * state without copying it. */
int pm_substep_record(const pm_params *prm, const pm_particles *P, const pm_particles *out, void *ws, size_t ws_bytes,
                      const pm_clock *clk, void *tape, size_t tape_bytes, int32_t slots, int32_t slot, void *stream);

/* Adjoint of the substep recorded in `slot`: pre is the state before it and
 * post the state after it (same material planes), adj_in the adjoint of the
 * post state, adj_out (distinct from adj_in) receives the adjoint of the pre
 * state, and grads accumulates the parameter gradients. */
int pm_substep_adjoint(const pm_params *prm, const pm_particles *pre, const pm_particles *post,
                       const pm_state_adj *adj_in, const pm_state_adj *adj_out, const pm_param_adj *grads,
                       void *tape, size_t tape_bytes, int32_t slots, int32_t slot, void *stream);

/* ---------------------------------------------------------------- batches */

/* Many independent scenes advanced by one set of launches per substep.  The
 * scenes' particles are concatenated (scene s owns particles
 * [sum n[<s], sum n[<=s]) of one pm_particles whose n is the total); each
 * scene keeps its own grid (n_grid from its pm_params), parameters, grips,
 * colliders, clock and damage cadence.  The scene parameters and the packing
 * tables are stored in the workspace by pm_batch_workspace_init (and
 * pm_batch_set_params), so pm_batch_substep reads no host data besides the
 * (n, n_grid) arrays that size its launches, which must equal those the
 * workspace was initialised for (the library keeps a host record per
 * workspace and returns PM_ERR_WORKSPACE otherwise).
 * Replaces a Python loop over many AnisoMPM objects calling run_frame
 * (anisompm.py:805-807) one scene at a time; the reference has no batch API. */
#define PM_MAX_BATCH_SCENES 4096

typedef struct pm_batch_layout {
    pm_ws_layout ws;                 /* ctrl holds one control block per scene */
    size_t params;                   /* pm_params[n_scenes] */
    size_t tables;                   /* int64 particle / node / sort-block / grid-block / CTA prefix tables */
    int64_t n_total, n_nodes, n_grid_blocks, n_sort_blocks, n_g2p_ctas;
} pm_batch_layout;

int pm_batch_workspace_size(int32_t n_scenes, const int64_t *n, const int32_t *n_grid, size_t *bytes);
int pm_batch_workspace_layout(int32_t n_scenes, const int64_t *n, const int32_t *n_grid, pm_batch_layout *out);

/* Zeroes the workspace and stores the scene tables and prms[n_scenes] (host
 * array).  Synchronises `stream`; not capturable. */
int pm_batch_workspace_init(void *ws, size_t ws_bytes, int32_t n_scenes, const int64_t *n, const pm_params *prms,
                            void *stream);
/* Replaces the stored parameters (same n and n_grid).  Synchronises `stream`. */
int pm_batch_set_params(void *ws, size_t ws_bytes, int32_t n_scenes, const int64_t *n, const pm_params *prms,
                        void *stream);
/* Forgets the host record of a workspace that is about to be freed. */
int pm_batch_workspace_release(const void *ws);

/* One substep of every scene: scene s reads its clock from dev_clocks[s]
 * (device memory, n_scenes consecutive pm_clock), so a graph captured over
 * rows of a device clock table replays with new times. */
int pm_batch_substep(int32_t n_scenes, const int64_t *n, const int32_t *n_grid, const pm_particles *P, void *ws,
                     size_t ws_bytes, const pm_clock *dev_clocks, void *stream);

/* Status counters of every scene into out[n_scenes] (n_active_blocks is the
 * batch total).  Synchronises `stream`. */
int pm_batch_read_status(const void *ws, size_t ws_bytes, int32_t n_scenes, const int64_t *n, const int32_t *n_grid,
                         pm_status_info *out, void *stream);

/* ---------------------------------------------------------------- observables */

/* Per-frame reductions of the reference's experiment loop (peel_test.py:263-307)
 * on the device, without a host synchronisation per frame.  Particles carry a
 * group id (group[p] in [0, n_groups), -1 = none; group NULL = all in group 0).
 * For each group g, row[g * PM_OBS_VALUES + k] accumulates (row zeroed by the
 * caller; one row per frame): k = 0 max phi, 1 max phi_shear, 2 sum of d,
 * 3 max d, 4 count of d > d_threshold, 5 count, 6 sum of y.  phi_peak /
 * phi_shear_peak (NULL to skip) keep per-particle running maxima.  status[1]
 * counts particles with non-finite x or d; status[0] (initialise to -1)
 * becomes the first frame whose group `onset_group` has a broken fraction
 * (k4 / k5) above onset_fraction, and at that frame d and x are copied to
 * snap_d / snap_x (3 planes of snap_stride; NULL to skip). */
#define PM_OBS_MAX_GROUPS 8
#define PM_OBS_VALUES 8
int pm_observe(const pm_particles *P, const int8_t *group, int32_t n_groups, float d_threshold, float *row,
               float *phi_peak, float *phi_shear_peak, int32_t *status, int32_t onset_group, float onset_fraction,
               int32_t frame, float *snap_d, float *snap_x, int64_t snap_stride, void *stream);

/* ---------------------------------------------------------------- renderer */

/* Gaussian-splat renderer of the reference's orange demo (render.py:71-162),
 * as CUDA kernels writing a headless (height, width, 3) float image in
 * [0, 1].  Camera: X_cam = X_world R + T (row vectors; the 3DGS convention of
 * Camera.world_to_cam), pinhole fx, fy, principal point at the image centre. */
typedef struct pm_camera {
    float R[9];                      /* row-major */
    float T[3];
    float fx, fy;
    int32_t width, height;
} pm_camera;

typedef struct pm_render_params {
    float bg[3];                     /* background colour */
    float scale_modifier;
    int32_t r_max;                   /* footprint radius cap in pixels */
    float tau;                       /* soft z-buffer depth scale; <= 0: 0.02 x median depth of the drawn splats */
    float near;                      /* splats with camera depth <= near are dropped */
    float max_raw_radius;            /* splats whose unclamped radius reaches this are dropped */
} pm_render_params;

/* Workspace of pm_render_gaussians for n gaussians, a width x height image and
 * footprint radii up to r_max (1..1024): per gaussian the projected splat and
 * the depth key, per 8x8 screen tile the list of splats whose footprint square
 * touches it (capacity n x (2 r_max / 8 + 2)^2 ids, at most the tile count). */
int pm_render_workspace_size(int64_t n, int32_t width, int32_t height, int32_t r_max, size_t *bytes);
/* xyz (n,3), cov3d (n,3,3) row-major, color (n,3): device float arrays.  The
 * reference's per-splat opacity does not enter its compositing, so it is not
 * an argument. */
int pm_render_gaussians(const pm_camera *cam, const pm_render_params *rp, const float *xyz, const float *cov3d,
                        const float *color, int64_t n, float *image, void *ws, size_t ws_bytes, void *stream);

/* Gaussian carrying (run_orange.py:116-133): gaussian i, bound to particle
 * bind[i] (device int32; an out-of-range id gives NaN outputs), gets position
 * affine (x) + F off0_i, covariance F cov0_i F^T and colour
 * color0_i (1 - crack_tint d) from its particle's current state; affine is a
 * device 3x4 row-major [A | t] (the demo's sim-to-world map); off0 (n,3),
 * cov0 (n,3,3), color0 (n,3), outputs pos (n,3), cov (n,3,3), color (n,3). */
int pm_carry_gaussians(const pm_particles *P, const int32_t *bind, const float *off0, const float *cov0,
                       const float *color0, int64_t g_n, const float *affine, float crack_tint, float *pos, float *cov,
                       float *color, void *stream);

/* ---------------------------------------------------------------- helpers */

/* Batched 3x3 symmetric eigendecomposition by cyclic Jacobi with `sweeps`
 * sweeps (the reference's default is 5; any count >= 0, 0 sorting the
 * symmetrised diagonal), A (n,3,3) row-major contiguous -> ascending evals
 * (n,3), eigenvector columns evecs (n,3,3).  Replaces sym_eig
 * (anisompm.py:48-95). */
int pm_sym_eig(const float *A, int64_t n, int32_t sweeps, float *evals, float *evecs, void *stream);

/* Binning only, in the reference's own numbering: keys_out = the sorted
 * _node_index of every particle's quadratic base cell (anisompm.py:544-548,
 * 586-590) and perm_out = the stable argsort of those keys, for positions x
 * (3 planes of stride `plane_stride`).  Uses the sort buffers at the start of
 * a substep workspace, so ws_bytes need only be pm_bin_workspace_size(n,
 * n_grid) (a full pm_workspace_size workspace also serves); keys_out /
 * perm_out must not alias the workspace. */
int pm_bin_workspace_size(int64_t n, int32_t n_grid, size_t *bytes);
int pm_bin_sort(const float *x, int64_t n, int64_t plane_stride, int32_t n_grid, double inv_dx,
                uint32_t *keys_out, int32_t *perm_out, void *ws, size_t ws_bytes, void *stream);

/* Binning exactly as pm_bin_sort, for callers that cannot allocate device
 * memory: a host application that owns every device allocation and hands a
 * plugin only its input and output buffers, or code that must not call
 * cudaMalloc/cudaFree (which can synchronise the whole device) in a
 * latency-bound loop.  The sort's scratch is a static array inside this
 * library (PM_BIN_STATIC_SCRATCH_BYTES on every GPU that loads it, held until
 * the process exits), so the caller passes only x, keys_out and perm_out.
 * n above PM_BIN_STATIC_MAX_N returns PM_ERR_ARG.  The first call on a device
 * looks up the array's device address; make it before any stream capture.
 * All calls share the array: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised by the caller.
 * No counterpart in the reference, which has no binning and never allocates
 * outside PyTorch. */
#define PM_BIN_STATIC_MAX_N 262144
#define PM_BIN_STATIC_SCRATCH_BYTES (16u * PM_BIN_STATIC_MAX_N + 4u * (512u * (PM_BIN_STATIC_MAX_N / 4096u) + 512u))
int pm_bin_sort_static(const float *x, int64_t n, int64_t plane_stride, int32_t n_grid, double inv_dx,
                       uint32_t *keys_out, int32_t *perm_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PEELMPM_H */
