// Per-frame observable reductions on the device, the step after the substep in
// the reference's experiment harness (peel_test.py:263-307): per particle
// group the peak damage drive phi and shear drive phi_shear, mean and max
// damage, the fraction of particles with d above a threshold, the mean height
// (y) of the group, the per-particle running maxima of phi and phi_shear, a
// non-finite count, and the delamination-onset frame (the first frame where
// the broken fraction of one group exceeds a limit) with a snapshot of d and x
// taken on the device at that frame.  Nothing is read back until the caller
// asks, so a frame costs three launches and no host synchronisation.
#include "pm_kernels.cuh"

namespace pm {
namespace {

constexpr int kObsMaxGroups = 8;

// order-preserving float max for non-negative floats through int atomics
__device__ __forceinline__ void atomic_max_nonneg(float *addr, float v) {
    if (v > 0.0f) atomicMax(reinterpret_cast<int *>(addr), __float_as_int(v));
}

__global__ void __launch_bounds__(256) k_observe(const Parts P, const int8_t *__restrict__ group, int n_groups,
                                                 float thr, float *__restrict__ row, float *__restrict__ phi_pp,
                                                 float *__restrict__ psh_pp, int *__restrict__ status) {
    __shared__ float s_acc[kObsMaxGroups][kObsValues];
    __shared__ int s_bad;
    for (int i = threadIdx.x; i < kObsMaxGroups * kObsValues; i += blockDim.x) (&s_acc[0][0])[i] = 0.0f;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < P.n) {
        const long long ps = P.ps;
        const float phi = P.phi ? P.phi[p] : 0.0f;
        const float psh = P.phi_shear ? P.phi_shear[p] : 0.0f;
        const float d = P.d[p];
        const float x0 = P.x[p], y = P.x[ps + p], z = P.x[2 * ps + p];
        if (!(isfinite(x0) && isfinite(y) && isfinite(z) && isfinite(d))) atomicAdd(&s_bad, 1);
        if (phi_pp && phi > phi_pp[p]) phi_pp[p] = phi;
        if (psh_pp && psh > psh_pp[p]) psh_pp[p] = psh;
        const int g = group ? (int)group[p] : 0;
        if (g >= 0 && g < n_groups) {
            float *a = s_acc[g];
            atomic_max_nonneg(&a[0], phi);
            atomic_max_nonneg(&a[1], psh);
            atomicAdd(&a[2], d);
            atomic_max_nonneg(&a[3], d);
            if (d > thr) atomicAdd(&a[4], 1.0f);
            atomicAdd(&a[5], 1.0f);
            atomicAdd(&a[6], y);
        }
    }
    __syncthreads();
    if (threadIdx.x < n_groups * kObsValues) {
        const int g = threadIdx.x / kObsValues, k = threadIdx.x % kObsValues;
        const float v = s_acc[g][k];
        if (k == 0 || k == 1 || k == 3)
            atomic_max_nonneg(&row[g * kObsValues + k], v);
        else if (k < 7 && v != 0.0f)
            atomicAdd(&row[g * kObsValues + k], v);
    }
    if (threadIdx.x == 0 && s_bad) atomicAdd(&status[1], s_bad);
}

// Onset: the first frame whose broken fraction of `onset_group` exceeds `frac`.
__global__ void k_onset(const float *row, int onset_group, float frac, int frame, int *status) {
    if (threadIdx.x == 0 && status[0] < 0 && onset_group >= 0) {
        const float *a = row + onset_group * kObsValues;
        if (a[5] > 0.0f && a[4] / a[5] > frac) status[0] = frame;
    }
}

// Snapshot of d and x (3 planes) at the onset frame, decided on the device.
__global__ void __launch_bounds__(256) k_snapshot(const Parts P, const int *status, int frame, float *snap_d,
                                                  float *snap_x, long long snap_stride) {
    if (status[0] != frame) return;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.n) return;
    if (snap_d) snap_d[p] = P.d[p];
    if (snap_x) {
#pragma unroll
        for (int a = 0; a < 3; ++a) snap_x[a * snap_stride + p] = P.x[a * P.ps + p];
    }
}

}  // namespace

int launch_observe(const Parts &P, const int8_t *group, int n_groups, float thr, float *row, float *phi_pp,
                   float *psh_pp, int *status, int onset_group, float onset_frac, int frame, float *snap_d,
                   float *snap_x, long long snap_stride, cudaStream_t s) {
    if (n_groups < 1 || n_groups > kObsMaxGroups) return 1;
    const unsigned blocks = (unsigned)((P.n + 255) / 256);
    if (blocks > 0) k_observe<<<blocks, 256, 0, s>>>(P, group, n_groups, thr, row, phi_pp, psh_pp, status);
    k_onset<<<1, 32, 0, s>>>(row, onset_group, onset_frac, frame, status);
    if (blocks > 0 && (snap_d || snap_x))
        k_snapshot<<<blocks, 256, 0, s>>>(P, status, frame, snap_d, snap_x, snap_stride);
    return 0;
}

}  // namespace pm
