// Launchers shared between the kernel files and the C ABI layer.
#pragma once

#include <algorithm>

#include "pm_common.cuh"

namespace pm {

void launch_keys(const WS &w, const Parts &P, int ng, float inv_dx, cudaStream_t s);
void launch_sort(const WS &w, long long n, cudaStream_t s, int *inv = nullptr);
void launch_compact(const WS &w, cudaStream_t s);
void prepare_p2g();
void launch_keys_only(const float *x, long long n, long long ps, int ng, float inv_dx, bool blocked, const WS &w,
                      cudaStream_t s);
void launch_p2g(const pm_params &prm, const Parts &P, const WS &w, cudaStream_t s, int range = 0);
void launch_grid(const pm_params &prm, const WS &w, cudaStream_t s);
void launch_g2p(const pm_params &prm, const Parts &P, const WS &w, cudaStream_t s);
void launch_set_clock(const pm_params &prm, const WS &w, const pm_clock &clk, cudaStream_t s);
void launch_set_clock_dev(const pm_params &prm, const WS &w, const pm_clock *dev, int row, cudaStream_t s);
int balanced_range(long long n, int slots, int max_range);
int resident_slots(const void *kernel, int threads, size_t smem);
void launch_sym_eig(const float *A, long long n, int sweeps, float *ev, float *V, cudaStream_t s);

}  // namespace pm
