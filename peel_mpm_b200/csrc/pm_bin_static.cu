// pm_bin_sort_static: the binning sort of pm_bin_sort with its scratch in a
// file-scope device array instead of a caller-provided workspace, for callers
// that cannot allocate device memory (see include/peelmpm.h).
//
// The array is a host-side symbol in this file: host code must never pass
// `g_sort_scratch` itself to a kernel (it names host memory there).  Its
// device address is looked up once per device with cudaGetSymbolAddress,
// with that device current, and cached.
#include <mutex>

#include "pm_kernels.cuh"

namespace pm {
int report_error(int code, const char *msg);
}

namespace {

constexpr long long kMaxN = PM_BIN_STATIC_MAX_N;
constexpr int kMaxTiles = (int)((kMaxN + pm::kSortTile - 1) / pm::kSortTile);
constexpr size_t kKeyBytes = 4u * (size_t)kMaxN;
constexpr size_t kBytes = 4 * kKeyBytes + 4u * ((size_t)pm::kRadixTop * kMaxTiles + pm::kRadixTop);
static_assert(kBytes == PM_BIN_STATIC_SCRATCH_BYTES, "header size must match the array");
static_assert(kKeyBytes % 256 == 0, "sub-buffers stay 256-byte aligned");

// keys_a | keys_b | ids_a | ids_b | tile histograms + digit totals
static __device__ __align__(256) unsigned char g_sort_scratch[kBytes];

std::mutex g_mu;
void *g_addr[64] = {nullptr};

int scratch_address(void **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return pm::report_error(PM_ERR_CUDA, "pm_bin_sort_static: no current CUDA device");
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_addr[dev] == nullptr) {
        int major = 0;
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        if (major != 10) return pm::report_error(PM_ERR_UNSUPPORTED, "peelmpm kernels are built for sm_100a only");
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return pm::report_error(PM_ERR_CUDA, "pm_bin_sort_static: cudaGetSymbolAddress failed");
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return PM_OK;
}

}  // namespace

extern "C" int pm_bin_sort_static(const float *x, int64_t n, int64_t plane_stride, int32_t n_grid, double inv_dx,
                                  uint32_t *keys_out, int32_t *perm_out, void *stream) {
    if (n < 0 || plane_stride < n || n_grid < 4 || n_grid > 1024 || !(inv_dx > 0.0))
        return pm::report_error(PM_ERR_ARG, "pm_bin_sort_static: bad size argument");
    if (n > kMaxN)
        return pm::report_error(PM_ERR_ARG, "pm_bin_sort_static: n exceeds PM_BIN_STATIC_MAX_N (262144)");
    if (n > 0 && (!x || !keys_out || !perm_out)) return pm::report_error(PM_ERR_ARG, "pm_bin_sort_static: NULL array");
    void *base = nullptr;
    int rc = scratch_address(&base);
    if (rc != PM_OK) return rc;
    if (n == 0) return PM_OK;
    char *b = (char *)base;
    pm::WS w{};
    w.keys_a = (unsigned *)(b);
    w.keys_b = (unsigned *)(b + kKeyBytes);
    w.vals_a = (int *)(b + 2 * kKeyBytes);
    w.vals_b = (int *)(b + 3 * kKeyBytes);
    w.hist = (unsigned *)(b + 4 * kKeyBytes);
    w.n_tiles = (int)((n + pm::kSortTile - 1) / pm::kSortTile);
    w.dtot = w.hist + (size_t)pm::kRadixTop * w.n_tiles;
    const pm::Layout L = pm::make_layout(n, n_grid);
    w.passes = L.passes;
    w.key_bits = L.key_bits;
    const unsigned *sorted = (w.passes & 1) ? w.keys_b : w.keys_a;
    const int *perm = (w.passes & 1) ? w.vals_b : w.vals_a;
    cudaStream_t s = (cudaStream_t)stream;
    // every scratch word the sort reads is written earlier in the same call
    // (keys/ids by the key kernel, histograms and totals by each pass), so the
    // previous call's contents need no clearing
    pm::launch_keys_only(x, n, plane_stride, n_grid, (float)inv_dx, false, w, s);
    pm::launch_sort(w, n, s);
    if (cudaMemcpyAsync(keys_out, sorted, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(perm_out, perm, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        cudaGetLastError();
        return pm::report_error(PM_ERR_CUDA, "pm_bin_sort_static: copy-out failed");
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return pm::report_error(PM_ERR_CUDA, cudaGetErrorString(e));
    return PM_OK;
}
