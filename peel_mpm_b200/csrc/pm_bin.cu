// Particle binning: per-substep cell keys and a stable LSD radix sort of
// (key, particle id), and the compaction of the active 4^3 grid blocks that
// P2G marks.
//
// Key = _node_index(base) of the quadratic base cell (anisompm.py:544-548,
// 586-590), x-major with z fastest.  The permutation equals the stable
// argsort of the keys, bit for bit.
#include "pm_kernels.cuh"

namespace pm {

// Keys, identity ids and allow.any().  blocked = false gives the reference's
// x-major cell index, true the block-major sort key.
__global__ void __launch_bounds__(256) k_keys(const float *__restrict__ x, long long n, long long ps, int ng,
                                              float inv_dx, bool blocked, unsigned *__restrict__ keys,
                                              int *__restrict__ vals, const unsigned char *__restrict__ allow,
                                              Ctrl *ctrl) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    bool any = false;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const float xp[3] = {x[p], x[ps + p], x[2 * ps + p]};
        int qb[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) qb[a] = sat_base(floorf(__fsub_rn(__fmul_rn(xp[a], inv_dx), 0.5f)), ng);
        keys[p] = blocked ? blocked_key(qb, ng) : cell_key(qb, ng);
        vals[p] = (int)p;
        if (allow != nullptr && allow[p]) any = true;
    }
    if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0 && ctrl != nullptr) ctrl->any_allow = 1;
}

// Substep keys: block-major sort key of the base cell, offset by the scene's
// first sort block; identity ids; allow.any() per scene; and the first radix
// pass's digit histogram.  One CTA per radix tile (kSortTile particles), so the
// tile's histogram column is complete when the CTA ends; each thread takes
// particles t, t + 256, ... of the tile, four at a time with their loads
// issued together.
template <class SC>
__global__ void __launch_bounds__(kSortThreads) k_keys_t(const SC sc, const float *__restrict__ x, long long n,
                                                         long long ps, unsigned *__restrict__ keys,
                                                         int *__restrict__ vals, const unsigned char *__restrict__ allow,
                                                         Ctrl *ctrl, unsigned *__restrict__ hist, int n_tiles) {
    __shared__ unsigned cnt[kRadix];
    for (int i = threadIdx.x; i < kRadix; i += kSortThreads) cnt[i] = 0;
    __syncthreads();
    const long long t0 = (long long)blockIdx.x * kSortTile;
    const int lane = threadIdx.x & 31;
    bool any_plain = false;
    int sid = 0;
    if (SC::batched) sid = sc.of_particle(min(t0 + threadIdx.x, n - 1));
    constexpr int G = 4;
#pragma unroll 1
    for (int k0 = 0; k0 < kSortItems; k0 += G) {
        float xp[G][3];
        unsigned char al[G];
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const long long p = t0 + (long long)(k0 + g) * kSortThreads + threadIdx.x;
            const bool ok = p < n;
#pragma unroll
            for (int a = 0; a < 3; ++a) xp[g][a] = ok ? x[a * ps + p] : 0.0f;
            al[g] = ok ? allow[p] : (unsigned char)0;
        }
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const long long p = t0 + (long long)(k0 + g) * kSortThreads + threadIdx.x;
            const bool ok = p < n;
            if (SC::batched && ok) {
                while (p >= sc.p_end(sid, n)) ++sid;   // particles of a thread come in increasing order
            }
            const pm_params &prm = sc.params(sid);
            const int ng = prm.n_grid;
            const float inv_dx = (float)prm.inv_dx;
            int qb[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) qb[a] = sat_base(floorf(__fsub_rn(__fmul_rn(xp[g][a], inv_dx), 0.5f)), ng);
            const unsigned key = (sc.sblock_base(sid) << kSortBlockBits) + blocked_key(qb, ng);
            if (ok) {
                keys[p] = key;
                vals[p] = (int)p;
                atomicAdd(&cnt[key & (kRadix - 1)], 1u);
            }
            const bool a = ok && al[g] != 0;
            if (SC::batched) {
                // a warp whose lanes share a scene votes once
                const int s0 = __shfl_sync(0xffffffffu, sid, 0);
                if (__all_sync(0xffffffffu, sid == s0)) {
                    if (__any_sync(0xffffffffu, a) && lane == 0) ctrl[s0].any_allow = 1;
                } else if (a) {
                    ctrl[sid].any_allow = 1;
                }
            } else {
                any_plain |= a;
            }
        }
    }
    if (!SC::batched) {
        if (__syncthreads_or(any_plain) && threadIdx.x == 0) ctrl->any_allow = 1;
    } else {
        __syncthreads();
    }
    for (int i = threadIdx.x; i < kRadix; i += kSortThreads) hist[(long long)i * n_tiles + blockIdx.x] = cnt[i];
}

// Compacts the marked blocks into block_list and clears the marks.
__global__ void __launch_bounds__(256) k_compact_blocks(unsigned char *__restrict__ block_mask, long long nb,
                                                        int *__restrict__ block_list, Ctrl *ctrl) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long start = (long long)blockIdx.x * blockDim.x;
    for (long long base = start; base < nb; base += stride) {
        const long long b = base + threadIdx.x;
        const bool on = (b < nb) && block_mask[b];
        const unsigned ball = __ballot_sync(0xffffffffu, on);
        unsigned slot0 = 0;
        if ((threadIdx.x & 31) == 0 && ball) slot0 = atomicAdd(&ctrl->n_active, (unsigned)__popc(ball));
        slot0 = __shfl_sync(0xffffffffu, slot0, 0);
        if (on) {
            const unsigned slot = slot0 + __popc(ball & lanemask_lt());
            if (slot < (unsigned long long)nb) block_list[slot] = (int)b;   // bounded even without a clock reset
            block_mask[b] = 0;
        }
    }
}

// ------------------------------------------------------------ radix sort
// Per tile (kSortTile keys) digit histogram -> hist[digit * n_tiles + tile]
// for RB-bit digits.  Full tiles load keys as uint4 (order does not matter for
// a histogram); int32 shared atomics aggregate equal addresses in hardware.
template <int RB>
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const unsigned *__restrict__ keys, long long n,
                                                             int shift, unsigned *__restrict__ hist, int n_tiles) {
    constexpr unsigned R = 1u << RB;
    __shared__ unsigned cnt[R];
    for (int i = threadIdx.x; i < (int)R; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    const long long t0 = (long long)blockIdx.x * kSortTile;
    if (t0 + kSortTile <= n) {
        const uint4 *k4 = reinterpret_cast<const uint4 *>(keys + t0);
        uint4 v[kSortItems / 4];
#pragma unroll
        for (int it = 0; it < kSortItems / 4; ++it) v[it] = k4[it * kSortThreads + threadIdx.x];
#pragma unroll
        for (int it = 0; it < kSortItems / 4; ++it) {
            atomicAdd(&cnt[(v[it].x >> shift) & (R - 1)], 1u);
            atomicAdd(&cnt[(v[it].y >> shift) & (R - 1)], 1u);
            atomicAdd(&cnt[(v[it].z >> shift) & (R - 1)], 1u);
            atomicAdd(&cnt[(v[it].w >> shift) & (R - 1)], 1u);
        }
    } else {
        for (int it = 0; it < kSortItems; ++it) {
            const long long i = t0 + (long long)it * kSortThreads + threadIdx.x;
            if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & (R - 1)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < (int)R; i += blockDim.x) hist[(long long)i * n_tiles + blockIdx.x] = cnt[i];
}

// Exclusive scan of each digit's row hist[d][0..n_tiles) in place; row totals
// go to dtot[d].  One CTA per digit.
__global__ void __launch_bounds__(256) k_radix_rowscan(unsigned *__restrict__ hist, int n_tiles,
                                                       unsigned *__restrict__ dtot) {
    __shared__ unsigned wsum[8];
    __shared__ unsigned carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    unsigned *row = hist + (long long)blockIdx.x * n_tiles;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n_tiles; base += 256) {
        const int i = base + tid;
        const unsigned v = i < n_tiles ? row[i] : 0u;
        unsigned incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        unsigned wpre = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) wpre += (w < wid) ? wsum[w] : 0u;
        const unsigned c = carry;
        if (i < n_tiles) row[i] = c + wpre + incl - v;
        __syncthreads();
        if (tid == 255) carry = c + wpre + incl;
        __syncthreads();
    }
    if (tid == 0) dtot[blockIdx.x] = carry;
}

// Stable scatter of one digit pass with RB-bit digits.  Warp w of a tile owns
// keys [w*512, w*512+512) of the tile and ranks them in 16 rounds of 32 in
// index order; per-warp digit counters are then offset by the earlier warps.
// The tile is first written to shared memory in (digit, rank) order, then
// copied out so that consecutive threads write consecutive addresses of one
// digit's run.  Shared memory (dynamic): per-warp digit counters, the tile's
// global and local digit starts and the staged tile (43 KB for 8-bit digits,
// 53 KB for 9-bit ones).
template <int RB>
constexpr size_t radix_scatter_smem() {
    return 4u * ((size_t)(kSortThreads / 32 + 2) * (1u << RB) + 2u * kSortTile);
}

template <int RB>
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const unsigned *__restrict__ kin,
                                                                const int *__restrict__ vin,
                                                                unsigned *__restrict__ kout, int *__restrict__ vout,
                                                                long long n, int shift,
                                                                const unsigned *__restrict__ offs, int n_tiles,
                                                                const unsigned *__restrict__ dtot,
                                                                int *__restrict__ inv) {
    constexpr int W = kSortThreads / 32;
    constexpr unsigned R = 1u << RB;
    constexpr int DPT = (int)R / kSortThreads;   // digits per thread in the prefix step
    static_assert(DPT >= 1 && (int)R == DPT * kSortThreads, "digits must fill the block");
    extern __shared__ unsigned sm_radix[];
    unsigned *wcnt = sm_radix;                   // [W][R]
    unsigned *gbase = wcnt + W * R;              // [R] global start of the tile's run of each digit
    unsigned *lbase = gbase + R;                 // [R] tile-local start of each digit
    unsigned *skey = lbase + R;                  // [kSortTile]
    int *sval = (int *)(skey + kSortTile);       // [kSortTile]
    __shared__ unsigned wv[W], wc[W];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < W * (int)R; i += blockDim.x) wcnt[i] = 0;
    __syncthreads();
    const long long tile0 = (long long)blockIdx.x * kSortTile;
    const int tile_len = (int)min((long long)kSortTile, n - tile0);
    const long long t0 = tile0 + (long long)wid * (32 * kSortItems);
    unsigned key[kSortItems];
    int val[kSortItems];
    unsigned rank[kSortItems];
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const long long i = t0 + r * 32 + lane;
        const bool ok = i < n;
        key[r] = ok ? kin[i] : 0u;
        val[r] = ok ? vin[i] : 0;
        const unsigned dg = ok ? (key[r] >> shift) & (R - 1) : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, dg);
        const int leader = __ffs(peers) - 1;
        unsigned before = 0;
        if (ok && lane == leader) {
            before = wcnt[wid * R + dg];
            wcnt[wid * R + dg] = before + (unsigned)__popc(peers);
        }
        before = __shfl_sync(0xffffffffu, before, leader);
        rank[r] = before + (unsigned)__popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();
    {   // per digit (DPT consecutive digits per thread): exclusive prefix over
        // warps and the tile count; then exclusive scans over all digits of the
        // global digit totals (dtot) and of the tile's own counts
        unsigned tc[DPT], gt[DPT];
        unsigned st = 0, sg = 0;
#pragma unroll
        for (int q = 0; q < DPT; ++q) {
            const int dg = threadIdx.x * DPT + q;
            unsigned run = 0;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const unsigned c = wcnt[w * R + dg];
                wcnt[w * R + dg] = run;
                run += c;
            }
            tc[q] = run;
            gt[q] = dtot[dg];
            st += run;
            sg += gt[q];
        }
        unsigned vi = sg, ci = st;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, vi, o);
            const unsigned z = __shfl_up_sync(0xffffffffu, ci, o);
            if (lane >= o) { vi += y; ci += z; }
        }
        if (lane == 31) { wv[wid] = vi; wc[wid] = ci; }
        __syncthreads();
        unsigned pv = 0, pc = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            pv += (w < wid) ? wv[w] : 0u;
            pc += (w < wid) ? wc[w] : 0u;
        }
        unsigned ag = pv + vi - sg, at = pc + ci - st;   // exclusive starts of this thread's first digit
#pragma unroll
        for (int q = 0; q < DPT; ++q) {
            const int dg = threadIdx.x * DPT + q;
            gbase[dg] = ag + offs[(long long)dg * n_tiles + blockIdx.x];
            lbase[dg] = at;
            ag += gt[q];
            at += tc[q];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const long long i = t0 + r * 32 + lane;
        if (i < n) {
            const unsigned dg = (key[r] >> shift) & (R - 1);
            const unsigned lp = lbase[dg] + wcnt[wid * R + dg] + rank[r];
            skey[lp] = key[r];
            sval[lp] = val[r];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tile_len; i += kSortThreads) {
        const unsigned k = skey[i];
        const unsigned dg = (k >> shift) & (R - 1);
        const unsigned gp = gbase[dg] + (unsigned)i - lbase[dg];
        kout[gp] = k;
        vout[gp] = sval[i];
        if (inv != nullptr) inv[sval[i]] = (int)gp;   // last pass: position of each particle in the order
    }
}

// One-time kernel attribute set-up for the current device (the 9-bit scatter
// needs more than 48 KB of dynamic shared memory); not a stream operation, so
// pm_prepare runs it before any capture.
void prepare_sort() {
    static int done[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || done[dev]) return;
    cudaFuncSetAttribute(k_radix_scatter<kRadixBitsTop>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)radix_scatter_smem<kRadixBitsTop>());
    done[dev] = 1;
}

template <int RB>
static void radix_pass(const WS &w, long long n, int tiles, int shift, bool need_hist, const unsigned *kin,
                       const int *vin, unsigned *kout, int *vout, int *inv, cudaStream_t s) {
    if (need_hist) k_radix_hist<RB><<<tiles, kSortThreads, 0, s>>>(kin, n, shift, w.hist, tiles);
    k_radix_rowscan<<<1u << RB, 256, 0, s>>>(w.hist, tiles, w.dtot);
    k_radix_scatter<RB><<<tiles, kSortThreads, radix_scatter_smem<RB>(), s>>>(kin, vin, kout, vout, n, shift, w.hist,
                                                                             tiles, w.dtot, inv);
}

void launch_sort(const WS &w, long long n, cudaStream_t s, int *inv, bool hist0_ready) {
    if (n <= 0) return;
    prepare_sort();
    const int tiles = (int)((n + kSortTile - 1) / kSortTile);
    unsigned *kin = w.keys_a, *kout = w.keys_b;
    int *vin = w.vals_a, *vout = w.vals_b;
    int shift = 0, rem = w.key_bits;
    for (int pass = 0; pass < w.passes; ++pass) {
        const int rb = radix_digit_bits(rem);
        // launch_keys leaves the first pass's 8-bit histogram
        const bool need_hist = pass > 0 || !hist0_ready || rb != kRadixBits;
        int *iv = pass == w.passes - 1 ? inv : nullptr;
        if (rb == kRadixBitsTop)
            radix_pass<kRadixBitsTop>(w, n, tiles, shift, need_hist, kin, vin, kout, vout, iv, s);
        else
            radix_pass<kRadixBits>(w, n, tiles, shift, need_hist, kin, vin, kout, vout, iv, s);
        shift += rb;
        rem -= rb;
        unsigned *tk = kin; kin = kout; kout = tk;
        int *tv = vin; vin = vout; vout = tv;
    }
}

template <class SC>
void launch_keys(const SC &sc, const WS &w, const Parts &P, cudaStream_t s) {
    if (P.n <= 0) return;
    const int tiles = (int)((P.n + kSortTile - 1) / kSortTile);
    k_keys_t<SC><<<tiles, kSortThreads, 0, s>>>(sc, P.x, P.n, P.ps, w.keys_a, w.vals_a, P.allow, w.ctrl, w.hist,
                                                tiles);
}
template void launch_keys<PlainScenes>(const PlainScenes &, const WS &, const Parts &, cudaStream_t);
template void launch_keys<BatchScenes>(const BatchScenes &, const WS &, const Parts &, cudaStream_t);

void launch_compact(const WS &w, cudaStream_t s) {
    const int cb = (int)std::min<long long>((w.n_blocks + 255) / 256, 148LL * 8);
    k_compact_blocks<<<cb > 0 ? cb : 1, 256, 0, s>>>(w.block_mask, w.n_blocks, w.block_list, w.ctrl);
}

void launch_keys_only(const float *x, long long n, long long ps, int ng, float inv_dx, bool blocked, const WS &w,
                      cudaStream_t s) {
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_keys<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(x, n, ps, ng, inv_dx, blocked, w.keys_a, w.vals_a, nullptr,
                                                  nullptr);
}

}  // namespace pm
