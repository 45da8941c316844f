// Gaussian-splat renderer (render.py:71-162 of the reference): EWA projection
// of 3D gaussians to screen-space gaussians, then the reference's two-pass
// soft z-buffer -- per pixel the nearest splat depth, then a blend of all
// splats weighted by exp(-(z - z_min) / tau) -- and coverage compositing over
// a background.  The image is a headless device buffer (H, W, 3).
//
// Screen tiles of 8x8 pixels.  k_splat_project (one thread per gaussian:
// camera transform, Jacobian, 2D covariance + 0.3 dilation, conic, radius,
// culling) packs each drawn splat into 48 bytes and counts it into every tile
// its (2r+1)^2 footprint square touches; a scan of the tile counts and
// k_splat_emit build per-tile splat lists; k_splat_tiles runs one warp per
// tile, two pixels per lane: the soft z-buffer walks the tile's list once from
// shared memory with the pixels' state in registers and each pixel is
// composed at the end -- no per-pixel atomics, no clear of pixel buffers.
// tau from the median depth uses the library's radix sort of the depth keys.
#include "pm_kernels.cuh"

namespace pm {
namespace {

constexpr int kTile = 8;                  // screen tile edge, pixels

struct RenderWS {
    float4 *sp;        // [3n] per splat: {u, v, c00, c01}, {c11, z, u0, v0 (int bits)}, {r, g, b, rad (int bits)}
    unsigned *count;   // [0] drawn splats, [1] list overflow (never set when the capacity bound holds)
    float *tau;        // [0] tau, [1] 1 / max(tau, 1e-6)
    unsigned *tcnt;    // [ntiles] splats per tile
    unsigned *tfill;   // [ntiles] emit cursors
    unsigned *tstart;  // [ntiles + 1] exclusive prefix of tcnt
    int *tlist;        // [cap] splat ids grouped by tile
    long long cap;
    int ntx, nty;
    WS sort;           // key / value buffers of the median sort
};

__device__ __forceinline__ void splat_tiles(int u0, int v0, int rad, int W, int H, int &tx0, int &ty0, int &nx,
                                            int &ny) {
    const int x0 = max(u0 - rad, 0), x1 = min(u0 + rad, W - 1);
    const int y0 = max(v0 - rad, 0), y1 = min(v0 + rad, H - 1);
    tx0 = x0 / kTile;
    ty0 = y0 / kTile;
    nx = x1 / kTile - tx0 + 1;
    ny = y1 / kTile - ty0 + 1;
}

__global__ void __launch_bounds__(256) k_splat_clear(RenderWS r, int ntiles) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 4) r.count[i] = 0;
    if (i < ntiles) {
        r.tcnt[i] = 0;
        r.tfill[i] = 0;
    }
}

// Each lane walks the tiles of its own splat; lanes of a warp that hit the
// same tile in the same step (neighbouring gaussians) add to it with one atomic.
__device__ __forceinline__ unsigned tile_reserve(unsigned act, unsigned *ctr, int t, bool on) {
    const unsigned peers = __match_any_sync(act, on ? t : -1);
    const int leader = __ffs(peers) - 1;
    const unsigned lane = threadIdx.x & 31;
    unsigned base = 0;
    if (on && (int)lane == leader) base = atomicAdd(&ctr[t], (unsigned)__popc(peers));
    base = __shfl_sync(act, base, leader);
    return base + (unsigned)__popc(peers & lanemask_lt());
}

__global__ void __launch_bounds__(256) k_splat_project(const pm_camera cam, const pm_render_params rp,
                                                       const float *__restrict__ xyz, const float *__restrict__ cov,
                                                       const float *__restrict__ color, long long n, RenderWS r) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float X[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    float Xc[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) Xc[j] = (X[0] * cam.R[j] + X[1] * cam.R[3 + j] + X[2] * cam.R[6 + j]) + cam.T[j];
    const float z = Xc[2];
    bool ok = z > rp.near;
    float u = 0.0f, v = 0.0f, c00 = 0.0f, c01 = 0.0f, c11 = 0.0f;
    int u0 = 0, v0 = 0, rad = 0;
    if (ok) {
        const float cx = 0.5f * (float)cam.width, cy = 0.5f * (float)cam.height;
        u = cam.fx * Xc[0] / z + cx;
        v = cam.fy * Xc[1] / z + cy;
        const float invz = 1.0f / z;
        // J (2x3): [fx/z, 0, -fx x / z^2; 0, fy/z, -fy y / z^2]
        const float J00 = cam.fx * invz, J02 = -cam.fx * Xc[0] * invz * invz;
        const float J11 = cam.fy * invz, J12 = -cam.fy * Xc[1] * invz * invz;
        // cov_cam = R^T cov R * s^2 (Rt = R^T)
        float Sg[9], T1[9], Cc[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) Sg[k] = cov[9 * i + k];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)   // T1 = Rt Sg, Rt[a][k] = R[k][a]
                T1[3 * a + b] = cam.R[a] * Sg[b] + cam.R[3 + a] * Sg[3 + b] + cam.R[6 + a] * Sg[6 + b];
        const float s2 = rp.scale_modifier * rp.scale_modifier;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)   // Cc = T1 Rt^T = T1 R, Rt^T[k][b] = R[k][b]
                Cc[3 * a + b] = (T1[3 * a] * cam.R[b] + T1[3 * a + 1] * cam.R[3 + b] + T1[3 * a + 2] * cam.R[6 + b]) * s2;
        // cov2d = J Cc J^T
        const float M00 = J00 * Cc[0] + J02 * Cc[6], M01 = J00 * Cc[1] + J02 * Cc[7], M02 = J00 * Cc[2] + J02 * Cc[8];
        const float M11 = J11 * Cc[4] + J12 * Cc[7], M12 = J11 * Cc[5] + J12 * Cc[8], M10 = J11 * Cc[3] + J12 * Cc[6];
        const float a = (M00 * J00 + M02 * J02) + 0.3f;
        const float b = M01 * J11 + M02 * J12;
        const float d = (M11 * J11 + M12 * J12) + 0.3f;
        (void)M10;
        const float det = a * d - b * b;
        const float mid = 0.5f * (a + d);
        const float disc = mid * mid - det;
        const float lam = mid + sqrtf(disc > 0.0f ? disc : 0.0f);
        const float raw = 3.0f * sqrtf(lam > 1e-6f ? lam : 1e-6f);
        u0 = (int)floorf(u);
        v0 = (int)floorf(v);
        rad = (int)ceilf(raw);
        rad = rad < 1 ? 1 : (rad > rp.r_max ? rp.r_max : rad);
        ok = det > 1e-9f && raw < rp.max_raw_radius && u0 + rad >= 0 && u0 - rad < cam.width && v0 + rad >= 0 &&
             v0 - rad < cam.height;
        if (ok) {
            const float inv_det = 1.0f / det;
            c00 = d * inv_det;
            c01 = -b * inv_det;
            c11 = a * inv_det;
        }
    }
    const int rd = ok ? rad : 0;
    r.sp[3 * i] = make_float4(u, v, c00, c01);
    r.sp[3 * i + 1] = make_float4(c11, z, __int_as_float(u0), __int_as_float(v0));
    if (ok)
        r.sp[3 * i + 2] = make_float4(color[3 * i], color[3 * i + 1], color[3 * i + 2], __int_as_float(rd));
    else
        r.sp[3 * i + 2] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(0));
    // depth key for the median of the drawn splats (z > near > 0: the float bits order like the values)
    r.sort.keys_a[i] = ok ? __float_as_uint(z) : 0xffffffffu;
    r.sort.vals_a[i] = (int)i;
    const unsigned act = __activemask(), drawn = __ballot_sync(act, ok);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(act) - 1) && drawn) atomicAdd(r.count, (unsigned)__popc(drawn));
    // tile counts of the footprint square
    int tx0 = 0, ty0 = 0, nx = 0, ny = 0;
    if (ok) splat_tiles(u0, v0, rd, cam.width, cam.height, tx0, ty0, nx, ny);
    const int nt = nx * ny;
    const int steps = __reduce_max_sync(act, nt);
    for (int k = 0; k < steps; ++k) {
        const bool on = k < nt;
        const int ky = on ? k / nx : 0;
        const int t = on ? (ty0 + ky) * r.ntx + tx0 + (k - ky * nx) : 0;
        tile_reserve(act, r.tcnt, t, on);
    }
}

// tau = 0.02 * median depth (torch.median: the lower middle element), or the given tau
__global__ void k_splat_tau(RenderWS r, float tau_given, const unsigned *sorted) {
    if (threadIdx.x != 0) return;
    float tau = tau_given;
    if (!(tau_given > 0.0f)) {
        const unsigned c = r.count[0];
        tau = c > 0 ? 0.02f * __uint_as_float(sorted[(c - 1) / 2]) : 1.0f;
    }
    r.tau[0] = tau;
    r.tau[1] = 1.0f / (tau > 1e-6f ? tau : 1e-6f);
}

// Exclusive scan of the tile counts (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) k_tile_scan(RenderWS r, int ntiles) {
    __shared__ unsigned wsum[32];
    __shared__ unsigned carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ntiles; base += 1024) {
        const int i = base + tid;
        const unsigned v = i < ntiles ? r.tcnt[i] : 0u;
        unsigned incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            unsigned w = wsum[lane], wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += y;
            }
            wsum[lane] = wi - w;   // exclusive over warps
        }
        __syncthreads();
        const unsigned c = carry;
        if (i < ntiles) r.tstart[i] = c + wsum[wid] + incl - v;
        __syncthreads();
        if (tid == 1023) carry = c + wsum[wid] + incl;
        __syncthreads();
    }
    if (tid == 0) r.tstart[ntiles] = carry;
}

// Per-tile lists: every drawn splat id into each tile of its footprint square.
__global__ void __launch_bounds__(256) k_splat_emit(const pm_camera cam, long long n, RenderWS r) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p1 = r.sp[3 * i + 1], p2 = r.sp[3 * i + 2];
    const int rd = __float_as_int(p2.w);
    int tx0 = 0, ty0 = 0, nx = 0, ny = 0;
    if (rd > 0) splat_tiles(__float_as_int(p1.z), __float_as_int(p1.w), rd, cam.width, cam.height, tx0, ty0, nx, ny);
    const int nt = nx * ny;
    const unsigned act = __activemask();
    const int steps = __reduce_max_sync(act, nt);
    for (int k = 0; k < steps; ++k) {
        const bool on = k < nt;
        const int ky = on ? k / nx : 0;
        const int t = on ? (ty0 + ky) * r.ntx + tx0 + (k - ky * nx) : 0;
        const unsigned slot = tile_reserve(act, r.tfill, t, on);
        if (on) {
            const long long at = (long long)r.tstart[t] + slot;
            if (slot < r.tcnt[t] && at < r.cap)
                r.tlist[at] = (int)i;
            else
                r.count[1] = 1;
        }
    }
}

// One warp per 8x8 tile (4 tiles per CTA), two pixels per lane (rows y and
// y + 4).  The warp walks its tile's list in batches of 32 splats staged in
// shared memory.  A splat counts at a pixel when the pixel lies in its
// footprint square and alpha = exp(min(power, 0)) exceeds 1/255 (a power below
// -6 gives exp(power) < 0.0025 < 1/255: dropped before the exponential with
// the same outcome).  The reference's two passes -- nearest depth z_min, then
// sums of c w and w with w = alpha exp(-(z - z_min) / tau) -- are done in one:
// the sums are kept relative to the nearest depth seen so far and rescaled by
// exp(-(z_old - z_new) / tau) when a nearer splat arrives, which is the same
// sum up to rounding.  The coverage 1 - exp(sum log(max(1 - alpha, 1e-6))) is
// taken as 1 - prod max(1 - alpha, 1e-6): the same quantity, and a product
// that underflows gives coverage 1.0f exactly as the sum of logs does.  The
// exponentials use the __expf intrinsic (a few ulp; the image tolerance is
// 1e-4 absolute).
constexpr int kTileWarps = 4;

struct PixAcc {
    float zmin, c0, c1, c2, w, rev;   // rev: prod max(1 - alpha, 1e-6)
};

__device__ __forceinline__ void pix_add(PixAcc &p, const float4 &A, const float4 &B, const float4 &Cc, int px, int py,
                                        float inv_tau) {
    const int rd = __float_as_int(Cc.w);
    if (abs(px - __float_as_int(B.z)) > rd || abs(py - __float_as_int(B.w)) > rd) return;
    const float dx = ((float)px + 0.5f) - A.x, dy = ((float)py + 0.5f) - A.y;
    const float power = -0.5f * (A.z * dx * dx + B.x * dy * dy) - A.w * dx * dy;
    if (power < -6.0f) return;
    const float ga = __expf(power < 0.0f ? power : 0.0f);
    if (!(ga > (1.0f / 255.0f))) return;
    float w;
    if (B.y < p.zmin) {
        const float sc = p.w > 0.0f ? __expf(-(p.zmin - B.y) * inv_tau) : 0.0f;
        p.c0 *= sc; p.c1 *= sc; p.c2 *= sc; p.w *= sc;
        p.zmin = B.y;
        w = ga;   // exp(0)
    } else {
        w = ga * __expf(-(B.y - p.zmin) * inv_tau);
    }
    p.c0 += Cc.x * w;
    p.c1 += Cc.y * w;
    p.c2 += Cc.z * w;
    p.w += w;
    const float om = 1.0f - ga;
    p.rev *= om > 1e-6f ? om : 1e-6f;
}

__device__ __forceinline__ void pix_store(const PixAcc &p, const pm_camera &cam, const pm_render_params &rp, int px,
                                          int py, float *img) {
    if (px >= cam.width || py >= cam.height) return;
    const float cover = 1.0f - p.rev;
    const float csum[3] = {p.c0, p.c1, p.c2};
    float *o = img + 3 * ((long long)py * cam.width + px);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float rgb = p.w > 1e-8f ? csum[c] / (p.w > 1e-8f ? p.w : 1e-8f) : rp.bg[c];
        const float v = rgb * cover + rp.bg[c] * (1.0f - cover);
        o[c] = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
    }
}

__global__ void __launch_bounds__(32 * kTileWarps) k_splat_tiles(const pm_camera cam, const pm_render_params rp,
                                                                 RenderWS r, float *__restrict__ img, int ntiles) {
    __shared__ float4 sA[kTileWarps][32], sB[kTileWarps][32], sC[kTileWarps][32];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * kTileWarps + wid;
    if (tile >= ntiles) return;   // whole warps only; no block-wide barrier below
    const int px = (tile % r.ntx) * kTile + (lane & (kTile - 1));
    const int py0 = (tile / r.ntx) * kTile + (lane >> 3), py1 = py0 + 4;
    const unsigned beg = r.tstart[tile], end = beg + r.tcnt[tile];
    const float inv_tau = r.tau[1];
    const float inf = __int_as_float(0x7f800000);
    PixAcc a = {inf, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f}, b = a;
    for (unsigned base = beg; base < end; base += 32) {
        const int cnt = (int)min(32u, end - base);
        __syncwarp();
        if (lane < cnt) {
            const long long g = r.tlist[base + lane];
            sA[wid][lane] = r.sp[3 * g];
            sB[wid][lane] = r.sp[3 * g + 1];
            sC[wid][lane] = r.sp[3 * g + 2];
        }
        __syncwarp();
        for (int j = 0; j < cnt; ++j) {
            const float4 A = sA[wid][j], B = sB[wid][j], Cc = sC[wid][j];
            pix_add(a, A, B, Cc, px, py0, inv_tau);
            pix_add(b, A, B, Cc, px, py1, inv_tau);
        }
    }
    pix_store(a, cam, rp, px, py0, img);
    pix_store(b, cam, rp, px, py1, img);
}

struct RenderLayout {
    Layout sort;
    size_t sp, count, tau, tcnt, tfill, tstart, tlist, total;
    long long cap;
    int ntx, nty;
};

// Tiles a footprint square of side 2 r_max + 1 can touch, per axis:
// floor(2 r_max / kTile) + 2, and never more than the screen has.
RenderLayout make_render_layout(long long n, int width, int height, int r_max) {
    RenderLayout R;
    R.ntx = (width + kTile - 1) / kTile;
    R.nty = (height + kTile - 1) / kTile;
    const long long ntiles = (long long)R.ntx * R.nty;
    const long long per_axis = 2LL * (r_max > 1 ? r_max : 1) / kTile + 2;
    const long long per = std::min(per_axis, (long long)R.ntx) * std::min(per_axis, (long long)R.nty);
    R.cap = std::max<long long>(1, n * per);
    R.sort = make_layout_sized(n, 0, 0, 32, 1, 0);
    const size_t A = 256, nn = (size_t)(n > 0 ? n : 1), nt = (size_t)ntiles;
    size_t o = R.sort.total;
    R.sp = o;     o = align_up(o + 48 * nn, A);
    R.count = o;  o = align_up(o + 16, A);
    R.tau = o;    o = align_up(o + 16, A);
    R.tcnt = o;   o = align_up(o + 4 * nt, A);
    R.tfill = o;  o = align_up(o + 4 * nt, A);
    R.tstart = o; o = align_up(o + 4 * (nt + 1), A);
    R.tlist = o;  o = align_up(o + 4 * (size_t)R.cap, A);
    R.total = o;
    return R;
}


// Gaussian carrying (run_orange.py:116-133): gaussian i bound to particle
// b = bind[i] moves with the particle's affine motion: position
// A (x_b) + t + F_b off0_i, covariance F_b cov0_i F_b^T, colour darkened by
// damage, color0_i (1 - tint d_b).
__global__ void __launch_bounds__(256) k_carry(const Parts P, const int *__restrict__ bind, const float *__restrict__ off0,
                                               const float *__restrict__ cov0, const float *__restrict__ color0,
                                               long long g_n, const float *__restrict__ affine, float tint,
                                               float *__restrict__ pos, float *__restrict__ cov,
                                               float *__restrict__ color) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g_n) return;
    const long long b = bind[i];
    if (b < 0 || b >= P.n) {   // an unbound gaussian: NaN outputs (the host wrapper rejects such bindings)
        const float q = __int_as_float(0x7fc00000);
#pragma unroll
        for (int k = 0; k < 3; ++k) pos[3 * i + k] = color[3 * i + k] = q;
#pragma unroll
        for (int k = 0; k < 9; ++k) cov[9 * i + k] = q;
        return;
    }
    const long long ps = P.ps;
    float F[9], xp[3];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = P.F[k * ps + b];
#pragma unroll
    for (int a = 0; a < 3; ++a) xp[a] = P.x[a * ps + b];
    const float o[3] = {off0[3 * i], off0[3 * i + 1], off0[3 * i + 2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float w = (affine[4 * a] * xp[0] + affine[4 * a + 1] * xp[1] + affine[4 * a + 2] * xp[2]) + affine[4 * a + 3];
        pos[3 * i + a] = w + (F[3 * a] * o[0] + F[3 * a + 1] * o[1] + F[3 * a + 2] * o[2]);
    }
    float S[9], T1[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) S[k] = cov0[9 * i + k];
    mm3(F, S, T1);
    mmt3(T1, F, S);
#pragma unroll
    for (int k = 0; k < 9; ++k) cov[9 * i + k] = S[k];
    const float shade = tint > 0.0f ? 1.0f - tint * P.d[b] : 1.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) color[3 * i + c] = color0[3 * i + c] * shade;
}

}  // namespace

void launch_carry(const Parts &P, const int *bind, const float *off0, const float *cov0, const float *color0,
                  long long g_n, const float *affine, float tint, float *pos, float *cov, float *color,
                  cudaStream_t s) {
    if (g_n <= 0) return;
    k_carry<<<(unsigned)((g_n + 255) / 256), 256, 0, s>>>(P, bind, off0, cov0, color0, g_n, affine, tint, pos, cov,
                                                          color);
}

size_t render_workspace_bytes(long long n, int width, int height, int r_max) {
    return make_render_layout(n, width, height, r_max).total;
}

void launch_render(const pm_camera &cam, const pm_render_params &rp, const float *xyz, const float *cov,
                   const float *color, long long n, float *img, void *ws, cudaStream_t s) {
    const RenderLayout L = make_render_layout(n, cam.width, cam.height, rp.r_max);
    char *b = (char *)ws;
    RenderWS r;
    r.sp = (float4 *)(b + L.sp);
    r.count = (unsigned *)(b + L.count);
    r.tau = (float *)(b + L.tau);
    r.tcnt = (unsigned *)(b + L.tcnt);
    r.tfill = (unsigned *)(b + L.tfill);
    r.tstart = (unsigned *)(b + L.tstart);
    r.tlist = (int *)(b + L.tlist);
    r.cap = L.cap;
    r.ntx = L.ntx;
    r.nty = L.nty;
    r.sort = make_ws(ws, L.sort);
    const int ntiles = L.ntx * L.nty;
    k_splat_clear<<<(unsigned)((std::max(ntiles, 4) + 255) / 256), 256, 0, s>>>(r, ntiles);
    if (n > 0) k_splat_project<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(cam, rp, xyz, cov, color, n, r);
    const bool median = !(rp.tau > 0.0f);
    if (median && n > 0) launch_sort(r.sort, n, s);
    k_splat_tau<<<1, 32, 0, s>>>(r, rp.tau, r.sort.sorted_keys);
    k_tile_scan<<<1, 1024, 0, s>>>(r, ntiles);
    if (n > 0) k_splat_emit<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(cam, n, r);
    k_splat_tiles<<<(unsigned)((ntiles + kTileWarps - 1) / kTileWarps), 32 * kTileWarps, 0, s>>>(cam, rp, r, img,
                                                                                                   ntiles);
}

}  // namespace pm
