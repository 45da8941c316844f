// Gaussian-splat renderer (render.py:71-162 of the reference): EWA projection
// of 3D gaussians to screen-space gaussians, then the reference's two-pass
// soft z-buffer -- per pixel the nearest splat depth, then a blend of all
// splats weighted by exp(-(z - z_min) / tau) -- and coverage compositing over
// a background.  The image is a headless device buffer (H, W, 3).
//
// Kernels: k_splat_project (one thread per gaussian: camera transform,
// Jacobian, 2D covariance + 0.3 dilation, conic, radius, culling; depth key
// for the median), the radix sort of the depth keys when tau is derived from
// the median depth, k_splat_zmin and k_splat_blend (one warp per gaussian,
// lanes over its footprint pixels, float atomics into the pixel buffers) and
// k_splat_compose (one thread per pixel).
#include "pm_kernels.cuh"

namespace pm {
namespace {

struct Splat {
    float u, v, z, c00, c01, c11;
    int u0, v0, rad;
};

struct RenderWS {
    float *u, *v, *z, *c00, *c01, *c11;
    int *u0, *v0, *rad;
    int *list;        // compacted drawn splats
    unsigned *count;  // [0] drawn splats
    float *tau;       // [0] tau, [1] 1 / tau
    float *zmin, *logrev;
    float4 *csum;     // per pixel: colour sums (x, y, z) and weight sum (w)
    WS sort;          // key / value buffers of the median sort
};

__global__ void __launch_bounds__(256) k_splat_clear(RenderWS r, long long npix, unsigned *count) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *count = 0;
    if (i < npix) {
        r.zmin[i] = __int_as_float(0x7f800000);   // +inf
        r.csum[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        r.logrev[i] = 0.0f;
    }
}

__global__ void __launch_bounds__(256) k_splat_project(const pm_camera cam, const pm_render_params rp,
                                                       const float *__restrict__ xyz, const float *__restrict__ cov,
                                                       long long n, RenderWS r) {
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
    r.u[i] = u; r.v[i] = v; r.z[i] = z;
    r.c00[i] = c00; r.c01[i] = c01; r.c11[i] = c11;
    r.u0[i] = u0; r.v0[i] = v0; r.rad[i] = ok ? rad : 0;
    // depth key for the median of the drawn splats (z > near > 0: the float bits order like the values)
    r.sort.keys_a[i] = ok ? __float_as_uint(z) : 0xffffffffu;
    r.sort.vals_a[i] = (int)i;
    if (ok) r.list[atomicAdd(r.count, 1u)] = (int)i;
}

// tau = 0.02 * median depth (torch.median: the lower middle element), or the given tau
__global__ void k_splat_tau(RenderWS r, float tau_given, const unsigned *sorted) {
    if (threadIdx.x != 0) return;
    float tau = tau_given;
    if (!(tau_given > 0.0f)) {
        const unsigned c = *r.count;
        tau = c > 0 ? 0.02f * __uint_as_float(sorted[(c - 1) / 2]) : 1.0f;
    }
    r.tau[0] = tau;
    r.tau[1] = 1.0f / (tau > 1e-6f ? tau : 1e-6f);
}

// One drawn splat, held in registers for its footprint loop.
struct SplatR {
    float u, v, z, c00, c01, c11;
    int u0, v0, rad, side;
    FastDiv fside;
};

__device__ __forceinline__ SplatR load_splat(const RenderWS &r, int g) {
    SplatR q;
    q.u = r.u[g]; q.v = r.v[g]; q.z = r.z[g];
    q.c00 = r.c00[g]; q.c01 = r.c01[g]; q.c11 = r.c11[g];
    q.u0 = r.u0[g]; q.v0 = r.v0[g]; q.rad = r.rad[g];
    q.side = 2 * q.rad + 1;
    q.fside = make_fastdiv(q.side);
    return q;
}

// Footprint pixel k of the splat: its screen coordinates and alpha
// exp(min(power, 0)), or false when the pixel is off screen or its alpha is
// not above 1/255.  A power below -6 gives exp(power) < 0.0025 < 1/255, so
// those pixels are dropped before the exponential with the same outcome.
__device__ __forceinline__ bool splat_pixel(const SplatR &q, int k, int W, int H, int &px, int &py, float &ga) {
    const int ky = fdiv(k, q.fside), kx = k - ky * q.side;
    px = q.u0 + kx - q.rad;
    py = q.v0 + ky - q.rad;
    if (px < 0 || px >= W || py < 0 || py >= H) return false;
    const float dx = (float)px + 0.5f - q.u, dy = (float)py + 0.5f - q.v;
    const float power = -0.5f * (q.c00 * dx * dx + q.c11 * dy * dy) - q.c01 * dx * dy;
    if (power < -6.0f) return false;
    ga = expf(power < 0.0f ? power : 0.0f);
    return ga > (1.0f / 255.0f);
}

// pass 1: nearest depth per pixel (z > 0: int ordering of the bits)
__global__ void __launch_bounds__(256) k_splat_zmin(const pm_camera cam, RenderWS r) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (warp >= (int)*r.count) return;
    const SplatR q = load_splat(r, r.list[warp]);
    const int zb = __float_as_int(q.z), W = cam.width, H = cam.height, nk = q.side * q.side;
    int *zmin = reinterpret_cast<int *>(r.zmin);
    for (int k = lane; k < nk; k += 32) {
        int px, py;
        float ga;
        if (!splat_pixel(q, k, W, H, px, py, ga)) continue;
        int *zp = zmin + (long long)py * W + px;
        if (zb < __ldcg(zp)) atomicMin(zp, zb);   // the stored depth only decreases: skip the atomic when nearer
    }
}

// pass 2: soft-z-buffer blend
__global__ void __launch_bounds__(256) k_splat_blend(const pm_camera cam, RenderWS r, const float *__restrict__ color) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (warp >= (int)*r.count) return;
    const int g = r.list[warp];
    const SplatR q = load_splat(r, g);
    const float inv_tau = r.tau[1];
    const float c0 = color[3 * g], c1 = color[3 * g + 1], c2 = color[3 * g + 2];
    const int W = cam.width, H = cam.height, nk = q.side * q.side;
    for (int k = lane; k < nk; k += 32) {
        int px, py;
        float ga;
        if (!splat_pixel(q, k, W, H, px, py, ga)) continue;
        const long long pix = (long long)py * W + px;
        const float w = ga * expf(-(q.z - __ldcg(&r.zmin[pix])) * inv_tau);
        atomicAdd(&r.csum[pix], make_float4(c0 * w, c1 * w, c2 * w, w));
        const float om = 1.0f - ga;
        atomicAdd(&r.logrev[pix], logf(om > 1e-6f ? om : 1e-6f));
    }
}

__global__ void __launch_bounds__(256) k_splat_compose(const pm_render_params rp, RenderWS r, long long npix,
                                                       float *__restrict__ img) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const float cover = 1.0f - expf(r.logrev[i]);
    const float4 cs = r.csum[i];
    const float ws = cs.w, csum[3] = {cs.x, cs.y, cs.z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float rgb = ws > 1e-8f ? csum[c] / (ws > 1e-8f ? ws : 1e-8f) : rp.bg[c];
        float o = rgb * cover + rp.bg[c] * (1.0f - cover);
        o = o < 0.0f ? 0.0f : (o > 1.0f ? 1.0f : o);
        img[3 * i + c] = o;
    }
}

struct RenderLayout {
    Layout sort;
    size_t u, v, z, c00, c01, c11, u0, v0, rad, list, count, tau, zmin, csum, logrev, total;
};

RenderLayout make_render_layout(long long n, long long npix) {
    RenderLayout R;
    R.sort = make_layout_sized(n, 0, 0, 32, 1, 0);
    const size_t A = 256, nn = (size_t)(n > 0 ? n : 1), np = (size_t)npix;
    size_t o = R.sort.total;
    R.u = o;      o = align_up(o + 4 * nn, A);
    R.v = o;      o = align_up(o + 4 * nn, A);
    R.z = o;      o = align_up(o + 4 * nn, A);
    R.c00 = o;    o = align_up(o + 4 * nn, A);
    R.c01 = o;    o = align_up(o + 4 * nn, A);
    R.c11 = o;    o = align_up(o + 4 * nn, A);
    R.u0 = o;     o = align_up(o + 4 * nn, A);
    R.v0 = o;     o = align_up(o + 4 * nn, A);
    R.rad = o;    o = align_up(o + 4 * nn, A);
    R.list = o;   o = align_up(o + 4 * nn, A);
    R.count = o;  o = align_up(o + 16, A);
    R.tau = o;    o = align_up(o + 16, A);
    R.zmin = o;   o = align_up(o + 4 * np, A);
    R.csum = o;   o = align_up(o + 16 * np, A);
    R.logrev = o; o = align_up(o + 4 * np, A);
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
    if (b < 0 || b >= P.n) return;
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

size_t render_workspace_bytes(long long n, long long npix) { return make_render_layout(n, npix).total; }

void launch_render(const pm_camera &cam, const pm_render_params &rp, const float *xyz, const float *cov,
                   const float *color, long long n, float *img, void *ws, cudaStream_t s) {
    const long long npix = (long long)cam.width * cam.height;
    const RenderLayout L = make_render_layout(n, npix);
    char *b = (char *)ws;
    RenderWS r;
    r.u = (float *)(b + L.u); r.v = (float *)(b + L.v); r.z = (float *)(b + L.z);
    r.c00 = (float *)(b + L.c00); r.c01 = (float *)(b + L.c01); r.c11 = (float *)(b + L.c11);
    r.u0 = (int *)(b + L.u0); r.v0 = (int *)(b + L.v0); r.rad = (int *)(b + L.rad);
    r.list = (int *)(b + L.list);
    r.count = (unsigned *)(b + L.count);
    r.tau = (float *)(b + L.tau);
    r.zmin = (float *)(b + L.zmin); r.csum = (float4 *)(b + L.csum);
    r.logrev = (float *)(b + L.logrev);
    r.sort = make_ws(ws, L.sort);
    const unsigned pb = (unsigned)((npix + 255) / 256);
    k_splat_clear<<<pb > 0 ? pb : 1, 256, 0, s>>>(r, npix, r.count);
    if (n > 0) k_splat_project<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(cam, rp, xyz, cov, n, r);
    const bool median = !(rp.tau > 0.0f);
    if (median && n > 0) launch_sort(r.sort, n, s);
    k_splat_tau<<<1, 32, 0, s>>>(r, rp.tau, r.sort.sorted_keys);
    if (n > 0) {
        const unsigned wb = (unsigned)((n * 32 + 255) / 256);   // one warp per gaussian (the drawn ones act)
        k_splat_zmin<<<wb, 256, 0, s>>>(cam, r);
        k_splat_blend<<<wb, 256, 0, s>>>(cam, r, color);
    }
    k_splat_compose<<<pb > 0 ? pb : 1, 256, 0, s>>>(rp, r, npix, img);
}

}  // namespace pm
