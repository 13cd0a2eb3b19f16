// M-step reconstruction on the device: the real-space map of a backprojection
// grid, the half-map FSC and the SSNR arrays.
//
// t2b_reconstruct follows BackProjector::reconstruct on the reference's default
// skip-gridding path (src/backprojector.cpp:1344-1530; skip_gridding =
// !--dont_skip_gridding, src/ml_optimiser.cpp:525): decenter (r^2 <= ROUND(r_max
// pad)^2), the MAP term 1 / (pad^3 tau2_fudge tau2) added to the weights
// (:1412-1455), the FP64 division by max(weight, radial average / 1000)
// (:1463-1531; the kernels of t2b_reconstruct_divide), then
// windowToOridimRealSpace (:2486-2620) and Projector::griddingCorrect
// (src/projector.cpp:489-522):
//   window the pad_size transform to pad * ori_size (src/fftw.h:736-790),
//   CenterFFTbySign, unnormalised inverse 3D FFT, real-space window to
//   ori_size, divide by pad^3 ori_size (2D particles), softMaskOutsideMap
//   (radius ori_size / 2, cosine width 3, average background), divide by
//   sinc^2(r / (ori_size pad)).
// The inverse transform is three passes of batched 1D FFTs in shared memory
// (fft_smem.cuh): columns along z, columns along y of the planes inside the
// real-space window, and the c2r rows of the window only; FP32 (the division
// before it and every sum after it are FP64).
//
// t2b_fsc_halves: getDownsampledAverage + calculateDownSampledFourierShellCorrelation
// (src/backprojector.cpp:933-1040).  t2b_update_ssnr: updateSSNRarrays
// (:1041-1205).  Both reduce the grid on the device (FP64 atomics into shell
// and down-sampled bins) and finish the per-shell arithmetic on the host.
#include "t2b_internal.cuh"
#include "fft_smem.cuh"

#include <array>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace t2b {

constexpr double PI_R = 3.14159265358979323846;

namespace {

constexpr int RC_THREADS = 256;
constexpr int RC_CX = 16;   // columns per CTA in the z and y passes
constexpr int RC_ROWS = 8;  // rows per CTA in the x pass

__device__ __forceinline__ int rround(double x) { return x > 0 ? (int)(x + 0.5) : (int)(x - 0.5); }

// the pad_size transform (FFTW layout, double2) -> the N = pad * ori_size half
// transform (float2), windowed (shrink: every output element; enlarge: input
// elements with r^2 <= (ps/2)^2) and centred by sign
__global__ void k_window(const double2* __restrict__ fc, int ps, int N, int dim, float2* __restrict__ G)
{
    const int h = N / 2 + 1, half = ps / 2, fx = ps / 2 + 1;
    const long long total = (long long)(dim == 3 ? N : 1) * N * h;   // 2D: one plane
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(n % h);
        const int i = (int)((n / h) % N);
        const int k = (int)(n / ((long long)h * N));
        const int kp = k < h ? k : k - N, ip = i < h ? i : i - N;
        float2 v = make_float2(0.f, 0.f);
        bool ok = kp >= -half && kp <= half && ip >= -half && ip <= half && j <= half;
        if (ok && N > ps) ok = kp * kp + ip * ip + j * j <= half * half;
        if (ok) {
            const double2 d = fc[((size_t)(kp < 0 ? kp + ps : kp) * ps + (ip < 0 ? ip + ps : ip)) * fx + j];
            const float sg = ((k ^ i ^ j) & 1) ? -1.f : 1.f;
            v = make_float2((float)d.x * sg, (float)d.y * sg);
        }
        G[n] = v;
    }
}

// inverse FFT of RC_CX columns along one axis: axis 0 = z (line index y = blockIdx.x),
// axis 1 = y (plane z = z0 + blockIdx.x); x tile = blockIdx.y
template <int NC>
__global__ void __launch_bounds__(RC_THREADS) k_cols3(float2* __restrict__ G, int Nrt, int axis, int z0,
                                                      const float2* __restrict__ tw, FftPlan plan)
{
    extern __shared__ float2 sm[];
    const int N = NC > 0 ? NC : Nrt, h = N / 2 + 1;
    float2* s_tw = sm;
    float2* A = sm + N;
    float2* B = A + RC_CX * N;
    for (int t = threadIdx.x; t < N; t += blockDim.x) s_tw[t] = tw[t];
    const int x0 = blockIdx.y * RC_CX;
    const size_t line = blockIdx.x;
    // element q of column c: axis 0: (q, line, x0 + c); axis 1: (z0 + line, q, x0 + c)
    auto idx = [&](int q, int c) -> size_t {
        return axis == 0 ? ((size_t)q * N + line) * h + x0 + c : (((size_t)z0 + line) * N + q) * h + x0 + c;
    };
    for (int e = threadIdx.x; e < RC_CX * N; e += blockDim.x) {
        const int c = e % RC_CX, q = e / RC_CX;
        A[c * N + q] = x0 + c < h ? G[idx(q, c)] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const float2* r = fft_any<NC, true>(A, B, RC_CX, plan, s_tw);
    for (int e = threadIdx.x; e < RC_CX * N; e += blockDim.x) {
        const int c = e % RC_CX, q = e / RC_CX;
        if (x0 + c < h) G[idx(q, c)] = r[c * N + q];
    }
}

// c2r rows (imaginary parts of x = 0 and N/2 dropped) of the real-space window:
// row (z0 + zw, z0 + yw) -> vol[zw][yw][0..ori) (2D: row z0 + yw of the single plane),
// divided by the FFT normalisation
template <int NC>
__global__ void __launch_bounds__(RC_THREADS) k_rows3(const float2* __restrict__ G, int Nrt, int ori, int z0,
                                                      float norm, const float2* __restrict__ tw, FftPlan plan,
                                                      float* __restrict__ vol, int dim)
{
    extern __shared__ float2 sm[];
    const int N = NC > 0 ? NC : Nrt, h = N / 2 + 1;
    float2* s_tw = sm;
    float2* A = sm + N;
    float2* B = A + RC_ROWS * N;
    for (int t = threadIdx.x; t < N; t += blockDim.x) s_tw[t] = tw[t];
    const int row0 = blockIdx.x * RC_ROWS;
    const int nrows = dim == 3 ? ori * ori : ori;
    for (int e = threadIdx.x; e < RC_ROWS * N; e += blockDim.x) {
        const int rr = e / N, k = e - rr * N, row = row0 + rr;
        float2 v = make_float2(0.f, 0.f);
        if (row < nrows) {
            const int zw = row / ori, yw = row - zw * ori;
            const float2* g = G + ((dim == 3 ? (size_t)z0 + zw : (size_t)0) * N + z0 + yw) * h;
            if (k == 0 || k == N / 2) v = make_float2(g[k].x, 0.f);
            else if (k < N / 2) v = g[k];
            else v = make_float2(g[N - k].x, -g[N - k].y);
        }
        A[e] = v;
    }
    __syncthreads();
    const float2* r = fft_any<NC, true>(A, B, RC_ROWS, plan, s_tw);
    for (int e = threadIdx.x; e < RC_ROWS * ori; e += blockDim.x) {
        const int rr = e / ori, x = e - rr * ori, row = row0 + rr;
        if (row < nrows) vol[(size_t)row * ori + x] = r[rr * N + z0 + x].x / norm;
    }
}

// soft-mask background (softMaskOutsideMap without a noise image), fixed-order FP64
// partial sums per block
__global__ void __launch_bounds__(RC_THREADS) k_mask_partial(const float* __restrict__ vol, int ori, int dim,
                                                             double radius, double width, double2* __restrict__ part)
{
    __shared__ double sw[RC_THREADS], sv[RC_THREADS];
    const long long total = (long long)ori * ori * (dim == 3 ? ori : 1);
    double aw = 0., av = 0.;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(n % ori), y = (int)((n / ori) % ori), z = (int)(n / ((long long)ori * ori));
        const double xl = x - ori / 2, yl = y - ori / 2, zl = dim == 3 ? z - ori / 2 : 0;
        const double r = sqrt(xl * xl + yl * yl + zl * zl);
        if (r < radius) continue;
        const double rp = radius + width;
        const double w = r > rp ? 1. : 0.5 + 0.5 * cos(PI_R * (rp - r) / width);
        aw += w;
        av += w * vol[n];
    }
    sw[threadIdx.x] = aw;
    sv[threadIdx.x] = av;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sw[threadIdx.x] += sw[threadIdx.x + o];
            sv[threadIdx.x] += sv[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = make_double2(sw[0], sv[0]);
}

// soft mask with the background, then the gridding correction (trilinear: sinc^2)
__global__ void k_mask_grid(const float* __restrict__ vol, int ori, int dim, int pad, double radius, double width,
                            const double2* __restrict__ part, int nparts, double* __restrict__ out)
{
    __shared__ double s_bg;
    if (threadIdx.x == 0) {
        double w = 0., v = 0.;
        for (int b = 0; b < nparts; ++b) {
            w += part[b].x;
            v += part[b].y;
        }
        s_bg = w > 0. ? v / w : 0.;
    }
    __syncthreads();
    const double bg = s_bg;
    const long long total = (long long)ori * ori * (dim == 3 ? ori : 1);
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(n % ori), y = (int)((n / ori) % ori), z = (int)(n / ((long long)ori * ori));
        const double xl = x - ori / 2, yl = y - ori / 2, zl = dim == 3 ? z - ori / 2 : 0;
        const double r = sqrt(xl * xl + yl * yl + zl * zl);
        double v = vol[n];
        if (r >= radius) {
            const double rp = radius + width;
            if (r > rp) v = bg;
            else {
                const double w = 0.5 + 0.5 * cos(PI_R * (rp - r) / width);
                v = (1. - w) * v + w * bg;
            }
        }
        if (r > 0.) {
            const double rv = r / ((double)ori * pad);
            const double sn = sin(PI_R * rv) / (PI_R * rv);
            v /= sn * sn;
        }
        out[n] = v;
    }
}

// ---------------------------------------------------------------- FSC and SSNR
__global__ void k_downsample(Volume g, const float2* __restrict__ data, const float* __restrict__ weight,
                             double* __restrict__ acc /* bins x 3 */)
{
    const int ds = 2 * (g.r_max + 1) + 1, dh = ds / 2;
    const long long total = (long long)g.zdim * g.ydim * g.xdim;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(n % g.xdim), i = (int)((n / g.xdim) % g.ydim), k = (int)(n / ((long long)g.xdim * g.ydim));
        const int kp = g.ref_dim == 3 ? rround((double)(k + g.initz) / g.pad) + dh : 0;   // 2D: one plane
        const int ip = rround((double)(i + g.inity) / g.pad) + dh;
        const int jp = rround((double)j / g.pad);
        if (kp < 0 || kp >= (g.ref_dim == 3 ? ds : 1) || ip < 0 || ip >= ds || jp > dh) continue;   // a grid larger than pad_size
        const size_t b = (((size_t)kp * ds + ip) * (dh + 1) + jp) * 3;
        const float2 d = data[n];
        const float w = weight[n];
        if (d.x != 0.f) atomicAdd(&acc[b], (double)d.x);
        if (d.y != 0.f) atomicAdd(&acc[b + 1], (double)d.y);
        if (w != 0.f) atomicAdd(&acc[b + 2], (double)w);
    }
}

// shell sums: FP64 shared-memory bins per block, one global atomic per bin and block
__device__ __forceinline__ void shell_init(double* sb, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) sb[i] = 0.;
    __syncthreads();
}
__device__ __forceinline__ void shell_flush(const double* sb, int n, double* acc)
{
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (sb[i] != 0.) atomicAdd(&acc[i], sb[i]);
}

__global__ void k_fsc_shells(int r_max, int nb, int dim, const double* __restrict__ a1, const double* __restrict__ a2,
                             double* __restrict__ sh /* nb x 3 */)
{
    extern __shared__ double sb[];
    shell_init(sb, 3 * nb);
    const int ds = 2 * (r_max + 1) + 1, dh = ds / 2;
    const long long total = (long long)(dim == 3 ? ds : 1) * ds * (dh + 1);
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(n % (dh + 1)), i = (int)((n / (dh + 1)) % ds) - dh;
        const int k = dim == 3 ? (int)(n / ((long long)(dh + 1) * ds)) - dh : 0;
        const double R = sqrt((double)(k * k + i * i + j * j));
        if (R > r_max) continue;
        const int idx = rround(R);
        const double w1 = a1[3 * n + 2], w2 = a2[3 * n + 2];
        const double r1 = w1 > 0. ? a1[3 * n] / w1 : 0., i1 = w1 > 0. ? a1[3 * n + 1] / w1 : 0.;
        const double r2 = w2 > 0. ? a2[3 * n] / w2 : 0., i2 = w2 > 0. ? a2[3 * n + 1] / w2 : 0.;
        atomicAdd(&sb[3 * idx], r1 * r2 + i1 * i2);
        atomicAdd(&sb[3 * idx + 1], r1 * r1 + i1 * i1);
        atomicAdd(&sb[3 * idx + 2], r2 * r2 + i2 * i2);
    }
    shell_flush(sb, 3 * nb, sh);
}

// pass 1 of updateSSNRarrays: per shell, sum of pad^3 weight and count (r^2 < max_r2)
__global__ void k_ssnr_sigma(Volume g, int nb, const float* __restrict__ weight, double oc, double* __restrict__ acc)
{
    extern __shared__ double sb[];
    shell_init(sb, 2 * nb);
    const int rp = g.r_max * g.pad;
    const long long total = (long long)g.zdim * g.ydim * g.xdim;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(n % g.xdim), i = (int)((n / g.xdim) % g.ydim) + g.inity, k = (int)(n / ((long long)g.xdim * g.ydim)) + g.initz;
        const int r2 = k * k + i * i + j * j;
        if (r2 >= rp * rp) continue;
        const int ires = rround(sqrt((double)r2) / g.pad);
        atomicAdd(&sb[2 * ires], oc * weight[n]);
        atomicAdd(&sb[2 * ires + 1], 1.);
    }
    shell_flush(sb, 2 * nb, acc);
}

// pass 2: per shell, sum of weight / invtau2 (data vs prior), coverage count, count
__global__ void k_ssnr_prior(Volume g, int nb, const float* __restrict__ weight, double oc, double tau2_fudge,
                             const double* __restrict__ tau2, const double* __restrict__ avgctf2, int correct_ctf2,
                             double* __restrict__ acc)
{
    extern __shared__ double sb[];
    shell_init(sb, 3 * nb);
    const int rp = g.r_max * g.pad;
    const long long total = (long long)g.zdim * g.ydim * g.xdim;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(n % g.xdim), i = (int)((n / g.xdim) % g.ydim) + g.inity, k = (int)(n / ((long long)g.xdim * g.ydim)) + g.initz;
        const int r2 = k * k + i * i + j * j;
        if (r2 >= rp * rp) continue;
        const int ires = rround(sqrt((double)r2) / g.pad);
        const double invw = weight[n];
        double invtau2;
        if (tau2[ires] > 0.) {
            invtau2 = 1. / (oc * tau2_fudge * tau2[ires]);
            if (correct_ctf2 && avgctf2[ires] > 0.) invtau2 *= 1. / avgctf2[ires];
        } else {
            invtau2 = 1. / (0.001 * invw);
        }
        const double ratio = invw / invtau2;
        atomicAdd(&sb[3 * ires], ratio);
        if (ratio >= 1.) atomicAdd(&sb[3 * ires + 1], 1.);
        atomicAdd(&sb[3 * ires + 2], 1.);
    }
    shell_flush(sb, 3 * nb, acc);
}

// BackProjector::enforceHermitianSymmetry (src/backprojector.cpp:2104-2121) on the x = 0
// plane: every Friedel pair (z, y) <-> (-z, -y) once (z < 0 with y >= 0, or z >= 0 with
// y >= 1), both members set to the data sum (conjugated on the partner) and the weight sum.
// The visited set and the partners' set are disjoint, so one thread per pair writes without
// conflicts.  Grids are centred: (z, y) at ((z - initz) * ydim + (y - inity)) * xdim.
__global__ void k_hermitian(Volume g, float2* __restrict__ data, float* __restrict__ weight)
{
    const int zlo = g.initz, zhi = g.initz + g.zdim - 1;
    const int ylo = g.inity, yhi = g.inity + g.ydim - 1;
    const int ny = yhi + 1;                       // y = 0 .. yhi
    const long long total = (long long)g.zdim * ny;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int z = zlo + (int)(i / ny), y = (int)(i % ny);
        if (z >= 0 && y == 0) continue;           // starty = (iz < 0) ? 0 : 1
        const int mz = -z, my = -y;
        if (mz < zlo || mz > zhi || my < ylo) continue;
        const size_t a = ((size_t)(z - g.initz) * g.ydim + (y - g.inity)) * g.xdim;
        const size_t b = ((size_t)(mz - g.initz) * g.ydim + (my - g.inity)) * g.xdim;
        const float2 da = data[a], db = data[b];
        const float2 f = make_float2(da.x + db.x, da.y - db.y);
        data[a] = f;
        data[b] = make_float2(f.x, -f.y);
        const float w = weight[a] + weight[b];
        weight[a] = w;
        weight[b] = w;
    }
}

// ---- gridding iterations (BackProjector::reconstruct with max_iter_preweight > 0,
// src/backprojector.cpp:1532-1655): weights w_n (FP64, FFTW layout of the pad_size box)
// start at 1 inside r^2 < max_r2; each iteration convolves w_n * weight with the blob
// through the Fourier transform of the full box (BackProjector::convoluteBlobRealSpace,
// :2439-2480) and divides w_n by max(1e-6, |result|) inside max_r2.  The half-complex grids
// are expanded to the full complex box by Hermitian symmetry (the box is odd: no Nyquist
// plane), transformed by the shared-memory FFTs along x, y and z, multiplied in real space
// by the blob's tabulated Fourier transform over its value at 0, and transformed back.
constexpr int GD_CX = 8;   // lines per CTA of the full-box transforms

// data and weight divided by `normalise`; w_n = 1 inside r^2 < max_r2, else 0
__global__ void k_gd_init(double2* __restrict__ fc, double* __restrict__ fw, double* __restrict__ fn, int ps, int nz,
                          int max_r2, double inv_norm)
{
    const int fx = ps / 2 + 1;
    const long long total = (long long)nz * ps * fx;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(n % fx), i = (int)((n / fx) % ps), k = (int)(n / ((long long)fx * ps));
        const int kp = k < fx ? k : k - ps, ip = i < fx ? i : i - ps;
        const double2 d = fc[n];
        fc[n] = make_double2(d.x * inv_norm, d.y * inv_norm);
        fw[n] *= inv_norm;
        fn[n] = kp * kp + ip * ip + j * j < max_r2 ? 1. : 0.;
    }
}

// the full box V[z][y][x] (2D: one plane) of w_n * weight (real), from the half by Hermitian
// symmetry: x > ps/2 reads (-z, -y, ps - x)
__global__ void k_gd_expand(const double* __restrict__ fn, const double* __restrict__ fw, int ps, int nz,
                            float2* __restrict__ V)
{
    const int fx = ps / 2 + 1;
    const long long total = (long long)nz * ps * ps;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(n % ps), y = (int)((n / ps) % ps), z = (int)(n / ((long long)ps * ps));
        size_t h;
        if (x < fx) h = ((size_t)z * ps + y) * fx + x;
        else h = ((size_t)(nz == 1 ? 0 : (ps - z) % ps) * ps + (ps - y) % ps) * fx + (ps - x);
        V[n] = make_float2((float)(fn[h] * fw[h]), 0.f);
    }
}

// FFT of GD_CX lines of the full box along one axis: axis 0 = x (rows blockIdx.x * GD_CX + c),
// axis 1 = y (plane z = blockIdx.x), axis 2 = z (row y = blockIdx.x); x tile blockIdx.y
template <bool INV>
__global__ void __launch_bounds__(RC_THREADS) k_gd_fft(float2* __restrict__ V, int N, int nz, int axis,
                                                       const float2* __restrict__ tw, FftPlan plan)
{
    extern __shared__ float2 sm[];
    float2* s_tw = sm;
    float2* A = sm + N;
    float2* B = A + GD_CX * N;
    for (int t = threadIdx.x; t < N; t += blockDim.x) s_tw[t] = tw[t];
    const long long nrows = (long long)nz * N;
    const size_t o = blockIdx.x;
    const int x0 = blockIdx.y * GD_CX;
    auto ok = [&](int c) -> bool { return axis == 0 ? (long long)o * GD_CX + c < nrows : x0 + c < N; };
    auto idx = [&](int q, int c) -> size_t {
        if (axis == 0) return ((size_t)o * GD_CX + c) * N + q;
        if (axis == 1) return (o * N + q) * N + x0 + c;
        return ((size_t)q * N + o) * N + x0 + c;
    };
    for (int e = threadIdx.x; e < GD_CX * N; e += blockDim.x) {
        // rows: consecutive threads along the row; columns: along x
        const int c = axis == 0 ? e / N : e % GD_CX, q = axis == 0 ? e % N : e / GD_CX;
        A[c * N + q] = ok(c) ? V[idx(q, c)] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const float2* r = fft_smem<INV, true>(A, B, GD_CX, plan, s_tw);
    for (int e = threadIdx.x; e < GD_CX * N; e += blockDim.x) {
        const int c = axis == 0 ? e / N : e % GD_CX, q = axis == 0 ? e % N : e / GD_CX;
        if (ok(c)) V[idx(q, c)] = r[c * N + q];
    }
}

// real space: multiply by the blob's tabulated Fourier transform at
// r = |(k, i, j)| / (ori_size pad) (coordinates k < ps/2 ? k : k - ps), entry floor(r / 5e-5),
// 0 beyond the table (TabFtBlob::operator(), src/tabfuncs.cpp:114-121); the imaginary part
// (rounding of a Hermitian transform) dropped
__global__ void k_gd_blob(float2* __restrict__ V, int N, int nz, const double* __restrict__ ratio, int ntab,
                          double ori_pad)
{
    const int ph = N / 2;
    const long long total = (long long)nz * N * N;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(n % N), y = (int)((n / N) % N), z = (int)(n / ((long long)N * N));
        const int kz = nz == 1 ? 0 : (z < ph ? z : z - N), ky = y < ph ? y : y - N, kx = x < ph ? x : x - N;
        const double rval = sqrt((double)(kz * kz + ky * ky + kx * kx)) / ori_pad;
        const int id = (int)(rval / (0.5 / (double)ntab));
        const double m = id < ntab ? ratio[id] : 0.;
        V[n] = make_float2((float)((double)V[n].x * m), 0.f);
    }
}

// w_n /= max(1e-6, |V| / N^d) inside r^2 < max_r2 (the forward transform's 1 / N^d here)
__global__ void k_gd_update(double* __restrict__ fn, const float2* __restrict__ V, int ps, int nz, int max_r2,
                            double inv_n)
{
    const int fx = ps / 2 + 1;
    const long long total = (long long)nz * ps * fx;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(n % fx), i = (int)((n / fx) % ps), k = (int)(n / ((long long)fx * ps));
        const int kp = k < fx ? k : k - ps, ip = i < fx ? i : i - ps;
        if (kp * kp + ip * ip + j * j >= max_r2) continue;
        const float2 v = V[((size_t)k * ps + i) * ps + j];
        const double a = sqrt((double)v.x * v.x + (double)v.y * v.y) * inv_n;
        fn[n] /= (a > 1e-6 ? a : 1e-6);
    }
}

// Fconv = data * w_n
__global__ void k_gd_apply(double2* __restrict__ fc, const double* __restrict__ fn, long long total)
{
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const double2 d = fc[n];
        fc[n] = make_double2(d.x * fn[n], d.y * fn[n]);
    }
}

// The blob's Fourier transform over its value at 0, 10,000 samples of [0, 0.5)
// (TabFtBlob::initialise(2 * 1.9, 15, 0, 10000), src/backprojector.h:111, src/tabfuncs.cpp:95-112):
// for the order-0 Kaiser-Bessel blob of radius a and taper alpha in 3D (Lewitt 1990),
// FT(w) = (2 pi)^(3/2) a^3 I_{3/2}(s) / (I_0(alpha) s^(3/2)), s = sqrt(alpha^2 - (2 pi a w)^2)
// (J_{3/2} of sqrt((2 pi a w)^2 - alpha^2) beyond 2 pi a w = alpha), with the half-integer
// Bessel functions in closed form.
std::vector<double> ftblob_ratio(int ntab)
{
    const double a = 3.8, alpha = 15.0;
    std::vector<double> t(ntab);
    for (int i = 0; i < ntab; ++i) {
        const double w = (double)i * (0.5 / (double)ntab);
        const double u = 2.0 * PI_R * a * w;
        const double sg = std::sqrt(std::fabs(alpha * alpha - u * u));
        const double pre = std::sqrt(2.0 / (PI_R * sg));
        const double bes = u > alpha ? pre * (std::sin(sg) / sg - std::cos(sg)) : pre * (std::cosh(sg) - std::sinh(sg) / sg);
        t[i] = bes / std::pow(sg, 1.5);   // the factor (2 pi)^(3/2) a^3 / I_0(alpha) cancels in the ratio
    }
    const double t0 = t[0];
    for (double& x : t) x /= t0;
    return t;
}

// ---- point-group symmetry (BackProjector::applyPointGroupSymmetry,
// src/backprojector.cpp:2279-2435): every voxel (x, y, z) of the grid inside r^2 <= ROUND(r_max pad)^2
// gets the sum, over the group's operators R other than the identity, of the grid read at
// R (x, y, z) by trilinear interpolation (the conjugate Friedel partner where the rotated x < 0),
// added to its own value; data and weight alike.  FP64 coordinates and sums, FP32 grids.
// With zsh (helical symmetry, BackProjector::applyHelicalSymmetry, src/backprojector.cpp:2122-2277),
// the data read for operator s is also multiplied by e^{2 pi i z zsh[s]} (z the voxel's own z;
// zsh[s] = hh rise / (-ori_size pad)), formed as the reference forms it: (ac - bd,
// (a + b)(c + d) - ac - bd).
__global__ void k_symmetrise(Volume g, const float2* __restrict__ data, const float* __restrict__ weight,
                             float2* __restrict__ sdata, float* __restrict__ sweight, const double* __restrict__ R,
                             const double* __restrict__ zsh, int nsym, int rmax2)
{
    const long long total = (long long)g.zdim * g.ydim * g.xdim;
    const size_t plane = (size_t)g.ydim * g.xdim;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < total; n += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(n % g.xdim), i = (int)((n / g.xdim) % g.ydim), k = (int)(n / (long long)plane);
        const int x = j, y = i + g.inity, z = k + g.initz;
        double sr = data[n].x, si = data[n].y, sw = weight[n];
        if (x * x + y * y + z * z <= rmax2) {
            for (int s = 0; s < nsym; ++s) {
                const double* m = R + 9 * s;
                // rounded products and sums in the reference's order (no contraction), so
                // that floor() and the sign test see the reference's coordinates
                double xp = __dadd_rn(__dadd_rn(__dmul_rn(x, m[0]), __dmul_rn(y, m[1])), __dmul_rn(z, m[2]));
                double yp = __dadd_rn(__dadd_rn(__dmul_rn(x, m[3]), __dmul_rn(y, m[4])), __dmul_rn(z, m[5]));
                double zp = __dadd_rn(__dadd_rn(__dmul_rn(x, m[6]), __dmul_rn(y, m[7])), __dmul_rn(z, m[8]));
                const bool neg = xp < 0;
                if (neg) { xp = -xp; yp = -yp; zp = -zp; }
                const int x0 = (int)floor(xp), y0f = (int)floor(yp), z0f = (int)floor(zp);
                const double fx = xp - x0, fy = yp - y0f, fz = zp - z0f;
                const int y0 = y0f - g.inity, z0 = z0f - g.initz;
                if (x0 < 0 || x0 + 1 >= g.xdim || y0 < 0 || y0 + 1 >= g.ydim || z0 < 0 || z0 + 1 >= g.zdim) continue;
                const size_t b = ((size_t)z0 * g.ydim + y0) * g.xdim + x0;
                const size_t c[8] = {b, b + 1, b + g.xdim, b + g.xdim + 1,
                                     b + plane, b + plane + 1, b + plane + g.xdim, b + plane + g.xdim + 1};
                // (z, y, x) corners: 000 001 010 011 100 101 110 111
                double dr[8], di[8], dw[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    dr[q] = data[c[q]].x;
                    di[q] = data[c[q]].y;
                    dw[q] = weight[c[q]];
                }
                const auto tri = [&](const double* d) {
                    const double x00 = d[0] + (d[1] - d[0]) * fx, x01 = d[4] + (d[5] - d[4]) * fx;
                    const double x10 = d[2] + (d[3] - d[2]) * fx, x11 = d[6] + (d[7] - d[6]) * fx;
                    const double y0v = x00 + (x10 - x00) * fy, y1v = x01 + (x11 - x01) * fy;
                    return y0v + (y1v - y0v) * fz;
                };
                double cr = tri(dr), ci = neg ? -tri(di) : tri(di);
                if (zsh && zsh[s] != 0.) {
                    double sn, cs;
                    sincos(2. * PI_R * (z * zsh[s]), &sn, &cs);
                    const double ac = cs * cr, bd = sn * ci, abcd = (cs + sn) * (cr + ci);
                    cr = ac - bd;
                    ci = abcd - ac - bd;
                }
                sr += cr;
                si += ci;
                sw += tri(dw);
            }
        }
        sdata[n] = make_float2((float)sr, (float)si);
        sweight[n] = (float)sw;
    }
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    explicit DevBuf(size_t n)
    {
        if (cudaMalloc(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            throw Error{T2B_ERR_NOMEM, "reconstruction buffers"};
        }
    }
    ~DevBuf() { cudaFree(p); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

using ColKernel = void (*)(float2*, int, int, int, const float2*, FftPlan);
using RowKernel = void (*)(const float2*, int, int, int, float, const float2*, FftPlan, float*, int);

void recon_kernels(int N, ColKernel& col, RowKernel& row)
{
    if (N == 256) { col = k_cols3<256>; row = k_rows3<256>; }
    else if (N == 128) { col = k_cols3<128>; row = k_rows3<128>; }
    else { col = k_cols3<0>; row = k_rows3<0>; }
}

int grid_of(long long total)
{
    return (int)std::min<long long>((total + RC_THREADS - 1) / RC_THREADS, 148LL * 16);
}

// the gridding iterations on (fc, fw) of the pad_size box, in place: fc becomes data * w_n
void gridding_weights(const Volume& v, int ori, int pad, int niter, double normalise, double2* fc, double* fw,
                      cudaStream_t st)
{
    const int ps = v.ydim, nz = v.ref_dim == 3 ? ps : 1, fx = ps / 2 + 1;
    const int rp = v.r_max * pad;
    const int max_r2 = rp * rp;
    const long long nh = (long long)nz * ps * fx, nf = (long long)nz * ps * ps;
    const size_t smem = sizeof(float2) * ((size_t)ps + 2 * (size_t)GD_CX * ps);
    T2B_REQUIRE(smem <= 227 * 1024, T2B_ERR_UNSUPPORTED, "pad_size box too large for the gridding transforms");
    const FftPlan plan = fft_plan(ps, true);
    constexpr int ntab = 10000;
    DevBuf<double> fn(nh), ratio(ntab);
    DevBuf<float2> V(nf), tw(ps);
    std::vector<float2> htw(ps);
    for (int t = 0; t < ps; ++t) {
        const double a = -2.0 * PI_R * (double)t / (double)ps;
        htw[t] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    const std::vector<double> hr = ftblob_ratio(ntab);
    T2B_CUDA(cudaMemcpyAsync(tw.p, htw.data(), ps * sizeof(float2), cudaMemcpyHostToDevice, st));
    T2B_CUDA(cudaMemcpyAsync(ratio.p, hr.data(), ntab * sizeof(double), cudaMemcpyHostToDevice, st));
    T2B_CUDA(cudaFuncSetAttribute((const void*)k_gd_fft<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    T2B_CUDA(cudaFuncSetAttribute((const void*)k_gd_fft<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int xt = (ps + GD_CX - 1) / GD_CX;
    const auto fft3 = [&](auto kern) {
        kern<<<(int)((nz * (long long)ps + GD_CX - 1) / GD_CX), RC_THREADS, smem, st>>>(V.p, ps, nz, 0, tw.p, plan);
        kern<<<dim3(nz, xt), RC_THREADS, smem, st>>>(V.p, ps, nz, 1, tw.p, plan);
        if (nz > 1) kern<<<dim3(ps, xt), RC_THREADS, smem, st>>>(V.p, ps, nz, 2, tw.p, plan);
    };
    const double inv_n = 1.0 / ((double)ps * ps * (nz > 1 ? ps : 1));
    k_gd_init<<<grid_of(nh), RC_THREADS, 0, st>>>(fc, fw, fn.p, ps, nz, max_r2, 1.0 / normalise);
    for (int it = 0; it < niter; ++it) {
        k_gd_expand<<<grid_of(nf), RC_THREADS, 0, st>>>(fn.p, fw, ps, nz, V.p);
        fft3(k_gd_fft<true>);
        k_gd_blob<<<grid_of(nf), RC_THREADS, 0, st>>>(V.p, ps, nz, ratio.p, ntab, (double)ori * pad);
        fft3(k_gd_fft<false>);
        k_gd_update<<<grid_of(nh), RC_THREADS, 0, st>>>(fn.p, V.p, ps, nz, max_r2, inv_n);
    }
    k_gd_apply<<<grid_of(nh), RC_THREADS, 0, st>>>(fc, fn.p, nh);
    T2B_CUDA(cudaGetLastError());
    T2B_CUDA(cudaStreamSynchronize(st));   // the buffers above are freed on return
}

const Volume& grid_volume(t2b_ctx* c, int ig)
{
    T2B_REQUIRE(ig >= 0 && ig < (int)c->gvol.size() && c->gdata[ig], T2B_ERR_ARG, "no such grid");
    const Volume& v = c->gvol[ig];
    T2B_REQUIRE(v.ref_dim == 3 || v.ref_dim == 2, T2B_ERR_UNSUPPORTED, "grids are 2D or 3D");
    return v;
}

// The operators of a point group, 3 x 3 row-major, the identity excluded, as SymList builds
// them (SymList::read_sym_file + compute_subgroup, src/symmetries.cpp:133-191, 243-325):
//  - a rotation axis of order n gives the rotations k * 360 / n about it, transposed, entries
//    below 1e-6 set to 0;
//  - a mirror plane with unit normal u gives I - 2 u u^T (the reference's A^T diag(1, 1, -1) A,
//    A turning u onto z), an inversion -I; the reference pairs every operator with a second
//    matrix L, diag(1, 1, -1) for the inversion and the identity otherwise, and so do we (lz);
//  - then every product in the reference's order: shells n = 0, 1, ..., the pairs (i, n) for
//    i = 0..n, then (n, j) for j = n-1..0 (found_not_tried), appended unless it is the identity
//    or equals a listed operator (L and R within 1e-6), zeroed below 1e-6.  The order fixes
//    which chain of products each operator comes from, and so its last digits (the generating
//    axes carry six to ten).
// The generators are the reference's (SymList::fill_symmetry_class, src/symmetries.cpp:606-725),
// the names as SymList::isSymmetryGroup reads them (:331-600: case-insensitive, orders of one or
// two digits): C1, Cn, Ci, Cs, Cnv, Cnh, Sn (n even), Dn, Dnv, Dnh, T, Td, Th, O, Oh, I, I1-I4,
// Ih, I1h-I4h.  I5 and I5h, which the reference does not implement either, are refused.
std::vector<std::array<double, 9>> point_group(const char* name)
{
    using M = std::array<double, 9>;
    struct Op { M r; int lz; };
    enum Kind { ROT, MIRROR, INVERSION };
    struct Gen { Kind kind; int fold; double ax, ay, az; };
    std::string g;
    for (const char* p = name; p && *p; ++p)
        if (*p != ' ') g += (char)std::toupper((unsigned char)*p);
    // order n of a name "<letter><n><suffix>", n of one or two digits; -1 if it does not match
    const auto order = [&](char lead, const char* suffix) -> int {
        const size_t ls = std::strlen(suffix);
        if (g.size() < 2 + ls || g.size() > 3 + ls || g[0] != lead) return -1;
        if (g.compare(g.size() - ls, ls, suffix) != 0) return -1;
        for (size_t i = 1; i < g.size() - ls; ++i)
            if (!std::isdigit((unsigned char)g[i])) return -1;
        return std::atoi(g.substr(1, g.size() - 1 - ls).c_str());
    };
    const std::vector<Gen> T_ = {{ROT, 3, 0., 0., 1.}, {ROT, 2, 0., 0.816496, 0.577350}};
    const std::vector<Gen> O_ = {{ROT, 3, .5773502, .5773502, .5773502}, {ROT, 4, 0, 0, 1}};
    const std::vector<Gen> I2_ = {{ROT, 2, 0, 0, 1}, {ROT, 5, 0.525731114, 0, 0.850650807},
                                  {ROT, 3, 0, 0.356822076, 0.934172364}};
    const std::vector<Gen> I1_ = {{ROT, 2, 1, 0, 0}, {ROT, 5, 0.85065080702670, 0, -0.5257311142635},
                                  {ROT, 3, 0.9341723640, 0.3568220765, 0}};
    const std::vector<Gen> I3_ = {{ROT, 2, -0.5257311143, 0, 0.8506508070}, {ROT, 5, 0., 0., 1.},
                                  {ROT, 3, -0.4911234778630044, 0.3568220764705179, 0.7946544753759428}};
    const std::vector<Gen> I4_ = {{ROT, 2, 0.5257311143, 0, 0.8506508070},
                                  {ROT, 5, 0.8944271932547096, 0, 0.4472135909903704},
                                  {ROT, 3, 0.4911234778630044, 0.3568220764705179, 0.7946544753759428}};
    const auto plus = [](std::vector<Gen> a, const Gen& b) {
        a.push_back(b);
        return a;
    };
    const auto dihedral = [&](int n) {
        std::vector<Gen> v;
        if (n > 1) v.push_back({ROT, n, 0, 0, 1});
        v.push_back({ROT, 2, 1, 0, 0});
        return v;
    };
    std::vector<Gen> gens;
    bool known = true;
    int n;
    if (g.empty() || g == "C1") return {};
    if ((n = order('C', "")) >= 1) gens = {{ROT, n, 0, 0, 1}};
    else if (g == "CI") gens = {{INVERSION, 0, 0, 0, 0}};
    else if (g == "CS") gens = {{MIRROR, 0, 0, 0, 1}};
    else if ((n = order('C', "V")) >= 1) gens = {{ROT, n, 0, 0, 1}, {MIRROR, 0, 0, 1, 0}};
    else if ((n = order('C', "H")) >= 1) gens = {{ROT, n, 0, 0, 1}, {MIRROR, 0, 0, 0, 1}};
    else if ((n = order('S', "")) >= 1) {
        if (n % 2) throw Error{T2B_ERR_ARG, "the order of an Sn group must be even"};
        gens = {{ROT, n / 2, 0, 0, 1}, {INVERSION, 0, 0, 0, 0}};
    } else if ((n = order('D', "")) >= 1) gens = dihedral(n);
    else if ((n = order('D', "V")) >= 1) gens = plus(dihedral(n), {MIRROR, 0, 1, 0, 0});
    else if ((n = order('D', "H")) >= 1) gens = plus(dihedral(n), {MIRROR, 0, 0, 0, 1});
    else if (g == "T") gens = T_;
    else if (g == "TD") gens = plus(T_, {MIRROR, 0, 1.4142136, 2.4494897, 0.0000000});
    else if (g == "TH") gens = {{ROT, 3, 0., 0., 1.}, {ROT, 2, 0., -0.816496, -0.577350}, {INVERSION, 0, 0, 0, 0}};
    else if (g == "O") gens = O_;
    else if (g == "OH") gens = plus(O_, {MIRROR, 0, 0, 1, 1});
    else if (g == "I" || g == "I2") gens = I2_;
    else if (g == "I1") gens = I1_;
    else if (g == "I3") gens = I3_;
    else if (g == "I4") gens = I4_;
    else if (g == "IH" || g == "I2H") gens = plus(I2_, {MIRROR, 0, 1, 0, 0});
    else if (g == "I1H") gens = plus(I1_, {MIRROR, 0, 0, 0, -1});
    else if (g == "I3H") gens = plus(I3_, {MIRROR, 0, 0.850650807, 0, 0.525731114});
    else if (g == "I4H") gens = plus(I4_, {MIRROR, 0, 0.850650807, 0, -0.525731114});
    else known = false;
    if (!known)
        throw Error{T2B_ERR_UNSUPPORTED, std::string("point group '") + (name ? name : "") +
                                             "' not supported: C1, Cn, Ci, Cs, Cnv, Cnh, Sn, Dn, Dnv, Dnh, T, Td, Th, "
                                             "O, Oh, I, I1-I4, Ih, I1h-I4h"};
    const auto clean = [](M& a) {
        for (double& v : a)
            if (std::fabs(v) < 1e-6) v = 0.;
    };
    const auto same = [](const Op& a, const Op& b) {
        if (a.lz != b.lz) return false;
        for (int i = 0; i < 9; ++i)
            if (std::fabs(a.r[i] - b.r[i]) > 1e-6) return false;
        return true;
    };
    const auto mul = [](const M& a, const M& b) {
        M r{};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) r[3 * i + j] += a[3 * i + k] * b[3 * k + j];
        return r;
    };
    const Op ident = {{1, 0, 0, 0, 1, 0, 0, 0, 1}, 1};
    std::vector<Op> ops;
    for (const Gen& ge : gens) {
        const double nrm = std::sqrt(ge.ax * ge.ax + ge.ay * ge.ay + ge.az * ge.az);
        const double a[3] = {ge.ax / nrm, ge.ay / nrm, ge.az / nrm};
        if (ge.kind == INVERSION) {
            ops.push_back({{-1, 0, 0, 0, -1, 0, 0, 0, -1}, -1});
        } else if (ge.kind == MIRROR) {
            M r;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) r[3 * i + j] = (i == j ? 1. : 0.) - 2. * a[i] * a[j];
            ops.push_back({r, 1});
        } else {
            for (int kk = 1; kk < ge.fold; ++kk) {
                const double ang = kk * (2.0 * PI_R / ge.fold), cs = std::cos(ang), sn = std::sin(ang);
                // rotation by ang about a (Rodrigues), transposed
                M r;
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        const double cross = (i == j) ? 0. : ((3 + j - i) % 3 == 1 ? -1. : 1.) * a[3 - i - j];
                        r[3 * j + i] = (i == j ? cs : 0.) + sn * cross + (1. - cs) * a[i] * a[j];
                    }
                clean(r);
                ops.push_back({r, 1});
            }
        }
    }
    const auto visit = [&](size_t i, size_t j) {
        Op p = {mul(ops[i].r, ops[j].r), ops[i].lz * ops[j].lz};
        if (same(p, ident)) return;
        for (const Op& o : ops)
            if (same(o, p)) return;
        clean(p.r);
        ops.push_back(p);
        T2B_REQUIRE(ops.size() < 1000, T2B_ERR_ARG, "point group does not close");
    };
    for (size_t q = 0; q < ops.size(); ++q) {
        for (size_t i = 0; i <= q; ++i) visit(i, q);
        for (size_t j = q; j-- > 0;) visit(q, j);
    }
    std::vector<M> out;
    for (const Op& o : ops) out.push_back(o.r);
    return out;
}

}  // namespace
}  // namespace t2b

using namespace t2b;

namespace t2b {
namespace {
// the grid of a class summed over operators (and, for helical symmetry, z phase shifts) in place:
// the sums go to the context's scratch (kept between calls: an M-step symmetrises every class of
// every iteration), copied back once the kernel has read the whole grid.  C1 (no operator) and
// 2D grids are left as they are, as the reference leaves them.
void symmetrise_grid(t2b_ctx* c, int iclass, const std::vector<std::array<double, 9>>& ops,
                     const std::vector<double>& zsh)
{
    const Volume& v = grid_volume(c, iclass);
    if (ops.empty() || v.ref_dim != 3) return;
    const int rp = v.r_max * v.pad;
    const size_t nv = v.nvox();
    cudaStream_t st = c->stream;
    std::vector<double> hr(9 * ops.size());
    for (size_t i = 0; i < ops.size(); ++i)
        for (int e = 0; e < 9; ++e) hr[9 * i + e] = ops[i][e];
    hr.insert(hr.end(), zsh.begin(), zsh.end());
    // [operators | sums of the data (float2) | sums of the weights], each part 256-byte aligned
    const size_t r_bytes = (hr.size() * sizeof(double) + 255) & ~size_t(255);
    const size_t d_bytes = (nv * sizeof(float2) + 255) & ~size_t(255);
    const size_t need = r_bytes + d_bytes + nv * sizeof(float);
    if (c->sym_bytes < need) {
        T2B_CUDA(cudaStreamSynchronize(st));
        cudaFree(c->sym_scratch);
        c->sym_scratch = nullptr;
        c->sym_bytes = 0;
        if (cudaMalloc(&c->sym_scratch, need) != cudaSuccess) {
            cudaGetLastError();
            throw Error{T2B_ERR_NOMEM, "symmetrisation scratch of " + std::to_string(need) + " bytes"};
        }
        c->sym_bytes = need;
    }
    char* base = static_cast<char*>(c->sym_scratch);
    double* R = reinterpret_cast<double*>(base);
    float2* sd = reinterpret_cast<float2*>(base + r_bytes);
    float* sw = reinterpret_cast<float*>(base + r_bytes + d_bytes);
    T2B_CUDA(cudaMemcpyAsync(R, hr.data(), hr.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    k_symmetrise<<<grid_of((long long)nv), RC_THREADS, 0, st>>>(v, c->gdata[iclass], c->gweight[iclass], sd, sw, R,
                                                               zsh.empty() ? nullptr : R + 9 * ops.size(),
                                                               (int)ops.size(), rp * rp);
    T2B_CUDA(cudaGetLastError());
    T2B_CUDA(cudaMemcpyAsync(c->gdata[iclass], sd, nv * sizeof(float2), cudaMemcpyDeviceToDevice, st));
    T2B_CUDA(cudaMemcpyAsync(c->gweight[iclass], sw, nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
    T2B_CUDA(cudaStreamSynchronize(st));   // the host table hr is read by the copy above
}
}  // namespace
}  // namespace t2b

extern "C" {

int t2b_reconstruct(t2b_ctx* c, int iclass, const t2b_recon_config* cf, double* vol_out)
{
    return guarded([&] {
        T2B_REQUIRE(c && cf && vol_out, T2B_ERR_ARG, "null argument");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        const Volume& v = grid_volume(c, iclass);
        const int ori = cf->ori_size, pad = v.pad;
        T2B_REQUIRE(ori >= 8 && ori % 2 == 0, T2B_ERR_ARG, "ori_size must be even and >= 8");
        T2B_REQUIRE(v.r_max <= ori / 2, T2B_ERR_ARG, "the grid's r_max exceeds ori_size / 2");
        T2B_REQUIRE(!cf->do_map || (cf->tau2 && cf->tau2_fudge > 0.), T2B_ERR_ARG, "do_map needs tau2 and tau2_fudge");
        int N = pad * ori;
        N += N % 2;
        T2B_REQUIRE(N <= 512, T2B_ERR_UNSUPPORTED, "pad * ori_size must be <= 512");
        const FftPlan plan = fft_plan(N);
        const int dim = v.ref_dim;
        const int ps = v.ydim, fx = ps / 2 + 1, h = N / 2 + 1;
        const size_t nps = (size_t)(dim == 3 ? ps : 1) * ps * fx;
        cudaStream_t st = c->stream;
        DevBuf<double2> fc(nps);
        DevBuf<double> fw(nps), rad(2 * (size_t)v.r_max), t2(ori / 2 + 1);
        if (cf->do_map)
            T2B_CUDA(cudaMemcpyAsync(t2.p, cf->tau2, (ori / 2 + 1) * sizeof(double), cudaMemcpyHostToDevice, st));
        const double tscale = (dim == 3 ? (double)pad * pad * pad : (double)pad * pad) * cf->tau2_fudge;
        if (cf->gridding_iter > 0) {
            // --dont_skip_gridding: the iterative weights in place of the division
            T2B_REQUIRE(cf->normalise > 0., T2B_ERR_ARG,
                        "gridding iterations need normalise > 0 (the class's sum of weights)");
            launch_decenter(v, c->gdata[iclass], c->gweight[iclass], fc.p, fw.p, rad.p, rad.p + v.r_max, st,
                            cf->do_map ? t2.p : nullptr, tscale, cf->minres_map);
            gridding_weights(v, ori, pad, cf->gridding_iter, cf->normalise, fc.p, fw.p, st);
        } else {
            launch_reconstruct(v, c->gdata[iclass], c->gweight[iclass], fc.p, fw.p, rad.p, rad.p + v.r_max, st,
                               cf->do_map ? t2.p : nullptr, tscale, cf->minres_map);
        }
        // window + centre by sign, inverse 3D FFT, real-space window
        DevBuf<float2> G((size_t)(dim == 3 ? N : 1) * N * h), tw(N);
        std::vector<float2> htw(N);
        for (int t = 0; t < N; ++t) {
            const double a = -2.0 * PI_R * (double)t / (double)N;
            htw[t] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        T2B_CUDA(cudaMemcpyAsync(tw.p, htw.data(), N * sizeof(float2), cudaMemcpyHostToDevice, st));
        k_window<<<grid_of((long long)(dim == 3 ? N : 1) * N * h), RC_THREADS, 0, st>>>(fc.p, ps, N, dim, G.p);
        ColKernel col;
        RowKernel row;
        recon_kernels(N, col, row);
        const size_t smc = sizeof(float2) * ((size_t)N + 2 * (size_t)RC_CX * N);
        const size_t smr = sizeof(float2) * ((size_t)N + 2 * (size_t)RC_ROWS * N);
        T2B_CUDA(cudaFuncSetAttribute((const void*)col, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc));
        T2B_CUDA(cudaFuncSetAttribute((const void*)row, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr));
        const int z0 = N / 2 - ori / 2, xt = (h + RC_CX - 1) / RC_CX;
        if (dim == 3) {
            col<<<dim3(N, xt), RC_THREADS, smc, st>>>(G.p, N, 0, 0, tw.p, plan);          // along z, every (y, x)
            col<<<dim3(ori, xt), RC_THREADS, smc, st>>>(G.p, N, 1, z0, tw.p, plan);       // along y, window planes
        } else {
            col<<<dim3(1, xt), RC_THREADS, smc, st>>>(G.p, N, 1, 0, tw.p, plan);          // along y, the one plane
        }
        const long long nv = (long long)ori * ori * (dim == 3 ? ori : 1);
        DevBuf<float> vol(nv);
        // normalisation of windowToOridimRealSpace for 2D particles: pad^3 ori (3D maps), pad^2 (2D)
        const float norm = dim == 3 ? (float)((double)pad * pad * pad * ori) : (float)((double)pad * pad);
        const int nrows = dim == 3 ? ori * ori : ori;
        row<<<(nrows + RC_ROWS - 1) / RC_ROWS, RC_THREADS, smr, st>>>(G.p, N, ori, z0, norm, tw.p, plan, vol.p, dim);
        // soft mask (radius ori/2, width 3, average background) and gridding correction
        const int nb = grid_of(nv);
        DevBuf<double2> part(nb);
        DevBuf<double> out(nv);
        k_mask_partial<<<nb, RC_THREADS, 0, st>>>(vol.p, ori, dim, ori / 2.0, 3.0, part.p);
        k_mask_grid<<<nb, RC_THREADS, 0, st>>>(vol.p, ori, dim, pad, ori / 2.0, 3.0, part.p, nb, out.p);
        T2B_CUDA(cudaGetLastError());
        T2B_CUDA(cudaMemcpyAsync(vol_out, out.p, nv * sizeof(double), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaStreamSynchronize(st));
    });
}

int t2b_backprojector_enforce_hermitian(t2b_ctx* c, int iclass)
{
    return guarded([&] {
        T2B_REQUIRE(c, T2B_ERR_ARG, "null argument");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        const Volume& v = grid_volume(c, iclass);
        T2B_REQUIRE(v.ref_dim == 2 || -v.initz == v.zdim / 2, T2B_ERR_ARG, "grid is not centred in z");
        T2B_REQUIRE(-v.inity == v.ydim / 2, T2B_ERR_ARG, "grid is not centred in y");
        const long long pairs = (long long)v.zdim * (v.ydim / 2 + 1);
        k_hermitian<<<grid_of(pairs), RC_THREADS, 0, c->stream>>>(v, c->gdata[iclass], c->gweight[iclass]);
        T2B_CUDA(cudaGetLastError());
        T2B_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int t2b_point_group(const char* group, double* mats, int cap, int* count)
{
    return guarded([&] {
        T2B_REQUIRE(count && (cap <= 0 || mats), T2B_ERR_ARG, "null argument");
        const auto ops = point_group(group);
        *count = (int)ops.size();
        for (int i = 0; i < (int)ops.size() && i < cap; ++i)
            for (int e = 0; e < 9; ++e) mats[9 * i + e] = ops[i][e];
    });
}

int t2b_backprojector_apply_symmetry(t2b_ctx* c, int iclass, const char* group)
{
    return guarded([&] {
        T2B_REQUIRE(c, T2B_ERR_ARG, "null argument");
        const auto ops = point_group(group);
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        symmetrise_grid(c, iclass, ops, {});
    });
}

int t2b_backprojector_apply_helical(t2b_ctx* c, int iclass, int nr_asu, double twist, double rise, int ori_size)
{
    return guarded([&] {
        T2B_REQUIRE(c, T2B_ERR_ARG, "null argument");
        T2B_REQUIRE(nr_asu < 2 || ori_size > 0, T2B_ERR_ARG, "ori_size must be positive");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        const Volume& v = grid_volume(c, iclass);
        std::vector<std::array<double, 9>> ops;
        std::vector<double> zsh;
        // the asymmetric units hh = -n/2 .. n/2 - 1 (+1 for odd n) other than 0: a rotation by
        // -hh twist degrees about z (rotation3DMatrix(ang, 'Z'), entries below 1e-6 zeroed) and
        // a shift of hh rise pixels along z
        const int h_min = -nr_asu / 2, h_max = -h_min + nr_asu % 2;
        for (int hh = h_min; nr_asu >= 2 && hh < h_max; ++hh) {
            if (hh == 0) continue;
            const double ang = (hh * -twist) * PI_R / 180.;
            std::array<double, 9> r = {std::cos(ang), -std::sin(ang), 0., std::sin(ang), std::cos(ang), 0., 0., 0., 1.};
            for (double& e : r)
                if (std::fabs(e) < 1e-6) e = 0.;
            ops.push_back(r);
            zsh.push_back(std::fabs(rise) > 0. ? (hh * rise) / (-ori_size * (double)v.pad) : 0.);
        }
        symmetrise_grid(c, iclass, ops, zsh);
    });
}

int t2b_fsc_halves(t2b_ctx* c, int grid_a, int grid_b, int ori_size, double* fsc)
{
    return guarded([&] {
        T2B_REQUIRE(c && fsc && ori_size >= 2, T2B_ERR_ARG, "bad argument");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        const Volume& a = grid_volume(c, grid_a);
        const Volume& b = grid_volume(c, grid_b);
        T2B_REQUIRE(a.xdim == b.xdim && a.ydim == b.ydim && a.zdim == b.zdim && a.r_max == b.r_max && a.pad == b.pad &&
                        a.ref_dim == b.ref_dim,
                    T2B_ERR_ARG, "the two grids differ in shape");
        T2B_REQUIRE(a.r_max <= ori_size / 2, T2B_ERR_ARG, "r_max exceeds ori_size / 2");
        const int ds = 2 * (a.r_max + 1) + 1, dh = ds / 2, nb = ori_size / 2 + 1;
        T2B_REQUIRE(nb <= 1024, T2B_ERR_ARG, "ori_size too large");
        const size_t bins = (size_t)(a.ref_dim == 3 ? ds : 1) * ds * (dh + 1);
        cudaStream_t st = c->stream;
        DevBuf<double> aa(3 * bins), ab(3 * bins), sh(3 * (size_t)nb);
        T2B_CUDA(cudaMemsetAsync(aa.p, 0, 3 * bins * sizeof(double), st));
        T2B_CUDA(cudaMemsetAsync(ab.p, 0, 3 * bins * sizeof(double), st));
        T2B_CUDA(cudaMemsetAsync(sh.p, 0, 3 * (size_t)nb * sizeof(double), st));
        const long long nvox = (long long)a.zdim * a.ydim * a.xdim;
        k_downsample<<<grid_of(nvox), RC_THREADS, 0, st>>>(a, c->gdata[grid_a], c->gweight[grid_a], aa.p);
        k_downsample<<<grid_of(nvox), RC_THREADS, 0, st>>>(b, c->gdata[grid_b], c->gweight[grid_b], ab.p);
        k_fsc_shells<<<grid_of((long long)bins), RC_THREADS, 3 * nb * sizeof(double), st>>>(a.r_max, nb, a.ref_dim, aa.p,
                                                                                             ab.p, sh.p);
        T2B_CUDA(cudaGetLastError());
        std::vector<double> h(3 * (size_t)nb);
        T2B_CUDA(cudaMemcpyAsync(h.data(), sh.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < nb; ++i) {
            const double d = h[3 * i + 1] * h[3 * i + 2];
            fsc[i] = d > 0. ? h[3 * i] / std::sqrt(d) : 0.;
        }
        fsc[0] = 1.;
    });
}

int t2b_update_ssnr(t2b_ctx* c, int iclass, const t2b_ssnr_config* cf, double* tau2, double* sigma2,
                    double* data_vs_prior, double* fourier_coverage)
{
    return guarded([&] {
        T2B_REQUIRE(c && cf && tau2 && sigma2 && data_vs_prior && fourier_coverage, T2B_ERR_ARG, "null argument");
        T2B_REQUIRE(!cf->update_tau2_with_fsc || cf->fsc, T2B_ERR_ARG, "update_tau2_with_fsc needs the FSC");
        T2B_REQUIRE(!cf->correct_tau2_by_avgctf2 || cf->avgctf2, T2B_ERR_ARG, "correct_tau2_by_avgctf2 needs avgctf2");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        const Volume& v = grid_volume(c, iclass);
        const int nb = cf->ori_size / 2 + 1;
        T2B_REQUIRE(v.r_max < nb && nb <= 1024, T2B_ERR_ARG, "r_max exceeds ori_size / 2 (or ori_size too large)");
        const double oc = v.ref_dim == 3 ? (double)v.pad * v.pad * v.pad : (double)v.pad * v.pad;
        cudaStream_t st = c->stream;
        DevBuf<double> acc(3 * (size_t)nb), t2d(nb), actf(nb);
        const long long nvox = (long long)v.zdim * v.ydim * v.xdim;
        // pass 1: sigma2 = count / sum(pad^3 weight) per shell (src/backprojector.cpp:1058-1088)
        T2B_CUDA(cudaMemsetAsync(acc.p, 0, 3 * (size_t)nb * sizeof(double), st));
        k_ssnr_sigma<<<grid_of(nvox), RC_THREADS, 2 * nb * sizeof(double), st>>>(v, nb, c->gweight[iclass], oc, acc.p);
        std::vector<double> h(3 * (size_t)nb);
        T2B_CUDA(cudaMemcpyAsync(h.data(), acc.p, 2 * (size_t)nb * sizeof(double), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaStreamSynchronize(st));
        std::vector<double> s2(nb), t(tau2, tau2 + nb), dvp(nb, 0.), cov(nb, 0.);
        for (int i = 0; i < nb; ++i) {
            const double sw = h[2 * i], cn = h[2 * i + 1];
            s2[i] = sw > 1e-10 ? cn / sw : 0.;
        }
        // tau2 from the FSC (:1101-1125)
        if (cf->update_tau2_with_fsc)
            for (int i = 0; i < nb; ++i) {
                double f = std::max(0.001, cf->fsc[i]);
                if (cf->is_whole_instead_of_half) f = std::sqrt(2. * f / (f + 1.));
                f = std::min(0.999, f);
                const double ssnr = f / (1. - f) * cf->tau2_fudge;
                t[i] = ssnr * s2[i];
                dvp[i] = ssnr;
            }
        // pass 2: data vs prior and Fourier coverage (:1127-1190)
        T2B_CUDA(cudaMemcpyAsync(t2d.p, t.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
        if (cf->correct_tau2_by_avgctf2)
            T2B_CUDA(cudaMemcpyAsync(actf.p, cf->avgctf2, nb * sizeof(double), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemsetAsync(acc.p, 0, 3 * (size_t)nb * sizeof(double), st));
        k_ssnr_prior<<<grid_of(nvox), RC_THREADS, 3 * nb * sizeof(double), st>>>(v, nb, c->gweight[iclass], oc,
                                                                                  cf->tau2_fudge, t2d.p, actf.p,
                                                                                  cf->correct_tau2_by_avgctf2, acc.p);
        T2B_CUDA(cudaGetLastError());
        T2B_CUDA(cudaMemcpyAsync(h.data(), acc.p, 3 * (size_t)nb * sizeof(double), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < nb; ++i) {
            const double ratio = h[3 * i], ncov = h[3 * i + 1], cn = h[3 * i + 2];
            if (!cf->update_tau2_with_fsc) dvp[i] = i > v.r_max ? 0. : (cn < 0.001 ? 999. : ratio / cn);
            cov[i] = cn > 0. ? ncov / cn : ncov;
        }
        for (int i = 0; i < nb; ++i) {
            tau2[i] = t[i];
            sigma2[i] = s2[i];
            data_vs_prior[i] = dvp[i];
            fourier_coverage[i] = cov[i];
        }
    });
}

}  // extern "C"
