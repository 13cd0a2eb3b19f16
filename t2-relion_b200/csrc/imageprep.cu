// Image preparation before the E-step, on the device: real-space particles ->
// the windowed Fourier images, CTF image, Minvsigma2 image and per-particle
// scalars that t2b_estep_batch_* reads.
//
// Follows MlOptimiser::getFourierTransformsAndCtfs (src/ml_optimiser.cpp:5689-6390;
// the accelerated path src/acc/acc_ml_optimiser_impl.h:96-1030 does the same
// steps with TranslateAndNormCorrect, softMaskBackgroundValue, cosineFilter,
// cuFFT and powerClass) and the Minvsigma2 part of
// precalculateShiftedImagesCtfsAndInvSigma2s (src/ml_optimiser.cpp:6680-6720):
//
//   norm correction, rounded old offset as an integer shift with zero fill
//   (selfTranslate DONT_WRAP), soft mask with the average background
//   (zero_mask) or a noise image of spectrum sigma2_fudge * sigma2_noise,
//   FFT (forward divided by N^2), power spectrum and highres_Xi2 over the full
//   transform, window to current_size, CenterFFTbySign, CTF image
//   (CTF::getFftwImage without padding), Minvsigma2.
//
// Layout: one 2D transform = a row pass and a column pass, each a batch of 1D
// FFTs held in shared memory (mixed-radix Stockham, radices 4, 2, 3, 5; any
// even N = 2^a 3^b 5^c up to 512).  The row pass transforms the masked and the
// unmasked row together as one complex sequence (masked + i * unmasked) and
// separates the two half spectra; the column pass only transforms the N/2 + 1
// columns of the half spectrum.  The intermediate half spectra stay in L2.
//
// Noise background: the reference draws the noise spectrum from rand() (CPU)
// or curand (GPU), neither reproducible across thread schedules; here it is a
// counter-based generator (one SplitMix64 draw per element from the particle's
// key random_seed + part_id and the element index, two 24-bit uniforms,
// Box-Muller) with the reference's spectrum, transformed back unnormalised like
// FFTW's c2r.
#include "t2b_internal.cuh"
#include "fft_smem.cuh"

#include <cmath>
#include <cstring>

namespace t2b {

constexpr double PI_D = 3.14159265358979323846;
constexpr int PREP_MAX_N = 512;
constexpr int PREP_THREADS = 256;

struct ImagePrep {
    t2b_prep_config cfg{};
    int N = 0, h = 0, s = 0, hs = 0, P = 0, max_batch = 0;
    int rpb = 0, cpb = 0, ncol_blocks = 0;
    bool fused = false;            // one CTA per particle (k_noise_fused, k_prep_fused)
    FftPlan plan{};
    double minv_dc = 0.;
    float2* tw = nullptr;          // N twiddles e^{-2 pi i t / N}
    double* noise_sig = nullptr;   // h: sqrt(sigma2_fudge * remapped sigma2_noise)
    float* minv = nullptr;         // P: Minvsigma2 window image
    int* ring_off = nullptr;       // h + 1: CSR offsets of the spectrum rings
    int* ring_pix = nullptr;       // pixels (i * h + kx) of rings 1 .. h-1
    float2* gm = nullptr;          // max_batch x N x h  masked half spectra (rows transformed)
    float2* gu = nullptr;          // max_batch x N x h  unmasked
    float2* gn = nullptr;          // max_batch x N x h  noise (columns transformed)
    float* noise = nullptr;        // max_batch x N x N  noise images
    float* pw = nullptr;           // max_batch x N x h  |F|^2 of the masked transform
    double* bg = nullptr;          // max_batch          average background
    // host batch staging
    float* h_img = nullptr;        // device copies of the host batch
    double* h_par = nullptr;
    long long* h_pid = nullptr;
    float* o_fimg = nullptr;
    float* o_fnm = nullptr;
    float* o_ctf = nullptr;
    float* o_minv = nullptr;
    double* o_sc = nullptr;
    double* o_pw = nullptr;
    std::vector<void*> allocs;
};

namespace {

__device__ __forceinline__ int relion_round(double x) { return x > 0 ? (int)(x + 0.5) : (int)(x - 0.5); }

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// ring index ROUND(sqrt(ky^2 + kx^2)): FP32 sqrt decides the rounding exactly for the
// integer radii of a box <= 512 (sqrt(r2) is never within 3e-4 of a half-integer)
__device__ __forceinline__ int ring_of(int ky, int kx)
{
    return (int)(sqrtf((float)(ky * ky + kx * kx)) + 0.5f);
}

// noise spectrum element: one SplitMix64 draw of the particle's key and the element
// index; two 24-bit uniforms u1 in (0, 1], u2 in [0, 1); Box-Muller
__device__ __forceinline__ float2 noise_value(unsigned long long key, unsigned long long c, float sig)
{
    const unsigned long long x = splitmix64(key + c);
    const float u1 = (float)((x >> 40) + 1ull) * 0x1.0p-24f;
    const float u2 = (float)((x >> 8) & 0xFFFFFFull) * 0x1.0p-24f;
    const float rad = sqrtf(-2.f * logf(u1)) * sig;
    float sn, cs;
    sincospif(2.f * u2, &sn, &cs);
    return make_float2(rad * cs, rad * sn);
}

struct PrepArgs {
    FftPlan plan;
    int N, h, s, hs, P, rpb, cpb;
    int zero_mask, do_ctf;
    int premult, do_abs, flip, intact;
    long long seed;
    float radius, width;
    double norm_on, avg_norm;
    double xs;                        // image_size * pixel_size
    double lam_k1, k2, k3;            // CTF constants of the optics group
    double minv_dc;
    const float2* tw;
    const double* noise_sig;
    const float* minv_img;
    const int* ring_off;
    const int* ring_pix;
    const float* img;
    const double* par;
    const long long* pid;
    float2* gm;
    float2* gu;
    float2* gn;
    float* noise;
    float* pw;
    double* bg;
    float* fimg;
    float* fnm;
    float* ctf;
    float* minv;
    double* sc;
    double* power;
};

constexpr int NPAR = T2B_PREP_NPARAM;

__device__ __forceinline__ void load_tw(float2* s_tw, const float2* tw, int N)
{
    for (int t = threadIdx.x; t < N; t += blockDim.x) s_tw[t] = tw[t];
}

// ------------------------------------------------------------ noise image
// columns: spectrum of the noise (rows i, columns kx), inverse FFT over y
__global__ void __launch_bounds__(PREP_THREADS) k_noise_cols(PrepArgs a)
{
    extern __shared__ float2 sm[];
    const int N = a.N, h = a.h, C = a.cpb;
    float2* s_tw = sm;
    float2* b0 = sm + N;
    float2* b1 = b0 + C * N;
    const int p = blockIdx.x, j0 = blockIdx.y * C;
    load_tw(s_tw, a.tw, N);
    const unsigned long long key = splitmix64((unsigned long long)(a.seed + a.pid[p]));
    for (int e = threadIdx.x; e < C * N; e += blockDim.x) {
        const int c = e % C, i = e / C, j = j0 + c;
        float2 v = make_float2(0.f, 0.f);
        if (j < h) {
            const int ky = i < h ? i : i - N;
            const int ires = ring_of(ky, j);
            if (ires < h) v = noise_value(key, (unsigned long long)i * h + j, (float)a.noise_sig[ires]);
        }
        b0[c * N + i] = v;
    }
    __syncthreads();
    const float2* r = fft_smem<true>(b0, b1, C, a.plan, s_tw);
    float2* out = a.gn + (size_t)p * N * h;
    for (int e = threadIdx.x; e < C * N; e += blockDim.x) {
        const int c = e % C, i = e / C, j = j0 + c;
        if (j < h) out[(size_t)i * h + j] = r[c * N + i];
    }
}

// rows: Hermitian extension (imaginary parts of kx = 0 and N/2 dropped), inverse FFT over x
__global__ void __launch_bounds__(PREP_THREADS) k_noise_rows(PrepArgs a)
{
    extern __shared__ float2 sm[];
    const int N = a.N, h = a.h, R = a.rpb;
    float2* s_tw = sm;
    float2* b0 = sm + N;
    float2* b1 = b0 + R * N;
    const int p = blockIdx.x, y0 = blockIdx.y * R;
    load_tw(s_tw, a.tw, N);
    const float2* g = a.gn + (size_t)p * N * h;
    for (int e = threadIdx.x; e < R * N; e += blockDim.x) {
        const int rr = e / N, k = e - rr * N, y = y0 + rr;
        float2 v = make_float2(0.f, 0.f);
        if (y < N) {
            if (k == 0 || k == N / 2) v = make_float2(g[(size_t)y * h + k].x, 0.f);
            else if (k < N / 2) v = g[(size_t)y * h + k];
            else {
                const float2 w = g[(size_t)y * h + (N - k)];
                v = make_float2(w.x, -w.y);
            }
        }
        b0[e] = v;
    }
    __syncthreads();
    const float2* r = fft_smem<true>(b0, b1, R, a.plan, s_tw);
    float* out = a.noise + (size_t)p * N * N;
    for (int e = threadIdx.x; e < R * N; e += blockDim.x) {
        const int rr = e / N, x = e - rr * N, y = y0 + rr;
        if (y < N) out[(size_t)y * N + x] = r[e].x;
    }
}

// ------------------------------------------------------------ pixel helpers
struct PixelCtx {
    int tx, ty;
    float scale;
};

__device__ __forceinline__ PixelCtx pixel_ctx(const PrepArgs& a, int p)
{
    const double* par = a.par + (size_t)p * NPAR;
    PixelCtx c;
    c.tx = relion_round(par[0]);
    c.ty = relion_round(par[1]);
    c.scale = a.norm_on ? (float)(a.avg_norm / par[4]) : 1.f;
    return c;
}

// translated, norm-corrected pixel (x, y) of particle p (zero outside)
__device__ __forceinline__ float shifted_pixel(const PrepArgs& a, const float* img, const PixelCtx& c, int x, int y)
{
    const int xs = x - c.tx, ys = y - c.ty;
    if (xs < 0 || ys < 0 || xs >= a.N || ys >= a.N) return 0.f;
    return img[(size_t)ys * a.N + xs] * c.scale;
}

// raised-cosine weight of the soft mask: <0 inside the radius, 1 beyond radius + width
__device__ __forceinline__ float mask_weight(const PrepArgs& a, int x, int y)
{
    const float xl = (float)(x - a.N / 2), yl = (float)(y - a.N / 2);
    const float r = sqrtf(xl * xl + yl * yl);
    if (r < a.radius) return -1.f;
    const float rp = a.radius + a.width;
    if (r > rp) return 1.f;
    return 0.5f + 0.5f * cospif((rp - r) / a.width);
}

// average background of the zero-mask path (softMaskOutsideMap without a noise
// image): sum of the weights and weighted pixels outside the radius; fixed-order
// reduction in FP64
__global__ void __launch_bounds__(PREP_THREADS) k_background(PrepArgs a)
{
    __shared__ double s_w[PREP_THREADS], s_v[PREP_THREADS];
    const int p = blockIdx.x, N = a.N;
    const PixelCtx c = pixel_ctx(a, p);
    const float* img = a.img + (size_t)p * N * N;
    double sw = 0., sv = 0.;
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
        const int y = e / N, x = e - y * N;
        const float w = mask_weight(a, x, y);
        if (w < 0.f) continue;
        sw += w;
        sv += (double)w * shifted_pixel(a, img, c, x, y);
    }
    s_w[threadIdx.x] = sw;
    s_v[threadIdx.x] = sv;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_w[threadIdx.x] += s_w[threadIdx.x + o];
            s_v[threadIdx.x] += s_v[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) a.bg[p] = s_w[0] > 0. ? s_v[0] / s_w[0] : 0.;
}

// ------------------------------------------------------------ row pass
// z = masked + i * unmasked, forward FFT over x, split into the two half spectra
__global__ void __launch_bounds__(PREP_THREADS) k_rows(PrepArgs a)
{
    extern __shared__ float2 sm[];
    const int N = a.N, h = a.h, R = a.rpb;
    float2* s_tw = sm;
    float2* b0 = sm + N;
    float2* b1 = b0 + R * N;
    const int p = blockIdx.x, y0 = blockIdx.y * R;
    load_tw(s_tw, a.tw, N);
    const PixelCtx c = pixel_ctx(a, p);
    const float* img = a.img + (size_t)p * N * N;
    const float bgv = a.zero_mask ? (float)a.bg[p] : 0.f;
    const float* noise = a.zero_mask ? nullptr : a.noise + (size_t)p * N * N;
    for (int e = threadIdx.x; e < R * N; e += blockDim.x) {
        const int rr = e / N, x = e - rr * N, y = y0 + rr;
        float2 v = make_float2(0.f, 0.f);
        if (y < N) {
            const float u = shifted_pixel(a, img, c, x, y);
            const float w = mask_weight(a, x, y);
            float m = u;
            if (w >= 0.f) {
                const float fill = a.zero_mask ? bgv : noise[(size_t)y * N + x];
                m = (w >= 1.f) ? fill : (1.f - w) * u + w * fill;
            }
            v = make_float2(m, u);
        }
        b0[e] = v;
    }
    __syncthreads();
    const float2* r = fft_smem<false>(b0, b1, R, a.plan, s_tw);
    float2* om = a.gm + (size_t)p * N * h;
    float2* ou = a.gu + (size_t)p * N * h;
    for (int e = threadIdx.x; e < R * h; e += blockDim.x) {
        const int rr = e / h, k = e - rr * h, y = y0 + rr;
        if (y >= N) continue;
        const float2 zk = r[rr * N + k];
        const float2 zc = r[rr * N + (N - k) % N];   // Z[N-k], conjugated below
        // masked = (Z[k] + conj Z[N-k]) / 2, unmasked = (Z[k] - conj Z[N-k]) / 2i
        om[(size_t)y * h + k] = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y - zc.y));
        ou[(size_t)y * h + k] = make_float2(0.5f * (zk.y + zc.y), -0.5f * (zk.x - zc.x));
    }
}

// ------------------------------------------------------------ column pass
__device__ __forceinline__ float ctf_value(const PrepArgs& a, const double* par, double Axx, double Axy, double Ayy,
                                           int kx, int ky)
{
    // CTF::getCTF (src/ctf.h:180-238) at X = kx / xs, Y = ky / xs
    const double X = kx / a.xs, Y = ky / a.xs;
    const double u2 = X * X + Y * Y;
    const double K4 = -par[8] / 4., K5 = par[10] * (PI_D / 180.);
    const double gamma = a.lam_k1 * (Axx * X * X + 2.0 * Axy * X * Y + Ayy * Y * Y) + a.k2 * u2 * u2 - K5 - a.k3;
    double v = (a.intact && fabs(gamma) < PI_D / 2.) ? 1. : -sin(gamma);
    v *= exp(K4 * u2);
    if (a.do_abs) v = fabs(v);
    else if (a.flip) v = (v < 0.) ? -1. : 1.;
    v *= par[9];
    if (fabs(v) < 1e-8) v = (v >= 0. ? 1. : -1.) * 1e-8;
    if (a.premult) v *= v;
    return (float)v;
}

__global__ void __launch_bounds__(PREP_THREADS) k_cols(PrepArgs a)
{
    extern __shared__ float2 sm[];
    const int N = a.N, h = a.h, C = a.cpb, s = a.s, hs = a.hs;
    float2* s_tw = sm;
    float2* b0 = sm + N;
    float2* b1 = b0 + 2 * C * N;
    const int p = blockIdx.x, j0 = blockIdx.y * C;
    load_tw(s_tw, a.tw, N);
    const float2* gm = a.gm + (size_t)p * N * h;
    const float2* gu = a.gu + (size_t)p * N * h;
    // sequences 0 .. C-1: masked columns; C .. 2C-1: unmasked
    for (int e = threadIdx.x; e < 2 * C * N; e += blockDim.x) {
        const int half = e / (C * N), q = e - half * C * N;
        const int c = q % C, i = q / C, j = j0 + c;
        float2 v = make_float2(0.f, 0.f);
        if (j < h) v = (half ? gu : gm)[(size_t)i * h + j];
        b0[(half * C + c) * N + i] = v;
    }
    __syncthreads();
    const float2* r = fft_smem<false>(b0, b1, 2 * C, a.plan, s_tw);
    const float inv = 1.f / ((float)N * (float)N);
    // |F|^2 of the masked transform, for the ring sums
    float* pw = a.pw + (size_t)p * N * h;
    for (int e = threadIdx.x; e < C * N; e += blockDim.x) {
        const int c = e % C, i = e / C, j = j0 + c;
        if (j >= h) continue;
        const float2 f = r[c * N + i];
        const float fr = f.x * inv, fi = f.y * inv;
        pw[(size_t)i * h + j] = fr * fr + fi * fi;
    }
    // window to s, CenterFFTbySign, CTF and Minvsigma2 on the window
    if (j0 >= hs) return;
    const double* par = a.par + (size_t)p * NPAR;
    const double az = par[7] * (PI_D / 180.);
    const double ca = cos(az), sa = sin(az);
    const double Axx = -par[5] * ca * ca - par[6] * sa * sa;
    const double Axy = (par[6] - par[5]) * ca * sa;
    const double Ayy = -par[5] * sa * sa - par[6] * ca * ca;
    const size_t o = (size_t)p * a.P;
    for (int e = threadIdx.x; e < C * s; e += blockDim.x) {
        const int c = e % C, iw = e / C, j = j0 + c;
        if (j >= hs) continue;
        const int ky = iw < hs ? iw : iw - s;
        const int i = ky >= 0 ? ky : ky + N;
        const float sg = ((iw ^ j) & 1) ? -inv : inv;
        const float2 fm = r[c * N + i], fu = r[(C + c) * N + i];
        const size_t w = o + (size_t)iw * hs + j;
        reinterpret_cast<float2*>(a.fimg)[w] = make_float2(fm.x * sg, fm.y * sg);
        reinterpret_cast<float2*>(a.fnm)[w] = make_float2(fu.x * sg, fu.y * sg);
        a.ctf[w] = a.do_ctf ? ctf_value(a, par, Axx, Axy, Ayy, j, ky) : 1.f;
        a.minv[w] = a.minv_img[(size_t)iw * hs + j];
    }
}

// power spectrum of the masked transform: one warp per ring, lanes over the
// ring's pixels, fixed-order shuffle reduction (deterministic)
__device__ __forceinline__ void ring_sums(const float* pw, const int* off, const int* pix, int h, double* spec,
                                          double* power)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int r = warp; r < h; r += nw) {
        double acc = 0.;
        for (int q = off[r] + lane; q < off[r + 1]; q += 32) acc += pw[pix[q]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            spec[r] = acc;
            if (power) power[r] = acc;
        }
    }
}

// ------------------------------------------------------------ spectrum and scalars
__global__ void __launch_bounds__(PREP_THREADS) k_final(PrepArgs a)
{
    __shared__ double s_spec[PREP_MAX_N / 2 + 1];
    const int p = blockIdx.x, h = a.h;
    const float* pw = a.pw + (size_t)p * a.N * h;
    ring_sums(pw, a.ring_off, a.ring_pix, h, s_spec, a.power ? a.power + (size_t)p * h : nullptr);
    __syncthreads();
    if (threadIdx.x != 0) return;
    double xi2 = 0.;
    if (a.s < a.N)
        for (int r = a.hs; r < h; ++r) xi2 += s_spec[r];
    const double* par = a.par + (size_t)p * NPAR;
    double* sc = a.sc + (size_t)p * 8;
    sc[0] = a.minv_dc;
    sc[1] = xi2;
    sc[2] = relion_round(par[0]);
    sc[3] = relion_round(par[1]);
    sc[4] = (par[2] > 998.99 && par[2] < 999.01) ? 0. : par[2];
    sc[5] = (par[3] > 998.99 && par[3] < 999.01) ? 0. : par[3];
    sc[6] = par[11];
    sc[7] = 0.;
}

// ------------------------------------------------------------ fused path: one CTA per particle
// When the particle's two half spectra fit in shared memory (N <= 136), the row
// and column passes run in one CTA per particle and the half spectra never
// leave the SM: rows in chunks of FQ (ping-pong scratch), unpacked into the
// masked and unmasked half spectra; then columns in chunks of FQ/2 of each.
constexpr int FQ = 16;
constexpr int FUSED_THREADS = 512;

size_t fused_prep_smem(int N)
{
    const size_t h = N / 2 + 1;
    return sizeof(float2) * (N + 2 * h * N + 2 * (size_t)FQ * N) + sizeof(float) * h * N + sizeof(double) * h;
}
size_t fused_noise_smem(int N)
{
    const size_t h = N / 2 + 1;
    return sizeof(float2) * (N + h * N + 2 * (size_t)FQ * N);
}

// noise image of one particle: spectrum -> inverse over y (columns) -> c2r over x (rows)
template <int NC>
__global__ void __launch_bounds__(FUSED_THREADS) k_noise_fused(PrepArgs a)
{
    extern __shared__ float2 sm[];
    const int N = NC > 0 ? NC : a.N, h = N / 2 + 1, p = blockIdx.x;
    float2* s_tw = sm;
    float2* S = s_tw + N;
    float2* A = S + (size_t)N * h;
    float2* B = A + FQ * N;
    load_tw(s_tw, a.tw, N);
    const unsigned long long key = splitmix64((unsigned long long)(a.seed + a.pid[p]));
    for (int e = threadIdx.x; e < N * h; e += blockDim.x) {
        const int i = e / h, j = e - i * h;
        const int ky = i < h ? i : i - N;
        const int ires = ring_of(ky, j);
        float2 v = make_float2(0.f, 0.f);
        if (ires < h) v = noise_value(key, (unsigned long long)e, (float)a.noise_sig[ires]);
        S[e] = v;
    }
    __syncthreads();
    for (int j0 = 0; j0 < h; j0 += FQ) {
        for (int e = threadIdx.x; e < FQ * N; e += blockDim.x) {
            const int i = e % N, c = e / N, j = j0 + c;
            A[e] = j < h ? S[(size_t)i * h + j] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        const float2* r = fft_any<NC, true>(A, B, FQ, a.plan, s_tw);
        for (int e = threadIdx.x; e < FQ * N; e += blockDim.x) {
            const int i = e % N, c = e / N, j = j0 + c;
            if (j < h) S[(size_t)i * h + j] = r[e];
        }
        __syncthreads();
    }
    float* out = a.noise + (size_t)p * N * N;
    for (int y0 = 0; y0 < N; y0 += FQ) {
        for (int e = threadIdx.x; e < FQ * N; e += blockDim.x) {
            const int rr = e / N, k = e - rr * N, y = y0 + rr;
            float2 v = make_float2(0.f, 0.f);
            if (y < N) {
                const float2* g = S + (size_t)y * h;
                if (k == 0 || k == N / 2) v = make_float2(g[k].x, 0.f);
                else if (k < N / 2) v = g[k];
                else v = make_float2(g[N - k].x, -g[N - k].y);
            }
            A[e] = v;
        }
        __syncthreads();
        const float2* r = fft_any<NC, true>(A, B, FQ, a.plan, s_tw);
        for (int e = threadIdx.x; e < FQ * N; e += blockDim.x) {
            const int rr = e / N, x = e - rr * N, y = y0 + rr;
            if (y < N) out[(size_t)y * N + x] = r[e].x;
        }
        __syncthreads();
    }
}

template <int NC>
__global__ void __launch_bounds__(FUSED_THREADS) k_prep_fused(PrepArgs a)
{
    extern __shared__ float2 sm[];
    __shared__ double s_w[FUSED_THREADS], s_v[FUSED_THREADS];
    const int N = NC > 0 ? NC : a.N, h = N / 2 + 1, p = blockIdx.x;
    constexpr int C = FQ / 2;
    float2* s_tw = sm;
    float2* SM = s_tw + N;
    float2* SU = SM + (size_t)N * h;
    float2* A = SU + (size_t)N * h;
    float2* B = A + FQ * N;
    float* PW = reinterpret_cast<float*>(B + FQ * N);
    load_tw(s_tw, a.tw, N);
    const PixelCtx pc = pixel_ctx(a, p);
    const float* img = a.img + (size_t)p * N * N;
    const float* noise = a.zero_mask ? nullptr : a.noise + (size_t)p * N * N;
    // average background (zero-mask path): fixed-order FP64 reduction
    float bgv = 0.f;
    if (a.zero_mask) {
        double sw = 0., sv = 0.;
        for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
            const int y = e / N, x = e - y * N;
            const float w = mask_weight(a, x, y);
            if (w < 0.f) continue;
            sw += w;
            sv += (double)w * shifted_pixel(a, img, pc, x, y);
        }
        s_w[threadIdx.x] = sw;
        s_v[threadIdx.x] = sv;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) {
                s_w[threadIdx.x] += s_w[threadIdx.x + o];
                s_v[threadIdx.x] += s_v[threadIdx.x + o];
            }
            __syncthreads();
        }
        bgv = s_w[0] > 0. ? (float)(s_v[0] / s_w[0]) : 0.f;
    }
    // rows: masked + i * unmasked, forward FFT over x, split into the two half spectra.
    // The pixels (and the noise outside the mask) of the next FQ rows are loaded into
    // registers before the current rows' FFT, so their latency overlaps it.
    constexpr int PMAX = (FQ * (NC > 0 ? NC : 136) + FUSED_THREADS - 1) / FUSED_THREADS;
    float ru[PMAX], rn[PMAX];
    auto fetch = [&](int y0) {
#pragma unroll
        for (int t = 0; t < PMAX; ++t) {
            const int e = threadIdx.x + t * FUSED_THREADS;
            const int rr = e / N, x = e - rr * N, y = y0 + rr;
            ru[t] = 0.f;
            rn[t] = 0.f;
            if (e < FQ * N && y < N) {
                ru[t] = shifted_pixel(a, img, pc, x, y);
                if (!a.zero_mask && mask_weight(a, x, y) >= 0.f) rn[t] = noise[(size_t)y * N + x];
            }
        }
    };
    fetch(0);
    for (int y0 = 0; y0 < N; y0 += FQ) {
#pragma unroll
        for (int t = 0; t < PMAX; ++t) {
            const int e = threadIdx.x + t * FUSED_THREADS;
            if (e >= FQ * N) continue;
            const int rr = e / N, x = e - rr * N, y = y0 + rr;
            const float u = ru[t];
            const float w = mask_weight(a, x, y);
            float m = u;
            if (w >= 0.f) {
                const float fill = a.zero_mask ? bgv : rn[t];
                m = (w >= 1.f) ? fill : (1.f - w) * u + w * fill;
            }
            A[e] = y < N ? make_float2(m, u) : make_float2(0.f, 0.f);
        }
        __syncthreads();
        if (y0 + FQ < N) fetch(y0 + FQ);
        const float2* r = fft_any<NC, false>(A, B, FQ, a.plan, s_tw);
        for (int e = threadIdx.x; e < FQ * h; e += blockDim.x) {
            const int rr = e / h, k = e - rr * h, y = y0 + rr;
            if (y >= N) continue;
            const float2 zk = r[rr * N + k];
            const float2 zc = r[rr * N + (N - k) % N];
            SM[(size_t)y * h + k] = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y - zc.y));
            SU[(size_t)y * h + k] = make_float2(0.5f * (zk.y + zc.y), -0.5f * (zk.x - zc.x));
        }
        __syncthreads();
    }
    // columns: C of each half spectrum per chunk, forward FFT over y
    const double* par = a.par + (size_t)p * NPAR;
    const double az = par[7] * (PI_D / 180.);
    const double ca = cos(az), sa = sin(az);
    const double Axx = -par[5] * ca * ca - par[6] * sa * sa;
    const double Axy = (par[6] - par[5]) * ca * sa;
    const double Ayy = -par[5] * sa * sa - par[6] * ca * ca;
    const float inv = 1.f / ((float)N * (float)N);
    const int s = a.s, hs = a.hs;
    const size_t o = (size_t)p * a.P;
    for (int j0 = 0; j0 < h; j0 += C) {
        for (int e = threadIdx.x; e < 2 * C * N; e += blockDim.x) {
            const int i = e % N, q = e / N, half = q / C, j = j0 + (q - half * C);
            A[e] = j < h ? (half ? SU : SM)[(size_t)i * h + j] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        const float2* r = fft_any<NC, false>(A, B, 2 * C, a.plan, s_tw);
        for (int e = threadIdx.x; e < C * N; e += blockDim.x) {
            const int i = e % N, c = e / N, j = j0 + c;
            if (j >= h) continue;
            const float2 f = r[e];
            const float fr = f.x * inv, fi = f.y * inv;
            PW[(size_t)i * h + j] = fr * fr + fi * fi;
        }
        if (j0 < hs)
            for (int e = threadIdx.x; e < C * s; e += blockDim.x) {
                const int c = e % C, iw = e / C, j = j0 + c;
                if (j >= hs) continue;
                const int ky = iw < hs ? iw : iw - s;
                const int i = ky >= 0 ? ky : ky + N;
                const float sg = ((iw ^ j) & 1) ? -inv : inv;
                const float2 fm = r[c * N + i], fu = r[(C + c) * N + i];
                const size_t w = o + (size_t)iw * hs + j;
                reinterpret_cast<float2*>(a.fimg)[w] = make_float2(fm.x * sg, fm.y * sg);
                reinterpret_cast<float2*>(a.fnm)[w] = make_float2(fu.x * sg, fu.y * sg);
                a.ctf[w] = a.do_ctf ? ctf_value(a, par, Axx, Axy, Ayy, j, ky) : 1.f;
                a.minv[w] = a.minv_img[(size_t)iw * hs + j];
            }
        __syncthreads();
    }
    // ring sums (fixed order per ring) and the scalars; the ring lists are staged in
    // the free row scratch (they fit for every N of this kernel)
    int* s_pix = reinterpret_cast<int*>(A);
    double* spec = reinterpret_cast<double*>(PW + (size_t)N * h);
    const int npix = a.ring_off[h];
    for (int q = threadIdx.x; q < npix; q += blockDim.x) s_pix[q] = a.ring_pix[q];
    __syncthreads();
    ring_sums(PW, a.ring_off, s_pix, h, spec, a.power ? a.power + (size_t)p * h : nullptr);
    __syncthreads();
    if (threadIdx.x == 0) {
        double xi2 = 0.;
        if (s < N)
            for (int r = hs; r < h; ++r) xi2 += spec[r];
        double* sc = a.sc + (size_t)p * 8;
        sc[0] = a.minv_dc;
        sc[1] = xi2;
        sc[2] = pc.tx;
        sc[3] = pc.ty;
        sc[4] = (par[2] > 998.99 && par[2] < 999.01) ? 0. : par[2];
        sc[5] = (par[3] > 998.99 && par[3] < 999.01) ? 0. : par[3];
        sc[6] = par[11];
        sc[7] = 0.;
    }
}

// ------------------------------------------------------------ host side

// compile-time sizes of the fused kernels (other sizes run the same kernels with the runtime plan)
#define T2B_PREP_SIZES(X) X(64) X(72) X(80) X(96) X(100) X(120) X(128)

using PrepKernel = void (*)(PrepArgs);
PrepKernel fused_kernel(int N, bool noise)
{
#define T2B_CASE(n) \
    if (N == n) return noise ? (PrepKernel)k_noise_fused<n> : (PrepKernel)k_prep_fused<n>;
    T2B_PREP_SIZES(T2B_CASE)
#undef T2B_CASE
    return noise ? (PrepKernel)k_noise_fused<0> : (PrepKernel)k_prep_fused<0>;
}

double host_round(double x) { return x > 0 ? (double)(int)(x + 0.5) : (double)(int)(x - 0.5); }

template <typename T>
T* dalloc(ImagePrep& G, size_t count)
{
    void* p = nullptr;
    if (count == 0) count = 1;
    T2B_CUDA(cudaMalloc(&p, count * sizeof(T)));
    G.allocs.push_back(p);
    return static_cast<T*>(p);
}

void free_prep(ImagePrep* G)
{
    if (!G) return;
    for (void* p : G->allocs) cudaFree(p);
    delete G;
}

size_t smem_rows(const ImagePrep& G) { return sizeof(float2) * ((size_t)G.N + 2 * (size_t)G.rpb * G.N); }
size_t smem_noise_cols(const ImagePrep& G) { return sizeof(float2) * ((size_t)G.N + 2 * (size_t)G.cpb * G.N); }
size_t smem_cols(const ImagePrep& G) { return sizeof(float2) * ((size_t)G.N + 4 * (size_t)G.cpb * G.N); }

PrepArgs make_args(const ImagePrep& G, int n, const float* img, const double* par, const long long* pid,
                   const t2b_prep_out& o)
{
    const t2b_prep_config& cf = G.cfg;
    PrepArgs a{};
    a.plan = G.plan;
    a.N = G.N;
    a.h = G.h;
    a.s = G.s;
    a.hs = G.hs;
    a.P = G.P;
    a.rpb = G.rpb;
    a.cpb = G.cpb;
    a.zero_mask = cf.zero_mask;
    a.do_ctf = cf.do_ctf_correction;
    a.premult = cf.ctf_premultiplied;
    a.do_abs = cf.ctf_phase_flipped;
    a.flip = cf.only_flip_phases;
    a.intact = cf.intact_ctf_first_peak;
    a.seed = cf.random_seed;
    a.radius = (float)cf.mask_radius;
    a.width = (float)cf.width_mask_edge;
    a.norm_on = cf.do_norm_correction ? 1. : 0.;
    a.avg_norm = cf.avg_norm_correction;
    a.xs = (double)G.N * cf.pixel_size;
    // CTF::initialise (src/ctf.cpp:206-235)
    const double kV = cf.voltage * 1e3;
    const double lam = 12.2643247 / std::sqrt(kV * (1. + kV * 0.978466e-6));
    a.lam_k1 = PI_D / 2 * 2 * lam;
    a.k2 = PI_D / 2 * (cf.cs * 1e7) * lam * lam * lam;
    a.k3 = std::atan(cf.q0 / std::sqrt(1 - cf.q0 * cf.q0));
    a.minv_dc = G.minv_dc;
    a.tw = G.tw;
    a.noise_sig = G.noise_sig;
    a.minv_img = G.minv;
    a.ring_off = G.ring_off;
    a.ring_pix = G.ring_pix;
    a.img = img;
    a.par = par;
    a.pid = pid;
    a.gm = G.gm;
    a.gu = G.gu;
    a.gn = G.gn;
    a.noise = G.noise;
    a.pw = G.pw;
    a.bg = G.bg;
    a.fimg = o.fimg;
    a.fnm = o.fimg_nomask;
    a.ctf = o.ctf;
    a.minv = o.minvsigma2;
    a.sc = o.scalars;
    a.power = o.power;
    (void)n;
    return a;
}

int enqueue_prep(const ImagePrep& G, const PrepArgs& a, int n, cudaStream_t st)
{
    int launches = 0;
    if (G.fused) {
        if (!G.cfg.zero_mask) {
            fused_kernel(G.N, true)<<<n, FUSED_THREADS, fused_noise_smem(G.N), st>>>(a);
            ++launches;
        }
        fused_kernel(G.N, false)<<<n, FUSED_THREADS, fused_prep_smem(G.N), st>>>(a);
        T2B_CUDA(cudaGetLastError());
        return launches + 1;
    }
    const dim3 grow(n, (G.N + G.rpb - 1) / G.rpb), gcol(n, G.ncol_blocks);
    if (!G.cfg.zero_mask) {
        k_noise_cols<<<gcol, PREP_THREADS, smem_noise_cols(G), st>>>(a);
        k_noise_rows<<<grow, PREP_THREADS, smem_rows(G), st>>>(a);
        launches += 2;
    } else {
        k_background<<<n, PREP_THREADS, 0, st>>>(a);
        launches += 1;
    }
    k_rows<<<grow, PREP_THREADS, smem_rows(G), st>>>(a);
    k_cols<<<gcol, PREP_THREADS, smem_cols(G), st>>>(a);
    k_final<<<n, PREP_THREADS, 0, st>>>(a);
    launches += 3;
    T2B_CUDA(cudaGetLastError());
    return launches;
}

void check_out(const t2b_prep_out* o)
{
    T2B_REQUIRE(o && o->fimg && o->fimg_nomask && o->ctf && o->minvsigma2 && o->scalars, T2B_ERR_ARG,
                "t2b_prep_out: fimg, fimg_nomask, ctf, minvsigma2 and scalars are required");
}

}  // namespace

void imageprep_release(t2b_ctx* c)
{
    free_prep(c->prep);
    c->prep = nullptr;
}

}  // namespace t2b

using namespace t2b;

extern "C" {

int t2b_prep_configure(t2b_ctx* c, const t2b_prep_config* cf)
{
    return guarded([&] {
        T2B_REQUIRE(c && cf, T2B_ERR_ARG, "null argument");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        const int N = cf->image_size, s = cf->current_size;
        T2B_REQUIRE(N >= 8 && N <= PREP_MAX_N && N % 2 == 0, T2B_ERR_UNSUPPORTED, "image_size must be even, 8..512");
        T2B_REQUIRE(s >= 2 && s <= N && s % 2 == 0, T2B_ERR_ARG, "current_size must be even and <= image_size");
        T2B_REQUIRE(cf->max_batch >= 1, T2B_ERR_ARG, "max_batch must be positive");
        T2B_REQUIRE(cf->sigma2_noise && cf->n_sigma2 >= 1, T2B_ERR_ARG, "sigma2_noise is required");
        T2B_REQUIRE(cf->sigma2_fudge > 0. && cf->pixel_size > 0. && cf->width_mask_edge > 0., T2B_ERR_ARG,
                    "sigma2_fudge, pixel_size and width_mask_edge must be positive");
        T2B_REQUIRE(cf->q0 >= 0. && cf->q0 < 1. && cf->voltage > 0., T2B_ERR_ARG, "bad optics (voltage, q0)");
        T2B_REQUIRE(!cf->do_norm_correction || cf->avg_norm_correction > 0., T2B_ERR_ARG,
                    "avg_norm_correction must be positive");
        const FftPlan plan = fft_plan(N);
        free_prep(c->prep);
        c->prep = nullptr;
        ImagePrep* G = new ImagePrep();
        try {
            G->cfg = *cf;
            G->cfg.sigma2_noise = nullptr;
            G->N = N;
            G->h = N / 2 + 1;
            G->s = s;
            G->hs = s / 2 + 1;
            G->P = s * G->hs;
            G->max_batch = cf->max_batch;
            G->plan = plan;
            G->rpb = std::max(1, std::min(16, 16384 / N));
            G->cpb = std::max(1, std::min(16, (96 * 1024) / (32 * N)));
            G->ncol_blocks = (G->h + G->cpb - 1) / G->cpb;
            const int h = G->h, hs = G->hs;
            // twiddles in FP64 on the host
            std::vector<float2> tw(N);
            for (int t = 0; t < N; ++t) {
                const double ang = -2.0 * PI_D * (double)t / (double)N;
                tw[t] = make_float2((float)std::cos(ang), (float)std::sin(ang));
            }
            // noise spectrum amplitude per ring (src/ml_optimiser.cpp:6196-6213)
            std::vector<double> rem(h, 0.), nsig(h, 0.);
            for (int i = 0; i < cf->n_sigma2; ++i) {
                const int ir = (int)host_round(cf->remap_noise * i);
                if (ir >= 0 && ir < h) rem[ir] = cf->sigma2_noise[i];
            }
            for (int i = 0; i < h; ++i) nsig[i] = std::sqrt(cf->sigma2_fudge * rem[i]);
            // Minvsigma2 of the window (src/ml_optimiser.cpp:6706-6719; Mresol :5628-5643)
            std::vector<float> minv(G->P, 0.f);
            for (int iw = 0; iw < s; ++iw)
                for (int j = 0; j < hs; ++j) {
                    const int ky = iw < hs ? iw : iw - s;
                    const int ires = (int)host_round(std::sqrt((double)(ky * ky + j * j)));
                    if (ires >= hs || (j == 0 && ky < 0) || ires <= 0) continue;
                    const int irr = (int)host_round(cf->remap_minv * ires);
                    if (irr < cf->n_sigma2) minv[(size_t)iw * hs + j] = (float)(1. / (cf->sigma2_fudge * cf->sigma2_noise[irr]));
                }
            G->minv_dc = cf->sigma2_noise[0] > 0. ? 1. / (cf->sigma2_fudge * cf->sigma2_noise[0]) : 0.;
            // spectrum rings of the full transform (src/ml_optimiser.cpp:6253-6266)
            std::vector<std::vector<int>> rings(h);
            for (int i = 0; i < N; ++i)
                for (int j = 0; j < h; ++j) {
                    const int ky = i < h ? i : i - N;
                    const int ires = (int)host_round(std::sqrt((double)(ky * ky + j * j)));
                    if (ires > 0 && ires < h && !(j == 0 && ky < 0)) rings[ires].push_back(i * h + j);
                }
            std::vector<int> off(h + 1, 0), pix;
            for (int r = 0; r < h; ++r) {
                off[r] = (int)pix.size();
                pix.insert(pix.end(), rings[r].begin(), rings[r].end());
            }
            off[h] = (int)pix.size();
            const size_t B = cf->max_batch, NH = (size_t)N * h;
            int optin = 0;
            T2B_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
            // static shared memory of k_prep_fused: the two FP64 reduction arrays
            // (the fused kernel stages the ring lists in its row scratch: 2 FQ N float2)
            G->fused = fused_prep_smem(N) + 2 * FUSED_THREADS * sizeof(double) <= (size_t)optin &&
                       pix.size() <= (size_t)4 * FQ * N;
            G->tw = dalloc<float2>(*G, N);
            G->noise_sig = dalloc<double>(*G, h);
            G->minv = dalloc<float>(*G, G->P);
            G->ring_off = dalloc<int>(*G, h + 1);
            G->ring_pix = dalloc<int>(*G, pix.size());
            G->bg = dalloc<double>(*G, B);
            if (!G->fused) {
                G->gm = dalloc<float2>(*G, B * NH);
                G->gu = dalloc<float2>(*G, B * NH);
                G->pw = dalloc<float>(*G, B * NH);
                if (!cf->zero_mask) G->gn = dalloc<float2>(*G, B * NH);
            }
            if (!cf->zero_mask) G->noise = dalloc<float>(*G, B * (size_t)N * N);
            T2B_CUDA(cudaMemcpy(G->tw, tw.data(), N * sizeof(float2), cudaMemcpyHostToDevice));
            T2B_CUDA(cudaMemcpy(G->noise_sig, nsig.data(), h * sizeof(double), cudaMemcpyHostToDevice));
            T2B_CUDA(cudaMemcpy(G->minv, minv.data(), G->P * sizeof(float), cudaMemcpyHostToDevice));
            T2B_CUDA(cudaMemcpy(G->ring_off, off.data(), (h + 1) * sizeof(int), cudaMemcpyHostToDevice));
            if (!pix.empty())
                T2B_CUDA(cudaMemcpy(G->ring_pix, pix.data(), pix.size() * sizeof(int), cudaMemcpyHostToDevice));
            if (G->fused) {
                T2B_CUDA(cudaFuncSetAttribute((const void*)fused_kernel(N, false),
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_prep_smem(N)));
                T2B_CUDA(cudaFuncSetAttribute((const void*)fused_kernel(N, true),
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_noise_smem(N)));
            } else {
                const int big = (int)std::max(smem_rows(*G), std::max(smem_cols(*G), smem_noise_cols(*G)));
                for (const void* k : {(const void*)k_rows, (const void*)k_cols, (const void*)k_noise_cols,
                                      (const void*)k_noise_rows})
                    T2B_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
            }
        } catch (...) {
            free_prep(G);
            throw;
        }
        c->prep = G;
    });
}

int t2b_prep_batch_device(t2b_ctx* c, const t2b_prep_batch* b, const t2b_prep_out* o, void* stream)
{
    return guarded([&] {
        T2B_REQUIRE(c && b, T2B_ERR_ARG, "null argument");
        check_out(o);
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        T2B_REQUIRE(c->prep, T2B_ERR_STATE, "t2b_prep_configure must be called first");
        const ImagePrep& G = *c->prep;
        T2B_REQUIRE(b->n >= 1 && b->n <= G.max_batch, T2B_ERR_ARG, "batch size out of range");
        T2B_REQUIRE(b->images && b->params && (b->part_id || G.cfg.zero_mask), T2B_ERR_ARG,
                    "images, params (and part_id for the noise background) are required");
        cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
        const PrepArgs a = make_args(G, b->n, b->images, b->params, b->part_id, *o);
        enqueue_prep(G, a, b->n, st);
    });
}

int t2b_prep_batch_host(t2b_ctx* c, const t2b_prep_batch* b, const t2b_prep_out* o)
{
    return guarded([&] {
        T2B_REQUIRE(c && b, T2B_ERR_ARG, "null argument");
        check_out(o);
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        T2B_REQUIRE(c->prep, T2B_ERR_STATE, "t2b_prep_configure must be called first");
        ImagePrep& G = *c->prep;
        const int n = b->n;
        T2B_REQUIRE(n >= 1 && n <= G.max_batch, T2B_ERR_ARG, "batch size out of range");
        T2B_REQUIRE(b->images && b->params && (b->part_id || G.cfg.zero_mask), T2B_ERR_ARG,
                    "images, params (and part_id for the noise background) are required");
        const size_t B = G.max_batch, NN = (size_t)G.N * G.N, P = G.P;
        if (!G.h_img) {
            G.h_img = dalloc<float>(G, B * NN);
            G.h_par = dalloc<double>(G, B * NPAR);
            G.h_pid = dalloc<long long>(G, B);
            G.o_fimg = dalloc<float>(G, B * 2 * P);
            G.o_fnm = dalloc<float>(G, B * 2 * P);
            G.o_ctf = dalloc<float>(G, B * P);
            G.o_minv = dalloc<float>(G, B * P);
            G.o_sc = dalloc<double>(G, B * 8);
            G.o_pw = dalloc<double>(G, B * G.h);
        }
        cudaStream_t st = c->stream;
        T2B_CUDA(cudaMemcpyAsync(G.h_img, b->images, n * NN * sizeof(float), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemcpyAsync(G.h_par, b->params, n * NPAR * sizeof(double), cudaMemcpyHostToDevice, st));
        if (b->part_id)
            T2B_CUDA(cudaMemcpyAsync(G.h_pid, b->part_id, n * sizeof(long long), cudaMemcpyHostToDevice, st));
        else
            T2B_CUDA(cudaMemsetAsync(G.h_pid, 0, n * sizeof(long long), st));
        t2b_prep_out d{G.o_fimg, G.o_fnm, G.o_ctf, G.o_minv, G.o_sc, o->power ? G.o_pw : nullptr};
        const PrepArgs a = make_args(G, n, G.h_img, G.h_par, G.h_pid, d);
        enqueue_prep(G, a, n, st);
        T2B_CUDA(cudaMemcpyAsync(o->fimg, G.o_fimg, n * 2 * P * sizeof(float), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaMemcpyAsync(o->fimg_nomask, G.o_fnm, n * 2 * P * sizeof(float), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaMemcpyAsync(o->ctf, G.o_ctf, n * P * sizeof(float), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaMemcpyAsync(o->minvsigma2, G.o_minv, n * P * sizeof(float), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaMemcpyAsync(o->scalars, G.o_sc, n * 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (o->power)
            T2B_CUDA(cudaMemcpyAsync(o->power, G.o_pw, n * (size_t)G.h * sizeof(double), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaStreamSynchronize(st));
    });
}

}  // extern "C"
