// E-step stages of libt2b for sm_100a.
//
// Data flow of one batch of particles (all on the device, no host sync):
//   prep      cvec = Minvsigma2 * scale * CTF * X, w2 = 0.5 * Minvsigma2 * (scale CTF)^2,
//             c0 = highres_Xi2/2 + sum 0.5 Minvsigma2 |X|^2
//   norms     N[b][oc] = sum_p w2[b][p] |P_oc[p]|^2
//   diff2     D[b][oc*T+t] = c0[b] + N[b][oc] - sum_p Re(P_oc[p] conj(cvec_b[p] ab_t[p]))
//             which equals highres_Xi2/2 + sum_p 0.5 M |scale CTF P - shift_t X|^2
//             (src/ml_optimiser.cpp:7251-7272; the reference GPU kernel splits the
//             same three terms, coarse_splitImg_BCF_PMO.cuh:139-693)
//   weights   w = pdf_o pdf_t exp(-(D - min)) in FP64, sum, significance threshold by
//             an exact MSB-first radix search on the FP64 bit patterns
//             (src/ml_optimiser.cpp:7770-7990, sort + cumulative sum)
//   compact   ordered list of significant coarse pairs per particle
//   fine      32 fine hypotheses per significant pair (8 rotations x 4 shifts)
//   weights   same on the fine set
//   wsum+BP   per (particle, significant orientation): weighted sums, sigma2 rings,
//             prior sums, then trilinear backprojection with float2 atomics
//             (src/ml_optimiser.cpp:8153-8700, src/backprojector.cpp:55-230)
#include "t2b_internal.cuh"
#include "project_pixel.cuh"
#include <map>
#include <algorithm>
#include <cfloat>
#include <type_traits>

namespace t2b {
namespace {

__device__ __forceinline__ unsigned f2key(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key2f(unsigned k)
{
    const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

template <typename T>
__device__ T block_sum(T v, T* sh /* >= 32 */)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : T(0);
    if (wid == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (threadIdx.x == 0) sh[0] = v;
    __syncthreads();
    const T r = sh[0];
    __syncthreads();
    return r;
}

// ------------------------------------------------------------------ prep
__global__ void k_prep(Tables tb, Work w)
{
    __shared__ double sh[32];
    const int b = blockIdx.x, P = tb.P;
    const double* sc = w.scal + 8 * (size_t)b;
    const float scale = (float)sc[6];
    double acc = 0.;
    for (int n = threadIdx.x; n < P; n += blockDim.x) {
        const float2 X = w.fimg[(size_t)b * P + n];
        const float M = w.minv[(size_t)b * P + n];
        const float c = w.ctf[(size_t)b * P + n] * scale;
        const float mc = M * c;
        w.cvec[(size_t)b * P + n] = make_float2(mc * X.x, mc * X.y);
        w.w2[(size_t)b * P + n] = 0.5f * M * c * c;
        acc += 0.5 * (double)M * ((double)X.x * X.x + (double)X.y * X.y);
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) {
        w.c0[b] = (float)(sc[1] / 2. + acc);
        w.minkey_c[b] = 0xffffffffu;
        w.minkey_f[b] = 0xffffffffu;
        w.sum_c[b] = 0.;
        w.sum_f[b] = 0.;
        w.status[b] = T2B_OK;
        SelState z{};
        z.argmax = 0x7fffffffffffffffLL;
        w.sel_c[b] = z;
        w.sel_f[b] = z;
        w.r_norm[b] = 0.; w.r_sumw[b] = 0.; w.r_sig_off[b] = 0.;
        if (w.r_xa) w.r_xa[b] = 0.;
        if (w.r_aa) w.r_aa[b] = 0.;
    }
    const int half = tb.ori_size / 2 + 1;
    for (int i = threadIdx.x; i < half; i += blockDim.x) w.r_sigma2[(size_t)b * half + i] = 0.;
    for (int i = threadIdx.x; i < tb.K; i += blockDim.x) w.r_pdf_class[(size_t)b * tb.K + i] = 0.;
    for (int i = threadIdx.x; i < tb.K * tb.n_dir; i += blockDim.x) w.r_pdf_dir[(size_t)b * tb.K * tb.n_dir + i] = 0.;
    for (int i = threadIdx.x; i < HIST_BINS; i += blockDim.x) {
        w.hist_cnt[(size_t)b * HIST_BINS + i] = 0;
        w.hist_sum[(size_t)b * HIST_BINS + i] = 0.;
    }
}

// ----------------------------------------------------------------- norms
// N[b][oc] = sum_p w2[b][p] |P_oc[p]|^2 ; tile 128 orientations x 64 particles,
// 4 x 8 outputs per thread, 16 pixels per shared-memory stage.
__global__ void __launch_bounds__(256) k_norms(Tables tb, Work w, const float2* __restrict__ proj, int nrows,
                                               float* __restrict__ out)
{
    __shared__ __align__(16) float Ps[16][132];
    __shared__ __align__(16) float Ws[16][68];
    const int o0 = blockIdx.x * 128, b0 = blockIdx.y * 64, P = tb.P;
    const int tx = threadIdx.x & 7, ty = threadIdx.x >> 3;  // 8 particle groups x 32 orientation groups
    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
    const int nk = tb.nk;
    for (int p0 = 0; p0 < nk; p0 += 16) {
        for (int idx = threadIdx.x; idx < 128 * 16; idx += 256) {
            const int oo = idx >> 4, pp = idx & 15;
            float v = 0.f;
            if (o0 + oo < nrows && p0 + pp < nk) {
                const float2 z = proj[(size_t)(o0 + oo) * P + tb.kpix[p0 + pp]];
                v = z.x * z.x + z.y * z.y;
            }
            Ps[pp][oo] = v;
        }
        for (int idx = threadIdx.x; idx < 64 * 16; idx += 256) {
            const int bb = idx >> 4, pp = idx & 15;
            Ws[pp][bb] = (b0 + bb < w.n && p0 + pp < nk) ? w.w2[(size_t)(b0 + bb) * P + tb.kpix[p0 + pp]] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int pp = 0; pp < 16; pp++) {
            const float4 pv = *reinterpret_cast<const float4*>(&Ps[pp][ty * 4]);
            const float4 w0 = *reinterpret_cast<const float4*>(&Ws[pp][tx * 8]);
            const float4 w1 = *reinterpret_cast<const float4*>(&Ws[pp][tx * 8 + 4]);
            const float a[4] = {pv.x, pv.y, pv.z, pv.w};
            const float c[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(a[i], c[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int bb = b0 + tx * 8 + j;
        if (bb >= w.n) continue;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int o = o0 + ty * 4 + i;
            if (o < nrows) out[(size_t)bb * nrows + o] = acc[i][j];
        }
    }
}

// --------------------------------------------------- plain FP32 diff2 GEMM
// C[oc][col] = sum_k Bm[oc][k] A[col][k], k over interleaved (re, im) of the P
// pixels, col = b*T + t.  A is built on the fly from cvec and the phase table.
// 128 x 128 tile, 256 threads, 8x8 register micro-tile, double-buffered smem.
constexpr int SB_M = 128, SB_N = 128, SB_KP = 8, SB_K = 16, SB_LD = 132;

__global__ void __launch_bounds__(256, 2) k_diff2_simt(Tables tb, Work w)
{
    __shared__ __align__(16) float Bs[2][SB_K][SB_LD];
    __shared__ __align__(16) float As[2][SB_K][SB_LD];
    __shared__ unsigned smin[SB_N + 2];
    const int P = tb.P, T = tb.T, KO = tb.K * tb.O;
    const int m0 = blockIdx.x * SB_M, n0 = blockIdx.y * SB_N;
    const int ncols = w.n * T;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int bfirst = n0 / T;

    // loader coordinates: thread loads rows/cols (tid>>3) + 32*j, pixel (tid & 7)
    const int lrow = tid >> 3, lp = tid & 7;
    int la_b[4], la_t[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int col = n0 + lrow + 32 * j;
        la_b[j] = col < ncols ? col / T : -1;
        la_t[j] = col < ncols ? col - (col / T) * T : 0;
    }
    float2 rb[4], ra[4];
    const int nk = tb.nk;
    auto gload = [&](int p0) {
        const bool in = p0 + lp < nk;
        const int p = in ? tb.kpix[p0 + lp] : 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int row = m0 + lrow + 32 * j;
            rb[j] = (row < KO && in) ? tb.proj_c[(size_t)row * P + p] : make_float2(0.f, 0.f);
            if (la_b[j] >= 0 && in) {
                const float2 c = w.cvec[(size_t)la_b[j] * P + p];
                const float2 ab = tb.ab_c[(size_t)la_t[j] * P + p];
                ra[j] = make_float2(c.x * ab.x - c.y * ab.y, c.x * ab.y + c.y * ab.x);
            } else {
                ra[j] = make_float2(0.f, 0.f);
            }
        }
    };
    auto sstore = [&](int buf) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            Bs[buf][2 * lp][lrow + 32 * j] = rb[j].x;
            Bs[buf][2 * lp + 1][lrow + 32 * j] = rb[j].y;
            As[buf][2 * lp][lrow + 32 * j] = ra[j].x;
            As[buf][2 * lp + 1][lrow + 32 * j] = ra[j].y;
        }
    };
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
    for (int i = tid; i < SB_N + 2; i += 256) smin[i] = 0xffffffffu;

    gload(0);
    sstore(0);
    __syncthreads();
    int buf = 0;
    for (int p0 = 0; p0 < nk; p0 += SB_KP) {
        const bool more = p0 + SB_KP < nk;
        if (more) gload(p0 + SB_KP);
#pragma unroll
        for (int k = 0; k < SB_K; k++) {
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][k][ty * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][k][64 + ty * 4]);
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][k][tx * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][k][64 + tx * 4]);
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(bv[i], av[j], acc[i][j]);
        }
        if (more) {
            sstore(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }
    // epilogue
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int oc = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (oc >= KO) continue;
        const bool skip = tb.skip[oc] != 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int col = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (col >= ncols) continue;
            const int b = col / T, t = col - b * T;
            float d;
            if (skip) {
                d = -999.f;
            } else {
                d = w.c0[b] + w.norms[(size_t)b * KO + oc] - acc[i][j];
                atomicMin(&smin[b - bfirst], f2key(d));
            }
            w.d2c[((size_t)b * KO + oc) * T + t] = d;
        }
    }
    __syncthreads();
    const int nb = min(SB_N / T + 2, SB_N + 2);
    for (int i = tid; i < nb; i += 256) {
        const int b = bfirst + i;
        if (b < w.n && smin[i] != 0xffffffffu) atomicMin(&w.minkey_c[b], smin[i]);
    }
}

// ---------------------------------------------------------------- priors
// pdf_offset of every coarse translation, normalised by its mean
// (src/ml_optimiser.cpp:7629-7716), and the per-particle bounds of
// log(pdf_orientation * pdf_offset) used to skip exp() outside a diff2 window.
// One CTA per particle.
__global__ void k_pdf_t(Tables tb, Work w)
{
    __shared__ double sh[32];
    __shared__ double smin[32], smax[32];
    const int b = blockIdx.x, T = tb.T;
    const double* sc = w.scal + 8 * (size_t)b;
    double local = 0.;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        const double ox = sc[2] + tb.trans_prior[2 * t], oy = sc[3] + tb.trans_prior[2 * t + 1];
        double td = (ox - sc[4]) * (ox - sc[4]) + (oy - sc[5]) * (oy - sc[5]);
        td *= tb.pixel_size * tb.pixel_size;
        double v;
        if (tb.sigma2_offset < 0.0001) v = td > 0. ? 0. : 1.;
        else v = exp(td / (-2. * tb.sigma2_offset)) / (2. * 3.14159265358979323846 * tb.sigma2_offset);
        w.pdf_t[(size_t)b * T + t] = v;
        local += v;
    }
    const double mean = block_sum(local, sh) / T;
    double lmin = INFINITY, lmax = -INFINITY;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        double v = w.pdf_t[(size_t)b * T + t];
        if (mean > 0.) v /= mean;
        w.pdf_t[(size_t)b * T + t] = v;
        const double lv = v > 0. ? log(v) : -INFINITY;
        lmin = fmin(lmin, lv);
        lmax = fmax(lmax, lv);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
        lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    }
    if ((threadIdx.x & 31) == 0) { smin[threadIdx.x >> 5] = lmin; smax[threadIdx.x >> 5] = lmax; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)((blockDim.x + 31) >> 5); i++) { lmin = fmin(lmin, smin[i]); lmax = fmax(lmax, smax[i]); }
        lmin = fmin(lmin, smin[0]);
        lmax = fmax(lmax, smax[0]);
        w.lbound[2 * b] = tb.lpo_min + lmin;
        w.lbound[2 * b + 1] = tb.lpo_max + lmax;
    }
}

// ------------------------------------------------------- weights (FP64)
// Coarse weights are never stored: every pass recomputes
//     w = pdf_o pdf_t exp(-(diff2 - min))      (0 if diff2 - min > 700)
// from the FP32 diff2 array, and skips the exp() outside the diff2 window in
// which w can fall into the range the pass looks for (bounds from the
// per-particle extremes of log(pdf_o pdf_t)).  Fine weights are stored (the
// weighted sums read them).
__device__ __forceinline__ double coarse_weight_ot(const Tables& tb, const Work& w, int b, long long oc, int t, float d,
                                                   double mn)
{
    if (d < 0.f) return 0.;
    const double dd = (double)d - mn;
    if (dd > 700.) return 0.;
    return tb.pdf_oc[oc] * w.pdf_t[(size_t)b * tb.T + t] * exp(-dd);
}

// Learned proposals: while *w.gate != 0 the coarse arrays of particle b hold
// kprop x T elements, proposal j being the global orientation w.prop[b*kprop+j];
// otherwise K*O x T elements in global orientation order.
__device__ __forceinline__ bool prop_mode(const Work& w) { return w.gate && *w.gate != 0; }
__device__ __forceinline__ long long coarse_n(const Tables& tb, const Work& w, bool pm)
{
    return pm ? (long long)w.kprop * tb.T : (long long)tb.K * tb.O * tb.T;
}
__device__ __forceinline__ long long glob_oc(const Work& w, int b, long long oc, bool pm)
{
    return pm ? (long long)w.prop[(size_t)b * w.kprop + oc] : oc;
}
__device__ __forceinline__ long long glob_il(const Tables& tb, const Work& w, int b, long long il, bool pm)
{
    if (!pm) return il;
    const long long j = il / tb.T;
    return glob_oc(w, b, j, true) * tb.T + (il - j * tb.T);
}

__device__ __forceinline__ double coarse_weight(const Tables& tb, const Work& w, int b, long long il, float d, double mn,
                                                bool pm)
{
    const long long oc = il / tb.T;
    return coarse_weight_ot(tb, w, b, glob_oc(w, b, oc, pm), (int)(il - oc * tb.T), d, mn);
}

// (orientation, translation) of consecutive coarse elements without divisions
struct OcT {
    long long oc;
    int t;
    __device__ __forceinline__ OcT(long long i, int T) : oc(i / T), t((int)(i - (i / T) * T)) {}
    __device__ __forceinline__ void next(int T)
    {
        if (++t == T) { t = 0; ++oc; }
    }
};

__device__ __forceinline__ double fine_prior(const Tables& tb, const Work& w, int b, long long i)
{
    const long long ih = w.pairs[i / ((long long)tb.R * tb.V)];
    const long long oc = ih / tb.T;
    const int t = (int)(ih - oc * tb.T);
    const int k = (int)(oc / tb.O), o = (int)(oc - (long long)k * tb.O), idir = o / tb.n_psi;
    return tb.pdf_o[k * tb.n_dir + idir] * w.pdf_t[(size_t)b * tb.T + t];
}

// diff2 window (lo, hi] outside which w cannot lie in [wlo, whi)
constexpr double WIN_EPS = 1e-6;
__device__ __forceinline__ void dwindow(double wlo, double whi, double mn, double Lmin, double Lmax, double& lo, double& hi)
{
    lo = (whi > 0. && whi < INFINITY && Lmin > -INFINITY) ? mn + Lmin - log(whi) - WIN_EPS : -INFINITY;
    hi = (wlo > 0.) ? mn + Lmax - log(wlo) + WIN_EPS : INFINITY;
}

__device__ __forceinline__ double bits2d(unsigned long long u)
{
    return u >= 0x7ff0000000000000ull ? INFINITY : __longlong_as_double((long long)u);
}

// digit layout of the radix search over the 64-bit pattern of positive doubles
__device__ __forceinline__ int digit_width(int shift) { return shift == 0 ? 4 : 12; }

struct Seg {
    long long beg, end;   // element range (coarse: local index; fine: global index into d2f / wf)
};

__device__ __forceinline__ Seg seg_of(const Tables& tb, const Work& w, bool fine, int b)
{
    Seg s;
    if (!fine) {
        s.beg = 0;
        s.end = coarse_n(tb, w, prop_mode(w));
    } else {
        const long long rv = (long long)tb.R * tb.V;
        s.beg = w.pair_off[b] * rv;
        s.end = w.pair_off[b + 1] * rv;
    }
    return s;
}

// 16 consecutive diff2 values starting at element i0 (float4 loads when
// aligned); elements at or past `end` read as -1 (no hypothesis).
__device__ __forceinline__ void load16(const float* __restrict__ base, long long i0, long long end, float v[16])
{
    const float* p = base + i0;
    if (i0 + 16 <= end && (reinterpret_cast<uintptr_t>(p) & 15u) == 0) {
        const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float4 f = __ldg(q + j);
            v[4 * j] = f.x; v[4 * j + 1] = f.y; v[4 * j + 2] = f.z; v[4 * j + 3] = f.w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] = (i0 + j < end) ? p[j] : -1.f;
    }
}

// Floor under which a weight can never reach the significance crossing:
// elements below tau hold less than n*tau <= (1-f) max <= (1-f) S of the mass,
// because the weight of the minimum-diff2 element is >= exp(Lmin).  They enter
// the sum but need no histogram entry.
__device__ __forceinline__ double hist_floor(const Tables& tb, const Work& w, int b, long long nseg)
{
    const double Lmin = w.lbound[2 * b];
    if (!(tb.adaptive_fraction < 1.) || !(Lmin > -INFINITY) || nseg <= 0) return 0.;
    return (1. - tb.adaptive_fraction) * exp(Lmin) / (double)nseg;
}

// pass 1: weights (stored for the fine set only), sum, max, level-0 histogram
__global__ void __launch_bounds__(256) k_weights(Tables tb, Work w, int fine)
{
    extern __shared__ unsigned char smem_raw[];
    unsigned* hc = reinterpret_cast<unsigned*>(smem_raw);
    double* hs = reinterpret_cast<double*>(smem_raw + HIST_BINS * sizeof(unsigned));
    __shared__ double sh[32];
    const int b = blockIdx.y;
    if ((fine ? w.sel_f[b] : w.sel_c[b]).fast == 2) return;   // selected by k_select_small
    if (fine && w.status[b] != T2B_OK) return;
    for (int i = threadIdx.x; i < HIST_BINS; i += blockDim.x) { hc[i] = 0; hs[i] = 0.; }
    __syncthreads();
    const Seg sg = seg_of(tb, w, fine, b);
    const bool pm = !fine && prop_mode(w);
    const double mn = (double)key2f(fine ? w.minkey_f[b] : w.minkey_c[b]);
    const float* dsrc = fine ? w.d2f : w.d2c + (size_t)b * (size_t)(sg.end - sg.beg);
    const double tau = hist_floor(tb, w, b, sg.end - sg.beg);
    // weights below exp(Lmin) e^-46 / n add < 1e-20 of the sum in total: no exp() for them
    const double Lmin = w.lbound[2 * b], Lmax = w.lbound[2 * b + 1];
    // and are below the histogram floor tau (so every pass agrees on the candidates)
    double cut = 700.;
    if (Lmin > -INFINITY && sg.end > sg.beg && tau > 0.)
        cut = fmin(700., fmax((Lmax - Lmin) + log((double)(sg.end - sg.beg)) + 46., Lmax - log(tau)));
    double lsum = 0.;
    unsigned long long lmax = 0;
    const long long stride = (long long)gridDim.x * blockDim.x * 16;
    for (long long i0 = sg.beg + ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 16; i0 < sg.end; i0 += stride) {
        float v[16];
        load16(dsrc, i0, sg.end, v);
        OcT ot(fine ? 0 : i0, tb.T);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const long long i = i0 + j;
            const float d = v[j];
            double wt = 0.;
            if (fine) {
                if (i >= sg.end) continue;
                if (d >= 0.f) {
                    const double dd = (double)d - mn;
                    if (dd <= 700.) wt = fine_prior(tb, w, b, i) * exp(-dd);
                }
                w.wf[i] = wt;
            } else {
                if (d >= 0.f && (double)d - mn <= cut) wt = coarse_weight_ot(tb, w, b, glob_oc(w, b, ot.oc, pm), ot.t, d, mn);
                ot.next(tb.T);
            }
            if (wt > 0.) {
                const unsigned long long bits = (unsigned long long)__double_as_longlong(wt);
                lsum += wt;
                lmax = max(lmax, bits);
                if (wt >= tau) {
                    const int dg = (int)(bits >> 52);
                    atomicAdd(&hc[dg], 1u);
                    atomicAdd(&hs[dg], wt);
                }
            }
        }
    }
    lsum = block_sum(lsum, sh);
    for (int o = 16; o > 0; o >>= 1) lmax = max(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    SelState* sel = fine ? &w.sel_f[b] : &w.sel_c[b];
    if ((threadIdx.x & 31) == 0 && lmax) atomicMax(&sel->maxbits, lmax);
    if (threadIdx.x == 0) atomicAdd(fine ? &w.sum_f[b] : &w.sum_c[b], lsum);
    __syncthreads();
    for (int i = threadIdx.x; i < HIST_BINS; i += blockDim.x)
        if (hc[i]) {
            atomicAdd(&w.hist_cnt[(size_t)b * HIST_BINS + i], hc[i]);
            atomicAdd(&w.hist_sum[(size_t)b * HIST_BINS + i], hs[i]);
        }
}

__global__ void k_sel_init(Work w, int fine, double frac)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= w.n) return;
    SelState* sel = fine ? &w.sel_f[b] : &w.sel_c[b];
    if (sel->fast == 2) return;   // selected by k_select_small
    const double S = fine ? w.sum_f[b] : w.sum_c[b];
    if (w.status[b] != T2B_OK) { sel->phase = 3; return; }
    if (!(S > 0.) || S != S) {
        sel->phase = 3;
        w.status[b] = T2B_ERR_NOSIGNIF;
        return;
    }
    sel->target = frac * S;
    sel->cum_above = 0.;
    sel->count_above = 0;
    sel->prefix = 0;
    sel->shift = 52;
    sel->phase = 0;
    sel->ncand = 0;
}

// Choose the digit bin that contains the crossing of the descending
// cumulative sum; narrow the prefix or move on to the gather.  One CTA per
// particle; bins are visited from the largest digit down.
// maxsig > 0 (coarse pass only, src/ml_optimiser.cpp:7945-7966): the walk also stops at
// the maxsig-th largest weight, so the threshold is the weight at rank
// min(crossing, maxsig - 1)
// cond (non-zero during graph capture, level 0 only): set when a particle still needs the
// multi-level search or the candidate gather, the condition of the graph node that holds them
__global__ void __launch_bounds__(1024) k_select(Work w, int fine, int maxsig, cudaGraphConditionalHandle cond)
{
    __shared__ double ssum[1024];
    __shared__ unsigned long long scnt[1024];
    __shared__ int chosen, lastne;
    const int b = blockIdx.x;
    SelState* sel = fine ? &w.sel_f[b] : &w.sel_c[b];
    if (sel->phase != 0) return;
    const int width = digit_width(sel->shift);
    const int nb = 1 << width;
    unsigned* hc = w.hist_cnt + (size_t)b * HIST_BINS;
    double* hs = w.hist_sum + (size_t)b * HIST_BINS;
    // thread i owns descending positions [i*per, (i+1)*per); position p is digit nb-1-p
    const int per = (nb + 1023) / 1024;
    double ls = 0.;
    unsigned long long lc = 0;
    for (int j = 0; j < per; j++) {
        const int pos = threadIdx.x * per + j;
        if (pos < nb) { ls += hs[nb - 1 - pos]; lc += hc[nb - 1 - pos]; }
    }
    ssum[threadIdx.x] = ls;
    scnt[threadIdx.x] = lc;
    if (threadIdx.x == 0) { chosen = 0x7fffffff; lastne = -1; }
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {  // inclusive scan
        double vs = 0.;
        unsigned long long vc = 0;
        if (threadIdx.x >= off) { vs = ssum[threadIdx.x - off]; vc = scnt[threadIdx.x - off]; }
        __syncthreads();
        ssum[threadIdx.x] += vs;
        scnt[threadIdx.x] += vc;
        __syncthreads();
    }
    const double base = sel->cum_above, target = sel->target;
    const unsigned long long cbase = sel->count_above;
    double before = threadIdx.x ? ssum[threadIdx.x - 1] : 0.;
    unsigned long long beforec = threadIdx.x ? scnt[threadIdx.x - 1] : 0;
    for (int j = 0; j < per; j++) {
        const int pos = threadIdx.x * per + j;
        if (pos >= nb) break;
        const double s = hs[nb - 1 - pos];
        const unsigned long long cn = hc[nb - 1 - pos];
        if (cn > 0) {
            atomicMax(&lastne, pos);
            if (base + before + s > target || (maxsig > 0 && cbase + beforec + cn >= (unsigned long long)maxsig)) {
                atomicMin(&chosen, pos);
                break;
            }
        }
        before += s;
        beforec += cn;
    }
    __syncthreads();
    // no crossing (adaptive_fraction ~ 1 under rounding): the lowest non-empty bin
    const int pos = chosen != 0x7fffffff ? chosen : lastne;
    if (pos >= 0 && pos >= threadIdx.x * per && pos < (threadIdx.x + 1) * per) {
        double bsum = threadIdx.x ? ssum[threadIdx.x - 1] : 0.;
        unsigned long long bc = threadIdx.x ? scnt[threadIdx.x - 1] : 0;
        for (int p = threadIdx.x * per; p < pos; p++) { bsum += hs[nb - 1 - p]; bc += hc[nb - 1 - p]; }
        const int digit = nb - 1 - pos;
        const unsigned long long cnt = hc[digit];
        sel->cum_above += bsum;
        sel->count_above += bc;
        sel->prefix = (sel->prefix << width) | (unsigned long long)digit;
        if (sel->shift == 52 && sel->count_above + cnt <= (unsigned long long)FAST_CAP) {
            sel->phase = 4;  // few candidates: gather the crossing bin and everything above it
            sel->ncand = 0;
        } else if (cnt <= (unsigned long long)CAND_CAP || sel->shift == 0) {
            sel->phase = 1;
            sel->ncand = 0;
        } else {
            sel->shift = sel->shift == 4 ? 0 : sel->shift - 12;
        }
    }
    if (pos < 0 && threadIdx.x == 0) { sel->phase = 3; w.status[b] = T2B_ERR_NOSIGNIF; }
    __syncthreads();
    if (cond && threadIdx.x == 0 && (sel->phase == 0 || sel->phase == 1)) cudaGraphSetConditional(cond, 1u);
    for (int i = threadIdx.x; i < HIST_BINS; i += blockDim.x) { hc[i] = 0; hs[i] = 0.; }
}

// level >= 1 histogram of the next digit among the elements under the prefix
__global__ void __launch_bounds__(256) k_hist_level(Tables tb, Work w, int fine)
{
    extern __shared__ unsigned char smem_raw[];
    unsigned* hc = reinterpret_cast<unsigned*>(smem_raw);
    double* hs = reinterpret_cast<double*>(smem_raw + HIST_BINS * sizeof(unsigned));
    const int b = blockIdx.y;
    const SelState* sel = fine ? &w.sel_f[b] : &w.sel_c[b];
    if (sel->phase != 0) return;
    const int shift = sel->shift, width = digit_width(shift);
    const unsigned long long prefix = sel->prefix;
    const int nb = 1 << width;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) { hc[i] = 0; hs[i] = 0.; }
    __syncthreads();
    const Seg sg = seg_of(tb, w, fine, b);
    const bool pm = !fine && prop_mode(w);
    const double mn = (double)key2f(fine ? w.minkey_f[b] : w.minkey_c[b]);
    const float* dsrc = fine ? w.d2f : w.d2c + (size_t)b * (size_t)(sg.end - sg.beg);
    const int sw = shift + width;
    double lo, hi;
    dwindow(bits2d(prefix << sw), bits2d((prefix + 1) << sw), mn, w.lbound[2 * b], w.lbound[2 * b + 1], lo, hi);
    const long long stride = (long long)gridDim.x * blockDim.x * 16;
    for (long long i0 = sg.beg + ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 16; i0 < sg.end; i0 += stride) {
        float v[16];
        if (!fine) load16(dsrc, i0, sg.end, v);
        OcT ot(fine ? 0 : i0, tb.T);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const long long i = i0 + j;
            const long long oc = ot.oc;
            const int t = ot.t;
            if (!fine) ot.next(tb.T);
            if (i >= sg.end) continue;
            double wt;
            if (fine) {
                wt = w.wf[i];
            } else {
                const double dd = (double)v[j];
                if (v[j] < 0.f || dd <= lo || dd > hi) continue;
                wt = coarse_weight_ot(tb, w, b, glob_oc(w, b, oc, pm), t, v[j], mn);
            }
            if (!(wt > 0.)) continue;
            const unsigned long long bits = (unsigned long long)__double_as_longlong(wt);
            if ((bits >> sw) != prefix) continue;
            const int dg = (int)((bits >> shift) & (unsigned long long)(nb - 1));
            atomicAdd(&hc[dg], 1u);
            atomicAdd(&hs[dg], wt);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
        if (hc[i]) {
            atomicAdd(&w.hist_cnt[(size_t)b * HIST_BINS + i], hc[i]);
            atomicAdd(&w.hist_sum[(size_t)b * HIST_BINS + i], hs[i]);
        }
}

__global__ void __launch_bounds__(256) k_gather(Tables tb, Work w, int fine)
{
    const int b = blockIdx.y;
    SelState* sel = fine ? &w.sel_f[b] : &w.sel_c[b];
    if (sel->phase != 1) return;
    const int shift = sel->shift;
    const unsigned long long prefix = sel->prefix;
    const Seg sg = seg_of(tb, w, fine, b);
    const bool pm = !fine && prop_mode(w);
    const double mn = (double)key2f(fine ? w.minkey_f[b] : w.minkey_c[b]);
    const float* dsrc = fine ? w.d2f : w.d2c + (size_t)b * (size_t)(sg.end - sg.beg);
    double lo, hi;
    dwindow(bits2d(prefix << shift), bits2d((prefix + 1) << shift), mn, w.lbound[2 * b], w.lbound[2 * b + 1], lo, hi);
    const long long stride = (long long)gridDim.x * blockDim.x * 16;
    for (long long i0 = sg.beg + ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 16; i0 < sg.end; i0 += stride) {
        float v[16];
        if (!fine) load16(dsrc, i0, sg.end, v);
        OcT ot(fine ? 0 : i0, tb.T);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const long long i = i0 + j;
            const long long oc = ot.oc;
            const int t = ot.t;
            if (!fine) ot.next(tb.T);
            if (i >= sg.end) continue;
            double wt;
            if (fine) {
                wt = w.wf[i];
            } else {
                const double dd = (double)v[j];
                if (v[j] < 0.f || dd <= lo || dd > hi) continue;
                wt = coarse_weight_ot(tb, w, b, glob_oc(w, b, oc, pm), t, v[j], mn);
            }
            if (!(wt > 0.)) continue;
            const unsigned long long bits = (unsigned long long)__double_as_longlong(wt);
            if ((bits >> shift) != prefix) continue;
            const long long pos = atomicAdd((unsigned long long*)&sel->ncand, 1ull);
            if (pos < CAND_CAP) w.cand[(size_t)b * CAND_CAP + pos] = wt;
        }
    }
}

// Sort the candidates (descending) and walk the cumulative sum
// (src/ml_optimiser.cpp:7905-7935).
__global__ void __launch_bounds__(1024) k_final(Work w, int fine, int ipass, int maxsig)
{
    __shared__ double c[CAND_CAP];
    const int b = blockIdx.x;
    SelState* sel = fine ? &w.sel_f[b] : &w.sel_c[b];
    if (sel->phase != 1) return;
    const long long nc = sel->ncand;
    if (nc <= 0) {  // nothing under the chosen prefix: inconsistent histogram
        if (threadIdx.x == 0) { sel->phase = 3; w.status[b] = T2B_ERR_NOSIGNIF; }
        return;
    }
    if (nc > CAND_CAP) {
        // only reachable with every remaining bit fixed: all candidates are equal
        if (threadIdx.x == 0) {
            const double v = w.cand[(size_t)b * CAND_CAP];
            long long need = (long long)floor((sel->target - sel->cum_above) / v) + 1;
            need = max(1LL, min(need, nc));
            if (maxsig > 0) need = max(1LL, min(need, (long long)maxsig - (long long)sel->count_above));
            sel->thr = v;
            sel->nr_sign = (long long)sel->count_above + need;
            sel->phase = 2;
        }
        return;
    }
    int m = 1;
    while (m < nc) m <<= 1;
    for (int i = threadIdx.x; i < m; i += blockDim.x) c[i] = i < nc ? w.cand[(size_t)b * CAND_CAP + i] : -1.;
    __syncthreads();
    // bitonic sort, descending
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const bool desc = (i & k) == 0;
                    const double a = c[i], bb = c[l];
                    if (desc ? (a < bb) : (a > bb)) { c[i] = bb; c[l] = a; }
                }
            }
            __syncthreads();
        }
    if (threadIdx.x == 0) {
        double cum = sel->cum_above;
        long long k = -1;
        for (long long i = 0; i < nc; i++) {
            cum += c[i];
            if (cum > sel->target || (maxsig > 0 && (long long)sel->count_above + i + 1 >= maxsig)) { k = i; break; }
        }
        if (k < 0) k = nc - 1;
        sel->thr = c[k];
        sel->nr_sign = ipass == 0 ? (long long)sel->count_above + k + 1 : 0;
        sel->phase = 2;
    }
}

// ------------------------------------------------- fast selection path
// When the crossing bin of the level-0 histogram and every bin above it hold
// at most FAST_CAP weights (the usual, concentrated posterior), one pass
// gathers all of them with their indices and one CTA per particle sorts them
// by weight, walks the cumulative sum exactly as src/ml_optimiser.cpp:
// 7905-7935 does, and emits the index-ordered significant list.
__global__ void __launch_bounds__(256) k_gather_fast(Tables tb, Work w, int fine)
{
    const int b = blockIdx.y;
    SelState* sel = fine ? &w.sel_f[b] : &w.sel_c[b];
    if (sel->phase != 4) return;
    const Seg sg = seg_of(tb, w, fine, b);
    const bool pm = !fine && prop_mode(w);
    const double mn = (double)key2f(fine ? w.minkey_f[b] : w.minkey_c[b]);
    const float* dsrc = fine ? w.d2f : w.d2c + (size_t)b * (size_t)(sg.end - sg.beg);
    const double wlo = fmax(bits2d(sel->prefix << 52), hist_floor(tb, w, b, sg.end - sg.beg));
    double lo, hi;
    dwindow(wlo, INFINITY, mn, w.lbound[2 * b], w.lbound[2 * b + 1], lo, hi);
    double* cw = w.fcand_w + (size_t)b * FAST_CAP;
    long long* ci = w.fcand_i + (size_t)b * FAST_CAP;
    const long long stride = (long long)gridDim.x * blockDim.x * 16;
    for (long long i0 = sg.beg + ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 16; i0 < sg.end; i0 += stride) {
        float v[16];
        if (!fine) load16(dsrc, i0, sg.end, v);
        OcT ot(fine ? 0 : i0, tb.T);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const long long i = i0 + j;
            const long long oc = ot.oc;
            const int t = ot.t;
            if (!fine) ot.next(tb.T);
            if (i >= sg.end) continue;
            double wt;
            if (fine) {
                wt = w.wf[i];
            } else {
                if (v[j] < 0.f || (double)v[j] > hi) continue;
                wt = coarse_weight_ot(tb, w, b, glob_oc(w, b, oc, pm), t, v[j], mn);
            }
            if (!(wt >= wlo) || !(wt > 0.)) continue;
            const long long pos = atomicAdd((unsigned long long*)&sel->ncand, 1ull);
            if (pos < FAST_CAP) { cw[pos] = wt; ci[pos] = i; }
        }
    }
}

// bitonic sort of n2 (power of two) (key, index) pairs in shared memory;
// by_weight: weight descending then index ascending; else index ascending
// The first n (<= blockDim.x) pairs sorted in place in bitonic_pairs' order -- by weight
// descending, ties by index ascending (by_weight), else by index ascending; the indices are
// distinct, so the order is total -- each thread placing its own pair at its rank (the
// number of pairs before it): one pass over the pairs, no sorting network.
__device__ void rank_pairs(double* kw, long long* ki, int n, bool by_weight)
{
    double mw = 0.;
    long long mi = 0;
    int rank = 0;
    const bool mine = (int)threadIdx.x < n;
    if (mine) {
        mw = kw[threadIdx.x];
        mi = ki[threadIdx.x];
        for (int j = 0; j < n; j++) {
            const double wj = kw[j];
            const long long ij = ki[j];
            rank += by_weight ? (wj > mw || (wj == mw && ij < mi)) : (ij < mi);
        }
    }
    __syncthreads();
    if (mine) {
        kw[rank] = mw;
        ki[rank] = mi;
    }
    __syncthreads();
}

__device__ void bitonic_pairs(double* kw, long long* ki, int n2, bool by_weight)
{
    for (int k = 2; k <= n2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n2; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    bool swap;
                    if (by_weight) {
                        const bool before = kw[l] > kw[i] || (kw[l] == kw[i] && ki[l] < ki[i]);  // l should precede i
                        swap = up ? before : !before;
                    } else {
                        swap = up ? (ki[l] < ki[i]) : (ki[l] > ki[i]);
                    }
                    if (swap) {
                        const double tw = kw[i]; kw[i] = kw[l]; kw[l] = tw;
                        const long long tx = ki[i]; ki[i] = ki[l]; ki[l] = tx;
                    }
                }
            }
            __syncthreads();
        }
}

__global__ void __launch_bounds__(1024) k_final_fast(Work w, int fine, int ipass, int maxsig)
{
    extern __shared__ unsigned char smem_raw[];
    double* sw = reinterpret_cast<double*>(smem_raw);
    long long* si = reinterpret_cast<long long*>(smem_raw + FAST_CAP * sizeof(double));
    __shared__ int msig;
    const int b = blockIdx.x;
    SelState* sel = fine ? &w.sel_f[b] : &w.sel_c[b];
    if (sel->phase != 4) return;
    const long long nc = sel->ncand;
    if (nc <= 0 || nc > FAST_CAP) {  // excluded by the histogram counts
        if (threadIdx.x == 0) { sel->phase = 3; w.status[b] = T2B_ERR_NOSIGNIF; }
        return;
    }
    int n2 = 1;
    while (n2 < nc) n2 <<= 1;
    for (int i = threadIdx.x; i < n2; i += blockDim.x) {
        sw[i] = i < nc ? w.fcand_w[(size_t)b * FAST_CAP + i] : -1.;
        si[i] = i < nc ? w.fcand_i[(size_t)b * FAST_CAP + i] : 0x7fffffffffffffffLL;
    }
    __syncthreads();
    bitonic_pairs(sw, si, n2, true);
    if (threadIdx.x == 0) {
        double cum = 0.;
        long long k = -1;
        for (long long i = 0; i < nc; i++) {
            cum += sw[i];
            if (cum > sel->target || (maxsig > 0 && i + 1 >= maxsig)) { k = i; break; }
        }
        if (k < 0) k = nc - 1;
        const double thr = sw[k];
        long long m = k + 1;
        while (m < nc && sw[m] >= thr) m++;
        sel->thr = thr;
        sel->nr_sign = ipass == 0 ? k + 1 : 0;
        sel->argmax = si[0];
        msig = (int)m;
    }
    __syncthreads();
    if (!fine) {
        const int m = msig;
        int m2 = 1;
        while (m2 < m) m2 <<= 1;
        for (int i = m + threadIdx.x; i < m2; i += blockDim.x) { sw[i] = 0.; si[i] = 0x7fffffffffffffffLL; }
        __syncthreads();
        bitonic_pairs(sw, si, m2, false);
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            w.flist_w[(size_t)b * FAST_CAP + i] = sw[i];
            w.flist_i[(size_t)b * FAST_CAP + i] = si[i];
        }
        if (threadIdx.x == 0) w.r_ncsig[b] = m;
    }
    if (threadIdx.x == 0) {
        sel->fast = 1;
        sel->phase = 2;
    }
}

// Selection of a particle whose hypotheses fit in shared memory (<= SMALL_CAP: the
// fine pass, and the coarse pass on the proposals), in one CTA: FP64 weights (the fine
// ones stored in wf, as k_weights), their sum and maximum, and the threshold where the
// cumulative sum of the weights sorted by weight (descending, then index) first exceeds
// adaptive_fraction * sum (src/ml_optimiser.cpp:7905-7935; the coarse pass also stops
// at the maxsig-th weight, :7945-7966).  Only the weights >= (1 - f) S / n can be
// reached before the crossing (all the others together hold less than (1 - f) S), so
// only they are sorted (up to 1,024 by rank counting, up to SMALL_SORT bitonically; more are
// left to the multi-kernel path); the prefix sum over them is a block scan in a fixed order.
// The coarse pass also emits the significant list in index order (as k_final_fast).  The
// particle is left marked (fast = 2) so the multi-kernel selection skips it; a coarse
// list longer than FAST_CAP is left to that path.
constexpr int SMALL_CAP = 8192;
constexpr int SMALL_PER = SMALL_CAP / 1024;   // hypotheses per thread
constexpr int SMALL_SORT = 4096;               // candidates the one-CTA selection sorts (shared memory)
__global__ void __launch_bounds__(1024, 2) k_select_small(Tables tb, Work w, int fine, int maxsig, double frac,
                                                       cudaGraphConditionalHandle cond)
{
    extern __shared__ unsigned char smem_raw[];
    double* sw = reinterpret_cast<double*>(smem_raw);
    long long* si = reinterpret_cast<long long*>(smem_raw + SMALL_SORT * sizeof(double));
    __shared__ double shd[32];
    __shared__ unsigned long long shu[32];
    __shared__ long long kmin;
    __shared__ int ncand;
    const int b = blockIdx.x;
    SelState* sel = fine ? &w.sel_f[b] : &w.sel_c[b];
    const bool pm = !fine && prop_mode(w);
    const Seg sg = seg_of(tb, w, fine, b);
    const long long n = sg.end - sg.beg;
    if (n > SMALL_CAP) {                            // the multi-kernel selection takes it
        if (cond && threadIdx.x == 0) cudaGraphSetConditional(cond, 1);
        return;
    }
    if (w.status[b] != T2B_OK) {
        if (threadIdx.x == 0) {
            sel->fast = 2;
            sel->phase = 3;
            if (!fine) w.r_ncsig[b] = 0;
        }
        return;
    }
    const float* dsrc = fine ? w.d2f + sg.beg : w.d2c + (size_t)b * (size_t)n;
    const double mn = (double)key2f(fine ? w.minkey_f[b] : w.minkey_c[b]);
    // this thread's hypotheses i = threadIdx.x + j * blockDim.x, weights in registers
    double wr[SMALL_PER];
    double lsum = 0.;
    unsigned long long lmax = 0;
#pragma unroll
    for (int j = 0; j < SMALL_PER; j++) {
        const long long i = threadIdx.x + (long long)j * blockDim.x;
        double wt = 0.;
        if (i < n) {
            const float d = dsrc[i];
            if (fine) {
                if (d >= 0.f) {
                    const double dd = (double)d - mn;
                    if (dd <= 700.) wt = fine_prior(tb, w, b, sg.beg + i) * exp(-dd);
                }
                w.wf[sg.beg + i] = wt;
            } else {
                wt = coarse_weight_ot(tb, w, b, glob_oc(w, b, i / tb.T, pm), (int)(i % tb.T), d, mn);
            }
            lsum += wt;
            lmax = max(lmax, (unsigned long long)__double_as_longlong(wt));
        }
        wr[j] = wt;
    }
    const double S = block_sum(lsum, shd);
    for (int o = 16; o > 0; o >>= 1) lmax = max(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if ((threadIdx.x & 31) == 0) shu[threadIdx.x >> 5] = lmax;
    if (threadIdx.x == 0) { kmin = 0x7fffffffffffffffLL; ncand = 0; }
    __syncthreads();
    unsigned long long maxbits = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) maxbits = max(maxbits, shu[i]);
    if (!(S > 0.) || S != S) {
        if (threadIdx.x == 0) {
            if (fine) w.sum_f[b] = S;
            else { w.sum_c[b] = S; w.r_ncsig[b] = 0; }
            sel->maxbits = maxbits;
            sel->fast = 2;
            sel->phase = 3;
            w.status[b] = T2B_ERR_NOSIGNIF;
        }
        return;
    }
    const double target = frac * S;
    const double floor_w = frac < 1. ? (1. - frac) * S / (double)n : 0.;
    // the candidates (weight >= floor_w, > 0) into the front of sw / si, in any order
#pragma unroll
    for (int j = 0; j < SMALL_PER; j++) {
        const long long i = threadIdx.x + (long long)j * blockDim.x;
        if (i < n && wr[j] > 0. && wr[j] >= floor_w) {
            const int pos = atomicAdd(&ncand, 1);
            if (pos < SMALL_SORT) {
                sw[pos] = wr[j];
                si[pos] = sg.beg + i;
            }
        }
    }
    __syncthreads();
    const int nc = ncand;
    if (nc > SMALL_SORT) {                          // too many to sort here: the multi-kernel selection
        if (cond && threadIdx.x == 0) cudaGraphSetConditional(cond, 1);
        return;
    }
    int n2 = 1;
    while (n2 < nc) n2 <<= 1;
    if (nc <= (int)blockDim.x) {
        rank_pairs(sw, si, nc, true);
    } else {
        for (int i = nc + threadIdx.x; i < n2; i += blockDim.x) { sw[i] = -1.; si[i] = 0x7fffffffffffffffLL; }
        __syncthreads();
        bitonic_pairs(sw, si, n2, true);
    }
    // inclusive prefix sums of the sorted candidates: runs of `per` per thread, then the
    // runs' exclusive offsets by a block scan
    const int per = (n2 + (int)blockDim.x - 1) / (int)blockDim.x;
    const int i0 = threadIdx.x * per, i1 = min(i0 + per, nc);
    double run = 0.;
    for (int i = i0; i < i1; i++) run += sw[i];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double incl = run;
    for (int o = 1; o < 32; o <<= 1) {
        const double x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
    }
    if (lane == 31) shd[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        double t = lane < (int)(blockDim.x >> 5) ? shd[lane] : 0.;
        for (int o = 1; o < 32; o <<= 1) {
            const double x = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += x;
        }
        shd[lane] = t;   // inclusive over warps
    }
    __syncthreads();
    double cum = (wid > 0 ? shd[wid - 1] : 0.) + incl - run;
    for (int i = i0; i < i1; i++) {
        cum += sw[i];
        if (cum > target || (!fine && maxsig > 0 && i + 1 >= maxsig)) { atomicMin(&kmin, (long long)i); break; }
    }
    __syncthreads();
    const long long k = kmin < nc ? kmin : nc - 1;
    const double thr = sw[k];
    const long long amax = si[0];
    if (!fine) {
        // the significant list: every weight >= thr (ties included), in index order
        int cnt = 0;
        for (int i = threadIdx.x; i < nc; i += blockDim.x) cnt += sw[i] >= thr;
        cnt = block_sum(cnt, reinterpret_cast<int*>(shu));
        if (cnt > FAST_CAP) {                        // too long for the list: left to the multi-kernel path
            if (cond && threadIdx.x == 0) cudaGraphSetConditional(cond, 1);
            return;
        }
        if (cnt <= (int)blockDim.x) {
            rank_pairs(sw, si, cnt, false);
        } else {
            int m2 = 1;
            while (m2 < cnt) m2 <<= 1;
            for (int i = cnt + threadIdx.x; i < m2; i += blockDim.x) { sw[i] = 0.; si[i] = 0x7fffffffffffffffLL; }
            __syncthreads();
            bitonic_pairs(sw, si, m2, false);
        }
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
            w.flist_w[(size_t)b * FAST_CAP + i] = sw[i];
            w.flist_i[(size_t)b * FAST_CAP + i] = si[i];
        }
        if (threadIdx.x == 0) w.r_ncsig[b] = cnt;
    }
    if (threadIdx.x == 0) {
        if (fine) w.sum_f[b] = S;
        else w.sum_c[b] = S;
        sel->maxbits = maxbits;
        sel->thr = thr;
        sel->nr_sign = fine ? 0 : k + 1;
        sel->argmax = amax;
        sel->fast = 2;
        sel->phase = 2;
    }
}

// copy the fast-path significant lists to their place in the batch pair list
__global__ void __launch_bounds__(256) k_write_fast(Tables tb, Work w, int gather_final)
{
    const int b = blockIdx.x;
    const SelState* sel = &w.sel_c[b];
    if (!sel->fast || sel->phase != 2 || w.status[b] != T2B_OK) return;
    const bool pm = prop_mode(w);
    const long long beg = w.pair_off[b], m = w.pair_off[b + 1] - beg;
    for (long long i = threadIdx.x; i < m; i += blockDim.x) {
        w.pairs[beg + i] = glob_il(tb, w, b, w.flist_i[(size_t)b * FAST_CAP + i], pm);
        w.pair_b[beg + i] = b;
        if (gather_final) w.wf[beg + i] = w.flist_w[(size_t)b * FAST_CAP + i];
    }
}

// ------------------------------------------------- ordered compaction
constexpr int CHUNK = 4096;

// significance predicate w >= thr of a coarse element, with the exp() only
// inside the ambiguous diff2 window
struct SigPred {
    double mn, thr, acc, rej;
    bool pm;
    __device__ bool operator()(const Tables& tb, const Work& w, int b, long long i, float d, double* wout) const
    {
        if (d < 0.f) return false;
        const double dd = (double)d;
        if (dd - mn > 700.) return false;
        if (dd > rej) return false;
        if (dd <= acc && !wout) return true;
        const double wt = coarse_weight(tb, w, b, i, d, mn, pm);
        if (wout) *wout = wt;
        return wt >= thr;
    }
};

__device__ __forceinline__ SigPred sig_pred(const Work& w, int b)
{
    SigPred p;
    p.mn = (double)key2f(w.minkey_c[b]);
    p.thr = w.sel_c[b].thr;
    const double lt = log(p.thr);
    p.acc = w.lbound[2 * b] > -INFINITY ? p.mn + w.lbound[2 * b] - lt - WIN_EPS : -INFINITY;
    p.rej = p.mn + w.lbound[2 * b + 1] - lt + WIN_EPS;
    p.pm = prop_mode(w);
    return p;
}

// Per chunk of 4096 coarse elements: number of significant ones (thread t
// covers 16 consecutive elements), and the index of the maximum weight.
__global__ void __launch_bounds__(256) k_count_sig(Tables tb, Work w)
{
    __shared__ int wsum[8];
    const int b = blockIdx.y;
    const SelState* sel = &w.sel_c[b];
    if (sel->phase != 2 || w.status[b] != T2B_OK || sel->fast) return;
    const SigPred pred = sig_pred(w, b);
    const long long n = coarse_n(tb, w, pred.pm);
    const int nch = (int)((n + CHUNK - 1) / CHUNK);
    const float* dsrc = w.d2c + (size_t)b * (size_t)n;
    const unsigned long long maxbits = sel->maxbits;
    const double wmax = __longlong_as_double((long long)maxbits);
    double alo, ahi;
    dwindow(wmax, wmax * (1. + 1e-12), pred.mn, w.lbound[2 * b], w.lbound[2 * b + 1], alo, ahi);
    for (int c = blockIdx.x; c < nch; c += gridDim.x) {
        const long long i0 = (long long)c * CHUNK + threadIdx.x * 16;
        float v[16];
        load16(dsrc, i0, n, v);
        int local = 0;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const long long i = i0 + j;
            const float d = v[j];
            if (d < 0.f) continue;
            if (pred(tb, w, b, i, d, nullptr)) local++;
            const double dd = (double)d;
            if (dd > alo && dd <= ahi) {
                const double wt = coarse_weight(tb, w, b, i, d, pred.mn, pred.pm);
                if ((unsigned long long)__double_as_longlong(wt) == maxbits) atomicMin((long long*)&w.sel_c[b].argmax, i);
            }
        }
        local = __reduce_add_sync(0xffffffffu, local);
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = local;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int j = 0; j < 8; j++) t += wsum[j];
            w.chunk_cnt[(size_t)b * w.max_chunks + c] = t;
        }
        __syncthreads();
    }
}

// exclusive scan of the chunk counts of one particle (one CTA per particle)
__global__ void __launch_bounds__(1024) k_scan_chunks(Tables tb, Work w)
{
    __shared__ long long sh[1024];
    const int b = blockIdx.x;
    const long long n = coarse_n(tb, w, prop_mode(w));
    const int nch = (int)((n + CHUNK - 1) / CHUNK);
    if (w.sel_c[b].fast) return;  // list and count come from the fast path
    const bool active = w.sel_c[b].phase == 2 && w.status[b] == T2B_OK;
    long long run = 0;
    for (int c0 = 0; c0 < nch; c0 += 1024) {
        const int c = c0 + threadIdx.x;
        const long long v = (active && c < nch) ? w.chunk_cnt[(size_t)b * w.max_chunks + c] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const long long u = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
            __syncthreads();
            sh[threadIdx.x] += u;
            __syncthreads();
        }
        if (c < nch) w.chunk_cnt[(size_t)b * w.max_chunks + c] = (int)(run + sh[threadIdx.x] - v);
        const long long tot = sh[1023];
        __syncthreads();
        run += tot;
    }
    if (threadIdx.x == 0) w.r_ncsig[b] = run;
}

// pair offsets of the batch (1 CTA); particles past the pair capacity are dropped
__global__ void __launch_bounds__(1024) k_pair_offsets(Work w)
{
    __shared__ long long sh[1024];
    __shared__ long long carry;
    if (threadIdx.x == 0) { carry = 0; w.pair_off[0] = 0; }
    __syncthreads();
    for (int b0 = 0; b0 < w.n; b0 += 1024) {
        const int b = b0 + threadIdx.x;
        long long v = b < w.n ? w.r_ncsig[b] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const long long u = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
            __syncthreads();
            sh[threadIdx.x] += u;
            __syncthreads();
        }
        long long end = carry + sh[threadIdx.x];
        if (b < w.n && end > w.pair_cap) {  // capacity exceeded: drop this particle
            w.status[b] = T2B_ERR_NOMEM;
            w.r_ncsig[b] = 0;
        }
        __syncthreads();
        // recompute with the dropped particles removed
        v = b < w.n ? w.r_ncsig[b] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const long long u = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
            __syncthreads();
            sh[threadIdx.x] += u;
            __syncthreads();
        }
        end = carry + sh[threadIdx.x];
        if (b < w.n) w.pair_off[b + 1] = end;
        __syncthreads();
        if (threadIdx.x == 1023) carry = end;
        __syncthreads();
    }
}

// Ordered compaction of the significant coarse pairs: thread t of a chunk
// owns 16 consecutive elements; a block scan of the per-thread counts keeps
// index order.
__global__ void __launch_bounds__(256) k_compact(Tables tb, Work w, int gather_final)
{
    __shared__ int wsum[8];
    const int b = blockIdx.y;
    const SelState* sel = &w.sel_c[b];
    if (sel->phase != 2 || w.status[b] != T2B_OK || sel->fast) return;
    const SigPred pred = sig_pred(w, b);
    const long long n = coarse_n(tb, w, pred.pm);
    const int nch = (int)((n + CHUNK - 1) / CHUNK);
    const float* dsrc = w.d2c + (size_t)b * (size_t)n;
    const long long pbase = w.pair_off[b], pend = w.pair_off[b + 1];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int c = blockIdx.x; c < nch; c += gridDim.x) {
        const long long i0 = (long long)c * CHUNK + threadIdx.x * 16;
        float v[16];
        load16(dsrc, i0, n, v);
        unsigned flags = 0;
        int local = 0;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            if (v[j] >= 0.f && pred(tb, w, b, i0 + j, v[j], nullptr)) { flags |= 1u << j; local++; }
        }
        int incl = local;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        int before = 0;
        for (int j = 0; j < wid; j++) before += wsum[j];
        long long pos = pbase + w.chunk_cnt[(size_t)b * w.max_chunks + c] + before + incl - local;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            if (!(flags & (1u << j))) continue;
            if (pos < pend) {
                w.pairs[pos] = glob_il(tb, w, b, i0 + j, pred.pm);
                w.pair_b[pos] = b;
                if (gather_final) w.wf[pos] = coarse_weight(tb, w, b, i0 + j, v[j], pred.mn, pred.pm);
            }
            pos++;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------- fine pass
// One work item per significant coarse pair, pulled from a device queue by a
// persistent grid: R fine orientations x V fine shifts against the pair
// (src/ml_optimiser.cpp:7090-7272 with exp_ipass == 1).
constexpr int MAXR = 8, MAXV = 4;

// ONFLY: the chunked configurations' build, which interpolates the fine projections itself.
// MINB: CTAs per SM the build is register-limited to (256 threads: 64 registers at 4, 85 at 3,
// 128 at 2).  With more registers all loads of a pixel are in flight at once; with fewer the 40
// accumulators leave room for only a few.  The tile autotuner picks the build.
template <bool ONFLY, int MINB>
__global__ void __launch_bounds__(256, MINB) k_fine(Tables tb, Work w)
{
    __shared__ long long item;
    __shared__ float red[8][MAXR * MAXV + MAXR];
    const int P = tb.P, R = tb.R, V = tb.V, T = tb.T;
    const long long total = w.pair_off[w.n];
    for (;;) {
        if (threadIdx.x == 0) item = (long long)atomicAdd(&w.counters[0], 1ull);
        __syncthreads();
        const long long q = item;
        __syncthreads();
        if (q >= total) break;
        const int b = w.pair_b[q];
        const long long ih = w.pairs[q];
        const int oc = (int)(ih / T), t = (int)(ih - (long long)oc * T);
        float cr[MAXR][MAXV], nr[MAXR];
#pragma unroll
        for (int r = 0; r < MAXR; r++) {
            nr[r] = 0.f;
#pragma unroll
            for (int v = 0; v < MAXV; v++) cr[r][v] = 0.f;
        }
        // only the pixels inside the projection radius: the projections, hence the
        // cross and norm terms, are zero outside
        for (int k = threadIdx.x; k < tb.nk; k += blockDim.x) {
            const int p = tb.kpix[k];
            // every load of this pixel first, then the arithmetic
            const float2 c = w.cvec[(size_t)b * P + p];
            const float wv = w.w2[(size_t)b * P + p];
            float2 ab[MAXV], pv[MAXR];
#pragma unroll
            for (int v = 0; v < MAXV; v++)
                ab[v] = v < V ? tb.ab_f[(size_t)(t * V + v) * P + p] : make_float2(0.f, 0.f);
#pragma unroll
            for (int r = 0; r < MAXR; r++) {
                if (r < R) {
                    // chunked configurations hold no fine table: the same interpolation, here
                    pv[r] = !ONFLY ? tb.proj_f[((size_t)oc * R + r) * P + p]
                                   : project_window_pixel((cudaTextureObject_t)tb.mtex[oc / tb.O],
                                                          tb.mvol[oc / tb.O],
                                                          tb.eul_f + 9 * ((size_t)(oc % tb.O) * R + r), p, tb.s);
                } else {
                    pv[r] = make_float2(0.f, 0.f);
                }
            }
            float2 a[MAXV];
#pragma unroll
            for (int v = 0; v < MAXV; v++)
                a[v] = make_float2(c.x * ab[v].x - c.y * ab[v].y, c.x * ab[v].y + c.y * ab[v].x);
#pragma unroll
            for (int r = 0; r < MAXR; r++) {
                if (r < R) {
                    nr[r] += wv * (pv[r].x * pv[r].x + pv[r].y * pv[r].y);
#pragma unroll
                    for (int v = 0; v < MAXV; v++) cr[r][v] += pv[r].x * a[v].x + pv[r].y * a[v].y;
                }
            }
        }
        // block reduction of the R*V cross terms and R norms
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
        for (int r = 0; r < MAXR; r++) {
#pragma unroll
            for (int v = 0; v < MAXV; v++) {
                float x = cr[r][v];
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == 0) red[wid][r * MAXV + v] = x;
            }
            float x = nr[r];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) red[wid][MAXR * MAXV + r] = x;
        }
        __syncthreads();
        if (threadIdx.x < R * V) {
            const int r = threadIdx.x / V, v = threadIdx.x - r * V;
            float cs = 0.f, ns = 0.f;
            for (int j = 0; j < 8; j++) { cs += red[j][r * MAXV + v]; ns += red[j][MAXR * MAXV + r]; }
            const float d = w.c0[b] + ns - cs;
            w.d2f[q * R * V + r * V + v] = d;
            atomicMin(&w.minkey_f[b], f2key(d));
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_argmax_fine(Tables tb, Work w)
{
    const int b = blockIdx.y;
    const SelState* sel = &w.sel_f[b];
    if (sel->phase != 2 || sel->fast) return;
    const long long rv = (long long)tb.R * tb.V;
    const long long beg = w.pair_off[b] * rv, end = w.pair_off[b + 1] * rv;
    for (long long i = beg + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < end;
         i += (long long)gridDim.x * blockDim.x)
        if ((unsigned long long)__double_as_longlong(w.wf[i]) == sel->maxbits)
            atomicMin((long long*)&w.sel_f[b].argmax, i);
}

// ---------------------------------------------- weighted sums + backprojection
constexpr int ENT_CAP = 512;

// Fire-and-forget FP32 reductions into the grids (red: no value comes back, so the
// warp does not hold a register for the reply as with an atomic whose result is unused)
__device__ __forceinline__ void red_add(float* p, float v)
{
    asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void red_add2(float2* p, float x, float y)
{
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(x), "f"(y) : "memory");
}

// The two x-neighbours (idx, idx + 1) of one row of a trilinear footprint, weights d0 and d1:
// from an even idx (the grids are separate cudaMalloc allocations, so 16-byte aligned at every
// even voxel for the complex values and 8-byte for the weights) one 16-byte reduction of the two
// complex values and one 8-byte of the two weights; from an odd idx two of each.  The same sums.
__device__ __forceinline__ void red_xpair(float2* gd, float* gw, size_t idx, float d0, float d1, float vr, float vi,
                                          float fw)
{
    if ((idx & 1) == 0) {
        asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(gd + idx), "f"(d0 * vr), "f"(d0 * vi),
                     "f"(d1 * vr), "f"(d1 * vi)
                     : "memory");
        asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(gw + idx), "f"(d0 * fw), "f"(d1 * fw) : "memory");
    } else {
        red_add2(gd + idx, d0 * vr, d0 * vi);
        red_add(gw + idx, d0 * fw);
        red_add2(gd + idx + 1, d1 * vr, d1 * vi);
        red_add(gw + idx + 1, d1 * fw);
    }
}

struct GridPtrs {
    float2* const* data;
    float* const* weight;
};

// First pair of every orientation group (consecutive pairs of one particle with
// the same coarse orientation) into w.groups; the count into w.counters[3].
__global__ void k_group_starts(Tables tb, Work w)
{
    const long long npairs = w.pair_off[w.n];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < npairs; q += (long long)gridDim.x * blockDim.x) {
        const int b = w.pair_b[q];
        const long long oc = w.pairs[q] / tb.T;
        if (q == w.pair_off[b] || w.pairs[q - 1] / tb.T != oc) {
            const unsigned long long i = atomicAdd(&w.counters[3], 1ull);
            w.groups[i] = q;
            // the group's end, found here (one thread per group) rather than by the consumer
            long long e = q + 1;
            const long long pend = w.pair_off[b + 1];
            while (e < pend && w.pairs[e] / tb.T == oc) e++;
            w.group_end[i] = e;
        }
    }
}

// SCL: with the scale-correction sums (a separate build: they cost the default path 16 registers);
// ONFLY: projections interpolated from the models (chunked configurations hold no table)
// MINB: CTAs per SM the build is register-limited to (as k_fine; the tile autotuner picks it)
template <bool SCL, bool ONFLY, int MINB>
__global__ void __launch_bounds__(256, MINB) k_wsum_bp(Tables tb, Work w, Volume g, GridPtrs gp)
{
    __shared__ long long item;
    __shared__ int nent;
    __shared__ float ent_w[ENT_CAP];
    __shared__ int ent_tv[ENT_CAP];
    __shared__ float ssig[1024];   // per-item ring sums (FP32, as the reference GPU path), FP64 across items
    __shared__ double shr[32];
    const int P = tb.P, T = tb.T, xh = tb.xh, s = tb.s;
    const int R = tb.ovs ? tb.R : 1, V = tb.ovs ? tb.V : 1;
    (void)xh;
    const unsigned long long nitems = w.counters[3] * (unsigned long long)R;   // (orientation group, rotation)
    const float2* proj = tb.ovs ? tb.proj_f : tb.proj_c;
    const float2* abt = tb.ovs ? tb.ab_f : tb.ab_c;
    const int nring = s / 2 + 1;
    __shared__ long long grp_end, grp_beg;
    for (;;) {
        if (threadIdx.x == 0) {
            item = (long long)atomicAdd(&w.counters[2], 1ull);
            // a work item is (orientation group, fine rotation); find the group's end
            grp_end = -1;
            if ((unsigned long long)item < nitems) {
                grp_beg = w.groups[item / R];
                grp_end = w.group_end[item / R];
            }
        }
        __syncthreads();
        const long long it = item;
        if ((unsigned long long)it >= nitems) break;
        const long long qa = grp_beg;
        const long long qb = grp_end;
        const int r = (int)(it % R);
        const int b = w.pair_b[qa];
        const int oc = (int)(w.pairs[qa] / T);
        const int k = oc / tb.O, o = oc - k * tb.O, idir = o / tb.n_psi;
        const long long tab = tb.ovs ? (long long)oc * R + r : oc;
        const double* A = tb.ovs ? tb.eul_f + 9 * ((size_t)o * R + r) : tb.eul_c + 9 * (size_t)o;
        const SelState* sel = tb.ovs ? &w.sel_f[b] : &w.sel_c[b];
        const double thr = sel->thr;
        const double S = tb.ovs ? w.sum_f[b] : w.sum_c[b];
        const double* sc = w.scal + 8 * (size_t)b;
        if (threadIdx.x == 0) nent = 0;
        for (int i = threadIdx.x; i < nring; i += blockDim.x) ssig[i] = 0.f;
        __syncthreads();
        if (w.status[b] == T2B_OK) {
            const long long nh = (qb - qa) * V;
            for (long long e0 = 0; e0 < nh; e0 += ENT_CAP) {
                // collect the significant hypotheses of this orientation
                for (long long e = e0 + threadIdx.x; e < min(nh, e0 + ENT_CAP); e += blockDim.x) {
                    const long long q = qa + e / V;
                    const int v = (int)(e % V);
                    const double wt = tb.ovs ? w.wf[q * R * V + r * V + v] : w.wf[q];
                    if (wt >= thr) {
                        const int t = (int)(w.pairs[q] - (long long)oc * T);
                        const double wn = wt / S;
                        const int pos = atomicAdd(&nent, 1);
                        ent_w[pos] = (float)wn;
                        ent_tv[pos] = t * V + v;
                        // scalar sums of src/ml_optimiser.cpp:8480-8540
                        atomicAdd(&w.r_sumw[b], wn);
                        atomicAdd(&w.r_pdf_class[(size_t)b * tb.K + k], wn);
                        atomicAdd(&w.r_pdf_dir[(size_t)b * tb.K * tb.n_dir + k * tb.n_dir + idir], wn);
                        const double* sh = tb.ovs ? tb.trans_f + 2 * (t * V + v) : tb.trans_c + 2 * t;
                        const double dx = sc[4] - sc[2] - sh[0], dy = sc[5] - sc[3] - sh[1];
                        atomicAdd(&w.r_sig_off[b], wn * tb.pixel_size * tb.pixel_size * (dx * dx + dy * dy));
                    }
                }
                __syncthreads();
                const int ne = nent;
                if (ne > 0) {
                    double nacc = 0., xacc = 0., aacc = 0.;
                    const float scale = (float)sc[6];
                    // scale-correction sums (src/ml_optimiser.cpp:8477-8486; the GPU path's
                    // per-pixel XA / AA of wavg.cuh:155-163): sum_e w'_e Re(A conj sX_e) and
                    // |A|^2 sum_e w'_e over the rings of this class with data_vs_prior > 3
                    const unsigned char* scl = SCL ? tb.scl_ring + (size_t)k * (tb.ori_size / 2 + 1) : nullptr;
                    float wsum_e = 0.f;
                    if (SCL)
                        for (int e = 0; e < ne; e++) wsum_e += ent_w[e];
                    for (int n = threadIdx.x; n < P; n += blockDim.x) {
                        const float2 pv = ONFLY ? project_window_pixel((cudaTextureObject_t)tb.mtex[k],
                                                                       tb.mvol[k], A, n, s)
                                                : proj[(size_t)tab * P + n];
                        const float c = w.ctf[(size_t)b * P + n] * scale;
                        const float frr = pv.x * c, fri = pv.y * c;
                        const float2 X = w.fimg[(size_t)b * P + n];
                        const float2 Xn = w.fimg_nm[(size_t)b * P + n];
                        const float minv = n == 0 ? (float)sc[0] : w.minv[(size_t)b * P + n];
                        const int ires = tb.mresol[n];
                        float fir = 0.f, fii = 0.f, fw = 0.f, wd = 0.f, xa = 0.f;
                        for (int e = 0; e < ne; e++) {
                            const float wn = ent_w[e];
                            const float2 ab = abt[(size_t)ent_tv[e] * P + n];
                            const float sr = ab.x * X.x - ab.y * X.y, si = ab.x * X.y + ab.y * X.x;
                            const float dr = frr - sr, di = fri - si;
                            wd += wn * (dr * dr + di * di);
                            if (SCL) xa += wn * (frr * sr + fri * si);
                            const float wx = wn * c * minv;
                            const float nr_ = ab.x * Xn.x - ab.y * Xn.y, ni = ab.x * Xn.y + ab.y * Xn.x;
                            fir += nr_ * wx;
                            fii += ni * wx;
                            fw += wx * c;
                        }
                        if (ires > -1) {
                            atomicAdd(&ssig[ires], wd);
                            nacc += wd;
                            if (SCL && scl[ires]) {
                                xacc += xa;
                                aacc += (frr * frr + fri * fri) * wsum_e;
                            }
                        }
                        // backprojection of this pixel (src/backprojector.cpp:140-228)
                        if (fw > 0.f && !w.no_bp) {
                            const int i = n / xh, x = n - i * xh;
                            const int y = (i < xh) ? i : i - s;
                            if (i >= xh && x == 0) continue;
                            if (x * x + y * y > g.r_max * g.r_max) continue;
                            double xp = rot_coord(A[0], A[3], g.pad, x, y);
                            double yp = rot_coord(A[1], A[4], g.pad, x, y);
                            double zp = rot_coord(A[2], A[5], g.pad, x, y);
                            float vr = fir, vi = fii;
                            if (xp < 0) { xp = -xp; yp = -yp; zp = -zp; vi = -vi; }
                            const int x0 = (int)floor(xp);
                            const float fx = (float)(xp - x0);
                            int y0 = (int)floor(yp);
                            const float fy = (float)(yp - y0);
                            y0 -= g.inity;
                            float2* gd = gp.data[k];
                            float* gw = gp.weight[k];
                            if (g.ref_dim == 3) {
                                int z0 = (int)floor(zp);
                                const float fz = (float)(zp - z0);
                                z0 -= g.initz;
                                if (x0 < 0 || x0 + 1 >= g.xdim || y0 < 0 || y0 + 1 >= g.ydim || z0 < 0 || z0 + 1 >= g.zdim) continue;
                                const float mfx = 1.f - fx, mfy = 1.f - fy, mfz = 1.f - fz;
                                const float dd[8] = {mfz * mfy * mfx, mfz * mfy * fx, mfz * fy * mfx, mfz * fy * fx,
                                                     fz * mfy * mfx,  fz * mfy * fx,  fz * fy * mfx,  fz * fy * fx};
#pragma unroll
                                for (int cc = 0; cc < 8; cc += 2) {
                                    const size_t idx = ((size_t)(z0 + (cc >> 2)) * g.ydim + y0 + ((cc >> 1) & 1)) * g.xdim + x0;
                                    red_xpair(gd, gw, idx, dd[cc], dd[cc + 1], vr, vi, fw);
                                }
                            } else {
                                if (x0 < 0 || x0 + 1 >= g.xdim || y0 < 0 || y0 + 1 >= g.ydim) continue;
                                const float mfx = 1.f - fx, mfy = 1.f - fy;
                                const float dd[4] = {mfy * mfx, mfy * fx, fy * mfx, fy * fx};
#pragma unroll
                                for (int cc = 0; cc < 4; cc += 2) {
                                    const size_t idx = (size_t)(y0 + (cc >> 1)) * g.xdim + x0;
                                    red_xpair(gd, gw, idx, dd[cc], dd[cc + 1], vr, vi, fw);
                                }
                            }
                        }
                    }
                    nacc = block_sum(nacc, shr);
                    if (threadIdx.x == 0) atomicAdd(&w.r_norm[b], nacc);
                    if (SCL) {
                        // divided by scale_correction and its square (src/ml_optimiser.cpp:8859-8860):
                        // the scale entered A through the CTF
                        xacc = block_sum(xacc, shr);
                        aacc = block_sum(aacc, shr);
                        if (threadIdx.x == 0) {
                            atomicAdd(&w.r_xa[b], xacc / sc[6]);
                            atomicAdd(&w.r_aa[b], aacc / (sc[6] * sc[6]));
                        }
                    }
                }
                __syncthreads();
                if (threadIdx.x == 0) nent = 0;
                __syncthreads();
            }
        }
        __syncthreads();
        const int half = tb.ori_size / 2 + 1;
        for (int i = threadIdx.x; i < nring && i < half; i += blockDim.x)
            if (ssig[i] != 0.f) atomicAdd(&w.r_sigma2[(size_t)b * half + i], (double)ssig[i]);
        __syncthreads();
    }
}

// ----------------------------------------------------------- results
__global__ void k_results(Tables tb, Work w)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= w.n) return;
    const SelState& sc = w.sel_c[b];
    const SelState& sf = tb.ovs ? w.sel_f[b] : w.sel_c[b];
    if (w.r_learned) w.r_learned[b] = prop_mode(w) ? 1 : 0;
    w.r_csum[b] = w.sum_c[b];
    w.r_csig[b] = sc.thr;
    w.r_nsign[b] = sc.nr_sign;
    const double S = tb.ovs ? w.sum_f[b] : w.sum_c[b];
    w.r_sum[b] = S;
    w.r_sig[b] = sf.thr;
    w.r_min[b] = (double)key2f(tb.ovs ? w.minkey_f[b] : w.minkey_c[b]);
    int* pose = w.r_pose + 5 * (size_t)b;
    if (*w.err != 0 && w.status[b] == T2B_OK) w.status[b] = *w.err;
    if (w.status[b] != T2B_OK || sf.phase != 2) {
        if (w.status[b] == T2B_OK) w.status[b] = T2B_ERR_NOSIGNIF;
        w.r_pmax[b] = -1.;
        for (int j = 0; j < 5; j++) pose[j] = -1;
        return;
    }
    const long long am = sf.argmax;
    const bool pm = prop_mode(w);
    const long long nfinal = tb.ovs ? (w.pair_off[w.n] * tb.R * tb.V) : coarse_n(tb, w, pm);
    if (am < 0 || am >= nfinal) {  // the maximum was not located: report, do not index
        w.status[b] = T2B_ERR_NOSIGNIF;
        w.r_pmax[b] = -1.;
        for (int j = 0; j < 5; j++) pose[j] = -1;
        return;
    }
    w.r_pmax[b] = __longlong_as_double((long long)sf.maxbits) / S;
    long long ih;
    int r = 0, v = 0;
    if (tb.ovs) {
        const long long rv = (long long)tb.R * tb.V;
        const long long q = am / rv;
        r = (int)((am % rv) / tb.V);
        v = (int)(am % tb.V);
        ih = w.pairs[q];
    } else {
        ih = glob_il(tb, w, b, am, pm);
    }
    const int oc = (int)(ih / tb.T);
    pose[0] = oc / tb.O;
    pose[1] = oc % tb.O;
    pose[2] = r;
    pose[3] = (int)(ih % tb.T);
    pose[4] = v;
}

// --------------------------------------------------- reconstruction (FP64)
__global__ void k_decenter(Volume g, const float2* __restrict__ data, const float* __restrict__ weight,
                           double2* __restrict__ fconv, double* __restrict__ fw, double* rad, double* cnt,
                           const double* __restrict__ tau2, double tscale, int minres_map)
{
    const int ps = g.ydim, fx = ps / 2 + 1, nz = g.ref_dim == 3 ? ps : 1;   // 2D grids: one plane
    const long long total = (long long)nz * ps * fx;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= total) return;
    const int j = (int)(n % fx);
    const int i = (int)((n / fx) % ps);
    const int k = (int)(n / ((long long)fx * ps));
    const int kp = k < fx ? k : k - ps, ip = i < fx ? i : i - ps, jp = j;
    const int rp = g.r_max * g.pad;
    const int r2 = kp * kp + ip * ip + jp * jp;
    double2 v = make_double2(0., 0.);
    double wv = 0.;
    if (r2 <= rp * rp) {
        const size_t src = ((size_t)(kp - g.initz) * g.ydim + (ip - g.inity)) * g.xdim + jp;
        const float2 d = data[src];
        v = make_double2(d.x, d.y);
        wv = weight[src];
    }
    // MAP term: the inverse tau2 spectrum added to the weight (src/backprojector.cpp:1412-1455)
    if (tau2 && r2 < rp * rp) {
        const double rr = sqrt((double)r2) / g.pad;
        const int im = rr > 0 ? (int)(rr + 0.5) : (int)(rr - 0.5);
        const double t = tau2[im];
        const double invtau2 = t > 0. ? 1. / (tscale * t) : (wv > 1e-20 ? 1. / (0.001 * wv) : 0.);
        if (im >= minres_map) wv += invtau2;
    }
    fconv[n] = v;
    fw[n] = wv;
    if (r2 < rp * rp) {
        const int ires = (int)floor(sqrt((double)r2) / g.pad);
        atomicAdd(&rad[ires], wv);
        atomicAdd(&cnt[ires], 1.);
    }
}

__global__ void k_radnorm(int r_max, double* rad, const double* cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < r_max && (cnt[i] > 0. || rad[i] > 0.)) rad[i] /= 1000. * cnt[i];
}

__global__ void k_divide(Volume g, double2* __restrict__ fconv, const double* __restrict__ fw, const double* rad)
{
    const int ps = g.ydim, fx = ps / 2 + 1, nz = g.ref_dim == 3 ? ps : 1;
    const long long total = (long long)nz * ps * fx;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= total) return;
    const int j = (int)(n % fx);
    const int i = (int)((n / fx) % ps);
    const int k = (int)(n / ((long long)fx * ps));
    const int kp = k < fx ? k : k - ps, ip = i < fx ? i : i - ps;
    const int r2 = kp * kp + ip * ip + j * j;
    const int ires = (int)floor(sqrt((double)r2) / g.pad);
    const double wv = fmax(fw[n], rad[ires < g.r_max ? ires : g.r_max - 1]);
    if (wv != 0.) {
        double2 v = fconv[n];
        v.x /= wv;
        v.y /= wv;
        fconv[n] = v;
    }
}

int sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

int grid_x_for(int nb)
{
    const int target = 4 * sm_count();
    return std::max(1, (target + nb - 1) / std::max(1, nb));
}

const size_t HIST_SMEM = HIST_BINS * (sizeof(unsigned) + sizeof(double));
const size_t FAST_SMEM = FAST_CAP * (sizeof(double) + sizeof(long long));
const size_t SMALL_SMEM = SMALL_SORT * (sizeof(double) + sizeof(long long));

// a stream per device and nesting depth to capture conditional-node bodies on
cudaStream_t body_stream(int depth)
{
    static std::mutex mu;
    static std::map<std::pair<int, int>, cudaStream_t> streams;
    int dev = 0;
    T2B_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    cudaStream_t& bs = streams[{dev, depth}];
    if (!bs) T2B_CUDA(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
    return bs;
}

// A condition for an IF node of the graph `st` is being captured into (reset to 0 at
// every launch of the graph); 0 when `st` is not capturing.
cudaGraphConditionalHandle cond_handle(cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    T2B_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr));
    cudaGraphConditionalHandle h = 0;
    if (cs == cudaStreamCaptureStatusActive && g != nullptr)
        T2B_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    return h;
}

// Enqueue body(stream): under capture (h != 0) as the body of an IF node on h, whose
// launches run only when a kernel before it set the condition; else directly on st.
template <class F>
void if_node(cudaStream_t st, cudaGraphConditionalHandle h, int depth, F body)
{
    if (!h) {
        body(st);
        return;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    T2B_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    T2B_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t bodyg = np.conditional.phGraph_out[0];
    T2B_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t bs = body_stream(depth);
    T2B_CUDA(cudaStreamBeginCaptureToGraph(bs, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        body(bs);
    } catch (...) {
        cudaGraph_t dummy = nullptr;
        cudaStreamEndCapture(bs, &dummy);
        throw;
    }
    cudaGraph_t done = nullptr;
    T2B_CUDA(cudaStreamEndCapture(bs, &done));
}

void run_selection(const Tables& tb, const Work& w, int fine, int ipass, cudaStream_t st, int depth)
{
    const int gx = grid_x_for(w.n);
    dim3 grid(gx, w.n);
    const int maxsig = fine ? 0 : tb.maxsig;   // the reference's count only grows in the coarse pass
    // under graph capture the multi-level search (levels 1-5, the candidate gather and sort)
    // is the body of an IF node whose condition the level-0 select sets when a particle needs
    // it, so the usual batch (every particle on the fast path) launches none of it
    const cudaGraphConditionalHandle h = cond_handle(st);
    k_sel_init<<<(w.n + 127) / 128, 128, 0, st>>>(w, fine, tb.adaptive_fraction);
    k_select<<<w.n, 1024, 0, st>>>(w, fine, maxsig, h);
    auto multilevel = [&](cudaStream_t s2) {
        for (int level = 1; level < 6; level++) {
            k_hist_level<<<grid, 256, HIST_SMEM, s2>>>(tb, w, fine);
            k_select<<<w.n, 1024, 0, s2>>>(w, fine, maxsig, 0);
        }
        k_gather<<<grid, 256, 0, s2>>>(tb, w, fine);
        k_final<<<w.n, 1024, 0, s2>>>(w, fine, ipass, maxsig);
    };
    if_node(st, h, depth, multilevel);
    k_gather_fast<<<grid, 256, 0, st>>>(tb, w, fine);
    k_final_fast<<<w.n, 1024, FAST_SMEM, st>>>(w, fine, ipass, maxsig);
}

}  // namespace

void launch_prep(const Tables& tb, const Work& w, cudaStream_t st)
{
    k_prep<<<w.n, 256, 0, st>>>(tb, w);
    k_pdf_t<<<w.n, 128, 0, st>>>(tb, w);
    T2B_CUDA(cudaGetLastError());
}

void launch_norms(const Tables& tb, const Work& w, cudaStream_t st)
{
    const int KO = tb.K * tb.O;
    dim3 grid((KO + 127) / 128, (w.n + 63) / 64);
    k_norms<<<grid, 256, 0, st>>>(tb, w, tb.proj_c, KO, w.norms);
    T2B_CUDA(cudaGetLastError());
}

void launch_diff2_simt(const Tables& tb, const Work& w, cudaStream_t st)
{
    const int KO = tb.K * tb.O;
    dim3 grid((KO + SB_M - 1) / SB_M, (w.n * tb.T + SB_N - 1) / SB_N);
    k_diff2_simt<<<grid, 256, 0, st>>>(tb, w);
    T2B_CUDA(cudaGetLastError());
}

void estep_init_attributes()
{
    T2B_CUDA(cudaFuncSetAttribute(k_weights, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HIST_SMEM));
    T2B_CUDA(cudaFuncSetAttribute(k_hist_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HIST_SMEM));
    T2B_CUDA(cudaFuncSetAttribute(k_final_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FAST_SMEM));
    T2B_CUDA(cudaFuncSetAttribute(k_select_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMALL_SMEM));
    (void)sm_count();
}

void launch_weights_coarse(const Tables& tb, const Work& w, int maxsig, cudaStream_t st)
{
    (void)maxsig;   // tb.maxsig
    const int gx = grid_x_for(w.n);
    dim3 grid(gx, w.n);
    const long long n = (long long)tb.K * tb.O * tb.T;
    const int nch = (int)((n + CHUNK - 1) / CHUNK);
    dim3 gc(std::min(nch, gx), w.n);
    // under capture, the multi-kernel selection and compaction are IF-node bodies that run
    // only when the one-CTA selection left a particle to them
    const cudaGraphConditionalHandle h = cond_handle(st);
    k_select_small<<<w.n, 1024, SMALL_SMEM, st>>>(tb, w, 0, tb.maxsig, tb.adaptive_fraction, h);
    if_node(st, h, 0, [&](cudaStream_t s) {
        k_weights<<<grid, 256, HIST_SMEM, s>>>(tb, w, 0);
        run_selection(tb, w, 0, 0, s, 1);
        k_count_sig<<<gc, 256, 0, s>>>(tb, w);
        k_scan_chunks<<<w.n, 1024, 0, s>>>(tb, w);
    });
    k_pair_offsets<<<1, 1024, 0, st>>>(w);
    k_compact<<<gc, 256, 0, st>>>(tb, w, tb.ovs ? 0 : 1);   // (a handle serves one IF node; this returns at once when unused)
    k_write_fast<<<w.n, 256, 0, st>>>(tb, w, tb.ovs ? 0 : 1);
    T2B_CUDA(cudaGetLastError());
}

void launch_fine(const Tables& tb, const Work& w, cudaStream_t st)
{
    const int per_sm = w.fine_ctas > 0 ? std::min(w.fine_ctas, 4) : 4;
    const int ctas = per_sm * sm_count();
    const auto run = [&](auto onfly) {
        constexpr bool F = decltype(onfly)::value;
        switch (per_sm) {
        case 1: k_fine<F, 1><<<ctas, 256, 0, st>>>(tb, w); break;
        case 2: k_fine<F, 2><<<ctas, 256, 0, st>>>(tb, w); break;
        case 3: k_fine<F, 3><<<ctas, 256, 0, st>>>(tb, w); break;
        default: k_fine<F, 4><<<ctas, 256, 0, st>>>(tb, w); break;
        }
    };
    if (tb.chunk) run(std::true_type{});
    else run(std::false_type{});
    T2B_CUDA(cudaGetLastError());
}

void launch_weights_fine(const Tables& tb, const Work& w, cudaStream_t st)
{
    const int gx = grid_x_for(w.n);
    dim3 grid(gx, w.n);
    const cudaGraphConditionalHandle h = cond_handle(st);
    k_select_small<<<w.n, 1024, SMALL_SMEM, st>>>(tb, w, 1, 0, tb.adaptive_fraction, h);
    if_node(st, h, 0, [&](cudaStream_t s) {
        k_weights<<<grid, 256, HIST_SMEM, s>>>(tb, w, 1);
        run_selection(tb, w, 1, 1, s, 1);
        k_argmax_fine<<<grid, 256, 0, s>>>(tb, w);
    });
    T2B_CUDA(cudaGetLastError());
}

void launch_wsum_bp(const Tables& tb, const Work& w, const Volume& g, float2* const* grid_data,
                    float* const* grid_weight, cudaStream_t st)
{
    GridPtrs gp{grid_data, grid_weight};
    k_group_starts<<<2 * sm_count(), 256, 0, st>>>(tb, w);
    const int per_sm = w.wsum_ctas > 0 ? std::min(w.wsum_ctas, 4) : 4;
    const int ctas = per_sm * sm_count();
    const bool scl = tb.scl_ring && w.r_xa && w.r_aa;
    const auto run = [&](auto sclv, auto onfly) {
        constexpr bool S = decltype(sclv)::value, F = decltype(onfly)::value;
        switch (per_sm) {
        case 1: k_wsum_bp<S, F, 1><<<ctas, 256, 0, st>>>(tb, w, g, gp); break;
        case 2: k_wsum_bp<S, F, 2><<<ctas, 256, 0, st>>>(tb, w, g, gp); break;
        case 3: k_wsum_bp<S, F, 3><<<ctas, 256, 0, st>>>(tb, w, g, gp); break;
        default: k_wsum_bp<S, F, 4><<<ctas, 256, 0, st>>>(tb, w, g, gp); break;
        }
    };
    if (tb.chunk) {
        if (scl) run(std::true_type{}, std::true_type{});
        else run(std::false_type{}, std::true_type{});
    } else if (scl) {
        run(std::true_type{}, std::false_type{});
    } else {
        run(std::false_type{}, std::false_type{});
    }
    k_results<<<(w.n + 127) / 128, 128, 0, st>>>(tb, w);
    T2B_CUDA(cudaGetLastError());
}

void launch_reconstruct(const Volume& g, const float2* data, const float* weight, double2* fconv,
                        double* fw, double* rad, double* cnt, cudaStream_t st, const double* tau2, double tscale,
                        int minres_map)
{
    const int ps = g.ydim, fx = ps / 2 + 1, nz = g.ref_dim == 3 ? ps : 1;
    const long long total = (long long)nz * ps * fx;
    T2B_CUDA(cudaMemsetAsync(rad, 0, sizeof(double) * g.r_max, st));
    T2B_CUDA(cudaMemsetAsync(cnt, 0, sizeof(double) * g.r_max, st));
    const int nb = (int)((total + 255) / 256);
    k_decenter<<<nb, 256, 0, st>>>(g, data, weight, fconv, fw, rad, cnt, tau2, tscale, minres_map);
    k_radnorm<<<(g.r_max + 255) / 256, 256, 0, st>>>(g.r_max, rad, cnt);
    k_divide<<<nb, 256, 0, st>>>(g, fconv, fw, rad);
    T2B_CUDA(cudaGetLastError());
}

void launch_decenter(const Volume& g, const float2* data, const float* weight, double2* fconv, double* fw,
                     double* rad, double* cnt, cudaStream_t st, const double* tau2, double tscale, int minres_map)
{
    const int ps = g.ydim, fx = ps / 2 + 1, nz = g.ref_dim == 3 ? ps : 1;
    const long long total = (long long)nz * ps * fx;
    T2B_CUDA(cudaMemsetAsync(rad, 0, sizeof(double) * g.r_max, st));
    T2B_CUDA(cudaMemsetAsync(cnt, 0, sizeof(double) * g.r_max, st));
    k_decenter<<<(int)((total + 255) / 256), 256, 0, st>>>(g, data, weight, fconv, fw, rad, cnt, tau2, tscale,
                                                          minres_map);
    T2B_CUDA(cudaGetLastError());
}

}  // namespace t2b
