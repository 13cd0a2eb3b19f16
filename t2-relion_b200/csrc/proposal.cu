// Learned orientation proposals for the coarse pass (sm_100a).
//
// A small network reads the lowest Fourier rings of each particle and ranks
// the K*O coarse orientations; the coarse diff2 then runs on the particle's
// top-k orientations only (tc_launch_prop), and the rest of the E-step
// (FP64 weights, significance, fine pass, weighted sums, backprojection) is
// unchanged.  A full coarse pass on every `every`-th particle (the audit)
// measures the posterior mass the proposals hold; below the threshold the
// batch falls back to the full coarse pass, decided on the device (a gate
// flag read by every kernel of both paths), so a captured CUDA graph serves
// both outcomes.  No counterpart in the reference.
//
// Network (BF16 weights, FP32 accumulation):
//   features  the 8 lowest rings of X * CTF * sqrt(Minvsigma2), as a 16 x 16
//             real image (inverse DFT of the half-plane), RMS-normalised
//   conv1     3x3, 1 -> 16 channels, ReLU            (16 x 16)
//   conv2     3x3 stride 2, 16 -> 32 channels, ReLU  (8 x 8 -> 2048)
//   fc1, fc2  2048 -> 1024 -> 1024, ReLU
//   fc3       1024 -> K*O logits
// Inference runs fc1..fc3 on the tcgen05 kernel (one BF16 product); training
// runs every layer through the SIMT kernels below, forward and backward, with
// Adam, on particles generated here from the current references (projection,
// CTF, shift, noise) and labelled with their true orientation and with the
// posterior of the plain E-step run on them.
#include "t2b_internal.cuh"
#include "project_pixel.cuh"
#include "proposal.cuh"
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

namespace t2b {
namespace {

using bf16 = __nv_bfloat16;
constexpr double PI = 3.14159265358979323846;

__device__ __forceinline__ float ldw(const bf16* th, size_t i) { return __bfloat162float(th[i]); }

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
__device__ T bsum(T v, T* sh /* >= 32 */)
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

__device__ __forceinline__ float bmax(float v, float* sh)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : -INFINITY;
    if (wid == 0)
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (threadIdx.x == 0) sh[0] = v;
    __syncthreads();
    const float r = sh[0];
    __syncthreads();
    return r;
}

// ------------------------------------------------------------ features
// img[b][u*16+v] = sum_k g_k Re(F_k e^{2 pi i (ky u + kx v)/16}),
// F = X CTF sqrt(Minvsigma2) over the ring pixels, g = 1 on the kx = 0 column
// (both ky signs are stored) and 2 elsewhere; then divided by its RMS.
// With `proj` set, F = P_oc CTF2 sqrt(Minvsigma2) of table row b instead (the
// noise-free template of orientation b under the mean squared CTF `ctf2`).
__global__ void __launch_bounds__(NET_NPIX) k_features(const float2* __restrict__ fimg, const float* __restrict__ ctf,
                                                      const float* __restrict__ minv, int P, const int* __restrict__ ring,
                                                      const int* __restrict__ ring_k, int nring, float* __restrict__ img,
                                                      const float2* __restrict__ proj, const float* __restrict__ ctf2)
{
    __shared__ float2 F[NET_MAX_RING];
    __shared__ int kk[NET_MAX_RING];
    __shared__ float cs[16], sn[16];
    __shared__ float red[32];
    const int b = blockIdx.x;
    if (threadIdx.x < 16) {
        double sv, cv;
        sincospi((double)threadIdx.x / 8., &sv, &cv);
        cs[threadIdx.x] = (float)cv;
        sn[threadIdx.x] = (float)sv;
    }
    for (int i = threadIdx.x; i < nring; i += blockDim.x) {
        const int n = ring[i];
        float2 X;
        float g;
        if (proj) {
            X = proj[(size_t)b * P + n];
            g = ctf2[n] * sqrtf(fmaxf(minv[n], 0.f));
        } else {
            X = fimg[(size_t)b * P + n];
            g = ctf[(size_t)b * P + n] * sqrtf(fmaxf(minv[(size_t)b * P + n], 0.f));
        }
        const int kx = ring_k[2 * i], ky = ring_k[2 * i + 1];
        const float wgt = kx == 0 ? 1.f : 2.f;
        F[i] = make_float2(wgt * g * X.x, wgt * g * X.y);
        kk[i] = (kx & 15) | ((ky & 15) << 4);
    }
    __syncthreads();
    const int u = threadIdx.x >> 4, v = threadIdx.x & 15;
    float acc = 0.f;
    for (int i = 0; i < nring; i++) {
        const int kx = kk[i] & 15, ky = kk[i] >> 4;
        const int m = (ky * u + kx * v) & 15;
        acc += F[i].x * cs[m] - F[i].y * sn[m];
    }
    const float ms = bsum(acc * acc, red) / NET_NPIX;
    img[(size_t)b * NET_NPIX + threadIdx.x] = ms > 0.f ? acc * rsqrtf(ms) : 0.f;
}

// ------------------------------------------------------------- convs
// conv1 (3x3, pad 1) + ReLU, conv2 (3x3, stride 2, pad 1) + ReLU; one CTA per
// particle.  x0 index = c2*64 + Y*8 + X.
__global__ void __launch_bounds__(256) k_conv_fwd(const float* __restrict__ img, const bf16* __restrict__ th, NetLayout L,
                                                  int n, float* __restrict__ a1_out, float* __restrict__ x0,
                                                  bf16* __restrict__ x0b)
{
    static_assert(NET_C2 == 32 && NET_H0 == NET_C2 * 64, "conv2 thread layout: 4 groups of 8 channels x 8 x 8");
    __shared__ float im[18][18];
    __shared__ float a1[NET_C1][18][18];
    __shared__ float w1[NET_C1 * 9 + NET_C1];
    __shared__ __align__(16) float w2t[NET_C1 * 9][NET_C2];   // conv2 weights as [tap][output channel]
    __shared__ float b2[NET_C2];
    const int b = blockIdx.x;
    if (b >= n) return;
    for (int i = threadIdx.x; i < 18 * 18; i += blockDim.x) (&im[0][0])[i] = 0.f;
    for (int i = threadIdx.x; i < NET_C1 * 18 * 18; i += blockDim.x) (&a1[0][0][0])[i] = 0.f;
    for (int i = threadIdx.x; i < NET_C1 * 9; i += blockDim.x) w1[i] = ldw(th, L.wc1 + i);
    for (int i = threadIdx.x; i < NET_C1; i += blockDim.x) w1[NET_C1 * 9 + i] = ldw(th, L.bc1 + i);
    for (int i = threadIdx.x; i < NET_C2 * NET_C1 * 9; i += blockDim.x) {
        const int c2 = i / (NET_C1 * 9), tap = i - c2 * (NET_C1 * 9);   // global layout [c2][c1][dy][dx]
        w2t[tap][c2] = ldw(th, L.wc2 + i);
    }
    for (int i = threadIdx.x; i < NET_C2; i += blockDim.x) b2[i] = ldw(th, L.bc2 + i);
    __syncthreads();
    {
        const int y = threadIdx.x >> 4, x = threadIdx.x & 15;
        im[y + 1][x + 1] = img[(size_t)b * NET_NPIX + threadIdx.x];
    }
    __syncthreads();
    {
        const int y = threadIdx.x >> 4, x = threadIdx.x & 15;
        for (int c = 0; c < NET_C1; c++) {
            float acc = w1[NET_C1 * 9 + c];
#pragma unroll
            for (int dy = 0; dy < 3; dy++)
#pragma unroll
                for (int dx = 0; dx < 3; dx++) acc += w1[c * 9 + dy * 3 + dx] * im[y + dy][x + dx];
            acc = fmaxf(acc, 0.f);
            a1[c][y + 1][x + 1] = acc;
            if (a1_out) a1_out[(size_t)b * NET_C1 * NET_NPIX + c * NET_NPIX + threadIdx.x] = acc;
        }
    }
    __syncthreads();
    // conv2: each thread one output position (Y, X) and eight output channels g*8 .. g*8+7, so
    // one read of a1 serves eight products and the weights of a tap come as two broadcast
    // 16-byte reads; every output sums its bias and taps in the order (c1, dy, dx) as before
    for (int e = threadIdx.x; e < NET_H0 / 8; e += blockDim.x) {
        const int pos = e & 63, g = e >> 6, Y = pos >> 3, X = pos & 7;
        float acc[8];
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] = b2[g * 8 + j];
        for (int c1 = 0; c1 < NET_C1; c1++)
#pragma unroll
            for (int dy = 0; dy < 3; dy++)
#pragma unroll
                for (int dx = 0; dx < 3; dx++) {
                    const float a = a1[c1][2 * Y + dy][2 * X + dx];
                    const float4 wa = *reinterpret_cast<const float4*>(&w2t[c1 * 9 + dy * 3 + dx][g * 8]);
                    const float4 wb = *reinterpret_cast<const float4*>(&w2t[c1 * 9 + dy * 3 + dx][g * 8 + 4]);
                    acc[0] += wa.x * a;
                    acc[1] += wa.y * a;
                    acc[2] += wa.z * a;
                    acc[3] += wa.w * a;
                    acc[4] += wb.x * a;
                    acc[5] += wb.y * a;
                    acc[6] += wb.z * a;
                    acc[7] += wb.w * a;
                }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int o = (g * 8 + j) * 64 + pos;   // output layout [c2][Y][X]
            const float v = fmaxf(acc[j], 0.f);
            if (x0) x0[(size_t)b * NET_H0 + o] = v;
            if (x0b) x0b[(size_t)b * NET_H0 + o] = __float2bfloat16_rn(v);
        }
    }
}

// out = act(sum_s y_s + bias) as FP32 and / or BF16 (rows x cols, row-major; the
// `slices` partial products of a split-K GEMM, rows * cols apart, summed in order)
__global__ void k_bias_act(const float* __restrict__ y, const bf16* __restrict__ bias, int rows, int cols, int relu,
                           float* __restrict__ outf, bf16* __restrict__ outb, int slices = 1)
{
    const size_t total = (size_t)rows * cols;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        // the slices' loads four at a time in flight, summed in slice order
        float acc = y[i];
        int s = 1;
        for (; s + 3 < slices; s += 4) {
            const float a0 = y[(size_t)s * total + i], a1 = y[(size_t)(s + 1) * total + i];
            const float a2 = y[(size_t)(s + 2) * total + i], a3 = y[(size_t)(s + 3) * total + i];
            acc += a0;
            acc += a1;
            acc += a2;
            acc += a3;
        }
        for (; s < slices; ++s) acc += y[(size_t)s * total + i];
        float v = acc + __bfloat162float(bias[i % cols]);
        if (relu) v = fmaxf(v, 0.f);
        if (outf) outf[i] = v;
        if (outb) outb[i] = __float2bfloat16_rn(v);
    }
}

// ------------------------------------------------------------- top-k
// The k largest logits (+ bias) of each particle, ranked (ties by index);
// orientations with a zero prior never enter.  Radix select over the ordered
// keys (four 8-bit digits) in shared memory, then a bitonic sort of the
// selected set.
__global__ void __launch_bounds__(1024) k_topk(const float* __restrict__ logits, const bf16* __restrict__ bias,
                                               const unsigned char* __restrict__ skip, int KO, int k,
                                               int* __restrict__ prop, int ranked)
{
    extern __shared__ unsigned keys[];
    __shared__ unsigned whist[8][256];   // sub-histograms: warps w and w + 8, + 16, + 24 share one
    __shared__ unsigned s_prefix, s_want, s_n;
    __shared__ unsigned long long cand[NET_TOPK_CAND];
    const int b = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    {
        // eight elements per thread in flight: all their loads issued before any key is formed
        const float* lg = logits + (size_t)b * KO;
        const int bd = blockDim.x;
        int i = threadIdx.x;
        for (; i + 7 * bd < KO; i += 8 * bd) {
            float v[8], bb[8];
            unsigned char sk[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                v[u] = lg[i + u * bd];
                bb[u] = __bfloat162float(bias[i + u * bd]);
                sk[u] = skip[i + u * bd];
            }
#pragma unroll
            for (int u = 0; u < 8; u++) keys[i + u * bd] = sk[u] ? 0u : f2key(v[u] + bb[u]);
        }
        for (; i < KO; i += bd) keys[i] = skip[i] ? 0u : f2key(lg[i] + __bfloat162float(bias[i]));
    }
    if (threadIdx.x == 0) { s_prefix = 0; s_want = (unsigned)k; s_n = 0; }
    __syncthreads();
    unsigned mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&whist[0][0])[i] = 0;
        __syncthreads();
        const unsigned prefix = s_prefix;
        unsigned* hw = whist[wid & 7];
        for (int i = threadIdx.x; i < KO; i += blockDim.x)
            if ((keys[i] & mask) == prefix) atomicAdd(&hw[(keys[i] >> shift) & 255u], 1u);
        __syncthreads();
        if (wid == 0) {
            // digit of the k-th largest: lane l holds bins 255-8l .. 248-8l (descending); a suffix
            // scan over the lanes finds the lane whose bins cross `want`, then the lane walks them
            const unsigned want0 = s_want;
            unsigned c[8], tot = 0;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int dg = 255 - 8 * lane - j;
                unsigned v = 0;
#pragma unroll
                for (int h = 0; h < 8; h++) v += whist[h][dg];
                c[j] = v;
                tot += v;
            }
            unsigned incl = tot;   // inclusive prefix over lanes 0..lane (higher digits first)
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned x = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += x;
            }
            const unsigned excl = incl - tot;
            const bool here = excl < want0 && incl >= want0;
            const unsigned ball = __ballot_sync(0xffffffffu, here);
            if (here && lane == __ffs(ball) - 1) {
                unsigned want = want0 - excl, d = 0;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    if (c[j] >= want) { d = 255u - 8u * lane - j; break; }
                    want -= c[j];
                }
                s_want = want;
                s_prefix = prefix | (d << shift);
            }
        }
        mask |= 255u << shift;
        __syncthreads();
    }
    const unsigned kth = s_prefix;
    if (!ranked) {
        // the set only, in index order: keys above the k-th, then the first ties at it;
        // thread t owns the contiguous index range [t*per, (t+1)*per)
        __shared__ unsigned wsum_hi[32], wsum_eq[32];
        const int per = (KO + blockDim.x - 1) / blockDim.x;
        const int i0 = threadIdx.x * per, i1 = min(KO, i0 + per);
        unsigned nhi = 0, neq = 0;
        for (int i = i0; i < i1; i++) { nhi += keys[i] > kth; neq += keys[i] == kth; }
        // prefix sums over the threads in order: within the warp by shuffles, then over the warps
        unsigned hi = nhi, eq = neq;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned a = __shfl_up_sync(0xffffffffu, hi, o), e = __shfl_up_sync(0xffffffffu, eq, o);
            if (lane >= o) { hi += a; eq += e; }
        }
        if (lane == 31) { wsum_hi[wid] = hi; wsum_eq[wid] = eq; }
        __syncthreads();
        const int nw = blockDim.x >> 5;
        if (wid == 0) {
            unsigned th = lane < nw ? wsum_hi[lane] : 0u, te = lane < nw ? wsum_eq[lane] : 0u;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned a = __shfl_up_sync(0xffffffffu, th, o), e = __shfl_up_sync(0xffffffffu, te, o);
                if (lane >= o) { th += a; te += e; }
            }
            if (lane < nw) { wsum_hi[lane] = th; wsum_eq[lane] = te; }   // inclusive over the warps
        }
        __syncthreads();
        const unsigned total_hi = wsum_hi[nw - 1];
        unsigned ph = (wid > 0 ? wsum_hi[wid - 1] : 0u) + hi - nhi, pe = (wid > 0 ? wsum_eq[wid - 1] : 0u) + eq - neq;
        for (int i = i0; i < i1; i++) {
            if (keys[i] > kth) {
                prop[(size_t)b * k + ph++] = i;
            } else if (keys[i] == kth) {
                const unsigned pos = total_hi + pe++;
                if (pos < (unsigned)k) prop[(size_t)b * k + pos] = i;
            }
        }
        return;
    }
    // every key above the k-th, and the ties at it
    for (int i = threadIdx.x; i < KO; i += blockDim.x)
        if (keys[i] >= kth) {
            const unsigned pos = atomicAdd(&s_n, 1u);
            if (pos < NET_TOPK_CAND) cand[pos] = ((unsigned long long)keys[i] << 32) | (unsigned)(0xffffffffu - (unsigned)i);
        }
    __syncthreads();
    const int nc = (int)min(s_n, (unsigned)NET_TOPK_CAND);
    int n2 = 1;
    while (n2 < nc) n2 <<= 1;
    for (int i = nc + threadIdx.x; i < n2; i += blockDim.x) cand[i] = 0ull;
    __syncthreads();
    // descending by key, then ascending index (the low word holds ~index)
    for (int kk = 2; kk <= n2; kk <<= 1)
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n2; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const bool desc = (i & kk) == 0;
                    const unsigned long long a = cand[i], c = cand[l];
                    if (desc ? (a < c) : (a > c)) { cand[i] = c; cand[l] = a; }
                }
            }
            __syncthreads();
        }
    for (int j = threadIdx.x; j < k; j += blockDim.x)
        prop[(size_t)b * k + j] = j < nc ? (int)(0xffffffffu - (unsigned)(cand[j] & 0xffffffffull)) : 0;
}

// ------------------------------------------------ low-resolution rescoring
// Exact low-resolution score of each of the network's K1 candidates: over the
// ring pixels only, d(j, t) = c0 + sum_q w2_q |P_j,q|^2 - Re(P_j,q conj(cvec_q ab_t,q))
// (the coarse diff2 restricted to the ring plus the particle's constant) and
// score_j = log sum_t pdf_t(t) exp(-d(j, t)) + log pdf_o(j), the log of the
// particle's low-resolution posterior of orientation j up to a constant.
// The contraction runs on the tensor cores (tc_launch_rescore: split-BF16, one
// 128 x 96 tile per 128 candidates of a particle) and its epilogue reduces each
// candidate's row to the score; the operands are the ring pixels as
// K = 2 x ring (re, im interleaved), zero padded to kr.
constexpr int RS_TMAX = 96;            // translations of one rescoring tile

// projections of every coarse orientation at the ring pixels: FP32 (norms) and
// split-BF16 rows (the contraction's A operand); once per configuration
__global__ void k_ring_table(const float2* __restrict__ proj, int P, const int* __restrict__ ring, int nring, int KO,
                             int kr, float2* __restrict__ projR, bf16* __restrict__ rh, bf16* __restrict__ rl)
{
    const size_t total = (size_t)KO * (kr / 2);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t oc = i / (kr / 2);
        const int q = (int)(i - oc * (kr / 2));
        float2 v = make_float2(0.f, 0.f);
        if (q < nring) {
            v = proj[oc * P + ring[q]];
            projR[oc * nring + q] = v;
        }
        const bf16 hx = __float2bfloat16_rn(v.x), hy = __float2bfloat16_rn(v.y);
        reinterpret_cast<__nv_bfloat162*>(rh)[i] = __halves2bfloat162(hx, hy);
        reinterpret_cast<__nv_bfloat162*>(rl)[i] = __halves2bfloat162(__float2bfloat16_rn(v.x - __bfloat162float(hx)),
                                                                      __float2bfloat16_rn(v.y - __bfloat162float(hy)));
    }
}

// per batch: the shifted ring images cvec_b ab_t as split-BF16 rows b*T + t (the
// contraction's B operand), and w2 at the ring pixels
// One CTA per particle: its ring pixels' indices and image values staged once in shared memory,
// then every (shift t, ring pixel q) of its T rows, four of them per thread in flight.
constexpr int RING_MAX = 512;   // kr / 2 (ring pixels + padding) at most
__global__ void __launch_bounds__(256) k_ring_images(Tables tb, Work w, const int* __restrict__ ring, int nring, int kr,
                                                     bf16* __restrict__ sh, bf16* __restrict__ sl, float* __restrict__ w2r)
{
    __shared__ int s_n[RING_MAX];
    __shared__ float2 s_c[RING_MAX];
    const int b = blockIdx.x, P = tb.P, T = tb.T, kh = kr / 2;
    if (b >= w.n || kh > RING_MAX) return;
    for (int q = threadIdx.x; q < kh; q += blockDim.x) {
        const int n = q < nring ? ring[q] : -1;
        s_n[q] = n;
        s_c[q] = n >= 0 ? w.cvec[(size_t)b * P + n] : make_float2(0.f, 0.f);
        if (n >= 0) w2r[(size_t)b * nring + q] = w.w2[(size_t)b * P + n];
    }
    __syncthreads();
    const int total = T * kh;
    const auto emit = [&](int e, float2 a) {
        const int t = e / kh, q = e - t * kh;
        const float2 c = s_c[q];
        const float2 v = make_float2(c.x * a.x - c.y * a.y, c.x * a.y + c.y * a.x);
        const size_t row = (size_t)b * T + t;
        const bf16 hx = __float2bfloat16_rn(v.x), hy = __float2bfloat16_rn(v.y);
        reinterpret_cast<__nv_bfloat162*>(sh + row * kr)[q] = __halves2bfloat162(hx, hy);
        reinterpret_cast<__nv_bfloat162*>(sl + row * kr)[q] =
            __halves2bfloat162(__float2bfloat16_rn(v.x - __bfloat162float(hx)), __float2bfloat16_rn(v.y - __bfloat162float(hy)));
    };
    const auto phase = [&](int e) -> float2 {   // ab_t at ring pixel q (zero for the padding)
        const int t = e / kh, n = s_n[e - t * kh];
        return n >= 0 ? tb.ab_c[(size_t)t * P + n] : make_float2(0.f, 0.f);
    };
    const int bd = blockDim.x;
    int e = threadIdx.x;
    for (; e + 3 * bd < total; e += 4 * bd) {
        const float2 a0 = phase(e), a1 = phase(e + bd), a2 = phase(e + 2 * bd), a3 = phase(e + 3 * bd);
        emit(e, a0);
        emit(e + bd, a1);
        emit(e + 2 * bd, a2);
        emit(e + 3 * bd, a3);
    }
    for (; e < total; e += bd) emit(e, phase(e));
}

// candidate rows (b*K1 + j) of the A operand and their ring norms; one warp per candidate
__global__ void __launch_bounds__(256) k_rescore_gather(int n, int k1, int nring, int kr, const int* __restrict__ cand,
                                                        const float2* __restrict__ projR, const bf16* __restrict__ rh,
                                                        const bf16* __restrict__ rl, const float* __restrict__ w2r,
                                                        bf16* __restrict__ ah, bf16* __restrict__ al,
                                                        float* __restrict__ rnorm)
{
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= (long long)n * k1) return;
    const int b = (int)(gw / k1);
    const size_t oc = (size_t)cand[gw];
    const uint4* sh = reinterpret_cast<const uint4*>(rh + oc * kr);
    const uint4* sl = reinterpret_cast<const uint4*>(rl + oc * kr);
    uint4* dh = reinterpret_cast<uint4*>(ah + (size_t)gw * kr);
    uint4* dl = reinterpret_cast<uint4*>(al + (size_t)gw * kr);
    float acc = 0.f;
    for (int v = lane; v < kr / 8; v += 32) {
        const uint4 hv = sh[v], lv = sl[v];
        dh[v] = hv;
        dl[v] = lv;
        const __nv_bfloat162* hp = reinterpret_cast<const __nv_bfloat162*>(&hv);
        const __nv_bfloat162* lp = reinterpret_cast<const __nv_bfloat162*>(&lv);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int q = 4 * v + e;   // ring pixel of this (re, im) pair; zero rows beyond nring
            if (q < nring) {
                const float2 hf = __bfloat1622float2(hp[e]), lf = __bfloat1622float2(lp[e]);
                const float re = hf.x + lf.x, im = hf.y + lf.y;
                acc += w2r[(size_t)b * nring + q] * (re * re + im * im);
            }
        }
    }
    (void)projR;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) rnorm[gw] = acc;
}

// the k best-scored candidates of each particle, ranked (ties by rank in the network's list):
// a bitonic sort of the keys (score, then the candidate's position), descending.  Up to 1,024
// candidates (the usual K1) one key per thread: the exchanges with a partner in the same warp
// (distance < 32) are shuffles, only the wider ones go through shared memory and a barrier
// (15 barriers instead of 55 for 1,024 keys); the same network, the same order.
__global__ void __launch_bounds__(1024) k_rescore_select(const int* __restrict__ cand, const float* __restrict__ score,
                                                         int k1, int k, int* __restrict__ prop)
{
    __shared__ unsigned long long key[NET_TOPK_CAND];
    const int b = blockIdx.x;
    const auto key_of = [&](int i) -> unsigned long long {
        // keys are > 0 (the low word holds ~i): padding with 0 sorts last
        return i < k1 ? ((unsigned long long)f2key(score[(size_t)b * k1 + i]) << 32) | (unsigned)(0xffffffffu - (unsigned)i)
                      : 0ull;
    };
    int n2 = 1;
    while (n2 < k1) n2 <<= 1;
    if (n2 <= (int)blockDim.x) {
        const int i = threadIdx.x;
        const int nb = blockDim.x;   // sorted as nb keys (the padding at the end)
        unsigned long long v = key_of(i);
        for (int kk = 2; kk <= nb; kk <<= 1)
            for (int jj = kk >> 1; jj > 0; jj >>= 1) {
                unsigned long long o;
                if (jj >= 32) {
                    key[i] = v;
                    __syncthreads();
                    o = key[i ^ jj];
                    __syncthreads();
                } else {
                    o = __shfl_xor_sync(0xffffffffu, v, jj);
                }
                // the pair (i, i ^ jj): in a descending block the lower index keeps the larger
                const bool keep_max = ((i & kk) == 0) == ((i & jj) == 0);
                v = keep_max ? (v > o ? v : o) : (v < o ? v : o);
            }
        key[i] = v;
        __syncthreads();
    } else {
        for (int i = threadIdx.x; i < n2; i += blockDim.x) key[i] = key_of(i);
        __syncthreads();
        for (int kk = 2; kk <= n2; kk <<= 1)
            for (int jj = kk >> 1; jj > 0; jj >>= 1) {
                for (int i = threadIdx.x; i < n2; i += blockDim.x) {
                    const int l = i ^ jj;
                    if (l > i) {
                        const bool desc = (i & kk) == 0;
                        const unsigned long long a = key[i], c = key[l];
                        if (desc ? (a < c) : (a > c)) { key[i] = c; key[l] = a; }
                    }
                }
                __syncthreads();
            }
    }
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        const int r = (int)(0xffffffffu - (unsigned)(key[j] & 0xffffffffull));
        prop[(size_t)b * k + j] = cand[(size_t)b * k1 + r];
    }
}

// ---------------------------------------------- proposal coarse operands
// A rows of the proposal contraction: for every (particle b, proposal j) the
// projection of orientation oc = prop[b][j] times the conjugate particle image,
// P_oc[p] conj(cvec_b[p]) over the in-radius pixels (P_oc = hi + lo of the
// configuration's split-BF16 coarse operand), split again into hi + lo; and, from the
// same values, the norm N = sum_p w2_p |P_oc[p]|^2.
// Row of (b, j): b * kslot + j, stored pre-swizzled and K-blocked (swz_offset: a
// tensor-core tile of 128 rows and one k-block is one contiguous 16 KB block).
// Runs while *gate != 0.
__global__ void __launch_bounds__(128) k_prop_gather(Work w, int P, const int* __restrict__ kpix, int nk, int kslot,
                                                     int rows, int kdim,
                                                     const bf16* __restrict__ bh, const bf16* __restrict__ bl,
                                                     bf16* __restrict__ ph, bf16* __restrict__ pl, float* __restrict__ nprop)
{
    __shared__ float red[32];
    if (!w.gate || *w.gate == 0) return;
    const int b = blockIdx.y, j = blockIdx.x;
    if (b >= w.n || j >= w.kprop) return;
    const size_t oc = (size_t)w.prop[(size_t)b * w.kprop + j];
    const size_t row = (size_t)b * kslot + j;
    float acc = 0.f;
    {
        const uint4* sh = reinterpret_cast<const uint4*>(bh + oc * kdim);
        const uint4* sl = reinterpret_cast<const uint4*>(bl + oc * kdim);
        const int4* kp4 = reinterpret_cast<const int4*>(kpix);
        const float2* cb = w.cvec + (size_t)b * P;
        const float* w2b = w.w2 + (size_t)b * P;
        uint4* dh = reinterpret_cast<uint4*>(ph);
        uint4* dl = reinterpret_cast<uint4*>(pl);
        for (int v = threadIdx.x; v < kdim / 8; v += blockDim.x) {
            const uint4 hv = sh[v], lv = sl[v];
            const __nv_bfloat162* hp = reinterpret_cast<const __nv_bfloat162*>(&hv);
            const __nv_bfloat162* lp = reinterpret_cast<const __nv_bfloat162*>(&lv);
            // pixel indices of these 4 values: one 16-byte load when all are in radius
            int kk[4];
            if (4 * v + 3 < nk) {
                const int4 k4 = kp4[v];
                kk[0] = k4.x; kk[1] = k4.y; kk[2] = k4.z; kk[3] = k4.w;
            } else {
#pragma unroll
                for (int e = 0; e < 4; e++) kk[e] = 4 * v + e < nk ? kpix[4 * v + e] : 0;
            }
            __nv_bfloat162 h[4], l[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                float2 a = make_float2(0.f, 0.f);
                if (4 * v + e < nk) {
                    const float2 hf = __bfloat1622float2(hp[e]), lf = __bfloat1622float2(lp[e]);
                    const float2 pv = make_float2(hf.x + lf.x, hf.y + lf.y);
                    const float2 c = cb[kk[e]];
                    a = make_float2(pv.x * c.x + pv.y * c.y, pv.y * c.x - pv.x * c.y);
                    acc += w2b[kk[e]] * (pv.x * pv.x + pv.y * pv.y);
                }
                const bf16 hx = __float2bfloat16_rn(a.x), hy = __float2bfloat16_rn(a.y);
                h[e] = __halves2bfloat162(hx, hy);
                l[e] = __halves2bfloat162(__float2bfloat16_rn(a.x - __bfloat162float(hx)),
                                          __float2bfloat16_rn(a.y - __bfloat162float(hy)));
            }
            const size_t o = swz_offset(row, 8 * v, rows) / 8;   // 16-byte group v of the row
            dh[o] = *reinterpret_cast<const uint4*>(h);
            dl[o] = *reinterpret_cast<const uint4*>(l);
        }
    }
    acc = bsum(acc, red);
    if (threadIdx.x == 0) nprop[(size_t)b * w.kprop + j] = acc;
}

// ------------------------------------------------------------- audit
// Choose the audited particles of the batch (every `every`-th particle of the
// stream), open the gate and reset the audit accumulators.  One CTA.
__global__ void k_audit_begin(PropState* ps, int* audit_b, int n, int every, int na_max, unsigned* minkeya,
                              double* asum, double* r_audit)
{
    if (threadIdx.x == 0) {
        // the stream positions seen + b that are multiples of `every`: an arithmetic progression
        int na = 0;
        const long long seen = ps->seen;
        const long long first = (every - seen % every) % every;
        for (long long b = first; b < n && na < na_max; b += every) audit_b[na++] = (int)b;
        ps->na = na;
        ps->seen = seen + n;
        ps->gate = 1;
    }
    __syncthreads();
    for (int a = threadIdx.x; a < na_max; a += blockDim.x) {
        minkeya[a] = 0xffffffffu;
        asum[2 * a] = 0.;
        asum[2 * a + 1] = 0.;
    }
    if (r_audit)
        for (int b = threadIdx.x; b < n; b += blockDim.x) r_audit[b] = -1.;
}

// image operand rows of the audited particles (cvec_b ab_t over the in-radius
// pixels, split-BF16, as the full pass's operand), their w2 and c0, into the
// audit slots
__global__ void __launch_bounds__(256) k_audit_operands(const PropState* ps, const int* audit_b, Work w, int T, int P,
                                                        const int* __restrict__ kpix, int nk, int kn,
                                                        int kdim, const float2* __restrict__ ab,
                                                        bf16* __restrict__ iah, bf16* __restrict__ ial,
                                                        bf16* __restrict__ wah, bf16* __restrict__ wal,
                                                        float* __restrict__ c0a)
{
    const int a = blockIdx.y;
    if (a >= ps->na) return;
    const int b = audit_b[a];
    const int t = blockIdx.x;  // t == T: the w2 / c0 row
    if (t < T) {
        const size_t dst = ((size_t)a * T + t) * kdim;
        const float2* cb = w.cvec + (size_t)b * P;
        const float2* at = ab + (size_t)t * P;
        __nv_bfloat162* dh = reinterpret_cast<__nv_bfloat162*>(iah + dst);
        __nv_bfloat162* dl = reinterpret_cast<__nv_bfloat162*>(ial + dst);
        for (int k = threadIdx.x; k < kdim / 2; k += blockDim.x) {
            float2 v = make_float2(0.f, 0.f);
            if (k < nk) {
                const int pp = kpix[k];
                const float2 c = cb[pp], e = at[pp];
                v = make_float2(c.x * e.x - c.y * e.y, c.x * e.y + c.y * e.x);
            }
            const bf16 hx = __float2bfloat16_rn(v.x), hy = __float2bfloat16_rn(v.y);
            dh[k] = __halves2bfloat162(hx, hy);
            dl[k] = __halves2bfloat162(__float2bfloat16_rn(v.x - __bfloat162float(hx)),
                                       __float2bfloat16_rn(v.y - __bfloat162float(hy)));
        }
    } else {
        for (int k = threadIdx.x; k < kn; k += blockDim.x) {
            const float v = k < nk ? w.w2[(size_t)b * P + kpix[k]] : 0.f;
            const bf16 h = __float2bfloat16_rn(v);
            wah[(size_t)a * kn + k] = h;
            wal[(size_t)a * kn + k] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
        if (threadIdx.x == 0) c0a[a] = w.c0[b];
    }
}

// posterior mass of the audited particles: total and inside the proposals
__global__ void __launch_bounds__(256) k_audit_mass(Tables tb, Work w, const PropState* ps, const int* audit_b,
                                                    const float* __restrict__ d2a, const unsigned* __restrict__ minkeya,
                                                    double* asum)
{
    extern __shared__ unsigned inprop[];  // KO bits
    __shared__ double red[32];
    const int a = blockIdx.y;
    if (a >= ps->na) return;
    const int b = audit_b[a];
    const int KO = tb.K * tb.O, T = tb.T;
    const int nwords = (KO + 31) / 32;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) inprop[i] = 0u;
    __syncthreads();
    for (int j = threadIdx.x; j < w.kprop; j += blockDim.x) {
        const int oc = w.prop[(size_t)b * w.kprop + j];
        atomicOr(&inprop[oc >> 5], 1u << (oc & 31));
    }
    __syncthreads();
    const double mn = (double)key2f(minkeya[a]);
    const long long n = (long long)KO * T;
    const float* d = d2a + (size_t)a * n;
    // hypotheses beyond this diff2 distance from the minimum weigh less than
    // e^-60 of the heaviest one (after the prior ratio); all of them together
    // are below 1e-18 of the sum
    const double cut = fmin(700., 60. + (w.lbound[2 * b + 1] - w.lbound[2 * b]));
    double sa = 0., sp = 0.;
    // 8 consecutive values per thread and pass (two 16-byte loads in flight; a slot's
    // n = K*O*T values start 16-byte aligned when n is a multiple of 4, else scalar loads)
    const bool vec = (n & 3) == 0;
    const long long step = (long long)gridDim.x * blockDim.x * 8;
    for (long long i0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 8; i0 < n; i0 += step) {
        float v[8];
        if (vec && i0 + 8 <= n) {
            const float4 a = *reinterpret_cast<const float4*>(d + i0), c = *reinterpret_cast<const float4*>(d + i0 + 4);
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = c.x; v[5] = c.y; v[6] = c.z; v[7] = c.w;
        } else {
#pragma unroll
            for (int e = 0; e < 8; e++) v[e] = i0 + e < n ? d[i0 + e] : -1.f;
        }
#pragma unroll
        for (int e = 0; e < 8; e++) {
            if (v[e] < 0.f) continue;
            const double dd = (double)v[e] - mn;
            if (dd > cut) continue;
            const long long i = i0 + e;
            const int oc = (int)(i / T), t = (int)(i - (long long)oc * T);
            const double wt = tb.pdf_oc[oc] * w.pdf_t[(size_t)b * T + t] * exp(-dd);
            sa += wt;
            if (inprop[oc >> 5] & (1u << (oc & 31))) sp += wt;
        }
    }
    sa = bsum(sa, red);
    sp = bsum(sp, red);
    if (threadIdx.x == 0) {
        atomicAdd(&asum[2 * a], sa);
        atomicAdd(&asum[2 * a + 1], sp);
    }
}

__global__ void k_audit_final(PropState* ps, const int* audit_b, const double* asum, double thr, double* r_audit)
{
    for (int a = threadIdx.x; a < ps->na; a += blockDim.x) {
        const double m = asum[2 * a] > 0. ? asum[2 * a + 1] / asum[2 * a] : 0.;
        if (r_audit) r_audit[audit_b[a]] = m;
        if (!(m >= thr)) atomicExch(&ps->gate, 0);
    }
}

// ------------------------------------------------- training particles
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
// uniform in [0, 1) from (seed, particle, stream): SplitMix64 finaliser
__device__ __forceinline__ double urand(unsigned long long seed, long long i, unsigned s)
{
    return (double)(mix64(seed ^ mix64((unsigned long long)i * 0x100000001b3ull + s)) >> 11) * (1.0 / 9007199254740992.0);
}

// One synthetic particle per CTA from the current references (the procedure
// of the reference's image simulator, src/apps/project.cpp:254-282):
// uniform random orientation and class, shift U(-max_shift, max_shift),
// defocus U(dmin, dmax) with astigmatism U(0, astig), CTF (src/ctf.h:181-238),
// X = CTF * P(A) * e^{+2 pi i k.t/N} + complex Gaussian noise of variance
// 1/Minvsigma2 per component (Box-Muller).  Writes the E-step inputs, the pose
// and class, and adds CTF^2 into ctf2_acc.
__global__ void __launch_bounds__(256) k_gen_particles(Tables tb, GenParams gp, const float2* const* mdl, const Volume* vol,
                                                       long long first, int n, float2* __restrict__ fimg,
                                                       float* __restrict__ ctf, float* __restrict__ minv,
                                                       double* __restrict__ scal, double* __restrict__ pose,
                                                       int* __restrict__ cls, float* __restrict__ ctf2_acc)
{
    __shared__ double A[9];
    __shared__ double prm[8];
    __shared__ int k_s;
    const int b = blockIdx.x;
    if (b >= n) return;
    const long long id = first + b;
    if (threadIdx.x == 0) {
        const int k = min(tb.K - 1, (int)(urand(gp.seed, id, 1) * tb.K));
        double rot, tilt, psi;
        if (tb.ref_dim == 3) {
            rot = -180. + 360. * urand(gp.seed, id, 2);
            tilt = acos(-1. + 2. * urand(gp.seed, id, 3)) * 180. / PI;
            psi = 360. * urand(gp.seed, id, 4);
        } else {
            rot = 0.;
            tilt = 0.;
            psi = 360. * urand(gp.seed, id, 4);
        }
        // Euler_angles2matrix (src/euler.cpp:52-91)
        double sa, ca, sb, cb, sg, cg;
        sincos(rot * PI / 180., &sa, &ca);
        sincos(tilt * PI / 180., &sb, &cb);
        sincos(psi * PI / 180., &sg, &cg);
        const double cc = cb * ca, cs = cb * sa, sc = sb * ca, ss = sb * sa;
        A[0] = cg * cc - sg * sa; A[1] = cg * cs + sg * ca; A[2] = -cg * sb;
        A[3] = -sg * cc - cg * sa; A[4] = -sg * cs + cg * ca; A[5] = sg * sb;
        A[6] = sc; A[7] = ss; A[8] = cb;
        prm[0] = gp.max_shift * (2. * urand(gp.seed, id, 5) - 1.);
        prm[1] = gp.max_shift * (2. * urand(gp.seed, id, 6) - 1.);
        const double du = gp.dmin + (gp.dmax - gp.dmin) * urand(gp.seed, id, 7);
        prm[2] = du;
        prm[3] = du - gp.astig * urand(gp.seed, id, 8);
        prm[4] = 180. * urand(gp.seed, id, 9);
        k_s = k;
        for (int j = 0; j < 9; j++) pose[(size_t)b * 9 + j] = A[j];
        cls[b] = k;
        double* sc8 = scal + (size_t)b * 8;
        for (int j = 0; j < 8; j++) sc8[j] = 0.;
        sc8[0] = gp.minv[0];
        sc8[6] = 1.;
    }
    __syncthreads();
    const int k = k_s;
    const Volume v = vol[k];
    const float2* m = mdl[k];
    // CTF constants (src/ctf.cpp:206-235)
    const double lam = 12.2643247 / sqrt(gp.kv * 1e3 * (1. + gp.kv * 1e3 * 0.978466e-6));
    const double K1 = PI / 2. * 2. * lam, K2 = PI / 2. * gp.cs * 1e7 * lam * lam * lam;
    const double K3 = atan(gp.q0 / sqrt(1. - gp.q0 * gp.q0));
    double saz, caz;
    sincos(prm[4] * PI / 180., &saz, &caz);
    const double Axx = -prm[2] * caz * caz - prm[3] * saz * saz;
    const double Axy = (prm[3] - prm[2]) * caz * saz;
    const double Ayy = -prm[2] * saz * saz - prm[3] * caz * caz;
    const int s = tb.s, xh = tb.xh, P = tb.P;
    const int rr = min(s / 2, v.r_max);
    for (int nn = threadIdx.x; nn < P; nn += blockDim.x) {
        const int i = nn / xh, x = nn - i * xh;
        const int y = (i < xh) ? i : i - s;
        const double X = x / (tb.ori_size * gp.angpix), Y = y / (tb.ori_size * gp.angpix);
        const double u2 = X * X + Y * Y;
        const double gamma = K1 * (Axx * X * X + 2. * Axy * X * Y + Ayy * Y * Y) + K2 * u2 * u2 - K3;
        double c = -sin(gamma);
        if (fabs(c) < 1e-8) c = c >= 0. ? 1e-8 : -1e-8;
        float2 pv = make_float2(0.f, 0.f);
        if (x * x + y * y <= rr * rr) pv = project_pixel(m, v, A, x, y);
        double ps_, pc_;
        sincos(2. * PI * (x * prm[0] + y * prm[1]) / tb.ori_size, &ps_, &pc_);
        double re = c * (pv.x * pc_ - pv.y * ps_), im = c * (pv.x * ps_ + pv.y * pc_);
        const float mv = gp.minv[nn];
        if (mv > 0.f) {
            const double sd = sqrt(1. / mv);
            const double u1 = fmax(urand(gp.seed, id, 1000 + 2 * nn), 1e-300), u2r = urand(gp.seed, id, 1001 + 2 * nn);
            const double r = sqrt(-2. * log(u1));
            double s2, c2;
            sincospi(2. * u2r, &s2, &c2);
            re += sd * r * c2;
            im += sd * r * s2;
        }
        fimg[(size_t)b * P + nn] = make_float2((float)re, (float)im);
        ctf[(size_t)b * P + nn] = (float)c;
        minv[(size_t)b * P + nn] = mv;
        if (ctf2_acc) atomicAdd(&ctf2_acc[nn], (float)(c * c));
    }
}

// class * O + the coarse orientation nearest to the true pose (largest trace(A_o^T A))
__global__ void __launch_bounds__(256) k_nearest(Tables tb, const double* __restrict__ pose, const int* __restrict__ cls,
                                                 int n, int* __restrict__ out)
{
    __shared__ double best[256];
    __shared__ int besti[256];
    const int b = blockIdx.x;
    if (b >= n) return;
    double A[9];
    for (int j = 0; j < 9; j++) A[j] = pose[(size_t)b * 9 + j];
    double bv = -1e300;
    int bi = 0;
    for (int o = threadIdx.x; o < tb.O; o += blockDim.x) {
        const double* E = tb.eul_c + 9 * (size_t)o;
        double tr = 0.;
        for (int j = 0; j < 9; j++) tr += E[j] * A[j];
        if (tr > bv) { bv = tr; bi = o; }
    }
    best[threadIdx.x] = bv;
    besti[threadIdx.x] = bi;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st) {
            const double o = best[threadIdx.x + st];
            const int oi = besti[threadIdx.x + st];
            if (o > best[threadIdx.x] || (o == best[threadIdx.x] && oi < besti[threadIdx.x])) {
                best[threadIdx.x] = o;
                besti[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[b] = cls[b] * tb.O + besti[0];
}

// marginal coarse posterior over orientations of the plain E-step just run on
// the batch in `w` (dense layout): marg[b][oc] = sum_t w(oc, t) / sum_c
__global__ void __launch_bounds__(256) k_marginal(Tables tb, Work w, double* __restrict__ marg)
{
    const int b = blockIdx.y;
    const int KO = tb.K * tb.O, T = tb.T;
    const int oc = blockIdx.x * blockDim.x + threadIdx.x;
    if (oc >= KO) return;
    const double mn = (double)key2f(w.minkey_c[b]);
    const double S = w.sum_c[b];
    const float* d = w.d2c + ((size_t)b * KO + oc) * T;
    double acc = 0.;
    for (int t = 0; t < T; t++) {
        const float v = d[t];
        if (v < 0.f) continue;
        const double dd = (double)v - mn;
        if (dd > 700.) continue;
        acc += tb.pdf_oc[oc] * w.pdf_t[(size_t)b * T + t] * exp(-dd);
    }
    marg[(size_t)b * KO + oc] = (S > 0. && w.status[b] == T2B_OK) ? acc / S : 0.;
}

// the NET_NPOST orientations of largest marginal posterior (oc, mass)
__global__ void __launch_bounds__(1024) k_post_top(const double* __restrict__ marg, int KO, int* __restrict__ top_oc,
                                                   float* __restrict__ top_w)
{
    __shared__ double bv[1024];
    __shared__ int bi[1024];
    __shared__ int taken[NET_NPOST];
    const int b = blockIdx.x;
    const double* m = marg + (size_t)b * KO;
    for (int r = 0; r < NET_NPOST; r++) {
        double v = -1.;
        int vi = -1;
        for (int i = threadIdx.x; i < KO; i += blockDim.x) {
            bool used = false;
            for (int q = 0; q < r; q++) used |= taken[q] == i;
            if (!used && m[i] > v) { v = m[i]; vi = i; }
        }
        bv[threadIdx.x] = v;
        bi[threadIdx.x] = vi;
        __syncthreads();
        for (int st = 512; st > 0; st >>= 1) {
            if (threadIdx.x < st) {
                const double o = bv[threadIdx.x + st];
                const int oi = bi[threadIdx.x + st];
                if (o > bv[threadIdx.x] || (o == bv[threadIdx.x] && oi >= 0 && (bi[threadIdx.x] < 0 || oi < bi[threadIdx.x]))) {
                    bv[threadIdx.x] = o;
                    bi[threadIdx.x] = oi;
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            taken[r] = bi[0];
            top_oc[(size_t)b * NET_NPOST + r] = bv[0] > 0. ? bi[0] : -1;
            top_w[(size_t)b * NET_NPOST + r] = bv[0] > 0. ? (float)bv[0] : 0.f;
        }
        __syncthreads();
    }
}

// posterior mass of the plain E-step held by each particle's proposals
__global__ void __launch_bounds__(256) k_capture(const double* __restrict__ marg, int KO, const int* __restrict__ prop,
                                                 int k, double* __restrict__ out)
{
    __shared__ double red[32];
    const int b = blockIdx.x;
    double acc = 0., tot = 0.;
    for (int j = threadIdx.x; j < k; j += blockDim.x) acc += marg[(size_t)b * KO + prop[(size_t)b * k + j]];
    for (int i = threadIdx.x; i < KO; i += blockDim.x) tot += marg[(size_t)b * KO + i];
    acc = bsum(acc, red);
    tot = bsum(tot, red);
    if (threadIdx.x == 0) out[b] = tot > 0. ? acc / tot : 0.;
}

// ----------------------------------------------------------- training
// C[m][n] (+)= sum_k A(m,k) B(k,n), A(m,k) = AT ? A[k*lda+m] : A[m*lda+k],
// B(k,n) = BT ? B[n*ldb+k] : B[k*ldb+n]; 64 x 64 tiles, 4 x 4 per thread.
// gridDim.z > 1 splits K (chunks of kchunk) and accumulates with atomics into
// a zeroed C.
template <bool AT, bool BT, typename TA, typename TB>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const TA* __restrict__ A, int lda,
                                               const TB* __restrict__ B, int ldb, float* __restrict__ C, int ldc,
                                               int kchunk)
{
    __shared__ __align__(16) float As[16][68];
    __shared__ __align__(16) float Bs[16][68];
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4] = {};
    for (int k0 = kbeg; k0 < kend; k0 += 16) {
        for (int e = 0; e < 4; e++) {
            const int idx = threadIdx.x * 4 + e;
            int mm, kk;
            if (AT) { mm = idx & 63; kk = idx >> 6; } else { kk = idx & 15; mm = idx >> 4; }
            const int m = m0 + mm, k = k0 + kk;
            float v = 0.f;
            if (m < M && k < kend) v = (float)(AT ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k]);
            As[kk][mm] = v;
            int nn, kb;
            if (BT) { kb = idx & 15; nn = idx >> 4; } else { nn = idx & 63; kb = idx >> 6; }
            const int n = n0 + nn, k2 = k0 + kb;
            float u = 0.f;
            if (n < N && k2 < kend) u = (float)(BT ? B[(size_t)n * ldb + k2] : B[(size_t)k2 * ldb + n]);
            Bs[kb][nn] = u;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
            const float4 a = *reinterpret_cast<const float4*>(&As[kk][ty * 4]);
            const float4 c = *reinterpret_cast<const float4*>(&Bs[kk][tx * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w}, cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], cv[j], acc[i][j]);
        }
        __syncthreads();
    }
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if (m >= M || n >= N) continue;
            if (gridDim.z > 1) atomicAdd(&C[(size_t)m * ldc + n], acc[i][j]);
            else C[(size_t)m * ldc + n] = acc[i][j];
        }
}

// Geometric target of a training particle: q(oc) proportional to
// exp(-angle(A_oc, A)^2 / (2 sigma^2)) over the orientations of its class
// (angle of the rotation between the coarse orientation and the true pose).
__device__ __forceinline__ float geo_q(const double* __restrict__ eul_c, int O, const float* geo, int cls, int oc,
                                       float inv2s2)
{
    if (oc / O != cls) return 0.f;
    const double* E = eul_c + 9 * (size_t)(oc - cls * O);
    float tr = 0.f;
    for (int j = 0; j < 9; j++) tr += (float)E[j] * geo[j];
    const float ang = acosf(fminf(1.f, fmaxf(-1.f, 0.5f * (tr - 1.f))));
    return expf(-ang * ang * inv2s2);
}

// Softmax cross-entropy against soft targets q = geo weight x normalised
// geometric target (geo: per row A[9] and its weight; null = none) + sparse
// (orientation, weight) pairs (NET_NTGT per row); the weights of a row sum to
// 1.  Logits (+ bias) are replaced by dL/dlogit = (softmax - q)/nb.
// Orientations with a zero prior are outside the softmax (gradient 0).
__global__ void __launch_bounds__(1024) k_softmax_ce(float* __restrict__ y, const bf16* __restrict__ bias,
                                                     const unsigned char* __restrict__ skip, int KO,
                                                     const int* __restrict__ tgt_oc, const float* __restrict__ tgt_w,
                                                     const float* __restrict__ geo, const int* __restrict__ gcls,
                                                     const double* __restrict__ eul_c, int O, float inv2s2, int nb,
                                                     double* loss)
{
    __shared__ float red[32];
    __shared__ double redd[32];
    const int b = blockIdx.x;
    float* row = y + (size_t)b * KO;
    const float* gb = geo ? geo + (size_t)b * 10 : nullptr;
    const float gw = gb ? gb[9] : 0.f;
    const int gc = geo ? gcls[b] : 0;
    float mx = -INFINITY;
    for (int i = threadIdx.x; i < KO; i += blockDim.x)
        if (!skip[i]) mx = fmaxf(mx, row[i] + __bfloat162float(bias[i]));
    mx = bmax(mx, red);
    double se = 0.;
    for (int i = threadIdx.x; i < KO; i += blockDim.x)
        if (!skip[i]) se += exp((double)(row[i] + __bfloat162float(bias[i]) - mx));
    se = bsum(se, redd);
    const double lse = log(se);
    double lq = 0.;
    for (int j = threadIdx.x; j < NET_NTGT; j += blockDim.x) {
        const int oc = tgt_oc[(size_t)b * NET_NTGT + j];
        const float q = tgt_w[(size_t)b * NET_NTGT + j];
        if (oc >= 0 && q > 0.f && !skip[oc]) lq += q * (lse - (double)(row[oc] + __bfloat162float(bias[oc]) - mx));
    }
    double gz = 0., gl = 0.;
    if (gw > 0.f) {
        for (int i = threadIdx.x; i < KO; i += blockDim.x)
            if (!skip[i]) {
                const float q = geo_q(eul_c, O, gb, gc, i, inv2s2);
                gz += q;
                gl += q * (lse - (double)(row[i] + __bfloat162float(bias[i]) - mx));
            }
        gz = bsum(gz, redd);
        gl = bsum(gl, redd);
        if (gz > 0.) lq += gw * gl / gz;
    }
    lq = bsum(lq, redd);
    if (threadIdx.x == 0) atomicAdd(loss, lq);
    __syncthreads();
    const float inv = 1.f / nb;
    const float gs = (gw > 0.f && gz > 0.) ? (float)(gw / gz) : 0.f;
    for (int i = threadIdx.x; i < KO; i += blockDim.x) {
        float v = skip[i] ? 0.f : (float)exp((double)(row[i] + __bfloat162float(bias[i]) - mx) - lse);
        if (gs > 0.f && !skip[i]) v -= gs * geo_q(eul_c, O, gb, gc, i, inv2s2);
        row[i] = v * inv;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < NET_NTGT; j += blockDim.x) {
        const int oc = tgt_oc[(size_t)b * NET_NTGT + j];
        const float q = tgt_w[(size_t)b * NET_NTGT + j];
        if (oc >= 0 && q > 0.f && !skip[oc]) atomicAdd(&row[oc], -q * inv);
    }
}

// d (rows x cols) *= (h > 0) when relu; db[c] += sum_r d[r][c]
__global__ void k_relu_back_bias(float* __restrict__ d, const float* __restrict__ h, int rows, int cols, int relu,
                                 float* __restrict__ db)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float acc = 0.f;
    for (int r = 0; r < rows; r++) {
        float v = d[(size_t)r * cols + c];
        if (relu && !(h[(size_t)r * cols + c] > 0.f)) { v = 0.f; d[(size_t)r * cols + c] = 0.f; }
        acc += v;
    }
    db[c] += acc;
}

// conv2 / conv1 backward of one particle per CTA: dx0 (2048, before the
// ReLU mask) -> conv weight and bias gradients (atomics into g)
__global__ void __launch_bounds__(256) k_conv_bwd(const float* __restrict__ img, const float* __restrict__ a1g,
                                                  const float* __restrict__ x0, const float* __restrict__ dx0,
                                                  const bf16* __restrict__ th, NetLayout L, float* __restrict__ g)
{
    __shared__ float im[18][18];
    __shared__ float a1[NET_C1][18][18];
    __shared__ float d2[NET_H0];
    __shared__ float da1[NET_C1][16][16];
    const int b = blockIdx.x;
    for (int i = threadIdx.x; i < 18 * 18; i += blockDim.x) (&im[0][0])[i] = 0.f;
    for (int i = threadIdx.x; i < NET_C1 * 18 * 18; i += blockDim.x) (&a1[0][0][0])[i] = 0.f;
    __syncthreads();
    {
        const int y = threadIdx.x >> 4, x = threadIdx.x & 15;
        im[y + 1][x + 1] = img[(size_t)b * NET_NPIX + threadIdx.x];
        for (int c = 0; c < NET_C1; c++) a1[c][y + 1][x + 1] = a1g[(size_t)b * NET_C1 * NET_NPIX + c * NET_NPIX + threadIdx.x];
    }
    for (int o = threadIdx.x; o < NET_H0; o += blockDim.x)
        d2[o] = x0[(size_t)b * NET_H0 + o] > 0.f ? dx0[(size_t)b * NET_H0 + o] : 0.f;
    __syncthreads();
    // conv2 weights: dW[c2][c1][dy][dx] = sum_{Y,X} d2[c2][Y][X] a1[c1][2Y+dy][2X+dx] (padded coordinates)
    for (int wi = threadIdx.x; wi < NET_C2 * NET_C1 * 9; wi += blockDim.x) {
        const int c2 = wi / (NET_C1 * 9), r = wi - c2 * NET_C1 * 9, c1 = r / 9, dy = (r % 9) / 3, dx = r % 3;
        float acc = 0.f;
        for (int Y = 0; Y < 8; Y++)
            for (int X = 0; X < 8; X++) acc += d2[c2 * 64 + Y * 8 + X] * a1[c1][2 * Y + dy][2 * X + dx];
        atomicAdd(&g[L.wc2 + wi], acc);
    }
    if (threadIdx.x < NET_C2) {
        float acc = 0.f;
        for (int q = 0; q < 64; q++) acc += d2[threadIdx.x * 64 + q];
        atomicAdd(&g[L.bc2 + threadIdx.x], acc);
    }
    // da1[c1][y][x]: every conv2 output reading padded position (y+1, x+1), masked by a1 > 0
    {
        const int y = threadIdx.x >> 4, x = threadIdx.x & 15;
        for (int c1 = 0; c1 < NET_C1; c1++) {
            float acc = 0.f;
            for (int dy = 0; dy < 3; dy++) {
                const int yy = y + 1 - dy;
                if (yy < 0 || (yy & 1)) continue;
                const int Y = yy >> 1;
                if (Y >= 8) continue;
                for (int dx = 0; dx < 3; dx++) {
                    const int xx = x + 1 - dx;
                    if (xx < 0 || (xx & 1)) continue;
                    const int X = xx >> 1;
                    if (X >= 8) continue;
                    for (int c2 = 0; c2 < NET_C2; c2++)
                        acc += d2[c2 * 64 + Y * 8 + X] * ldw(th, L.wc2 + ((size_t)c2 * NET_C1 + c1) * 9 + dy * 3 + dx);
                }
            }
            da1[c1][y][x] = a1[c1][y + 1][x + 1] > 0.f ? acc : 0.f;
        }
    }
    __syncthreads();
    // conv1 weights and bias
    for (int wi = threadIdx.x; wi < NET_C1 * 9; wi += blockDim.x) {
        const int c1 = wi / 9, dy = (wi % 9) / 3, dx = wi % 3;
        float acc = 0.f;
        for (int y = 0; y < 16; y++)
            for (int x = 0; x < 16; x++) acc += da1[c1][y][x] * im[y + dy][x + dx];
        atomicAdd(&g[L.wc1 + wi], acc);
    }
    if (threadIdx.x < NET_C1) {
        float acc = 0.f;
        for (int q = 0; q < 256; q++) acc += (&da1[threadIdx.x][0][0])[q];
        atomicAdd(&g[L.bc1 + threadIdx.x], acc);
    }
}

// Adam (bias-corrected), then the BF16 copy every forward pass reads
__global__ void k_adam(float* __restrict__ th, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       bf16* __restrict__ thb, size_t n, float lr, float c1, float c2)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = 0.9f * m[i] + 0.1f * gi;
        const float vi = 0.999f * v[i] + 0.001f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float t = th[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
        th[i] = t;
        thb[i] = __float2bfloat16_rn(t);
    }
}

__global__ void k_to_bf16(const float* __restrict__ x, bf16* __restrict__ y, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(x[i]);
}

// training batch: images and targets of the sampled indices.  Target: 1/2
// geometric (true pose) + 1/2 plain-E-step posterior where the particle has
// one, the geometric target alone otherwise.
__global__ void k_batch_gather(const int* __restrict__ idx, int nb, const float* __restrict__ imgs,
                               const float* __restrict__ poses, const int* __restrict__ pcls,
                               const int* __restrict__ post_oc, const float* __restrict__ post_w,
                               float* __restrict__ bimg, float* __restrict__ geo, int* __restrict__ gcls,
                               int* __restrict__ tgt_oc, float* __restrict__ tgt_w)
{
    const int r = blockIdx.x;
    if (r >= nb) return;
    const int i = idx[r];
    for (int p = threadIdx.x; p < NET_NPIX; p += blockDim.x) bimg[(size_t)r * NET_NPIX + p] = imgs[(size_t)i * NET_NPIX + p];
    if (threadIdx.x == 0) {
        float ps = 0.f;
        for (int j = 0; j < NET_NPOST; j++) ps += post_oc[(size_t)i * NET_NPOST + j] >= 0 ? post_w[(size_t)i * NET_NPOST + j] : 0.f;
        const float a = ps > 0.f ? 0.5f : 1.f;
        for (int j = 0; j < 9; j++) geo[(size_t)r * 10 + j] = poses[(size_t)i * 9 + j];
        geo[(size_t)r * 10 + 9] = a;
        gcls[r] = pcls[i];
        tgt_oc[(size_t)r * NET_NTGT] = -1;
        tgt_w[(size_t)r * NET_NTGT] = 0.f;
        for (int j = 0; j < NET_NPOST; j++) {
            const int oc = post_oc[(size_t)i * NET_NPOST + j];
            const float wv = (ps > 0.f && oc >= 0) ? (1.f - a) * post_w[(size_t)i * NET_NPOST + j] / ps : 0.f;
            tgt_oc[(size_t)r * NET_NTGT + 1 + j] = oc;
            tgt_w[(size_t)r * NET_NTGT + 1 + j] = wv;
        }
    }
}

// pose (double, 9) -> float training store
__global__ void k_pose_store(const double* __restrict__ pose, const int* __restrict__ cls, int n, float* __restrict__ out,
                             int* __restrict__ out_cls)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * 9) return;
    out[i] = (float)pose[i];
    if (i % 9 == 0) out_cls[i / 9] = cls[i / 9];
}

// fc3 rows of the matched-filter initialisation: W3[oc][2p] = alpha T_oc[p] / 16,
// W3[oc][2p+1] = -alpha T_oc[p] / 16 (T_oc the template feature image, RMS 1),
// every other input of the row 0; b3 = 0
__global__ void k_init_w3(const float* __restrict__ tmpl, int KO, float alpha, float* __restrict__ w3,
                          float* __restrict__ b3)
{
    const size_t total = (size_t)KO * NET_H2;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t oc = i / NET_H2;
        const int c = (int)(i - oc * NET_H2);
        float v = 0.f;
        if (c < 2 * NET_NPIX) {
            const float t = alpha * tmpl[oc * NET_NPIX + (c >> 1)] / 16.f;
            v = (c & 1) ? -t : t;
        }
        w3[i] = v;
        if (c == 0) b3[oc] = 0.f;
    }
}

}  // namespace

// ===================================================================== host
NetLayout net_layout(int KO)
{
    NetLayout L{};
    auto al = [](size_t x) { return (x + 63) / 64 * 64; };
    size_t o = 0;
    L.wc1 = o; o = al(o + NET_C1 * 9);
    L.bc1 = o; o = al(o + NET_C1);
    L.wc2 = o; o = al(o + (size_t)NET_C2 * NET_C1 * 9);
    L.bc2 = o; o = al(o + NET_C2);
    L.b1 = o; o = al(o + NET_H1);
    L.b2 = o; o = al(o + NET_H2);
    L.b3 = o; o = al(o + (size_t)KO);
    L.w1 = o; o = al(o + (size_t)NET_H1 * NET_H0);
    L.w2 = o; o = al(o + (size_t)NET_H2 * NET_H1);
    L.w3 = o; o += (size_t)KO * NET_H2;
    L.total = o;
    L.KO = KO;
    L.KOpad = (KO + 127) / 128 * 128;
    L.alloc = L.w3 + (size_t)L.KOpad * NET_H2;
    return L;
}

namespace {

int gridsz(size_t n, int threads = 256)
{
    return (int)std::max<size_t>(1, std::min<size_t>((n + threads - 1) / threads, 148 * 16));
}

void* net_dalloc(std::vector<void*>& owner, size_t bytes)
{
    void* p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) {
        cudaGetLastError();
        throw Error{T2B_ERR_NOMEM, "proposal network: cudaMalloc of " + std::to_string(bytes) + " bytes failed"};
    }
    owner.push_back(p);
    return p;
}

void free_list(std::vector<void*>& v)
{
    for (void* p : v) cudaFree(p);
    v.clear();
}

// Initial parameters: small uniform noise everywhere (PyTorch's default bound
// 1/sqrt(fan_in), times 0.01), overwritten by an identity path that carries
// +x and -x of every feature pixel through both ReLU convolutions and both
// ReLU dense layers:
//   conv1 channels 0/1: +x, -x (centre tap)
//   conv2 channels 2q+s: sign s of the sub-pixel q = 2(y%2) + (x%2) of each
//         2x2 block (taps (1,1), (1,2), (2,1), (2,2) of the stride-2 kernel)
//   fc1, fc2 rows 2p / 2p+1: relu(+v_p), relu(-v_p) of pixel p
// so that with fc3 rows alpha (T_oc, -T_oc) / 16 (k_init_w3) the network starts
// as the matched filter of the feature image against the templates T_oc.
void init_params_host(const NetLayout& L, unsigned long long seed, std::vector<float>& h)
{
    h.assign(L.alloc, 0.f);
    std::mt19937_64 rng(seed ^ 0x5eed5eedull);
    auto fill = [&](size_t off, size_t cnt, int fan_in) {
        const float bnd = 0.01f / std::sqrt((float)fan_in);
        std::uniform_real_distribution<float> u(-bnd, bnd);
        for (size_t i = 0; i < cnt; i++) h[off + i] = u(rng);
    };
    fill(L.wc1, NET_C1 * 9, 9);
    fill(L.bc1, NET_C1, 9);
    fill(L.wc2, (size_t)NET_C2 * NET_C1 * 9, NET_C1 * 9);
    fill(L.bc2, NET_C2, NET_C1 * 9);
    fill(L.w1, (size_t)NET_H1 * NET_H0, NET_H0);
    fill(L.b1, NET_H1, NET_H0);
    fill(L.w2, (size_t)NET_H2 * NET_H1, NET_H1);
    fill(L.b2, NET_H2, NET_H1);
    for (int c = 0; c < 2; c++) {
        for (int t = 0; t < 9; t++) h[L.wc1 + c * 9 + t] = 0.f;
        h[L.wc1 + c * 9 + 4] = c == 0 ? 1.f : -1.f;
        h[L.bc1 + c] = 0.f;
    }
    const int taps[4][2] = {{1, 1}, {1, 2}, {2, 1}, {2, 2}};
    for (int q = 0; q < 4; q++)
        for (int sg = 0; sg < 2; sg++) {
            const int ch = 2 * q + sg;
            for (int t = 0; t < NET_C1 * 9; t++) h[L.wc2 + (size_t)ch * NET_C1 * 9 + t] = 0.f;
            h[L.wc2 + (size_t)ch * NET_C1 * 9 + sg * 9 + taps[q][0] * 3 + taps[q][1]] = 1.f;
            h[L.bc2 + ch] = 0.f;
        }
    auto x0_index = [](int y, int x, int sg) {
        const int q = 2 * (y & 1) + (x & 1);
        return (2 * q + sg) * 64 + (y >> 1) * 8 + (x >> 1);
    };
    for (int r = 0; r < 2 * NET_NPIX; r++) {
        for (int i = 0; i < NET_H0; i++) h[L.w1 + (size_t)r * NET_H0 + i] = 0.f;
        for (int i = 0; i < NET_H1; i++) h[L.w2 + (size_t)r * NET_H1 + i] = 0.f;
        h[L.b1 + r] = 0.f;
        h[L.b2 + r] = 0.f;
    }
    for (int p = 0; p < NET_NPIX; p++) {
        const int y = p >> 4, x = p & 15;
        const int ip = x0_index(y, x, 0), im = x0_index(y, x, 1);
        h[L.w1 + (size_t)(2 * p) * NET_H0 + ip] = 1.f;
        h[L.w1 + (size_t)(2 * p) * NET_H0 + im] = -1.f;
        h[L.w1 + (size_t)(2 * p + 1) * NET_H0 + ip] = -1.f;
        h[L.w1 + (size_t)(2 * p + 1) * NET_H0 + im] = 1.f;
        h[L.w2 + (size_t)(2 * p) * NET_H1 + 2 * p] = 1.f;
        h[L.w2 + (size_t)(2 * p) * NET_H1 + 2 * p + 1] = -1.f;
        h[L.w2 + (size_t)(2 * p + 1) * NET_H1 + 2 * p] = -1.f;
        h[L.w2 + (size_t)(2 * p + 1) * NET_H1 + 2 * p + 1] = 1.f;
    }
}

ProposalNet& net_params(t2b_ctx* c, int KO)
{
    if (!c->net) c->net = new ProposalNet();
    ProposalNet& N = *c->net;
    if (N.th && N.KO == KO) return N;
    free_list(N.ws);
    N.ready = false;
    N.enabled = false;
    free_list(N.owned);
    N.L = net_layout(KO);
    N.KO = KO;
    const size_t n = N.L.alloc;
    N.th = (float*)net_dalloc(N.owned, n * sizeof(float));
    N.g = (float*)net_dalloc(N.owned, n * sizeof(float));
    N.m = (float*)net_dalloc(N.owned, n * sizeof(float));
    N.v = (float*)net_dalloc(N.owned, n * sizeof(float));
    N.thb = net_dalloc(N.owned, n * sizeof(bf16));
    std::vector<float> h;
    init_params_host(N.L, 1, h);
    T2B_CUDA(cudaMemcpy(N.th, h.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    T2B_CUDA(cudaMemset(N.g, 0, n * sizeof(float)));
    T2B_CUDA(cudaMemset(N.m, 0, n * sizeof(float)));
    T2B_CUDA(cudaMemset(N.v, 0, n * sizeof(float)));
    k_to_bf16<<<gridsz(n), 256>>>(N.th, (bf16*)N.thb, n);
    T2B_CUDA(cudaDeviceSynchronize());
    N.adam_t = 0;
    N.trained = false;
    return N;
}

// workspace of the inference path and of the audit (na_max audited particles per batch)
void net_setup(t2b_ctx* c, int na_max)
{
    ProposalNet& N = *c->net;
    if (N.ready && N.na_max >= na_max) return;
    free_list(N.ws);
    N.ready = false;
    const Tables& tb = c->tb;
    const TcOperands& op = c->tc;
    const int B = c->cfg.max_batch, KO = tb.K * tb.O, P = tb.P, s = tb.s, xh = tb.xh;
    T2B_REQUIRE(KO <= NET_MAX_KO, T2B_ERR_UNSUPPORTED, "learned proposals need nr_classes*n_dir*n_psi <= 49152");
    T2B_REQUIRE(c->cfg.diff2_mode == T2B_DIFF2_SPLIT_BF16, T2B_ERR_UNSUPPORTED,
                "learned proposals run with diff2_mode T2B_DIFF2_SPLIT_BF16");
    T2B_REQUIRE(tb.T <= 256, T2B_ERR_UNSUPPORTED, "learned proposals need n_trans <= 256");
    auto& W = N.ws;
    // ring pixels of the window
    const int R = std::min(NET_RING, s / 2);
    std::vector<int> ring, rk;
    for (int n = 0; n < P; n++) {
        const int i = n / xh, x = n - i * xh, y = (i < xh) ? i : i - s;
        if (x * x + y * y <= R * R) {
            ring.push_back(n);
            rk.push_back(x);
            rk.push_back(y);
        }
    }
    T2B_REQUIRE((int)ring.size() <= NET_MAX_RING, T2B_ERR_STATE, "ring table");
    N.nring = (int)ring.size();
    N.ring = (int*)net_dalloc(W, ring.size() * sizeof(int));
    N.ring_k = (int*)net_dalloc(W, rk.size() * sizeof(int));
    T2B_CUDA(cudaMemcpy(N.ring, ring.data(), ring.size() * sizeof(int), cudaMemcpyHostToDevice));
    T2B_CUDA(cudaMemcpy(N.ring_k, rk.data(), rk.size() * sizeof(int), cudaMemcpyHostToDevice));
    N.b_pad = (B + 255) / 256 * 256;
    N.img = (float*)net_dalloc(W, (size_t)std::max(B, 1024) * NET_NPIX * sizeof(float));
    N.x0b = net_dalloc(W, (size_t)N.b_pad * NET_H0 * sizeof(bf16));
    N.h1b = net_dalloc(W, (size_t)N.b_pad * NET_H1 * sizeof(bf16));
    N.h2b = net_dalloc(W, (size_t)N.b_pad * NET_H2 * sizeof(bf16));
    T2B_CUDA(cudaMemset(N.x0b, 0, (size_t)N.b_pad * NET_H0 * sizeof(bf16)));
    T2B_CUDA(cudaMemset(N.h1b, 0, (size_t)N.b_pad * NET_H1 * sizeof(bf16)));
    T2B_CUDA(cudaMemset(N.h2b, 0, (size_t)N.b_pad * NET_H2 * sizeof(bf16)));
    N.y1 = (float*)net_dalloc(W, (size_t)NET_KSPLIT * B * NET_H1 * sizeof(float));   // split-K partials
    N.y2 = (float*)net_dalloc(W, (size_t)NET_KSPLIT * B * NET_H2 * sizeof(float));
    N.logits = (float*)net_dalloc(W, (size_t)B * KO * sizeof(float));
    N.prop = (int*)net_dalloc(W, (size_t)B * 128 * sizeof(int));
    T2B_CUDA(cudaMemset(N.prop, 0, (size_t)B * 128 * sizeof(int)));
    N.cand1 = (int*)net_dalloc(W, (size_t)B * NET_TOPK_CAND * sizeof(int));
    N.score1 = (float*)net_dalloc(W, (size_t)B * NET_TOPK_CAND * sizeof(float));
    // low-resolution rescoring operands (K = 2 x ring pixels, padded to a multiple of 64)
    N.kr = (2 * N.nring + 63) / 64 * 64;
    T2B_REQUIRE(N.kr / 2 <= RING_MAX, T2B_ERR_UNSUPPORTED, "too many low-resolution ring pixels");
    N.projR = (float2*)net_dalloc(W, (size_t)KO * N.nring * sizeof(float2));
    N.rth = net_dalloc(W, (size_t)KO * N.kr * sizeof(bf16));
    N.rtl = net_dalloc(W, (size_t)KO * N.kr * sizeof(bf16));
    k_ring_table<<<gridsz((size_t)KO * N.kr / 2), 256>>>(tb.proj_c, P, N.ring, N.nring, KO, N.kr, N.projR, (bf16*)N.rth,
                                                         (bf16*)N.rtl);
    N.w2r = (float*)net_dalloc(W, (size_t)B * N.nring * sizeof(float));
    const size_t ra_rows = (size_t)B * NET_MAX_K1, rb_rows = ((size_t)B * tb.T + RS_TMAX + 255) / 256 * 256;
    N.rah = net_dalloc(W, ra_rows * N.kr * sizeof(bf16));
    N.ral = net_dalloc(W, ra_rows * N.kr * sizeof(bf16));
    N.rbh = net_dalloc(W, rb_rows * N.kr * sizeof(bf16));
    N.rbl = net_dalloc(W, rb_rows * N.kr * sizeof(bf16));
    T2B_CUDA(cudaMemset(N.rbh, 0, rb_rows * N.kr * sizeof(bf16)));
    T2B_CUDA(cudaMemset(N.rbl, 0, rb_rows * N.kr * sizeof(bf16)));
    N.rnorm = (float*)net_dalloc(W, ra_rows * sizeof(float));
    const int rs = tc_slot_rescore();
    tc_set_map_box(c->tc, rs, N.rah, (int)ra_rows, N.kr, 128);
    tc_set_map_box(c->tc, rs + 1, N.ral, (int)ra_rows, N.kr, 128);
    tc_set_map_box(c->tc, rs + 2, N.rbh, (int)rb_rows, N.kr, RS_TMAX);
    tc_set_map_box(c->tc, rs + 3, N.rbl, (int)rb_rows, N.kr, RS_TMAX);
    // tensor maps of the dense layers: W1, X0b, W2, H1b, W3, H2b, then the three activations
    // again with a 128-row box (batches of <= 128 particles: 128-column tiles)
    unsigned char blobs[9][128];
    const bf16* thb = (const bf16*)N.thb;
    tc_encode((void*)(thb + N.L.w1), NET_H1, NET_H0, true, blobs[0]);
    tc_encode(N.x0b, N.b_pad, NET_H0, false, blobs[1]);
    tc_encode((void*)(thb + N.L.w2), NET_H2, NET_H1, true, blobs[2]);
    tc_encode(N.h1b, N.b_pad, NET_H1, false, blobs[3]);
    tc_encode((void*)(thb + N.L.w3), N.L.KOpad, NET_H2, true, blobs[4]);
    tc_encode(N.h2b, N.b_pad, NET_H2, false, blobs[5]);
    tc_encode(N.x0b, N.b_pad, NET_H0, false, blobs[6], 128);
    tc_encode(N.h1b, N.b_pad, NET_H1, false, blobs[7], 128);
    tc_encode(N.h2b, N.b_pad, NET_H2, false, blobs[8], 128);
    N.maps = net_dalloc(W, sizeof(blobs));
    T2B_CUDA(cudaMemcpy(N.maps, blobs, sizeof(blobs), cudaMemcpyHostToDevice));
    // restricted coarse pass operands: up to 128 proposal rows per particle
    const size_t pg_rows = (size_t)B * 128;
    N.pg_h = net_dalloc(W, pg_rows * op.kdim * sizeof(bf16));
    N.pg_l = net_dalloc(W, pg_rows * op.kdim * sizeof(bf16));
    T2B_CUDA(cudaMemset(N.pg_h, 0, pg_rows * op.kdim * sizeof(bf16)));
    T2B_CUDA(cudaMemset(N.pg_l, 0, pg_rows * op.kdim * sizeof(bf16)));
    N.nprop = (float*)net_dalloc(W, (size_t)B * 128 * sizeof(float));
    N.pg_rows = (int)pg_rows;   // pre-swizzled K-blocked (swz_offset), read by bulk copies
    // the B operand of the proposal tiles: the phase rows, zero beyond T
    const int ab_rows = (tb.T + 31) / 32 * 32;
    N.ab_h = net_dalloc(W, (size_t)ab_rows * op.kdim * sizeof(bf16));
    N.ab_l = net_dalloc(W, (size_t)ab_rows * op.kdim * sizeof(bf16));
    tc_split_phases(tb, op, ab_rows, N.ab_h, N.ab_l, 0);   // pre-swizzled K-blocked, read by bulk copies
    // split-K exchange buffers of the proposal tiles: up to half the SMs' worth of m-tiles
    int nsm = 0;
    T2B_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    N.part_tiles = std::max(1, nsm / 2);
    N.part = (float*)net_dalloc(W, (size_t)N.part_tiles * 2 * 4 * (ab_rows / 32) * 1024 * sizeof(float));
    N.fix = (int*)net_dalloc(W, (size_t)N.part_tiles * 4 * sizeof(int));
    // audit
    N.na_max = std::max(1, std::min(B, na_max));
    const int ia_rows = (N.na_max * tb.T + 255) / 256 * 256;
    N.ps = (PropState*)net_dalloc(W, sizeof(PropState));
    T2B_CUDA(cudaMemset(N.ps, 0, sizeof(PropState)));
    N.audit_b = (int*)net_dalloc(W, (size_t)N.na_max * sizeof(int));
    N.ia_h = net_dalloc(W, (size_t)ia_rows * op.kdim * sizeof(bf16));
    N.ia_l = net_dalloc(W, (size_t)ia_rows * op.kdim * sizeof(bf16));
    T2B_CUDA(cudaMemset(N.ia_h, 0, (size_t)ia_rows * op.kdim * sizeof(bf16)));
    T2B_CUDA(cudaMemset(N.ia_l, 0, (size_t)ia_rows * op.kdim * sizeof(bf16)));
    const int tn_f = tc_audit_tn(N.na_max, tb.T);
    tc_set_map_box(c->tc, tc_slot_audit(), N.ia_h, ia_rows, op.kdim, tn_f);
    tc_set_map_box(c->tc, tc_slot_audit() + 1, N.ia_l, ia_rows, op.kdim, tn_f);
    if (const int tn_n = tc_audit_narrow_tn(N.na_max, tb.T)) {
        tc_set_map_box(c->tc, tc_slot_audit_narrow(), N.ia_h, ia_rows, op.kdim, tn_n);
        tc_set_map_box(c->tc, tc_slot_audit_narrow() + 1, N.ia_l, ia_rows, op.kdim, tn_n);
    }
    const int wa_rows = (N.na_max + 31) / 32 * 32;
    N.wa_h = net_dalloc(W, (size_t)wa_rows * op.kn * sizeof(bf16));
    N.wa_l = net_dalloc(W, (size_t)wa_rows * op.kn * sizeof(bf16));
    T2B_CUDA(cudaMemset(N.wa_h, 0, (size_t)wa_rows * op.kn * sizeof(bf16)));
    T2B_CUDA(cudaMemset(N.wa_l, 0, (size_t)wa_rows * op.kn * sizeof(bf16)));
    tc_set_map_box(c->tc, tc_slot_audit_w2(), N.wa_h, wa_rows, op.kn, 32);
    tc_set_map_box(c->tc, tc_slot_audit_w2() + 1, N.wa_l, wa_rows, op.kn, 32);
    N.c0a = (float*)net_dalloc(W, (size_t)N.na_max * sizeof(float));
    N.norma = (float*)net_dalloc(W, (size_t)N.na_max * KO * sizeof(float));
    N.d2a = (float*)net_dalloc(W, (size_t)N.na_max * KO * tb.T * sizeof(float));
    N.minkeya = (unsigned*)net_dalloc(W, (size_t)N.na_max * sizeof(unsigned));
    N.asum = (double*)net_dalloc(W, (size_t)N.na_max * 2 * sizeof(double));
    T2B_CUDA(cudaMemset(N.c0a, 0, (size_t)N.na_max * sizeof(float)));
    T2B_CUDA(cudaMemset(N.norma, 0, (size_t)N.na_max * KO * sizeof(float)));
    T2B_CUDA(cudaFuncSetAttribute(k_topk, cudaFuncAttributeMaxDynamicSharedMemorySize, KO * (int)sizeof(unsigned)));
    T2B_CUDA(cudaDeviceSynchronize());
    N.ready = true;
}

// Proposal tiles: 128 rows of (particle, proposal), 64 rows per particle when
// k <= 64 (two particles per tile), else 128, against the T phase rows padded to a
// multiple of 32 columns.
void set_tile_shape(ProposalNet& N, int T)
{
    N.kslot = N.kprop <= 64 ? 64 : 128;
    N.tn = (T + 31) / 32 * 32;
}

// dense layers of the inference path: x0b (n rows) -> logits (n x KO, no bias)
// fc1 and fc2 have only 8 output tiles of 128 features: K is split into NET_KSPLIT
// slices (128 CTAs), the partial products summed in a fixed order with the bias;
// batches of <= 128 particles use 128-column tiles
void infer_dense(ProposalNet& N, int n, int* err, cudaStream_t st)
{
    const bf16* thb = (const bf16*)N.thb;
    const bool narrow = n <= 128;
    const int tn = narrow ? 128 : 256;
    const int s1 = tc_gemm_raw(N.maps, 0, narrow ? 6 : 1, NET_H1, n, NET_H0, N.y1, 1, err, st, NET_KSPLIT, tn);
    k_bias_act<<<gridsz((size_t)n * NET_H1), 256, 0, st>>>(N.y1, thb + N.L.b1, n, NET_H1, 1, nullptr, (bf16*)N.h1b, s1);
    const int s2 = tc_gemm_raw(N.maps, 2, narrow ? 7 : 3, NET_H2, n, NET_H1, N.y2, 1, err, st, NET_KSPLIT, tn);
    k_bias_act<<<gridsz((size_t)n * NET_H2), 256, 0, st>>>(N.y2, thb + N.L.b2, n, NET_H2, 1, nullptr, (bf16*)N.h2b, s2);
    tc_gemm_raw(N.maps, 4, narrow ? 8 : 5, N.KO, n, NET_H2, N.logits, 1, err, st, 1, tn);
    T2B_CUDA(cudaGetLastError());
}

template <bool AT, bool BT, typename TA, typename TB>
void sgemm(int M, int N, int K, const TA* A, int lda, const TB* B, int ldb, float* C, int ldc, int splitk,
           cudaStream_t st)
{
    const int kchunk = ((K + splitk - 1) / splitk + 15) / 16 * 16;
    const int z = (K + kchunk - 1) / kchunk;
    if (z > 1) T2B_CUDA(cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * ldc, st));
    dim3 grid((N + 63) / 64, (M + 63) / 64, z);
    k_sgemm<AT, BT, TA, TB><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, kchunk);
    T2B_CUDA(cudaGetLastError());
}

// buffers of one training minibatch of nb particles
struct TrainBufs {
    std::vector<void*> mem;
    int nb = 0;
    float *bimg, *a1, *x0, *h1, *h2, *y, *dh2, *dh1, *dx0, *tgt_w, *geo;
    int *tgt_oc, *gcls;
    double* loss;
    TrainBufs(int nb_, int KO) : nb(nb_)
    {
        auto f = [&](size_t n) { return (float*)net_dalloc(mem, n * sizeof(float)); };
        bimg = f((size_t)nb * NET_NPIX);
        a1 = f((size_t)nb * NET_C1 * NET_NPIX);
        x0 = f((size_t)nb * NET_H0);
        h1 = f((size_t)nb * NET_H1);
        h2 = f((size_t)nb * NET_H2);
        y = f((size_t)nb * KO);
        dh2 = f((size_t)nb * NET_H2);
        dh1 = f((size_t)nb * NET_H1);
        dx0 = f((size_t)nb * NET_H0);
        tgt_w = f((size_t)nb * NET_NTGT);
        geo = f((size_t)nb * 10);
        tgt_oc = (int*)net_dalloc(mem, (size_t)nb * NET_NTGT * sizeof(int));
        gcls = (int*)net_dalloc(mem, (size_t)nb * sizeof(int));
        loss = (double*)net_dalloc(mem, sizeof(double));
    }
    ~TrainBufs() { free_list(mem); }
};

// forward + backward of one minibatch (bimg and targets filled): gradient in
// N.g, summed loss added to *t.loss; use_geo: the rows' geometric targets count
float inv2s2_of(double sigma_deg)
{
    const double s = sigma_deg * PI / 180.;
    return (float)(1. / (2. * s * s));
}

void train_fwd_bwd(ProposalNet& N, TrainBufs& t, const Tables& tb, bool use_geo, float inv2s2, cudaStream_t st)
{
    const NetLayout& L = N.L;
    const int nb = t.nb, KO = N.KO;
    const bf16* thb = (const bf16*)N.thb;
    float* g = N.g;
    k_conv_fwd<<<nb, 256, 0, st>>>(t.bimg, thb, L, nb, t.a1, t.x0, nullptr);
    sgemm<false, true>(nb, NET_H1, NET_H0, t.x0, NET_H0, thb + L.w1, NET_H0, t.h1, NET_H1, 1, st);
    k_bias_act<<<gridsz((size_t)nb * NET_H1), 256, 0, st>>>(t.h1, thb + L.b1, nb, NET_H1, 1, t.h1, nullptr);
    sgemm<false, true>(nb, NET_H2, NET_H1, t.h1, NET_H1, thb + L.w2, NET_H1, t.h2, NET_H2, 1, st);
    k_bias_act<<<gridsz((size_t)nb * NET_H2), 256, 0, st>>>(t.h2, thb + L.b2, nb, NET_H2, 1, t.h2, nullptr);
    sgemm<false, true>(nb, KO, NET_H2, t.h2, NET_H2, thb + L.w3, NET_H2, t.y, KO, 1, st);
    k_softmax_ce<<<nb, 1024, 0, st>>>(t.y, thb + L.b3, tb.skip, KO, t.tgt_oc, t.tgt_w, use_geo ? t.geo : nullptr,
                                      t.gcls, tb.eul_c, tb.O, inv2s2, nb, t.loss);
    // backward: t.y now holds dL/dlogits
    T2B_CUDA(cudaMemsetAsync(g, 0, L.alloc * sizeof(float), st));
    k_relu_back_bias<<<(KO + 255) / 256, 256, 0, st>>>(t.y, nullptr, nb, KO, 0, g + L.b3);
    sgemm<true, false>(KO, NET_H2, nb, t.y, KO, t.h2, NET_H2, g + L.w3, NET_H2, 1, st);
    sgemm<false, false>(nb, NET_H2, KO, t.y, KO, thb + L.w3, NET_H2, t.dh2, NET_H2, 32, st);
    k_relu_back_bias<<<(NET_H2 + 255) / 256, 256, 0, st>>>(t.dh2, t.h2, nb, NET_H2, 1, g + L.b2);
    sgemm<true, false>(NET_H2, NET_H1, nb, t.dh2, NET_H2, t.h1, NET_H1, g + L.w2, NET_H1, 1, st);
    sgemm<false, false>(nb, NET_H1, NET_H2, t.dh2, NET_H2, thb + L.w2, NET_H1, t.dh1, NET_H1, 4, st);
    k_relu_back_bias<<<(NET_H1 + 255) / 256, 256, 0, st>>>(t.dh1, t.h1, nb, NET_H1, 1, g + L.b1);
    sgemm<true, false>(NET_H1, NET_H0, nb, t.dh1, NET_H1, t.x0, NET_H0, g + L.w1, NET_H0, 1, st);
    sgemm<false, false>(nb, NET_H0, NET_H1, t.dh1, NET_H1, thb + L.w1, NET_H0, t.dx0, NET_H0, 4, st);
    k_conv_bwd<<<nb, 256, 0, st>>>(t.bimg, t.a1, t.x0, t.dx0, thb, L, g);
    T2B_CUDA(cudaGetLastError());
}

struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(size_t bytes)
    {
        if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) {
            cudaGetLastError();
            throw Error{T2B_ERR_NOMEM, "proposal training: cudaMalloc of " + std::to_string(bytes) + " bytes failed"};
        }
    }
    ~DevBuf() { cudaFree(p); }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace

// ------------------------------------------------ per-batch entry points
void proposal_infer(t2b_ctx* c, const Work& w, cudaStream_t st)
{
    ProposalNet& N = *c->net;
    const Tables& tb = c->tb;
    k_features<<<w.n, NET_NPIX, 0, st>>>(w.fimg, w.ctf, w.minv, tb.P, N.ring, N.ring_k, N.nring, N.img, nullptr, nullptr);
    k_conv_fwd<<<w.n, 256, 0, st>>>(N.img, (const bf16*)N.thb, N.L, w.n, nullptr, nullptr, (bf16*)N.x0b);
    infer_dense(N, w.n, w.err, st);
    if (N.k1 > 0) {
        // network top-k1, exact low-resolution rescoring, top-kprop of those
        k_topk<<<w.n, 1024, N.KO * sizeof(unsigned), st>>>(N.logits, (const bf16*)N.thb + N.L.b3, tb.skip, N.KO, N.k1,
                                                           N.cand1, 0);
        const long long nc = (long long)w.n * N.k1;
        k_ring_images<<<w.n, 256, 0, st>>>(tb, w, N.ring, N.nring, N.kr, (bf16*)N.rbh, (bf16*)N.rbl, N.w2r);
        k_rescore_gather<<<(int)((nc * 32 + 255) / 256), 256, 0, st>>>(w.n, N.k1, N.nring, N.kr, N.cand1, N.projR,
                                                                       (const bf16*)N.rth, (const bf16*)N.rtl, N.w2r,
                                                                       (bf16*)N.rah, (bf16*)N.ral, N.rnorm);
        T2B_CUDA(cudaGetLastError());
        tc_launch_rescore(w.n, N.k1, tb.T, N.kr, c->tc, N.rnorm, tb.skip, N.cand1, w.pdf_t, tb.pdf_oc, N.score1, w.err,
                          st);
        k_rescore_select<<<w.n, 1024, 0, st>>>(N.cand1, N.score1, N.k1, N.kprop, N.prop);
    } else {
        k_topk<<<w.n, 1024, N.KO * sizeof(unsigned), st>>>(N.logits, (const bf16*)N.thb + N.L.b3, tb.skip, N.KO,
                                                           N.kprop, N.prop, 1);
    }
    T2B_CUDA(cudaGetLastError());
}

void proposal_audit(t2b_ctx* c, const Work& w, cudaStream_t st, cudaEvent_t* ev)
{
    proposal_audit_contract(c, w, st, ev);
    proposal_audit_mass(c, w, st);
}

void proposal_audit_contract(t2b_ctx* c, const Work& w, cudaStream_t st, cudaEvent_t* ev)
{
    ProposalNet& N = *c->net;
    const Tables& tb = c->tb;
    TcOperands& op = c->tc;
    k_audit_begin<<<1, 256, 0, st>>>(N.ps, N.audit_b, w.n, N.every, N.na_max, N.minkeya, N.asum, w.r_audit);
    k_audit_operands<<<dim3(tb.T + 1, N.na_max), 256, 0, st>>>(N.ps, N.audit_b, w, tb.T, tb.P, tb.kpix, tb.nk, op.kn,
                                                               op.kdim, tb.ab_c, (bf16*)N.ia_h,
                                                               (bf16*)N.ia_l, (bf16*)N.wa_h, (bf16*)N.wa_l, N.c0a);
    tc_launch_audit_norms(tb, op, N.na_max, N.norma, w.err, st);
    T2B_CUDA(cudaGetLastError());
    if (ev) cudaEventRecord(ev[0], st);
    tc_launch_audit(tb, op, N.na_max, &N.ps->na, N.c0a, N.norma, N.d2a, N.minkeya, w.err, st);
    if (ev) cudaEventRecord(ev[1], st);
    T2B_CUDA(cudaGetLastError());
}

void proposal_audit_mass(t2b_ctx* c, const Work& w, cudaStream_t st)
{
    ProposalNet& N = *c->net;
    const Tables& tb = c->tb;
    const int KO = tb.K * tb.O;
    k_audit_mass<<<dim3(2 * 148, N.na_max), 256, ((KO + 31) / 32) * sizeof(unsigned), st>>>(tb, w, N.ps, N.audit_b, N.d2a,
                                                                                     N.minkeya, N.asum);
    k_audit_final<<<1, 1024, 0, st>>>(N.ps, N.audit_b, N.asum, N.thr, w.r_audit);
    T2B_CUDA(cudaGetLastError());
}

void proposal_coarse(t2b_ctx* c, const Work& w, cudaStream_t st, cudaEvent_t* ev)
{
    ProposalNet& N = *c->net;
    const Tables& tb = c->tb;
    const TcOperands& op = c->tc;
    k_prop_gather<<<dim3(N.kprop, w.n), 128, 0, st>>>(w, tb.P, tb.kpix, tb.nk, N.kslot, N.pg_rows, op.kdim,
                                                      (const bf16*)op.bh, (const bf16*)op.bl, (bf16*)N.pg_h,
                                                      (bf16*)N.pg_l, N.nprop);
    T2B_CUDA(cudaGetLastError());
    if (ev) cudaEventRecord(ev[0], st);
    tc_launch_prop(tb, w, c->tc, N.kslot, N.tn, N.nprop, N.pg_h, N.pg_l, N.pg_rows, N.ab_h, N.ab_l, N.part, N.fix,
                   N.part_tiles, st);
    if (ev) cudaEventRecord(ev[1], st);
}

void proposal_invalidate(t2b_ctx* c)
{
    if (!c->net) return;
    free_list(c->net->ws);
    c->net->ready = false;
    c->net->enabled = false;
}

void proposal_release(t2b_ctx* c)
{
    if (!c->net) return;
    free_list(c->net->ws);
    free_list(c->net->owned);
    delete c->net;
    c->net = nullptr;
}

}  // namespace t2b

using namespace t2b;

namespace {

void drop_graph(t2b_ctx* c) { c->drop_graphs(); }

long long real_params(int KO)
{
    return (long long)NET_C1 * 9 + NET_C1 + (long long)NET_C2 * NET_C1 * 9 + NET_C2 + (long long)NET_H1 * NET_H0 +
           NET_H1 + (long long)NET_H2 * NET_H1 + NET_H2 + (long long)KO * NET_H2 + KO;
}

// re-initialise the parameters (identity path + noise) and set fc3 from the
// template feature images of every coarse orientation under the mean CTF^2
void init_from_templates(t2b_ctx* c, ProposalNet& N, unsigned long long seed, const float* ctf2, const float* minv,
                         float alpha, cudaStream_t st)
{
    const Tables& tb = c->tb;
    std::vector<float> h;
    init_params_host(N.L, seed, h);
    T2B_CUDA(cudaMemcpyAsync(N.th, h.data(), N.L.alloc * sizeof(float), cudaMemcpyHostToDevice, st));
    DevBuf tmpl((size_t)N.KO * NET_NPIX * sizeof(float));
    for (int k = 0; k < tb.K; k++)
        k_features<<<tb.O, NET_NPIX, 0, st>>>(nullptr, nullptr, minv, tb.P, N.ring, N.ring_k, N.nring,
                                              tmpl.as<float>() + (size_t)k * tb.O * NET_NPIX,
                                              tb.proj_c + (size_t)k * tb.O * tb.P, ctf2);
    k_init_w3<<<gridsz((size_t)N.KO * NET_H2), 256, 0, st>>>(tmpl.as<float>(), N.KO, alpha, N.th + N.L.w3, N.th + N.L.b3);
    T2B_CUDA(cudaMemsetAsync(N.m, 0, N.L.alloc * sizeof(float), st));
    T2B_CUDA(cudaMemsetAsync(N.v, 0, N.L.alloc * sizeof(float), st));
    k_to_bf16<<<gridsz(N.L.alloc), 256, 0, st>>>(N.th, (bf16*)N.thb, N.L.alloc);
    T2B_CUDA(cudaGetLastError());
    T2B_CUDA(cudaStreamSynchronize(st));
    N.adam_t = 0;
}

}  // namespace

extern "C" {

int t2b_proposal_train(t2b_ctx* c, const t2b_proposal_train_config* cfg, t2b_proposal_report* rep)
{
    return guarded([&] {
        T2B_REQUIRE(c && cfg && rep, T2B_ERR_ARG, "null argument");
        T2B_REQUIRE(c->configured, T2B_ERR_STATE, "t2b_configure must be called before t2b_proposal_train");
        T2B_REQUIRE(!c->tb.chunk, T2B_ERR_UNSUPPORTED,
                    "learned proposals need the resident projection tables (this configuration is chunked)");
        const t2b_proposal_train_config& f = *cfg;
        T2B_REQUIRE(f.batch >= 8 && f.batch <= 1024 && f.n_train >= f.batch && f.epochs >= 0 && f.n_val >= 0 &&
                        f.n_posterior >= 0 && f.topk >= 1 && f.topk <= 128 && f.minvsigma2 && f.lr >= 0.f &&
                        f.defocus_max >= f.defocus_min && f.voltage > 0. && f.q0 >= 0. && f.q0 < 1.,
                    T2B_ERR_ARG, "bad proposal training configuration");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        c->quiesce();   // training reallocates buffers that host batches in flight still use
        cudaStream_t st = c->stream;
        drop_graph(c);
        const Tables& tb = c->tb;
        const int KO = tb.K * tb.O, B = c->cfg.max_batch, P = tb.P;
        T2B_REQUIRE(KO <= NET_MAX_KO, T2B_ERR_UNSUPPORTED, "learned proposals need nr_classes*n_dir*n_psi <= 49152");
        ProposalNet& N = net_params(c, KO);
        N.enabled = false;
        N.trained = false;
        N.kprop = f.topk;
        N.k1 = 0;
        set_tile_shape(N, tb.T);
        net_setup(c, std::max(1, N.na_max));
        T2B_REQUIRE(f.rescore == 0 || (f.rescore >= f.topk && f.rescore <= NET_MAX_K1 && f.rescore % 128 == 0 && f.rescore <= KO &&
                                       tb.T <= RS_TMAX),
                    T2B_ERR_ARG, "bad rescore candidate count");
        *rep = t2b_proposal_report{};
        rep->params = real_params(KO);

        DevBuf minv_d((size_t)P * sizeof(float)), ctf2((size_t)P * sizeof(float));
        T2B_CUDA(cudaMemcpy(minv_d.p, f.minvsigma2, (size_t)P * sizeof(float), cudaMemcpyHostToDevice));
        T2B_CUDA(cudaMemset(ctf2.p, 0, (size_t)P * sizeof(float)));
        DevBuf mdl_tab(tb.K * sizeof(float2*)), vol_tab(tb.K * sizeof(Volume));
        T2B_CUDA(cudaMemcpy(mdl_tab.p, c->mdl.data(), tb.K * sizeof(float2*), cudaMemcpyHostToDevice));
        T2B_CUDA(cudaMemcpy(vol_tab.p, c->mvol.data(), tb.K * sizeof(Volume), cudaMemcpyHostToDevice));
        const long long ntr = f.n_train;
        DevBuf imgs((size_t)ntr * NET_NPIX * sizeof(float)), poses((size_t)ntr * 9 * sizeof(float));
        DevBuf pcls((size_t)ntr * sizeof(int));
        DevBuf poc((size_t)ntr * NET_NPOST * sizeof(int)), pw((size_t)ntr * NET_NPOST * sizeof(float));
        T2B_CUDA(cudaMemset(poc.p, 0xff, (size_t)ntr * NET_NPOST * sizeof(int)));
        T2B_CUDA(cudaMemset(pw.p, 0, (size_t)ntr * NET_NPOST * sizeof(float)));
        DevBuf pose((size_t)B * 9 * sizeof(double)), cls((size_t)B * sizeof(int)), marg((size_t)B * KO * sizeof(double));
        DevBuf cap((size_t)2 * B * sizeof(double)), vlab((size_t)B * sizeof(int));
        GenParams gp{f.seed, f.defocus_min, f.defocus_max, f.astig_max, f.voltage, f.cs, f.q0, tb.pixel_size,
                     f.max_shift, minv_d.as<float>()};
        Work wg = c->wk;
        float2* gf = const_cast<float2*>(c->wk.fimg);
        float* gc = const_cast<float*>(c->wk.ctf);
        float* gm = const_cast<float*>(c->wk.minv);
        double* gs = const_cast<double*>(c->wk.scal);
        wg.fimg_nm = wg.fimg;
        wg.no_bp = 1;
        auto gen = [&](long long first, int cnt, unsigned long long seed, float* acc) {
            gp.seed = seed;
            k_gen_particles<<<cnt, 256, 0, st>>>(tb, gp, mdl_tab.as<const float2*>(), vol_tab.as<Volume>(), first, cnt,
                                                 gf, gc, gm, gs, pose.as<double>(), cls.as<int>(), acc);
            T2B_CUDA(cudaGetLastError());
        };
        auto plain_estep = [&](int cnt) {
            Work we = wg;
            we.n = cnt;
            enqueue_estep(c, we, st, false, false);
            k_marginal<<<dim3((KO + 255) / 256, cnt), 256, 0, st>>>(tb, we, marg.as<double>());
            T2B_CUDA(cudaGetLastError());
        };
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        auto elapsed = [&]() {
            float ms = 0.f;
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
            return (double)ms;
        };
        try {
            // 1. training particles: feature images, true poses, mean CTF^2
            cudaEventRecord(e0, st);
            for (long long s0 = 0; s0 < ntr; s0 += B) {
                const int cnt = (int)std::min<long long>(B, ntr - s0);
                gen(s0, cnt, f.seed, ctf2.as<float>());
                k_features<<<cnt, NET_NPIX, 0, st>>>(gf, gc, gm, P, N.ring, N.ring_k, N.nring,
                                                     imgs.as<float>() + s0 * NET_NPIX, nullptr, nullptr);
                k_pose_store<<<(cnt * 9 + 255) / 256, 256, 0, st>>>(pose.as<double>(), cls.as<int>(), cnt,
                                                                    poses.as<float>() + s0 * 9, pcls.as<int>() + s0);
            }
            T2B_CUDA(cudaGetLastError());
            {
                std::vector<float> h(P);
                T2B_CUDA(cudaMemcpyAsync(h.data(), ctf2.p, P * sizeof(float), cudaMemcpyDeviceToHost, st));
                T2B_CUDA(cudaStreamSynchronize(st));
                for (auto& x : h) x /= (float)ntr;
                T2B_CUDA(cudaMemcpy(ctf2.p, h.data(), P * sizeof(float), cudaMemcpyHostToDevice));
            }
            rep->gen_ms = elapsed();
            // 2. plain E-step posteriors of the first n_posterior particles (regenerated)
            cudaEventRecord(e0, st);
            const long long npost = std::min<long long>(f.n_posterior, ntr);
            for (long long s0 = 0; s0 < npost; s0 += B) {
                const int cnt = (int)std::min<long long>(B, npost - s0);
                gen(s0, cnt, f.seed, nullptr);
                plain_estep(cnt);
                k_post_top<<<cnt, 1024, 0, st>>>(marg.as<double>(), KO, poc.as<int>() + s0 * NET_NPOST,
                                                  pw.as<float>() + s0 * NET_NPOST);
            }
            T2B_CUDA(cudaGetLastError());
            rep->label_ms = elapsed();
            // 3. initial network: the matched filter of the references
            init_from_templates(c, N, f.seed, ctf2.as<float>(), minv_d.as<float>(), f.alpha > 0.f ? f.alpha : 3.f, st);
            // held-out particles: posterior mass of the plain E-step inside the top-k
            auto validate = [&](double* mean, double* mn, double* frac, double* hit, double* frac_cand = nullptr) {
                const int nv = f.n_val;
                if (nv <= 0) return;
                double sum = 0., lo = INFINITY;
                long long ok = 0, hits = 0, ok_cand = 0;
                std::vector<double> hcc(B);
                std::vector<double> hc(B);
                std::vector<int> hp((size_t)B * N.kprop), hl(B);
                for (int v0 = 0; v0 < nv; v0 += B) {
                    const int cnt = std::min(B, nv - v0);
                    gen(v0, cnt, f.seed ^ 0x9e3779b97f4a7c15ull, nullptr);
                    plain_estep(cnt);
                    Work wi = wg;
                    wi.n = cnt;
                    proposal_infer(c, wi, st);
                    k_capture<<<cnt, 256, 0, st>>>(marg.as<double>(), KO, N.prop, N.kprop, cap.as<double>());
                    if (frac_cand && N.k1 > 0) {
                        k_capture<<<cnt, 256, 0, st>>>(marg.as<double>(), KO, N.cand1, N.k1, cap.as<double>() + B);
                        T2B_CUDA(cudaMemcpyAsync(hcc.data(), cap.as<double>() + B, cnt * sizeof(double),
                                                 cudaMemcpyDeviceToHost, st));
                    }
                    k_nearest<<<cnt, 256, 0, st>>>(tb, pose.as<double>(), cls.as<int>(), cnt, vlab.as<int>());
                    T2B_CUDA(cudaMemcpyAsync(hc.data(), cap.p, cnt * sizeof(double), cudaMemcpyDeviceToHost, st));
                    T2B_CUDA(cudaMemcpyAsync(hp.data(), N.prop, (size_t)cnt * N.kprop * sizeof(int),
                                             cudaMemcpyDeviceToHost, st));
                    T2B_CUDA(cudaMemcpyAsync(hl.data(), vlab.p, cnt * sizeof(int), cudaMemcpyDeviceToHost, st));
                    T2B_CUDA(cudaStreamSynchronize(st));
                    for (int i = 0; i < cnt; i++) {
                        if (frac_cand && N.k1 > 0) ok_cand += hcc[i] >= 0.999;
                        sum += hc[i];
                        lo = std::min(lo, hc[i]);
                        ok += hc[i] >= 0.999;
                        for (int j = 0; j < N.kprop; j++)
                            if (hp[(size_t)i * N.kprop + j] == hl[i]) { hits++; break; }
                    }
                }
                if (mean) *mean = sum / nv;
                if (mn) *mn = lo;
                if (frac) *frac = (double)ok / nv;
                if (hit) *hit = (double)hits / nv;
                if (frac_cand) *frac_cand = (double)ok_cand / nv;
            };
            validate(&rep->val_mass_init, nullptr, nullptr, nullptr);
            // 4. Adam epochs over shuffled minibatches
            cudaEventRecord(e0, st);
            TrainBufs t(f.batch, KO);
            std::vector<int> perm((size_t)ntr);
            std::iota(perm.begin(), perm.end(), 0);
            std::mt19937_64 rng(f.seed ^ 0x7261696eull);
            DevBuf perm_d((size_t)ntr * sizeof(int));
            const long long nbat = ntr / f.batch;
            const float inv2s2 = inv2s2_of(f.sigma_deg > 0. ? f.sigma_deg : 8.);
            for (int e = 0; e < f.epochs; e++) {
                std::shuffle(perm.begin(), perm.end(), rng);
                T2B_CUDA(cudaMemcpyAsync(perm_d.p, perm.data(), (size_t)ntr * sizeof(int), cudaMemcpyHostToDevice, st));
                T2B_CUDA(cudaMemsetAsync(t.loss, 0, sizeof(double), st));
                for (long long i = 0; i < nbat; i++) {
                    k_batch_gather<<<f.batch, 256, 0, st>>>(perm_d.as<int>() + i * f.batch, f.batch, imgs.as<float>(),
                                                            poses.as<float>(), pcls.as<int>(), poc.as<int>(),
                                                            pw.as<float>(), t.bimg, t.geo, t.gcls, t.tgt_oc, t.tgt_w);
                    train_fwd_bwd(N, t, tb, true, inv2s2, st);
                    N.adam_t++;
                    const float c1 = 1.f - std::pow(0.9f, (float)N.adam_t), c2 = 1.f - std::pow(0.999f, (float)N.adam_t);
                    k_adam<<<gridsz(N.L.alloc), 256, 0, st>>>(N.th, N.g, N.m, N.v, (bf16*)N.thb, N.L.alloc, f.lr, c1, c2);
                }
                double l = 0.;
                T2B_CUDA(cudaMemcpyAsync(&l, t.loss, sizeof(double), cudaMemcpyDeviceToHost, st));
                T2B_CUDA(cudaStreamSynchronize(st));
                if (e < 64) rep->loss[e] = nbat > 0 ? l / ((double)nbat * f.batch) : 0.;
            }
            rep->train_ms = elapsed();
            N.trained = true;
            validate(&rep->val_mass_trained, &rep->val_mass_min, &rep->val_frac_999, &rep->val_true_hit);
            if (f.rescore > 0) {
                N.k1 = f.rescore;
                validate(&rep->val_mass_rescored, &rep->val_mass_min_rescored, &rep->val_frac_999_rescored, nullptr,
                         &rep->val_frac_999_candidates);
                N.k1 = 0;
            }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        T2B_CUDA(cudaStreamSynchronize(st));
    });
}

int t2b_proposal_enable(t2b_ctx* c, int topk, int rescore, int audit_every, double audit_mass)
{
    return guarded([&] {
        T2B_REQUIRE(c, T2B_ERR_ARG, "null context");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        c->quiesce();   // buffers of the network and of slot 0 may be in use by host batches in flight
        drop_graph(c);
        if (topk == 0) {
            if (c->net) c->net->enabled = false;
            return;
        }
        T2B_REQUIRE(c->configured, T2B_ERR_STATE, "t2b_configure must be called before t2b_proposal_enable");
        T2B_REQUIRE(!c->tb.chunk || topk <= 0, T2B_ERR_UNSUPPORTED,
                    "learned proposals need the resident projection tables (this configuration is chunked)");
        const int KO = c->tb.K * c->tb.O;
        T2B_REQUIRE(c->net && c->net->trained && c->net->KO == KO, T2B_ERR_STATE,
                    "no trained proposal network for this orientation sampling");
        T2B_REQUIRE(topk >= 1 && topk <= 128 && topk <= KO && audit_every >= 1 && audit_mass > 0. && audit_mass <= 1.,
                    T2B_ERR_ARG, "bad proposal settings");
        T2B_REQUIRE(rescore == 0 || (rescore >= topk && rescore <= NET_MAX_K1 && rescore % 128 == 0 && rescore <= KO), T2B_ERR_ARG,
                    "rescore must be 0 or a multiple of 128 in [topk, min(1024, nr_classes*n_dir*n_psi)]");
        ProposalNet& N = *c->net;
        const int B = c->cfg.max_batch;
        // at most ceil(B / every) multiples of `every` in any B consecutive stream positions
        net_setup(c, std::min(B, (B + audit_every - 1) / audit_every));
        T2B_REQUIRE(rescore == 0 || c->tb.T <= RS_TMAX,
                    T2B_ERR_UNSUPPORTED, "the low-resolution rescoring takes at most 96 translations");
        N.k1 = rescore;
        N.kprop = topk;
        N.every = audit_every;
        N.thr = audit_mass;
        set_tile_shape(N, c->tb.T);
        T2B_CUDA(cudaMemset(N.ps, 0, sizeof(PropState)));
        N.enabled = true;
    });
}

int t2b_proposal_params(t2b_ctx* c, float* get, const float* set, long long* count)
{
    return guarded([&] {
        T2B_REQUIRE(c && count, T2B_ERR_ARG, "null argument");
        T2B_REQUIRE(c->configured, T2B_ERR_STATE, "t2b_configure must be called first");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        ProposalNet& N = net_params(c, c->tb.K * c->tb.O);
        *count = (long long)N.L.total;
        if (get || set) c->quiesce();   // the copies run outside the context's streams
        if (get) T2B_CUDA(cudaMemcpy(get, N.th, N.L.total * sizeof(float), cudaMemcpyDeviceToHost));
        if (set) {
            drop_graph(c);
            T2B_CUDA(cudaMemcpy(N.th, set, N.L.total * sizeof(float), cudaMemcpyHostToDevice));
            k_to_bf16<<<gridsz(N.L.alloc), 256, 0, c->stream>>>(N.th, (bf16*)N.thb, N.L.alloc);
            T2B_CUDA(cudaMemsetAsync(N.m, 0, N.L.alloc * sizeof(float), c->stream));
            T2B_CUDA(cudaMemsetAsync(N.v, 0, N.L.alloc * sizeof(float), c->stream));
            T2B_CUDA(cudaStreamSynchronize(c->stream));
            N.adam_t = 0;
            N.trained = true;
        }
    });
}

int t2b_proposal_features(t2b_ctx* c, const t2b_batch* b, float* imgs)
{
    return guarded([&] {
        T2B_REQUIRE(c && b && imgs && b->fimg && b->ctf && b->minvsigma2, T2B_ERR_ARG, "null argument");
        T2B_REQUIRE(c->configured && b->n >= 1 && b->n <= c->cfg.max_batch, T2B_ERR_ARG, "batch size out of range");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        c->quiesce();   // buffers of the network and of slot 0 may be in use by host batches in flight
        ProposalNet& N = net_params(c, c->tb.K * c->tb.O);
        net_setup(c, std::max(1, N.na_max));
        cudaStream_t st = c->stream;
        const int n = b->n, P = c->tb.P;
        Work& w = c->wk;
        T2B_CUDA(cudaMemcpyAsync((void*)w.fimg, b->fimg, (size_t)n * P * sizeof(float2), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemcpyAsync((void*)w.ctf, b->ctf, (size_t)n * P * sizeof(float), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemcpyAsync((void*)w.minv, b->minvsigma2, (size_t)n * P * sizeof(float), cudaMemcpyHostToDevice, st));
        k_features<<<n, NET_NPIX, 0, st>>>(w.fimg, w.ctf, w.minv, P, N.ring, N.ring_k, N.nring, N.img, nullptr, nullptr);
        T2B_CUDA(cudaGetLastError());
        T2B_CUDA(cudaMemcpyAsync(imgs, N.img, (size_t)n * NET_NPIX * sizeof(float), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaStreamSynchronize(st));
    });
}

int t2b_proposal_logits(t2b_ctx* c, const float* imgs, int n, float* logits)
{
    return guarded([&] {
        T2B_REQUIRE(c && imgs && logits, T2B_ERR_ARG, "null argument");
        T2B_REQUIRE(c->configured && n >= 1 && n <= c->cfg.max_batch, T2B_ERR_ARG, "n out of range");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        c->quiesce();   // buffers of the network and of slot 0 may be in use by host batches in flight
        ProposalNet& N = net_params(c, c->tb.K * c->tb.O);
        net_setup(c, std::max(1, N.na_max));
        cudaStream_t st = c->stream;
        T2B_CUDA(cudaMemcpyAsync(N.img, imgs, (size_t)n * NET_NPIX * sizeof(float), cudaMemcpyHostToDevice, st));
        k_conv_fwd<<<n, 256, 0, st>>>(N.img, (const bf16*)N.thb, N.L, n, nullptr, nullptr, (bf16*)N.x0b);
        infer_dense(N, n, c->wk.err, st);
        k_bias_act<<<gridsz((size_t)n * N.KO), 256, 0, st>>>(N.logits, (const bf16*)N.thb + N.L.b3, n, N.KO, 0, N.logits,
                                                            nullptr);
        T2B_CUDA(cudaGetLastError());
        T2B_CUDA(cudaMemcpyAsync(logits, N.logits, (size_t)n * N.KO * sizeof(float), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaStreamSynchronize(st));
    });
}

int t2b_proposal_grad(t2b_ctx* c, const float* imgs, const int* tgt_oc, const float* tgt_w, int n, double* loss,
                      float* grad)
{
    return guarded([&] {
        T2B_REQUIRE(c && imgs && tgt_oc && tgt_w && loss && grad, T2B_ERR_ARG, "null argument");
        T2B_REQUIRE(c->configured && n >= 1 && n <= 1024, T2B_ERR_ARG, "n out of range");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        c->quiesce();   // buffers of the network and of slot 0 may be in use by host batches in flight
        const int KO = c->tb.K * c->tb.O;
        ProposalNet& N = net_params(c, KO);
        for (int i = 0; i < n * NET_NTGT; i++)
            T2B_REQUIRE(tgt_oc[i] >= -1 && tgt_oc[i] < KO, T2B_ERR_ARG, "target orientation out of range");
        cudaStream_t st = c->stream;
        TrainBufs t(n, KO);
        T2B_CUDA(cudaMemcpyAsync(t.bimg, imgs, (size_t)n * NET_NPIX * sizeof(float), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemcpyAsync(t.tgt_oc, tgt_oc, (size_t)n * NET_NTGT * sizeof(int), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemcpyAsync(t.tgt_w, tgt_w, (size_t)n * NET_NTGT * sizeof(float), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemsetAsync(t.loss, 0, sizeof(double), st));
        train_fwd_bwd(N, t, c->tb, false, 0.f, st);
        double l = 0.;
        T2B_CUDA(cudaMemcpyAsync(&l, t.loss, sizeof(double), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaMemcpyAsync(grad, N.g, N.L.total * sizeof(float), cudaMemcpyDeviceToHost, st));
        T2B_CUDA(cudaStreamSynchronize(st));
        *loss = l / n;
    });
}

}  // extern "C"
