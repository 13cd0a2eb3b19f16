// Batched 1D FFTs in shared memory (libt2b): mixed-radix Stockham autosort
// over nfft sequences of length N, ping-ponging between two shared buffers;
// radix-4, 2, 3, 5, 7 stages with a runtime plan, any other prime factor p by a
// direct length-p DFT (the odd padded boxes of the reconstruction's gridding
// iterations, e.g. 259 = 7 x 37): as the first stage in conjugate output pairs,
// later ones one output per thread (N p work for that stage), or, for a
// size known at compile time, radix-16 and radix-8 register butterflies first
// and constant index arithmetic.  Twiddles tw[t] = e^{-2 pi i t / N} (a table
// the caller stages in shared memory); the inverse transform uses their
// conjugates and is unnormalised.  Used by the image preparation
// (imageprep.cu) and the reconstruction's inverse 3D transform (recon.cu).
#pragma once
#include "t2b_internal.cuh"

namespace t2b {

constexpr int FFT_MAX_STAGES = 12;

struct FftPlan {
    int n = 0;
    int nst = 0;
    int rad[FFT_MAX_STAGES] = {};
};

// runtime plan: radices 4, then 2, 3, 5; with any_prime, the prime factors >= 7 come first,
// largest first, so that the largest one runs as the first stage (no input twiddles there:
// fft_stage_prime_first), the others by the radix-7 or the generic stage
inline FftPlan fft_plan(int N, bool any_prime = false)
{
    FftPlan pl;
    pl.n = N;
    int n = N;
    auto take = [&](int r) {
        while (n % r == 0 && pl.nst < FFT_MAX_STAGES) {
            pl.rad[pl.nst++] = r;
            n /= r;
        }
    };
    if (any_prime) {
        int m = N, primes[FFT_MAX_STAGES], np = 0;
        for (int p : {2, 3, 5})
            while (m % p == 0) m /= p;
        for (int p = 7; m > 1 && np < FFT_MAX_STAGES; p += 2)
            while (m % p == 0 && np < FFT_MAX_STAGES) {
                primes[np++] = p;
                m /= p;
            }
        for (int i = np - 1; i >= 0; --i) take(primes[i]);
    }
    take(4);
    take(2);
    take(3);
    take(5);
    T2B_REQUIRE(n == 1, T2B_ERR_UNSUPPORTED,
                any_prime ? "transform size has too many prime factors" : "transform sizes must be products of 2, 3 and 5");
    return pl;
}

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

template <bool INV>
__device__ __forceinline__ float2 twid(const float2* tw, int t)
{
    const float2 w = tw[t];
    return INV ? make_float2(w.x, -w.y) : w;
}

// DFT of R points in registers: out[q] = sum_r v[r] W^{q r}, W = e^{-+2 pi i / R}
// (tw[t] = e^{-2 pi i t / N}, NR = N / R).
template <int R, bool INV>
__device__ __forceinline__ void dft_small(float2* v, const float2* tw, int NR)
{
    if (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        const float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        const float2 c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
        // forward: X1 = b - i d, X3 = b + i d; inverse swaps them
        const float2 mid = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);   // -+ i d
        v[0] = cadd(a, c);
        v[2] = csub(a, c);
        v[1] = cadd(b, mid);
        v[3] = csub(b, mid);
    } else if (R == 8) {
        // 8 = 2 x 4: DFT4 of the even and odd points, X[k] = E[k] + W8^k O[k], X[k+4] = E[k] - W8^k O[k]
        float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        dft_small<4, INV>(e, tw, NR);
        dft_small<4, INV>(o, tw, NR);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 t = k == 0 ? o[0] : cmul(o[k], twid<INV>(tw, k * NR));
            v[k] = cadd(e[k], t);
            v[k + 4] = csub(e[k], t);
        }
    } else if (R == 16) {
        // 16 = 4 x 4: Y_l = DFT4 over m of v[4m + l]; X[k1 + 4 k2] = DFT4 over l of W16^{l k1} Y_l[k1]
        float2 y[4][4];
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            float2 t[4] = {v[l], v[4 + l], v[8 + l], v[12 + l]};
            dft_small<4, INV>(t, tw, NR);
#pragma unroll
            for (int k1 = 0; k1 < 4; ++k1) y[l][k1] = t[k1];
        }
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            float2 z[4];
#pragma unroll
            for (int l = 0; l < 4; ++l) z[l] = (l * k1 == 0) ? y[l][k1] : cmul(y[l][k1], twid<INV>(tw, l * k1 * NR));
            dft_small<4, INV>(z, tw, NR);
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = z[k2];
        }
    } else {
        float2 o[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            float2 acc = v[0];
#pragma unroll
            for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(v[r], twid<INV>(tw, ((q * r) % R) * NR)));
            o[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = o[q];
    }
}

// One Stockham stage over nfft sequences of length N: a -> b.
template <int R, bool INV>
__device__ __forceinline__ void fft_stage(const float2* a, float2* b, int nfft, int N, int Ns, const float2* tw)
{
    const int NR = N / R;
    const int tstride = N / (Ns * R);
    for (int e = threadIdx.x; e < nfft * NR; e += blockDim.x) {
        const int f = e / NR, j = e - f * NR;
        const float2* in = a + f * N;
        float2* out = b + f * N;
        const int k = j % Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = in[j + r * NR];
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid<INV>(tw, k * r * tstride));
        dft_small<R, INV>(v, tw, NR);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) out[base + r * Ns] = v[r];
    }
}

// The same stage for a radix R known only at run time (a prime >= 7): one thread per output,
// X[m Ns R + q Ns + k] = sum_r in[m Ns + k + r N/R] e^{-+2 pi i (k r N/(Ns R) + (q r mod R) N/R) / N},
// the Stockham twiddle and the length-R DFT's root folded into one table entry.
template <bool INV>
__device__ __forceinline__ void fft_stage_gen(const float2* a, float2* b, int nfft, int N, int Ns, int R,
                                              const float2* tw)
{
    const int NR = N / R;
    const int tstride = N / (Ns * R);
    for (int e = threadIdx.x; e < nfft * N; e += blockDim.x) {
        const int f = e / N, o = e - f * N;
        const int k = o % Ns, q = (o / Ns) % R, m = o / (Ns * R);
        const float2* in = a + f * N + m * Ns + k;
        float2 acc = make_float2(0.f, 0.f);
        int qr = 0;   // (q r) mod R
        for (int r = 0; r < R; ++r) {
            int t = k * r * tstride + qr * NR;
            if (t >= N) t -= N;
            acc = cadd(acc, cmul(in[r * NR], twid<INV>(tw, t)));
            qr += q;
            if (qr >= R) qr -= R;
        }
        b[f * N + o] = acc;
    }
}

// The first stage (Ns = 1: no input twiddles) for an odd prime radix R >= 7: one thread per
// (sequence, group m, pair u), X[u] and X[R - u] from the same sums over r = 1 .. (R - 1) / 2 of
// S_r = x_r + x_{R-r} and D_r = x_r - x_{R-r}: X[u] = x_0 + A -+ i B, X[R - u] = x_0 + A +- i B
// with A = sum_r cos(2 pi u r / R) S_r, B = sum_r sin(2 pi u r / R) D_r (upper signs forward);
// u = 0 gives X[0] = x_0 + sum_r S_r.  About a quarter of the generic stage's loads and products.
template <bool INV>
__device__ __forceinline__ void fft_stage_prime_first(const float2* a, float2* b, int nfft, int N, int R,
                                                      const float2* tw)
{
    const int NR = N / R, h = (R - 1) / 2, per = NR * (h + 1);
    for (int e = threadIdx.x; e < nfft * per; e += blockDim.x) {
        const int f = e / per, rem = e - f * per;
        const int m = rem / (h + 1), u = rem - m * (h + 1);
        const float2* in = a + f * N + m;
        float2* out = b + f * N + m * R;
        const float2 x0 = in[0];
        float2 A = make_float2(0.f, 0.f), Bs = make_float2(0.f, 0.f);
        int ur = 0;   // (u r) mod R
        for (int r = 1; r <= h; ++r) {
            ur += u;
            if (ur >= R) ur -= R;
            const float2 xr = in[r * NR], xm = in[(R - r) * NR];
            const float2 S = cadd(xr, xm), D = csub(xr, xm);
            const float2 w = tw[ur * NR];   // (cos, -sin) of 2 pi u r / R
            A.x = fmaf(w.x, S.x, A.x);
            A.y = fmaf(w.x, S.y, A.y);
            Bs.x = fmaf(-w.y, D.x, Bs.x);
            Bs.y = fmaf(-w.y, D.y, Bs.y);
        }
        const float2 c0 = cadd(x0, A);
        if (u == 0) {
            out[0] = c0;
        } else {
            const float2 mib = make_float2(Bs.y, -Bs.x);   // -i B
            out[u] = INV ? csub(c0, mib) : cadd(c0, mib);
            out[R - u] = INV ? cadd(c0, mib) : csub(c0, mib);
        }
    }
}

// All stages; returns the buffer holding the transform (natural order).  PRIMES (the plans of
// fft_plan(N, true)): the radix-7 register stage and the first-stage pairs for larger primes,
// compiled only into the kernels that take such plans (they cost the others registers).
template <bool INV, bool PRIMES = false>
__device__ float2* fft_smem(float2* a, float2* b, int nfft, const FftPlan& pl, const float2* tw)
{
    int Ns = 1;
    for (int st = 0; st < pl.nst; ++st) {
        const int R = pl.rad[st];
        switch (R) {
        case 4: fft_stage<4, INV>(a, b, nfft, pl.n, Ns, tw); break;
        case 2: fft_stage<2, INV>(a, b, nfft, pl.n, Ns, tw); break;
        case 3: fft_stage<3, INV>(a, b, nfft, pl.n, Ns, tw); break;
        case 5: fft_stage<5, INV>(a, b, nfft, pl.n, Ns, tw); break;
        default:
            if constexpr (PRIMES) {
                if (R == 7) fft_stage<7, INV>(a, b, nfft, pl.n, Ns, tw);
                else if (Ns == 1) fft_stage_prime_first<INV>(a, b, nfft, pl.n, R, tw);
                else fft_stage_gen<INV>(a, b, nfft, pl.n, Ns, R, tw);
            } else {
                fft_stage_gen<INV>(a, b, nfft, pl.n, Ns, R, tw);
            }
            break;
        }
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}


// ---- the same FFT with the size known at compile time (the common box sizes):
// constant radix plan (radix-16 and radix-8 register butterflies first), constant
// index arithmetic, unrolled stage sequence
constexpr int ct_radix(int N, int st)
{
    int n = N, k = 0;
    for (int r : {16, 8, 4, 2, 3, 5})
        while (n % r == 0) {
            if (k == st) return r;
            n /= r;
            ++k;
        }
    return 0;
}
constexpr int ct_ns(int N, int st)
{
    int ns = 1;
    for (int k = 0; k < st; ++k) ns *= ct_radix(N, k);
    return ns;
}

template <int R, bool INV, int N, int Ns>
__device__ __forceinline__ void fft_stage_ct(const float2* a, float2* b, int nfft, const float2* tw)
{
    constexpr int NR = N / R;
    constexpr int tstride = N / (Ns * R);
    for (int e = threadIdx.x; e < nfft * NR; e += blockDim.x) {
        const int f = e / NR, j = e - f * NR;
        const float2* in = a + f * N;
        float2* out = b + f * N;
        const int k = j % Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = in[j + r * NR];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid<INV>(tw, k * r * tstride));
        }
        dft_small<R, INV>(v, tw, NR);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) out[base + r * Ns] = v[r];
    }
}

template <int N, bool INV, int ST>
__device__ __forceinline__ float2* fft_ct(float2* a, float2* b, int nfft, const float2* tw)
{
    if constexpr (ct_radix(N, ST) == 0) {
        return a;
    } else {
        fft_stage_ct<ct_radix(N, ST), INV, N, ct_ns(N, ST)>(a, b, nfft, tw);
        __syncthreads();
        return fft_ct<N, INV, ST + 1>(b, a, nfft, tw);
    }
}

// compile-time size when NC > 0, the runtime plan otherwise
template <int NC, bool INV>
__device__ __forceinline__ float2* fft_any(float2* a, float2* b, int nfft, const FftPlan& pl, const float2* tw)
{
    if constexpr (NC > 0) return fft_ct<NC, INV, 0>(a, b, nfft, tw);
    else return fft_smem<INV>(a, b, nfft, pl, tw);
}

}  // namespace
}  // namespace t2b
