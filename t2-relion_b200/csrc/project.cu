// Projection and phase tables of libt2b.
//
// Coarse orientations do not depend on the particle (no per-particle priors),
// so every projection of an iteration is computed once here and kept resident
// in HBM (K*O x P complex FP32 for the coarse pass, K*O*R x P for the fine
// pass) instead of being re-interpolated for every particle as the reference
// kernels do (orientation_matrix_handler.cuh:99-126, tex3D per particle).
//
// Interpolation follows the TRILINEAR branch of Projector::project
// (src/projector.cpp:566-650) and AccProjectorKernel::project3Dmodel
// (src/acc/acc_projectorkernel_impl.h:179-250): mirror + conjugate for
// xp < 0, origin at (0, inity, initz).  Coordinates and weights are FP64 so the
// table matches the FP64 oracle to float rounding; the radius test is the exact
// integer test x*x + y*y <= r_max*r_max (the reference's float test of the
// rotated radius keeps or drops the pixels lying on the circle by rounding).
#include "t2b_internal.cuh"
#include <cmath>

namespace t2b {
namespace {

__device__ __forceinline__ void lerp_c(double a, double lr, double li, double hr, double hi, double& r, double& i)
{
    r = lr + (hr - lr) * a;
    i = li + (hi - li) * a;
}

__global__ void k_project3d(const float2* __restrict__ mdl, Volume v, const double* __restrict__ eul,
                            int s, float2* __restrict__ out)
{
    const int xh = s / 2 + 1, P = s * xh;
    const int o = blockIdx.y;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P) return;
    const int i = n / xh, x = n - i * xh;
    const int y = (i < xh) ? i : i - s;
    const int rmo = s / 2;
    float2 res = make_float2(0.f, 0.f);
    const double* A = eul + 9 * (size_t)o;
    if (x * x + y * y <= rmo * rmo && x * x + y * y <= v.r_max * v.r_max) {
        double xp = (A[0] * x + A[3] * y) * v.pad;
        double yp = (A[1] * x + A[4] * y) * v.pad;
        double zp = (A[2] * x + A[5] * y) * v.pad;
        const bool neg = xp < 0;
        if (neg) { xp = -xp; yp = -yp; zp = -zp; }
        const int x0 = (int)floor(xp);
        const double fx = xp - x0;
        int y0 = (int)floor(yp);
        const double fy = yp - y0;
        y0 -= v.inity;
        int z0 = (int)floor(zp);
        const double fz = zp - z0;
        z0 -= v.initz;
        if (!(x0 < 0 || x0 + 1 >= v.xdim || y0 < 0 || y0 + 1 >= v.ydim || z0 < 0 || z0 + 1 >= v.zdim)) {
            const size_t b00 = ((size_t)z0 * v.ydim + y0) * v.xdim + x0;
            const size_t b01 = b00 + v.xdim;                            // y0+1
            const size_t b10 = b00 + (size_t)v.ydim * v.xdim;           // z0+1
            const size_t b11 = b10 + v.xdim;
            const float2 d000 = mdl[b00], d001 = mdl[b00 + 1];
            const float2 d010 = mdl[b01], d011 = mdl[b01 + 1];
            const float2 d100 = mdl[b10], d101 = mdl[b10 + 1];
            const float2 d110 = mdl[b11], d111 = mdl[b11 + 1];
            double x00r, x00i, x01r, x01i, x10r, x10i, x11r, x11i, y0r, y0i, y1r, y1i, rr, ri;
            lerp_c(fx, d000.x, d000.y, d001.x, d001.y, x00r, x00i);
            lerp_c(fx, d100.x, d100.y, d101.x, d101.y, x01r, x01i);
            lerp_c(fx, d010.x, d010.y, d011.x, d011.y, x10r, x10i);
            lerp_c(fx, d110.x, d110.y, d111.x, d111.y, x11r, x11i);
            lerp_c(fy, x00r, x00i, x10r, x10i, y0r, y0i);
            lerp_c(fy, x01r, x01i, x11r, x11i, y1r, y1i);
            lerp_c(fz, y0r, y0i, y1r, y1i, rr, ri);
            res = make_float2((float)rr, (float)(neg ? -ri : ri));
        }
    }
    out[(size_t)o * P + n] = res;
}

// Projector::rotate2D (src/projector.cpp:904-1016), bilinear, 2D references.
__global__ void k_project2d(const float2* __restrict__ mdl, Volume v, const double* __restrict__ eul,
                            int s, float2* __restrict__ out)
{
    const int xh = s / 2 + 1, P = s * xh;
    const int o = blockIdx.y;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P) return;
    const int i = n / xh, x = n - i * xh;
    const int y = (i < xh) ? i : i - s;
    const int rmo = s / 2;
    float2 res = make_float2(0.f, 0.f);
    const double* A = eul + 9 * (size_t)o;
    if (x * x + y * y <= rmo * rmo && x * x + y * y <= v.r_max * v.r_max) {
        double xp = (A[0] * x + A[3] * y) * v.pad;
        double yp = (A[1] * x + A[4] * y) * v.pad;
        const bool neg = xp < 0;
        if (neg) { xp = -xp; yp = -yp; }
        const int x0 = (int)floor(xp);
        const double fx = xp - x0;
        int y0 = (int)floor(yp);
        const double fy = yp - y0;
        y0 -= v.inity;
        if (!(x0 < 0 || x0 + 1 >= v.xdim || y0 < 0 || y0 + 1 >= v.ydim)) {
            const size_t b0 = (size_t)y0 * v.xdim + x0, b1 = b0 + v.xdim;
            const float2 d00 = mdl[b0], d01 = mdl[b0 + 1], d10 = mdl[b1], d11 = mdl[b1 + 1];
            double a0r, a0i, a1r, a1i, rr, ri;
            lerp_c(fx, d00.x, d00.y, d01.x, d01.y, a0r, a0i);
            lerp_c(fx, d10.x, d10.y, d11.x, d11.y, a1r, a1i);
            lerp_c(fy, a0r, a0i, a1r, a1i, rr, ri);
            res = make_float2((float)rr, (float)(neg ? -ri : ri));
        }
    }
    out[(size_t)o * P + n] = res;
}

// e^{-2 pi i (kx sx + ky sy)/N} for every pixel of the window
// (shiftImageInFourierTransform, src/fftw.cpp:874-918; AB matrices,
// src/ml_optimiser.cpp:3751-3830), FP64 then rounded to float.
__global__ void k_phase(const double* __restrict__ shifts, int s, int ori, float2* __restrict__ out)
{
    const int xh = s / 2 + 1, P = s * xh;
    const int t = blockIdx.y;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P) return;
    const int i = n / xh, x = n - i * xh;
    const int y = (i < xh) ? i : i - s;
    const double xs = -shifts[2 * t] / ori, ys = -shifts[2 * t + 1] / ori;
    const double dotp = 2 * 3.14159265358979323846 * (x * xs + y * ys);
    double sn, cs;
    sincos(dotp, &sn, &cs);
    out[(size_t)t * P + n] = make_float2((float)cs, (float)sn);
}

}  // namespace

void launch_project_table(const Volume& v, const float2* mdl, const double* eul9, int n, int s,
                          float2* out, cudaStream_t st)
{
    const int P = s * (s / 2 + 1);
    for (int o0 = 0; o0 < n; o0 += 65535) {
        const int cnt = std::min(65535, n - o0);
        dim3 grid((P + 255) / 256, cnt);
        if (v.ref_dim == 3)
            k_project3d<<<grid, 256, 0, st>>>(mdl, v, eul9 + 9 * (size_t)o0, s, out + (size_t)o0 * P);
        else
            k_project2d<<<grid, 256, 0, st>>>(mdl, v, eul9 + 9 * (size_t)o0, s, out + (size_t)o0 * P);
    }
    T2B_CUDA(cudaGetLastError());
}

void launch_phase_table(const double* shifts, int n, int s, int ori_size, float2* out, cudaStream_t st)
{
    const int P = s * (s / 2 + 1);
    dim3 grid((P + 255) / 256, n);
    k_phase<<<grid, 256, 0, st>>>(shifts, s, ori_size, out);
    T2B_CUDA(cudaGetLastError());
}

}  // namespace t2b
