// One Fourier-slice sample of a centred half-complex model (device inline).
//
// TRILINEAR branch of Projector::project (src/projector.cpp:566-650) and
// AccProjectorKernel::project3Dmodel (src/acc/acc_projectorkernel_impl.h:
// 179-250) for 3D models, Projector::rotate2D (src/projector.cpp:904-1016)
// bilinear for 2D: rotate the window pixel (x, y) by A^T (A row-major, the
// Euler matrix of the orientation), scale by the padding factor, mirror and
// conjugate when xp < 0, interpolate from the origin (0, inity, initz).  FP64
// coordinates and weights, FP32 result; zero outside the grid.  The caller
// applies the radius test.
#pragma once
#include "t2b_internal.cuh"

namespace t2b {

__device__ __forceinline__ void pp_lerp(double a, double lr, double li, double hr, double hi, double& r, double& i)
{
    r = lr + (hr - lr) * a;
    i = li + (hi - li) * a;
}

// One coordinate of the padded, rotated window pixel (x, y): (a pad) x + (b pad) y with
// a, b a column of A (A^-1 = A^T), the padding factor folded into the matrix first and
// each product and the sum rounded on their own, as the reference CPU path evaluates it
// (Ainv *= padding_factor; xp = Ainv(0,0) x + Ainv(0,1) y, src/backprojector.cpp:79-83,
// 215; src/projector.cpp:566-590).  No fused multiply-add: on the x = 0 plane the sign
// of xp is rounding noise, and it decides which Friedel partner a backprojected pixel
// lands on, so the device takes the same decision as the CPU path.
__device__ __forceinline__ double rot_coord(double a, double b, int pad, int x, int y)
{
    return __dadd_rn(__dmul_rn(a * (double)pad, (double)x), __dmul_rn(b * (double)pad, (double)y));
}

__device__ __forceinline__ float2 project_pixel(const float2* __restrict__ mdl, const Volume& v,
                                                const double* A, int x, int y)
{
    double xp = rot_coord(A[0], A[3], v.pad, x, y);
    double yp = rot_coord(A[1], A[4], v.pad, x, y);
    double zp = v.ref_dim == 3 ? rot_coord(A[2], A[5], v.pad, x, y) : 0.;
    const bool neg = xp < 0;
    if (neg) { xp = -xp; yp = -yp; zp = -zp; }
    const int x0 = (int)floor(xp);
    const double fx = xp - x0;
    int y0 = (int)floor(yp);
    const double fy = yp - y0;
    y0 -= v.inity;
    double rr, ri;
    if (v.ref_dim == 3) {
        int z0 = (int)floor(zp);
        const double fz = zp - z0;
        z0 -= v.initz;
        if (x0 < 0 || x0 + 1 >= v.xdim || y0 < 0 || y0 + 1 >= v.ydim || z0 < 0 || z0 + 1 >= v.zdim)
            return make_float2(0.f, 0.f);
        const size_t b00 = ((size_t)z0 * v.ydim + y0) * v.xdim + x0;
        const size_t b01 = b00 + v.xdim;                            // y0+1
        const size_t b10 = b00 + (size_t)v.ydim * v.xdim;           // z0+1
        const size_t b11 = b10 + v.xdim;
        const float2 d000 = mdl[b00], d001 = mdl[b00 + 1];
        const float2 d010 = mdl[b01], d011 = mdl[b01 + 1];
        const float2 d100 = mdl[b10], d101 = mdl[b10 + 1];
        const float2 d110 = mdl[b11], d111 = mdl[b11 + 1];
        double x00r, x00i, x01r, x01i, x10r, x10i, x11r, x11i, y0r, y0i, y1r, y1i;
        pp_lerp(fx, d000.x, d000.y, d001.x, d001.y, x00r, x00i);
        pp_lerp(fx, d100.x, d100.y, d101.x, d101.y, x01r, x01i);
        pp_lerp(fx, d010.x, d010.y, d011.x, d011.y, x10r, x10i);
        pp_lerp(fx, d110.x, d110.y, d111.x, d111.y, x11r, x11i);
        pp_lerp(fy, x00r, x00i, x10r, x10i, y0r, y0i);
        pp_lerp(fy, x01r, x01i, x11r, x11i, y1r, y1i);
        pp_lerp(fz, y0r, y0i, y1r, y1i, rr, ri);
    } else {
        if (x0 < 0 || x0 + 1 >= v.xdim || y0 < 0 || y0 + 1 >= v.ydim) return make_float2(0.f, 0.f);
        const size_t b0 = (size_t)y0 * v.xdim + x0, b1 = b0 + v.xdim;
        const float2 d00 = mdl[b0], d01 = mdl[b0 + 1], d10 = mdl[b1], d11 = mdl[b1 + 1];
        double a0r, a0i, a1r, a1i;
        pp_lerp(fx, d00.x, d00.y, d01.x, d01.y, a0r, a0i);
        pp_lerp(fx, d10.x, d10.y, d11.x, d11.y, a1r, a1i);
        pp_lerp(fy, a0r, a0i, a1r, a1i, rr, ri);
    }
    return make_float2((float)rr, (float)(neg ? -ri : ri));
}

// Window pixel px (FFTW layout of the s-window) of the projection for Euler matrix A: zero
// outside the window's circle and the model's r_max (the exact integer radius test), else
// project_pixel.  The resident tables (k_project) and the on-the-fly projections of the
// chunked mode both call this, so they hold the same values.
__device__ __forceinline__ float2 project_window_pixel(const float2* __restrict__ mdl, const Volume& v,
                                                       const double* A, int px, int s)
{
    const int xh = s / 2 + 1;
    const int i = px / xh, x = px - i * xh;
    const int y = (i < xh) ? i : i - s;
    const int rmo = s / 2;
    const bool inside = x * x + y * y <= rmo * rmo && x * x + y * y <= v.r_max * v.r_max;
    return inside ? project_pixel(mdl, v, A, x, y) : make_float2(0.f, 0.f);
}

}  // namespace t2b
