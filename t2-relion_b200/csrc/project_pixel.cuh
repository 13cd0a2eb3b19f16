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

// A model as the interpolation reads it: the centred half-complex grid in linear memory (the
// resident tables' projection), or the same values in a 3D CUDA array read through the texture
// path with point sampling (the chunked configurations, which interpolate every class-orientation
// of every batch: the array's block-linear layout keeps a slice's corners in fewer cache lines,
// and the loads leave the LSU's queue).  Each fetch returns the 2 x 2 corners (z, y..y+1,
// x..x+1) of grid index (x, y, z) (0-based): d[0] = (y, x), d[1] = (y, x+1), d[2] = (y+1, x),
// d[3] = (y+1, x+1).  The values are the same, so is every projection.
struct GridFetch {
    const float2* __restrict__ mdl;
    __device__ __forceinline__ void operator()(const Volume& v, int x, int y, int z, float2* d) const
    {
        const size_t b = ((size_t)z * v.ydim + y) * v.xdim + x;
        d[0] = mdl[b];
        d[1] = mdl[b + 1];
        d[2] = mdl[b + v.xdim];
        d[3] = mdl[b + v.xdim + 1];
    }
};

struct TexFetch {
    cudaTextureObject_t t;   // float2 texels, point sampling, unnormalised coordinates
    __device__ __forceinline__ void operator()(const Volume&, int x, int y, int z, float2* d) const
    {
        // texel centres: a point-sampled fetch at i + 0.5 returns texel i exactly
        const float fx = (float)x + 0.5f, fy = (float)y + 0.5f, fz = (float)z + 0.5f;
        d[0] = tex3D<float2>(t, fx, fy, fz);
        d[1] = tex3D<float2>(t, fx + 1.f, fy, fz);
        d[2] = tex3D<float2>(t, fx, fy + 1.f, fz);
        d[3] = tex3D<float2>(t, fx + 1.f, fy + 1.f, fz);
    }
};

template <typename Fetch>
__device__ __forceinline__ float2 project_pixel_t(const Fetch& fetch, const Volume& v, const double* A, int x, int y)
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
        float2 d0[4], d1[4];
        fetch(v, x0, y0, z0, d0);                            // z0: (y0, x0) (y0, x0+1) (y0+1, x0) (y0+1, x0+1)
        fetch(v, x0, y0, z0 + 1, d1);                        // z0 + 1
        double x00r, x00i, x01r, x01i, x10r, x10i, x11r, x11i, y0r, y0i, y1r, y1i;
        pp_lerp(fx, d0[0].x, d0[0].y, d0[1].x, d0[1].y, x00r, x00i);
        pp_lerp(fx, d1[0].x, d1[0].y, d1[1].x, d1[1].y, x01r, x01i);
        pp_lerp(fx, d0[2].x, d0[2].y, d0[3].x, d0[3].y, x10r, x10i);
        pp_lerp(fx, d1[2].x, d1[2].y, d1[3].x, d1[3].y, x11r, x11i);
        pp_lerp(fy, x00r, x00i, x10r, x10i, y0r, y0i);
        pp_lerp(fy, x01r, x01i, x11r, x11i, y1r, y1i);
        pp_lerp(fz, y0r, y0i, y1r, y1i, rr, ri);
    } else {
        if (x0 < 0 || x0 + 1 >= v.xdim || y0 < 0 || y0 + 1 >= v.ydim) return make_float2(0.f, 0.f);
        float2 d[4];
        fetch(v, x0, y0, 0, d);
        double a0r, a0i, a1r, a1i;
        pp_lerp(fx, d[0].x, d[0].y, d[1].x, d[1].y, a0r, a0i);
        pp_lerp(fx, d[2].x, d[2].y, d[3].x, d[3].y, a1r, a1i);
        pp_lerp(fy, a0r, a0i, a1r, a1i, rr, ri);
    }
    return make_float2((float)rr, (float)(neg ? -ri : ri));
}

__device__ __forceinline__ float2 project_pixel(const float2* __restrict__ mdl, const Volume& v,
                                                const double* A, int x, int y)
{
    return project_pixel_t(GridFetch{mdl}, v, A, x, y);
}

// Window pixel px (FFTW layout of the s-window) of the projection for Euler matrix A: zero
// outside the window's circle and the model's r_max (the exact integer radius test), else
// project_pixel.  The resident tables (k_project) and the on-the-fly projections of the
// chunked mode both call this, so they hold the same values.
template <typename Fetch>
__device__ __forceinline__ float2 project_window_pixel_t(const Fetch& fetch, const Volume& v, const double* A, int px,
                                                         int s)
{
    const int xh = s / 2 + 1;
    const int i = px / xh, x = px - i * xh;
    const int y = (i < xh) ? i : i - s;
    const int rmo = s / 2;
    const bool inside = x * x + y * y <= rmo * rmo && x * x + y * y <= v.r_max * v.r_max;
    return inside ? project_pixel_t(fetch, v, A, x, y) : make_float2(0.f, 0.f);
}

__device__ __forceinline__ float2 project_window_pixel(const float2* __restrict__ mdl, const Volume& v,
                                                       const double* A, int px, int s)
{
    return project_window_pixel_t(GridFetch{mdl}, v, A, px, s);
}

// the same from a model's 3D array (chunked configurations)
__device__ __forceinline__ float2 project_window_pixel(cudaTextureObject_t t, const Volume& v, const double* A, int px,
                                                       int s)
{
    return project_window_pixel_t(TexFetch{t}, v, A, px, s);
}

}  // namespace t2b
