// Projection and phase tables of libt2b.
//
// Coarse orientations do not depend on the particle (no per-particle priors),
// so every projection of an iteration is computed once here and kept resident
// in HBM (K*O x P complex FP32 for the coarse pass, K*O*R x P for the fine
// pass) instead of being re-interpolated for every particle as the reference
// kernels do (orientation_matrix_handler.cuh:99-126, tex3D per particle).
//
// Interpolation: project_pixel (project_pixel.cuh).  Coordinates and weights
// are FP64 so the table matches the FP64 oracle to float rounding; the radius
// test is the exact integer test x*x + y*y <= r_max*r_max (the reference's
// float test of the rotated radius keeps or drops the pixels lying on the
// circle by rounding).
#include "t2b_internal.cuh"
#include "project_pixel.cuh"
#include <cmath>

namespace t2b {
namespace {

// projection tile: blockDim.x window pixels x `orients` orientations per CTA (rows
// blockIdx.y * orients ...), one pixel per thread; the tile shape is chosen by
// t2b_autotune and does not change any value
__global__ void k_project(const float2* __restrict__ mdl, Volume v, const double* __restrict__ eul,
                          int s, int n, int orients, float2* __restrict__ out)
{
    const int xh = s / 2 + 1, P = s * xh;
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    if (px >= P) return;
    const int o0 = blockIdx.y * orients, o1 = min(n, o0 + orients);
    for (int o = o0; o < o1; ++o) out[(size_t)o * P + px] = project_window_pixel(mdl, v, eul + 9 * (size_t)o, px, s);
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

void make_model_texture(const Volume& v, const float2* mdl, cudaArray_t* arr, cudaTextureObject_t* tex,
                        cudaStream_t st)
{
    int dev = 0, m3 = 0;
    T2B_CUDA(cudaGetDevice(&dev));
    T2B_CUDA(cudaDeviceGetAttribute(&m3, cudaDevAttrMaxTexture3DWidth, dev));
    T2B_REQUIRE(v.xdim <= m3 && v.ydim <= m3 && v.zdim <= m3, T2B_ERR_UNSUPPORTED, "model larger than a 3D texture");
    const cudaChannelFormatDesc cd = cudaCreateChannelDesc<float2>();
    const cudaExtent ext = make_cudaExtent(v.xdim, v.ydim, v.zdim);
    cudaArray_t a = nullptr;
    if (cudaMalloc3DArray(&a, &cd, ext) != cudaSuccess) {
        cudaGetLastError();
        throw Error{T2B_ERR_NOMEM, "3D array allocation failed"};
    }
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr(const_cast<float2*>(mdl), (size_t)v.xdim * sizeof(float2), v.xdim, v.ydim);
    cp.dstArray = a;
    cp.extent = ext;
    cp.kind = cudaMemcpyDeviceToDevice;
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = a;
    cudaTextureDesc td = {};
    for (int i = 0; i < 3; i++) td.addressMode[i] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    cudaError_t e = cudaMemcpy3DAsync(&cp, st);
    if (e == cudaSuccess) e = cudaCreateTextureObject(&t, &rd, &td, nullptr);
    if (e != cudaSuccess) {
        cudaFreeArray(a);
        T2B_CUDA(e);
    }
    *arr = a;
    *tex = t;
}

void launch_project_table(const Volume& v, const float2* mdl, const double* eul9, int n, int s,
                          float2* out, cudaStream_t st, int px, int orients)
{
    const int P = s * (s / 2 + 1);
    T2B_REQUIRE(px >= 32 && px <= 1024 && px % 32 == 0 && orients >= 1 && orients <= 64, T2B_ERR_ARG,
                "projection tile shape");
    const int per_launch = 65535 * orients;
    for (int o0 = 0; o0 < n; o0 += per_launch) {
        const int cnt = std::min(per_launch, n - o0);
        dim3 grid((P + px - 1) / px, (cnt + orients - 1) / orients);
        k_project<<<grid, px, 0, st>>>(mdl, v, eul9 + 9 * (size_t)o0, s, cnt, orients, out + (size_t)o0 * P);
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
