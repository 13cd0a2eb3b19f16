// Skip-gridding reconstruction division that allocates no device memory.
//
// Some callers cannot call cudaMalloc: RELION's GPU path reserves most of the
// device's free memory for its own arena allocator when it sets up
// (CudaCustomAllocator, -DNEWMEM), so code running inside that process finds
// little or nothing left to allocate; and cudaMalloc / cudaFree synchronise
// the whole device, which a caller overlapping this step with work on other
// streams must avoid.  t2b_reconstruct_divide_noalloc computes the same FP64
// division as t2b_reconstruct_divide from caller-owned device buffers (grid
// in, FFTW-ordered transform out); its only scratch -- the radial weight
// averages, 2 x r_max doubles -- lives in the file-scope array below.
//
// The array is one per device, shared by every call on that device, and keeps
// the previous call's contents (each call clears it first).  Calls on one
// device whose kernels overlap on the GPU race on it: serialise them (one
// stream, or events).  r_max is limited to T2B_NOALLOC_MAX_RMAX.
//
// The set-up of a device -- the device address of the array (cudaGetSymbolAddress,
// with that device current), cached, and the loading of the division's four kernels
// (with CUDA's lazy module loading, the first launch of a kernel loads its module,
// which takes device memory for the code and the array and can synchronise the
// context) -- runs once per device: in t2b_create for the context's device, else in
// the entry point's first call on that device.  A caller without a context makes that
// first call at its own set-up: before any stream capture, and before an arena
// allocator reserves the device's free memory.
#include "t2b_internal.cuh"
#include <mutex>

namespace t2b {
namespace {

constexpr int MAX_RMAX = 2048;
// radial sums [0, MAX_RMAX) and counts [MAX_RMAX, 2*MAX_RMAX)
static __device__ __align__(256) double g_noalloc_scratch[2 * MAX_RMAX];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double* g_addr[MAX_DEVICES] = {};

struct Geo {
    int xdim, ydim, zdim, inity, initz, r_max, pad;
};

__global__ void k_na_clear(double* scratch, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) scratch[i] = 0.;
}

// radial average of the decentred weight (src/backprojector.cpp:1480-1505)
__global__ void k_na_radial(Geo g, const float* __restrict__ weight, double* rad, double* cnt)
{
    const int ps = g.ydim, fx = ps / 2 + 1;
    const long long total = (long long)ps * ps * fx;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= total) return;
    const int j = (int)(n % fx);
    const int i = (int)((n / fx) % ps);
    const int k = (int)(n / ((long long)fx * ps));
    const int kp = k < fx ? k : k - ps, ip = i < fx ? i : i - ps;
    const int rp = g.r_max * g.pad;
    const int r2 = kp * kp + ip * ip + j * j;
    if (r2 >= rp * rp) return;
    const size_t src = ((size_t)(kp - g.initz) * g.ydim + (ip - g.inity)) * g.xdim + j;
    const int ires = (int)floor(sqrt((double)r2) / g.pad);
    atomicAdd(&rad[ires], (double)weight[src]);
    atomicAdd(&cnt[ires], 1.);
}

__global__ void k_na_radnorm(int r_max, double* rad, const double* cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < r_max && (cnt[i] > 0. || rad[i] > 0.)) rad[i] /= 1000. * cnt[i];
}

// decenter + divide by max(weight, radial average) (src/backprojector.cpp:1506-1531)
__global__ void k_na_divide(Geo g, const float2* __restrict__ data, const float* __restrict__ weight,
                            const double* __restrict__ rad, double2* __restrict__ out)
{
    const int ps = g.ydim, fx = ps / 2 + 1;
    const long long total = (long long)ps * ps * fx;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= total) return;
    const int j = (int)(n % fx);
    const int i = (int)((n / fx) % ps);
    const int k = (int)(n / ((long long)fx * ps));
    const int kp = k < fx ? k : k - ps, ip = i < fx ? i : i - ps;
    const int rp = g.r_max * g.pad;
    const int r2 = kp * kp + ip * ip + j * j;
    double2 v = make_double2(0., 0.);
    double w = 0.;
    if (r2 <= rp * rp) {
        const size_t src = ((size_t)(kp - g.initz) * g.ydim + (ip - g.inity)) * g.xdim + j;
        const float2 d = data[src];
        v = make_double2(d.x, d.y);
        w = weight[src];
    }
    const int ires = (int)floor(sqrt((double)r2) / g.pad);
    const double wv = fmax(w, rad[ires < g.r_max ? ires : g.r_max - 1]);
    if (wv != 0.) {
        v.x /= wv;
        v.y /= wv;
    }
    out[n] = v;
}

// Set-up of the current device (once): the scratch array's device address, and every
// kernel of the division loaded (cudaFuncGetAttributes loads a kernel's module).
double* scratch_for_current_device()
{
    int dev = 0;
    T2B_CUDA(cudaGetDevice(&dev));
    T2B_REQUIRE(dev >= 0 && dev < MAX_DEVICES, T2B_ERR_UNSUPPORTED, "device index beyond the scratch table");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw Error{T2B_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)};
        cudaFuncAttributes fa;
        for (const void* k : {(const void*)k_na_clear, (const void*)k_na_radial, (const void*)k_na_radnorm,
                              (const void*)k_na_divide})
            T2B_CUDA(cudaFuncGetAttributes(&fa, k));
        g_addr[dev] = static_cast<double*>(p);
    }
    return g_addr[dev];
}

}  // namespace

// t2b_create's part of the set-up: the context's device is current.
void noalloc_prepare_current_device()
{
    (void)scratch_for_current_device();
}

}  // namespace t2b

using namespace t2b;

extern "C" int t2b_reconstruct_divide_noalloc(const float* data, const float* weight, int xdim, int ydim, int zdim,
                                              int inity, int initz, int r_max, int padding_factor, double* fconv,
                                              void* stream)
{
    try {
        T2B_REQUIRE(data && weight && fconv, T2B_ERR_ARG, "null device pointer");
        T2B_REQUIRE(r_max >= 1 && r_max <= MAX_RMAX, T2B_ERR_ARG,
                    "r_max out of range: t2b_reconstruct_divide_noalloc supports 1 <= r_max <= "
                    "T2B_NOALLOC_MAX_RMAX (2048)");
        T2B_REQUIRE(padding_factor >= 1 && ydim > 1 && zdim == ydim && xdim == ydim / 2 + 1 &&
                        inity == -(ydim / 2) && initz == -(zdim / 2) && r_max * padding_factor + 1 < xdim,
                    T2B_ERR_ARG, "grid must be a centred 3D half-complex grid holding r_max*padding_factor");
        double* scratch = scratch_for_current_device();
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const Geo g{xdim, ydim, zdim, inity, initz, r_max, padding_factor};
        const long long total = (long long)ydim * ydim * (ydim / 2 + 1);
        const int nb = (int)((total + 255) / 256);
        k_na_clear<<<(2 * MAX_RMAX + 255) / 256, 256, 0, st>>>(scratch, 2 * MAX_RMAX);
        k_na_radial<<<nb, 256, 0, st>>>(g, weight, scratch, scratch + MAX_RMAX);
        k_na_radnorm<<<(r_max + 255) / 256, 256, 0, st>>>(r_max, scratch, scratch + MAX_RMAX);
        k_na_divide<<<nb, 256, 0, st>>>(g, reinterpret_cast<const float2*>(data), weight, scratch,
                                        reinterpret_cast<double2*>(fconv));
        T2B_CUDA(cudaGetLastError());
        return T2B_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    }
}
