// C ABI of libt2b: context, model / grid management, configuration, the
// batched E-step and its host <-> device plumbing.
//
// Replaces the reference's per-particle task graph
// (src/acc/cuda/cuda_ml_optimiser.cu:101-1130), its arena allocators
// (custom_allocator.cuh) and the host packer (acc_boo.h) by one preallocated
// workspace per context and a fixed sequence of batched kernels with no host
// synchronisation between the coarse pass and the backprojection.
#include "t2b_internal.cuh"
#include "proposal.cuh"
#include <algorithm>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <new>

namespace t2b {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }

template <typename T>
static T* dalloc(t2b_ctx* c, size_t n)
{
    void* p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{T2B_ERR_NOMEM, "cudaMalloc of " + std::to_string(n * sizeof(T)) + " bytes failed"};
    }
    c->allocs.push_back(p);
    return static_cast<T*>(p);
}

static void free_allocs(t2b_ctx* c)
{
    c->drop_graphs();
    for (void* p : c->allocs) cudaFree(p);
    c->allocs.clear();
    for (cudaTextureObject_t t : c->mtex) cudaDestroyTextureObject(t);
    for (cudaArray_t a : c->marr) cudaFreeArray(a);
    c->mtex.clear();
    c->marr.clear();
    c->configured = false;
}

static void check_volume(int ref_dim, int xdim, int ydim, int zdim, int inity, int initz, int r_max, int pad)
{
    T2B_REQUIRE(ref_dim == 2 || ref_dim == 3, T2B_ERR_ARG, "ref_dim must be 2 or 3");
    T2B_REQUIRE(xdim > 1 && ydim > 1 && zdim >= 1 && r_max > 0 && pad >= 1, T2B_ERR_ARG, "bad volume dimensions");
    T2B_REQUIRE(xdim == ydim / 2 + 1, T2B_ERR_ARG, "xdim must be ydim/2+1 (half-complex)");
    T2B_REQUIRE(ref_dim == 2 ? zdim == 1 : zdim == ydim, T2B_ERR_ARG, "zdim must equal ydim (3D) or 1 (2D)");
    T2B_REQUIRE(inity == -(ydim / 2) && (ref_dim == 2 || initz == -(zdim / 2)), T2B_ERR_ARG,
                "origin must be at the centre (inity = -ydim/2)");
    T2B_REQUIRE(r_max * pad + 1 < xdim, T2B_ERR_ARG, "r_max*padding_factor must fit the grid");
}

}  // namespace t2b

using namespace t2b;

extern "C" {

const char* t2b_last_error(void) { return g_err.c_str(); }
const char* t2b_version(void) { return "t2b 0.1 sm_100a"; }

int t2b_create(int device, t2b_ctx** out)
{
    return guarded([&] {
        T2B_REQUIRE(out != nullptr, T2B_ERR_ARG, "null output pointer");
        int n = 0;
        T2B_CUDA(cudaGetDeviceCount(&n));
        T2B_REQUIRE(device >= 0 && device < n, T2B_ERR_ARG, "no such CUDA device");
        DeviceGuard g(device);
        cudaDeviceProp prop;
        T2B_CUDA(cudaGetDeviceProperties(&prop, device));
        T2B_REQUIRE(prop.major >= 10, T2B_ERR_UNSUPPORTED, "libt2b is built for sm_100a (Blackwell)");
        auto* c = new t2b_ctx();
        c->device = device;
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->d2h_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking);
        for (cudaEvent_t* ev : {&c->fork[0], &c->fork[1]})
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
        for (auto& s : c->in)
            for (cudaEvent_t* ev : {&s.copied, &s.consumed, &s.done})
                if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            for (auto& s : c->in)
                for (cudaEvent_t ev : {s.copied, s.consumed, s.done})
                    if (ev) cudaEventDestroy(ev);
            for (cudaEvent_t ev : c->fork)
                if (ev) cudaEventDestroy(ev);
            if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
            if (c->d2h_stream) cudaStreamDestroy(c->d2h_stream);
            if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
            if (c->stream) cudaStreamDestroy(c->stream);
            delete c;
            T2B_CUDA(e);
        }
        for (auto& ev : c->ev) cudaEventCreate(&ev);
        for (auto& ev : c->handoff) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        // the allocation-free division's once-per-device set-up, here where allocating is fine
        try {
            noalloc_prepare_current_device();
        } catch (...) {
            t2b_destroy(c);
            throw;
        }
        *out = c;
    });
}

void t2b_destroy(t2b_ctx* c)
{
    if (!c) return;
    {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamSynchronize(c->stream);
        cudaStreamSynchronize(c->aux_stream);
        cudaStreamSynchronize(c->d2h_stream);
        free_allocs(c);
        proposal_release(c);
        imageprep_release(c);
        for (auto p : c->mdl) cudaFree(p);
        for (auto p : c->gdata) cudaFree(p);
        for (auto p : c->gweight) cudaFree(p);
        cudaFree(c->sym_scratch);
        for (auto& ev : c->ev) cudaEventDestroy(ev);
        for (auto& ev : c->handoff) cudaEventDestroy(ev);
        for (auto& s : c->in)
            for (cudaEvent_t ev : {s.copied, s.consumed, s.done}) cudaEventDestroy(ev);
        for (cudaEvent_t ev : c->fork) cudaEventDestroy(ev);
        cudaStreamDestroy(c->aux_stream);
        cudaStreamDestroy(c->d2h_stream);
        cudaStreamDestroy(c->copy_stream);
        cudaStreamDestroy(c->stream);
        if (prev >= 0) cudaSetDevice(prev);
    }
    delete c;
}

int t2b_projector_set(t2b_ctx* c, int iclass, int ref_dim, int xdim, int ydim, int zdim, int inity, int initz,
                      int r_max, int pad, const float* mdl)
{
    return guarded([&] {
        T2B_REQUIRE(c && mdl && iclass >= 0 && iclass < 4096, T2B_ERR_ARG, "bad projector arguments");
        check_volume(ref_dim, xdim, ydim, zdim, inity, initz, r_max, pad);
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        if ((int)c->mvol.size() <= iclass) { c->mvol.resize(iclass + 1); c->mdl.resize(iclass + 1, nullptr); }
        Volume v;
        v.ref_dim = ref_dim; v.xdim = xdim; v.ydim = ydim; v.zdim = zdim;
        v.inity = inity; v.initz = initz; v.r_max = r_max; v.pad = pad;
        if (c->mdl[iclass] && c->mvol[iclass].nvox() != v.nvox()) { cudaFree(c->mdl[iclass]); c->mdl[iclass] = nullptr; }
        if (!c->mdl[iclass]) {
            void* p = nullptr;
            if (cudaMalloc(&p, v.nvox() * sizeof(float2)) != cudaSuccess) {
                cudaGetLastError();
                throw Error{T2B_ERR_NOMEM, "model allocation failed"};
            }
            c->mdl[iclass] = (float2*)p;
        }
        c->mvol[iclass] = v;
        T2B_CUDA(cudaMemcpyAsync(c->mdl[iclass], mdl, v.nvox() * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        c->configured = false;  // projection tables are stale
    });
}

int t2b_backprojector_init(t2b_ctx* c, int iclass, int ref_dim, int xdim, int ydim, int zdim, int inity, int initz,
                           int r_max, int pad)
{
    return guarded([&] {
        T2B_REQUIRE(c && iclass >= 0 && iclass < 4096, T2B_ERR_ARG, "bad backprojector arguments");
        check_volume(ref_dim, xdim, ydim, zdim, inity, initz, r_max, pad);
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        if ((int)c->gvol.size() <= iclass) {
            c->gvol.resize(iclass + 1);
            c->gdata.resize(iclass + 1, nullptr);
            c->gweight.resize(iclass + 1, nullptr);
        }
        Volume v;
        v.ref_dim = ref_dim; v.xdim = xdim; v.ydim = ydim; v.zdim = zdim;
        v.inity = inity; v.initz = initz; v.r_max = r_max; v.pad = pad;
        if (c->gdata[iclass] && c->gvol[iclass].nvox() != v.nvox()) {
            cudaFree(c->gdata[iclass]); cudaFree(c->gweight[iclass]);
            c->gdata[iclass] = nullptr; c->gweight[iclass] = nullptr;
        }
        if (!c->gdata[iclass]) {
            void *p = nullptr, *q = nullptr;
            if (cudaMalloc(&p, v.nvox() * sizeof(float2)) != cudaSuccess || cudaMalloc(&q, v.nvox() * sizeof(float)) != cudaSuccess) {
                cudaGetLastError();
                if (p) cudaFree(p);
                throw Error{T2B_ERR_NOMEM, "grid allocation failed"};
            }
            c->gdata[iclass] = (float2*)p;
            c->gweight[iclass] = (float*)q;
        }
        c->gvol[iclass] = v;
        T2B_CUDA(cudaMemsetAsync(c->gdata[iclass], 0, v.nvox() * sizeof(float2), c->stream));
        T2B_CUDA(cudaMemsetAsync(c->gweight[iclass], 0, v.nvox() * sizeof(float), c->stream));
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        c->configured = false;  // grid pointer table is stale
    });
}

int t2b_backprojector_clear(t2b_ctx* c, int iclass)
{
    return guarded([&] {
        T2B_REQUIRE(c && iclass >= 0 && iclass < (int)c->gvol.size() && c->gdata[iclass], T2B_ERR_ARG, "no such grid");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        const Volume& v = c->gvol[iclass];
        T2B_CUDA(cudaMemsetAsync(c->gdata[iclass], 0, v.nvox() * sizeof(float2), c->stream));
        T2B_CUDA(cudaMemsetAsync(c->gweight[iclass], 0, v.nvox() * sizeof(float), c->stream));
        T2B_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int t2b_backprojector_get(t2b_ctx* c, int iclass, float* real, float* imag, float* weight)
{
    return guarded([&] {
        T2B_REQUIRE(c && iclass >= 0 && iclass < (int)c->gvol.size() && c->gdata[iclass], T2B_ERR_ARG, "no such grid");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        const Volume& v = c->gvol[iclass];
        std::vector<float2> tmp(v.nvox());
        T2B_CUDA(cudaMemcpyAsync(tmp.data(), c->gdata[iclass], v.nvox() * sizeof(float2), cudaMemcpyDeviceToHost, c->stream));
        if (weight)
            T2B_CUDA(cudaMemcpyAsync(weight, c->gweight[iclass], v.nvox() * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        for (size_t i = 0; i < v.nvox(); i++) {
            if (real) real[i] = tmp[i].x;
            if (imag) imag[i] = tmp[i].y;
        }
    });
}

int t2b_backprojector_device_ptrs(t2b_ctx* c, int iclass, float** data, float** weight)
{
    return guarded([&] {
        T2B_REQUIRE(c && iclass >= 0 && iclass < (int)c->gvol.size() && c->gdata[iclass], T2B_ERR_ARG, "no such grid");
        if (data) *data = reinterpret_cast<float*>(c->gdata[iclass]);
        if (weight) *weight = c->gweight[iclass];
    });
}

int t2b_configure(t2b_ctx* c, const t2b_config* cfg)
{
    return guarded([&] {
        T2B_REQUIRE(c && cfg, T2B_ERR_ARG, "null argument");
        const t2b_config& f = *cfg;
        T2B_REQUIRE(f.ori_size > 0 && f.current_size > 0 && f.current_size % 2 == 0 && f.current_size <= f.ori_size,
                    T2B_ERR_ARG, "current_size must be even and <= ori_size");
        T2B_REQUIRE(f.ref_dim == 2 || f.ref_dim == 3, T2B_ERR_ARG, "ref_dim must be 2 or 3");
        T2B_REQUIRE(f.nr_classes >= 1 && f.n_dir >= 1 && f.n_psi >= 1 && f.n_trans >= 1, T2B_ERR_ARG, "empty sampling");
        T2B_REQUIRE(f.adaptive_oversampling == 0 || f.adaptive_oversampling == 1, T2B_ERR_ARG,
                    "adaptive_oversampling must be 0 or 1");
        const int R = f.adaptive_oversampling ? f.nover_rot : 1, V = f.adaptive_oversampling ? f.nover_trans : 1;
        T2B_REQUIRE(R >= 1 && R <= 8 && V >= 1 && V <= 4, T2B_ERR_ARG, "oversampling factors must be <= 8 (rot), <= 4 (trans)");
        T2B_REQUIRE(f.diff2_mode == T2B_DIFF2_PLAIN_FP32 || f.diff2_mode == T2B_DIFF2_SPLIT_BF16, T2B_ERR_ARG, "bad diff2_mode");
        T2B_REQUIRE(f.diff2_mode != T2B_DIFF2_SPLIT_BF16 || tc_supported(), T2B_ERR_UNSUPPORTED,
                    "split-BF16 tcgen05 contraction unavailable in this build");
        T2B_REQUIRE(f.max_batch >= 1 && f.max_batch <= 4096, T2B_ERR_ARG, "max_batch must be in [1, 4096]");
        T2B_REQUIRE(f.eul_coarse && f.trans_px && f.trans_prior && f.pdf_direction && f.pdf_class && f.mresol,
                    T2B_ERR_ARG, "missing sampling arrays");
        T2B_REQUIRE(!f.adaptive_oversampling || (f.eul_fine && f.trans_px_fine), T2B_ERR_ARG, "missing fine sampling arrays");
        T2B_REQUIRE(f.adaptive_fraction > 0. && f.adaptive_fraction <= 1., T2B_ERR_ARG, "adaptive_fraction must be in (0,1]");
        T2B_REQUIRE(f.pixel_size > 0., T2B_ERR_ARG, "pixel_size must be positive");
        T2B_REQUIRE((int)c->mvol.size() >= f.nr_classes && (int)c->gvol.size() >= f.nr_classes, T2B_ERR_STATE,
                    "set projectors and backprojectors of every class before t2b_configure");
        for (int k = 0; k < f.nr_classes; k++) {
            T2B_REQUIRE(c->mdl[k] && c->gdata[k], T2B_ERR_STATE, "projector/backprojector of a class is missing");
            T2B_REQUIRE(c->mvol[k].ref_dim == f.ref_dim && c->gvol[k].ref_dim == f.ref_dim, T2B_ERR_ARG, "ref_dim mismatch");
            T2B_REQUIRE(c->gvol[k].nvox() == c->gvol[0].nvox() && c->gvol[k].r_max == c->gvol[0].r_max, T2B_ERR_ARG,
                        "all backprojection grids must share one geometry");
        }
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        c->quiesce();
        free_allocs(c);
        proposal_invalidate(c);
        estep_init_attributes();
        if (f.diff2_mode == T2B_DIFF2_SPLIT_BF16) tc_init_attributes();
        c->cfg = f;
        const int s = f.current_size, xh = s / 2 + 1, P = s * xh;
        const int K = f.nr_classes, O = f.n_dir * f.n_psi, T = f.n_trans, B = f.max_batch;
        const long long KO = (long long)K * O;
        Tables& tb = c->tb;
        tb = Tables{};
        tb.s = s; tb.xh = xh; tb.P = P; tb.ori_size = f.ori_size;
        tb.K = K; tb.n_dir = f.n_dir; tb.n_psi = f.n_psi; tb.O = O; tb.T = T;
        tb.R = R; tb.V = V; tb.ovs = f.adaptive_oversampling; tb.ref_dim = f.ref_dim;
        tb.sigma2_offset = f.sigma2_offset; tb.pixel_size = f.pixel_size; tb.adaptive_fraction = f.adaptive_fraction;
        tb.maxsig = f.maximum_significants > 0 ? f.maximum_significants : 0;
        cudaStream_t st = c->stream;
        // host-side tables: normalised pdf_orientation and the skip mask
        std::vector<double> pdf_o((size_t)K * f.n_dir);
        double om = 0.;
        for (int k = 0; k < K; k++)
            for (int d = 0; d < f.n_dir; d++) om += f.pdf_direction[k * f.n_dir + d] * f.n_psi;
        om /= (double)(K * f.n_dir * f.n_psi);
        std::vector<unsigned char> skip(KO);
        double lpo_min = INFINITY, lpo_max = -INFINITY;
        for (int k = 0; k < K; k++)
            for (int d = 0; d < f.n_dir; d++) {
                double v = f.pdf_direction[k * f.n_dir + d];
                const bool sk = !(f.pdf_class[k] > 0.) || !(v > 0.);
                if (om != 0.) v /= om;
                pdf_o[(size_t)k * f.n_dir + d] = v;
                if (!sk) { lpo_min = std::min(lpo_min, std::log(v)); lpo_max = std::max(lpo_max, std::log(v)); }
                for (int p = 0; p < f.n_psi; p++) skip[(size_t)k * O + d * f.n_psi + p] = sk;
            }
        auto up = [&](const void* h, size_t bytes) {
            void* d = dalloc<unsigned char>(c, bytes);
            T2B_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
            return d;
        };
        T2B_REQUIRE(lpo_max > -INFINITY, T2B_ERR_ARG, "every orientation has a zero prior");
        tb.lpo_min = lpo_min;
        tb.lpo_max = lpo_max;
        tb.pdf_o = (const double*)up(pdf_o.data(), pdf_o.size() * sizeof(double));
        {
            std::vector<double> poc((size_t)K * O);
            for (int k = 0; k < K; k++)
                for (int o = 0; o < O; o++) poc[(size_t)k * O + o] = pdf_o[(size_t)k * f.n_dir + o / f.n_psi];
            tb.pdf_oc = (const double*)up(poc.data(), poc.size() * sizeof(double));
        }
        tb.skip = (const unsigned char*)up(skip.data(), skip.size());
        if (f.data_vs_prior) {
            // do_scale_correction: rings of each class whose data_vs_prior exceeds 3 enter the
            // XA / AA sums (src/ml_optimiser.cpp:8477)
            const int half = f.ori_size / 2 + 1;
            std::vector<unsigned char> ring((size_t)K * half);
            for (size_t i = 0; i < ring.size(); i++) ring[i] = f.data_vs_prior[i] > 3. ? 1 : 0;
            tb.scl_ring = (const unsigned char*)up(ring.data(), ring.size());
        }
        tb.mresol = (const int*)up(f.mresol, (size_t)P * sizeof(int));
        {
            // pixels inside the largest projection radius of all classes
            int rr = 0;
            for (int k = 0; k < K; k++) rr = std::max(rr, std::min(s / 2, c->mvol[k].r_max));
            std::vector<int> kp;
            for (int n = 0; n < P; n++) {
                const int i = n / xh, x = n - i * xh, y = (i < xh) ? i : i - s;
                if (x * x + y * y <= rr * rr) kp.push_back(n);
            }
            tb.nk = (int)kp.size();
            tb.kpix = (const int*)up(kp.data(), kp.size() * sizeof(int));
        }
        // resident projection tables, or one chunk of the coarse orientations per batch step
        int chunk = 0;
        {
            const double kd = (double)tc_kdim(tb.nk), kn = (double)tc_kn(tb.nk);
            const double resident = (double)KO * P * 8. * (1 + (tb.ovs ? R : 0)) +
                                    (f.diff2_mode == T2B_DIFF2_SPLIT_BF16 ? (double)KO * (kd + kn) * 4. : 0.);
            size_t fr = 0, tot = 0;
            T2B_CUDA(cudaMemGetInfo(&fr, &tot));
            T2B_REQUIRE(f.orientation_chunk >= 0, T2B_ERR_ARG, "orientation_chunk must be >= 0");
            if (f.orientation_chunk > 0) chunk = f.orientation_chunk;
            else if (resident > 0.6 * (double)fr) chunk = 16384;
            if (chunk >= KO) chunk = 0;
            chunk = std::min({chunk, O, 32768});   // chunks never straddle two classes; one launch row each
        }
        T2B_REQUIRE(chunk == 0 || f.diff2_mode == T2B_DIFF2_SPLIT_BF16, T2B_ERR_UNSUPPORTED,
                    "projection tables do not fit (or orientation_chunk was set): the chunked coarse pass "
                    "runs on the split-BF16 contraction only");
        tb.chunk = chunk;
        tb.eul_c = (const double*)up(f.eul_coarse, (size_t)O * 9 * sizeof(double));
        tb.trans_c = (const double*)up(f.trans_px, (size_t)T * 2 * sizeof(double));
        tb.trans_prior = (const double*)up(f.trans_prior, (size_t)T * 2 * sizeof(double));
        if (tb.ovs) {
            tb.eul_f = (const double*)up(f.eul_fine, (size_t)O * R * 9 * sizeof(double));
            tb.trans_f = (const double*)up(f.trans_px_fine, (size_t)T * V * 2 * sizeof(double));
        } else {
            tb.eul_f = tb.eul_c;
            tb.trans_f = tb.trans_c;
        }
        for (int k = 0; k < K; k++)
            T2B_REQUIRE(c->mvol[k].r_max * c->mvol[k].pad + 1 < c->mvol[k].xdim, T2B_ERR_ARG, "projector too small");
        if (chunk) {
            // one chunk of coarse projections, filled inside each batch; the fine pass and the
            // weighted sums interpolate from the models
            tb.proj_c = nullptr;   // projections go straight into the chunk's operands
            tb.proj_f = nullptr;
            std::vector<Volume> mv(c->mvol.begin(), c->mvol.begin() + K);
            tb.mvol = (const Volume*)up(mv.data(), K * sizeof(Volume));
            // the models as 3D arrays, read through the texture path (point sampling)
            std::vector<unsigned long long> mt(K);
            for (int k = 0; k < K; k++) {
                cudaArray_t a = nullptr;
                cudaTextureObject_t t = 0;
                make_model_texture(c->mvol[k], c->mdl[k], &a, &t, st);
                c->marr.push_back(a);
                c->mtex.push_back(t);
                mt[k] = (unsigned long long)t;
            }
            tb.mtex = (const unsigned long long*)up(mt.data(), K * sizeof(unsigned long long));
        } else {
            // projection tables (per class, resident)
            float2* pc = dalloc<float2>(c, (size_t)KO * P);
            for (int k = 0; k < K; k++)
                launch_project_table(c->mvol[k], c->mdl[k], tb.eul_c, O, s, pc + (size_t)k * O * P, st,
                                     c->tune.proj_px, c->tune.proj_orients);
            tb.proj_c = pc;
            if (tb.ovs) {
                float2* pf = dalloc<float2>(c, (size_t)KO * R * P);
                for (int k = 0; k < K; k++)
                    launch_project_table(c->mvol[k], c->mdl[k], tb.eul_f, O * R, s, pf + (size_t)k * O * R * P, st,
                                         c->tune.proj_px, c->tune.proj_orients);
                tb.proj_f = pf;
            } else {
                tb.proj_f = pc;
            }
        }
        float2* abc = dalloc<float2>(c, (size_t)T * P);
        launch_phase_table(tb.trans_c, T, s, f.ori_size, abc, st);
        tb.ab_c = abc;
        if (tb.ovs) {
            float2* abf = dalloc<float2>(c, (size_t)T * V * P);
            launch_phase_table(tb.trans_f, T * V, s, f.ori_size, abf, st);
            tb.ab_f = abf;
        } else {
            tb.ab_f = abc;
        }
        // workspace
        Work& w = c->wk;
        w = Work{};
        w.fine_ctas = c->tune.fine_ctas;
        w.wsum_ctas = c->tune.wsum_ctas;
        const long long KOT = KO * T;
        w.cvec = dalloc<float2>(c, (size_t)B * P);
        w.w2 = dalloc<float>(c, (size_t)B * P);
        w.c0 = dalloc<float>(c, B);
        w.norms = dalloc<float>(c, (size_t)B * KO);
        w.d2c = dalloc<float>(c, (size_t)B * KOT);
        w.lbound = dalloc<double>(c, (size_t)B * 2);
        w.minkey_c = dalloc<unsigned>(c, B);
        w.minkey_f = dalloc<unsigned>(c, B);
        w.pdf_t = dalloc<double>(c, (size_t)B * T);
        w.sum_c = dalloc<double>(c, B);
        w.sum_f = dalloc<double>(c, B);
        w.sel_c = dalloc<SelState>(c, B);
        w.sel_f = dalloc<SelState>(c, B);
        w.hist_cnt = dalloc<unsigned>(c, (size_t)B * HIST_BINS);
        w.hist_sum = dalloc<double>(c, (size_t)B * HIST_BINS);
        w.cand = dalloc<double>(c, (size_t)B * CAND_CAP);
        w.fcand_w = dalloc<double>(c, (size_t)B * FAST_CAP);
        w.fcand_i = dalloc<long long>(c, (size_t)B * FAST_CAP);
        w.flist_w = dalloc<double>(c, (size_t)B * FAST_CAP);
        w.flist_i = dalloc<long long>(c, (size_t)B * FAST_CAP);
        const size_t fine_cap = f.fine_capacity ? f.fine_capacity : (size_t)32 << 20;
        w.pair_cap = std::max<long long>((long long)(fine_cap / (size_t)(R * V)), (long long)B * 64);
        w.pairs = dalloc<long long>(c, w.pair_cap);
        w.pair_b = dalloc<int>(c, w.pair_cap);
        w.pair_off = dalloc<long long>(c, B + 1);
        w.max_chunks = (int)((KOT + 4095) / 4096);
        w.chunk_cnt = dalloc<int>(c, (size_t)B * w.max_chunks);
        w.d2f = dalloc<float>(c, (size_t)w.pair_cap * R * V);
        w.wf = dalloc<double>(c, (size_t)w.pair_cap * R * V);
        w.groups = dalloc<long long>(c, w.pair_cap);
        w.group_end = dalloc<long long>(c, w.pair_cap);
        w.group_b = dalloc<int>(c, w.pair_cap);
        w.group_off = dalloc<long long>(c, B + 1);
        w.counters = dalloc<unsigned long long>(c, 16);
        w.err = dalloc<int>(c, 1);
        w.status = dalloc<int>(c, B);
        w.r_learned = dalloc<int>(c, B);
        w.r_audit = dalloc<double>(c, B);
        // staging of host inputs and internal results
        w.fimg = dalloc<float2>(c, (size_t)B * P);
        w.fimg_nm = dalloc<float2>(c, (size_t)B * P);
        w.ctf = dalloc<float>(c, (size_t)B * P);
        w.minv = dalloc<float>(c, (size_t)B * P);
        w.scal = dalloc<double>(c, (size_t)B * 8);
        c->in[0].fimg = const_cast<float2*>(w.fimg);
        c->in[0].fimg_nm = const_cast<float2*>(w.fimg_nm);
        c->in[0].ctf = const_cast<float*>(w.ctf);
        c->in[0].minv = const_cast<float*>(w.minv);
        c->in[0].scal = const_cast<double*>(w.scal);
        c->in[1].fimg = dalloc<float2>(c, (size_t)B * P);
        c->in[1].fimg_nm = dalloc<float2>(c, (size_t)B * P);
        c->in[1].ctf = dalloc<float>(c, (size_t)B * P);
        c->in[1].minv = dalloc<float>(c, (size_t)B * P);
        c->in[1].scal = dalloc<double>(c, (size_t)B * 8);
        w.r_min = dalloc<double>(c, B); w.r_sum = dalloc<double>(c, B); w.r_sig = dalloc<double>(c, B);
        w.r_csum = dalloc<double>(c, B); w.r_csig = dalloc<double>(c, B); w.r_pmax = dalloc<double>(c, B);
        w.r_nsign = dalloc<long long>(c, B); w.r_ncsig = dalloc<long long>(c, B);
        w.r_pose = dalloc<int>(c, (size_t)B * 5);
        w.r_norm = dalloc<double>(c, B); w.r_sumw = dalloc<double>(c, B); w.r_sig_off = dalloc<double>(c, B);
        w.r_sigma2 = dalloc<double>(c, (size_t)B * (f.ori_size / 2 + 1));
        w.r_pdf_class = dalloc<double>(c, (size_t)B * K);
        w.r_pdf_dir = dalloc<double>(c, (size_t)B * K * f.n_dir);
        w.r_xa = dalloc<double>(c, B); w.r_aa = dalloc<double>(c, B);
        // results of the two host slots: slot 0 the workspace's, slot 1 a second set
        for (int i = 0; i < 2; i++) {
            t2b_ctx::InSlot& s = c->in[i];
            const bool own = i == 0;
            s.r_min = own ? w.r_min : dalloc<double>(c, B);
            s.r_sum = own ? w.r_sum : dalloc<double>(c, B);
            s.r_sig = own ? w.r_sig : dalloc<double>(c, B);
            s.r_csum = own ? w.r_csum : dalloc<double>(c, B);
            s.r_csig = own ? w.r_csig : dalloc<double>(c, B);
            s.r_pmax = own ? w.r_pmax : dalloc<double>(c, B);
            s.r_nsign = own ? w.r_nsign : dalloc<long long>(c, B);
            s.r_ncsig = own ? w.r_ncsig : dalloc<long long>(c, B);
            s.r_pose = own ? w.r_pose : dalloc<int>(c, (size_t)B * 5);
            s.r_norm = own ? w.r_norm : dalloc<double>(c, B);
            s.r_sumw = own ? w.r_sumw : dalloc<double>(c, B);
            s.r_sig_off = own ? w.r_sig_off : dalloc<double>(c, B);
            s.r_sigma2 = own ? w.r_sigma2 : dalloc<double>(c, (size_t)B * (f.ori_size / 2 + 1));
            s.r_pdf_class = own ? w.r_pdf_class : dalloc<double>(c, (size_t)B * K);
            s.r_pdf_dir = own ? w.r_pdf_dir : dalloc<double>(c, (size_t)B * K * f.n_dir);
            s.status = own ? w.status : dalloc<int>(c, B);
            s.r_learned = own ? w.r_learned : dalloc<int>(c, B);
            s.r_audit = own ? w.r_audit : dalloc<double>(c, B);
            s.r_xa = own ? w.r_xa : dalloc<double>(c, B);
            s.r_aa = own ? w.r_aa : dalloc<double>(c, B);
        }
        // grid pointer tables
        float2** gd = dalloc<float2*>(c, K);
        float** gw = dalloc<float*>(c, K);
        T2B_CUDA(cudaMemcpyAsync(gd, c->gdata.data(), K * sizeof(float2*), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemcpyAsync(gw, c->gweight.data(), K * sizeof(float*), cudaMemcpyHostToDevice, st));
        c->gd_table = gd;
        c->gw_table = gw;
        c->tc = TcOperands{};
        c->tc.dense_tn = c->tune.dense_tn;
        c->tc.group_m = c->tune.group_m;
        if (f.diff2_mode == T2B_DIFF2_SPLIT_BF16) {
            TcOperands& op = c->tc;
            op.kdim = (int)tc_kdim(tb.nk);
            op.chunk = chunk;
            op.m_pad = (int)(((chunk ? chunk : KO) + 127) / 128 * 128);
            op.n_pad = (B * T + 255) / 256 * 256;
            op.bh = dalloc<uint16_t>(c, (size_t)op.m_pad * op.kdim);
            op.bl = dalloc<uint16_t>(c, (size_t)op.m_pad * op.kdim);
            op.ah = dalloc<uint16_t>(c, (size_t)op.n_pad * op.kdim);
            op.al = dalloc<uint16_t>(c, (size_t)op.n_pad * op.kdim);
            op.kn = (int)tc_kn(tb.nk);
            op.b_pad = (B + 255) / 256 * 256;
            op.nh = dalloc<uint16_t>(c, (size_t)op.m_pad * op.kn);
            op.nl = dalloc<uint16_t>(c, (size_t)op.m_pad * op.kn);
            op.wh = dalloc<uint16_t>(c, (size_t)op.b_pad * op.kn);
            op.wl = dalloc<uint16_t>(c, (size_t)op.b_pad * op.kn);
            op.maps = dalloc<uint8_t>(c, TC_MAP_SLOTS * 128);
            tc_prepare_projections(tb, op, st);
        }
        T2B_CUDA(cudaStreamSynchronize(st));
        c->configured = true;
    });
}

}  // extern "C"

namespace t2b {

// Enqueue the whole E-step of the batch in `w` on `st`.  Stage events are
// recorded only outside stream capture (a captured batch is timed as a whole).
// With learned proposals enabled the network ranks the orientations, the
// audit sets the device gate, and both coarse paths are enqueued: each of
// their kernels runs or returns on the gate.
void enqueue_estep(t2b_ctx* c, Work& w, cudaStream_t st, bool stage_events, bool allow_prop)
{
    const Tables& tb = c->tb;
    const bool tc = c->cfg.diff2_mode == T2B_DIFF2_SPLIT_BF16;
    const bool pm = allow_prop && tc && c->net && c->net->enabled && c->net->ready;
    if (pm) {
        w.gate = &c->net->ps->gate;
        w.prop = c->net->prop;
        w.kprop = c->net->kprop;
    } else {
        w.gate = nullptr;
        w.prop = nullptr;
        w.kprop = 0;
    }
    T2B_CUDA(cudaMemsetAsync(w.counters, 0, 16 * sizeof(unsigned long long), st));
    T2B_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    if (stage_events) cudaEventRecord(c->ev[0], st);
    launch_prep(tb, w, st);
    if (pm && !stage_events) {
        // the audit's contraction (tensor cores) needs the prepared images only: a second
        // branch beside the proposal inference (mostly latency-bound), joined before the
        // audit mass reads the proposals.  Timed stages keep the two in sequence.
        T2B_CUDA(cudaEventRecord(c->fork[0], st));
        T2B_CUDA(cudaStreamWaitEvent(c->aux_stream, c->fork[0], 0));
        proposal_audit_contract(c, w, c->aux_stream);
        proposal_infer(c, w, st);
        T2B_CUDA(cudaEventRecord(c->fork[1], c->aux_stream));
        T2B_CUDA(cudaStreamWaitEvent(st, c->fork[1], 0));
        proposal_audit_mass(c, w, st);
    } else {
        if (pm) proposal_infer(c, w, st);
        if (stage_events) cudaEventRecord(c->ev[1], st);
        if (pm) proposal_audit(c, w, st, stage_events ? c->ev + 8 : nullptr);
    }
    if (tc) tc_split_images(tb, w, c->tc, st, w.gate);   // the full pass's operand: skipped while proposals hold
    if (tb.chunk) {
        // chunked coarse pass: per chunk of one class's orientations, its projections, their
        // split-BF16 operands, the norms and the contraction into the batch's diff2 rows
        if (stage_events) cudaEventRecord(c->ev[2], st);
        bool first = true;
        for (int k = 0; k < tb.K; k++)
            for (int o0 = 0; o0 < tb.O; o0 += tb.chunk) {
                const int n = std::min(tb.chunk, tb.O - o0);
                tc_project_split(tb, c->tc, c->mtex[k], c->mvol[k], tb.eul_c + 9 * (size_t)o0, n, st);
                RowChunk ch;
                ch.row0 = k * tb.O + o0;
                ch.rows = n;
                tc_launch_norms(tb, w, c->tc, st, nullptr, 0, ch, first);
                tc_launch_diff2(tb, w, c->tc, st, nullptr, 0, ch);
                first = false;
            }
    } else {
        if (tc) tc_launch_norms(tb, w, c->tc, st, w.gate, 0);
        else launch_norms(tb, w, st);
        if (stage_events) cudaEventRecord(c->ev[2], st);
        if (pm) proposal_coarse(c, w, st, stage_events ? c->ev + 10 : nullptr);
        if (tc) tc_launch_diff2(tb, w, c->tc, st, w.gate, 0);
        else launch_diff2_simt(tb, w, st);
    }
    if (stage_events) cudaEventRecord(c->ev[3], st);
    launch_weights_coarse(tb, w, c->cfg.maximum_significants, st);
    if (stage_events) cudaEventRecord(c->ev[4], st);
    if (tb.ovs) launch_fine(tb, w, st);
    if (stage_events) cudaEventRecord(c->ev[5], st);
    if (tb.ovs) launch_weights_fine(tb, w, st);
    if (stage_events) cudaEventRecord(c->ev[6], st);
    launch_wsum_bp(tb, w, c->gvol[0], c->gd_table, c->gw_table, st);
    if (stage_events) cudaEventRecord(c->ev[7], st);
    if (stage_events) c->prop_events = pm;
}

static void check_batch(t2b_ctx* c, const t2b_batch* b, const t2b_result* r)
{
    T2B_REQUIRE(c && b && r, T2B_ERR_ARG, "null argument");
    T2B_REQUIRE(c->configured, T2B_ERR_STATE, "t2b_configure must be called before the E-step");
    T2B_REQUIRE(b->n >= 1 && b->n <= c->cfg.max_batch, T2B_ERR_ARG, "batch size out of range");
    T2B_REQUIRE(b->fimg && b->ctf && b->minvsigma2 && b->scalars, T2B_ERR_ARG, "missing batch inputs");
}

static void collect_stage_ms(t2b_ctx* c)
{
    for (int i = 0; i < 7; i++) {
        if (c->last_kernels >= 0 || cudaEventElapsedTime(&c->stage_ms[i], c->ev[i], c->ev[i + 1]) != cudaSuccess) {
            cudaGetLastError();  // do not leave the failure as the runtime's last error
            c->stage_ms[i] = -1.f;
        }
    }
    for (int i = 0; i < 2; i++) {
        if (c->last_kernels >= 0 || !c->prop_events ||
            cudaEventElapsedTime(&c->stage_ms[7 + i], c->ev[8 + 2 * i], c->ev[9 + 2 * i]) != cudaSuccess) {
            cudaGetLastError();
            c->stage_ms[7 + i] = -1.f;
        }
    }
}

}  // namespace t2b

namespace t2b {

// Enqueue the batch in `w` on `st` as a CUDA graph: captured once per key
// (batch shape, buffers, stream, proposal settings) into slot `g`, replayed
// afterwards.  Returns the kernel nodes of the graph.
static int replay_graph(t2b_ctx* c, Work& w, cudaStream_t st, const std::vector<const void*>& key,
                        t2b_ctx::GraphSlot& g)
{
    if (!g.exec || key != g.key) {
        if (g.exec) { cudaGraphExecDestroy(g.exec); g.exec = nullptr; }
        cudaGraph_t graph = nullptr;
        T2B_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_estep(c, w, st, false, true);
        } catch (...) {
            cudaStreamEndCapture(st, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        T2B_CUDA(cudaStreamEndCapture(st, &graph));
        size_t nn = 0;
        T2B_CUDA(cudaGraphGetNodes(graph, nullptr, &nn));
        std::vector<cudaGraphNode_t> nodes(nn);
        T2B_CUDA(cudaGraphGetNodes(graph, nodes.data(), &nn));
        int kn = 0;
        for (auto nd : nodes) {
            // this runtime reports conditional nodes (the selection's multi-kernel path) as an
            // error: they are not kernel nodes either way, and their bodies run only when needed
            cudaGraphNodeType ty;
            if (cudaGraphNodeGetType(nd, &ty) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            if (ty == cudaGraphNodeTypeKernel) kn++;
        }
        const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        T2B_CUDA(ie);
        g.key = key;
        g.kernels = kn;
    }
    T2B_CUDA(cudaGraphLaunch(g.exec, st));
    return g.kernels;
}

// Enqueue one host batch: inputs into staging slot (ticket & 1) on the copy stream once
// that slot's previous batch has read its own, the batch on the context's stream once they
// are in and that batch's results have left the slot, and the results back to host memory
// on the read-back stream after it.  Returns the ticket.
static long long submit_host(t2b_ctx* c, const t2b_batch* b, const t2b_result* r)
{
    cudaStream_t st = c->stream, cs = c->copy_stream, ds = c->d2h_stream;
    const long long ticket = c->submitted;
    t2b_ctx::InSlot& in = c->in[ticket & 1];
    Work w = c->wk;
    const int n = b->n, P = c->tb.P;
    w.n = n;
    w.fimg = in.fimg;
    w.fimg_nm = b->fimg_nomask ? in.fimg_nm : in.fimg;   // no separate unmasked image: the masked one serves both
    w.ctf = in.ctf;
    w.minv = in.minv;
    w.scal = in.scal;
    w.r_min = in.r_min; w.r_sum = in.r_sum; w.r_sig = in.r_sig; w.r_csum = in.r_csum; w.r_csig = in.r_csig;
    w.r_pmax = in.r_pmax; w.r_nsign = in.r_nsign; w.r_ncsig = in.r_ncsig; w.r_pose = in.r_pose;
    w.r_norm = in.r_norm; w.r_sumw = in.r_sumw; w.r_sig_off = in.r_sig_off; w.r_sigma2 = in.r_sigma2;
    w.r_pdf_class = in.r_pdf_class; w.r_pdf_dir = in.r_pdf_dir; w.status = in.status;
    w.r_learned = in.r_learned; w.r_audit = in.r_audit; w.r_xa = in.r_xa; w.r_aa = in.r_aa;
    T2B_CUDA(cudaStreamWaitEvent(cs, in.consumed, 0));
    T2B_CUDA(cudaMemcpyAsync(in.fimg, b->fimg, (size_t)n * P * sizeof(float2), cudaMemcpyHostToDevice, cs));
    if (b->fimg_nomask)
        T2B_CUDA(cudaMemcpyAsync(in.fimg_nm, b->fimg_nomask, (size_t)n * P * sizeof(float2), cudaMemcpyHostToDevice, cs));
    T2B_CUDA(cudaMemcpyAsync(in.ctf, b->ctf, (size_t)n * P * sizeof(float), cudaMemcpyHostToDevice, cs));
    T2B_CUDA(cudaMemcpyAsync(in.minv, b->minvsigma2, (size_t)n * P * sizeof(float), cudaMemcpyHostToDevice, cs));
    T2B_CUDA(cudaMemcpyAsync(in.scal, b->scalars, (size_t)n * 8 * sizeof(double), cudaMemcpyHostToDevice, cs));
    T2B_CUDA(cudaEventRecord(in.copied, cs));
    T2B_CUDA(cudaStreamWaitEvent(st, in.copied, 0));
    T2B_CUDA(cudaStreamWaitEvent(st, in.done, 0));
    // the batch computation itself: a replayed graph unless stage timing is on
    const bool graph = c->cfg.use_graph && !c->stage_timing;
    if (graph) {
        const std::vector<const void*> key = {(const void*)(intptr_t)n, (const void*)st, (const void*)w.fimg_nm,
                                              (const void*)(intptr_t)(c->net && c->net->enabled ? c->net->kprop : 0)};
        c->last_kernels = replay_graph(c, w, st, key, in.g);
    } else {
        enqueue_estep(c, w, st, true, true);
        c->last_kernels = -1;
    }
    T2B_CUDA(cudaEventRecord(in.consumed, st));
    T2B_CUDA(cudaStreamWaitEvent(ds, in.consumed, 0));
    const int K = c->tb.K, half = c->cfg.ori_size / 2 + 1;
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        if (dst) T2B_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ds));
    };
    d2h(r->min_diff2, w.r_min, n * sizeof(double));
    d2h(r->sum_weight, w.r_sum, n * sizeof(double));
    d2h(r->sig_weight, w.r_sig, n * sizeof(double));
    d2h(r->coarse_sum_weight, w.r_csum, n * sizeof(double));
    d2h(r->coarse_sig_weight, w.r_csig, n * sizeof(double));
    d2h(r->nr_sign, w.r_nsign, n * sizeof(long long));
    d2h(r->n_coarse_sig, w.r_ncsig, n * sizeof(long long));
    d2h(r->pmax, w.r_pmax, n * sizeof(double));
    d2h(r->pose, w.r_pose, n * 5 * sizeof(int));
    d2h(r->wsum_norm, w.r_norm, n * sizeof(double));
    d2h(r->sumw, w.r_sumw, n * sizeof(double));
    d2h(r->wsum_sigma2_offset, w.r_sig_off, n * sizeof(double));
    d2h(r->wsum_sigma2, w.r_sigma2, (size_t)n * half * sizeof(double));
    d2h(r->wsum_pdf_class, w.r_pdf_class, (size_t)n * K * sizeof(double));
    d2h(r->wsum_pdf_dir, w.r_pdf_dir, (size_t)n * K * c->tb.n_dir * sizeof(double));
    d2h(r->status, w.status, n * sizeof(int));
    d2h(r->learned, w.r_learned, n * sizeof(int));
    d2h(r->audit_mass, w.r_audit, n * sizeof(double));
    d2h(r->wsum_scale_xa, w.r_xa, n * sizeof(double));
    d2h(r->wsum_scale_aa, w.r_aa, n * sizeof(double));
    T2B_CUDA(cudaEventRecord(in.done, ds));
    c->last_n = n;
    return c->submitted++;
}

// Block until the batch of `ticket` (every batch when ticket < 0) is done.
static void wait_host(t2b_ctx* c, long long ticket)
{
    cudaEvent_t ev = nullptr;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        T2B_REQUIRE(ticket < c->submitted, T2B_ERR_ARG, "no batch was submitted with this ticket");
        if (ticket >= 0) ev = c->in[ticket & 1].done;
    }
    DeviceGuard g(c->device);
    // a slot's event recorded again by a later batch completes after this one: stream order
    if (ev) T2B_CUDA(cudaEventSynchronize(ev));
    else {
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        T2B_CUDA(cudaStreamSynchronize(c->d2h_stream));
    }
}

}  // namespace t2b

extern "C" {

int t2b_estep_batch_host(t2b_ctx* c, const t2b_batch* b, const t2b_result* r)
{
    return guarded([&] {
        check_batch(c, b, r);
        long long ticket;
        {
            std::lock_guard<std::mutex> lk(c->mu);
            DeviceGuard g(c->device);
            ticket = submit_host(c, b, r);
        }
        wait_host(c, ticket);
        std::lock_guard<std::mutex> lk(c->mu);
        collect_stage_ms(c);
    });
}

int t2b_estep_submit_host(t2b_ctx* c, const t2b_batch* b, const t2b_result* r, long long* ticket)
{
    return guarded([&] {
        check_batch(c, b, r);
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        const long long t = submit_host(c, b, r);
        if (ticket) *ticket = t;
    });
}

int t2b_estep_wait(t2b_ctx* c, long long ticket)
{
    return guarded([&] {
        T2B_REQUIRE(c, T2B_ERR_ARG, "null argument");
        wait_host(c, ticket);
    });
}

int t2b_estep_batch_device(t2b_ctx* c, const t2b_batch* b, const t2b_result* r, void* stream)
{
    return guarded([&] {
        check_batch(c, b, r);
        T2B_REQUIRE(r->min_diff2 && r->sum_weight && r->sig_weight && r->coarse_sum_weight && r->coarse_sig_weight &&
                        r->nr_sign && r->n_coarse_sig && r->pmax && r->pose && r->wsum_norm && r->sumw &&
                        r->wsum_sigma2_offset && r->wsum_sigma2 && r->wsum_pdf_class && r->wsum_pdf_dir && r->status,
                    T2B_ERR_ARG, "the device variant needs every result array");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
        // the batch shares the context's workspace with host batches still in flight on the
        // context's stream: the caller's stream waits for them, and they for it
        const bool other = st != c->stream;
        if (other) {
            T2B_CUDA(cudaEventRecord(c->handoff[0], c->stream));
            T2B_CUDA(cudaStreamWaitEvent(st, c->handoff[0], 0));
        }
        Work w = c->wk;
        w.n = b->n;
        w.fimg = (const float2*)b->fimg;
        w.fimg_nm = (const float2*)(b->fimg_nomask ? b->fimg_nomask : b->fimg);
        w.ctf = b->ctf;
        w.minv = b->minvsigma2;
        w.scal = b->scalars;
        w.r_min = r->min_diff2; w.r_sum = r->sum_weight; w.r_sig = r->sig_weight;
        w.r_csum = r->coarse_sum_weight; w.r_csig = r->coarse_sig_weight; w.r_pmax = r->pmax;
        w.r_nsign = r->nr_sign; w.r_ncsig = r->n_coarse_sig; w.r_pose = r->pose;
        w.r_norm = r->wsum_norm; w.r_sumw = r->sumw; w.r_sig_off = r->wsum_sigma2_offset;
        w.r_sigma2 = r->wsum_sigma2; w.r_pdf_class = r->wsum_pdf_class; w.r_pdf_dir = r->wsum_pdf_dir;
        w.status = r->status;
        w.r_learned = r->learned;
        w.r_audit = r->audit_mass;
        w.r_xa = r->wsum_scale_xa;
        w.r_aa = r->wsum_scale_aa;
        if (c->cfg.use_graph) {
            const std::vector<const void*> key = {(const void*)(intptr_t)b->n, b->fimg, b->fimg_nomask, b->ctf,
                                                  b->minvsigma2, b->scalars, r->min_diff2, r->sum_weight, r->sig_weight,
                                                  r->coarse_sum_weight, r->coarse_sig_weight, r->nr_sign,
                                                  r->n_coarse_sig, r->pmax, r->pose, r->wsum_norm, r->sumw,
                                                  r->wsum_sigma2_offset, r->wsum_sigma2, r->wsum_pdf_class,
                                                  r->wsum_pdf_dir, r->status, r->learned, r->audit_mass,
                                                  r->wsum_scale_xa, r->wsum_scale_aa, (const void*)st,
                                                  (const void*)(intptr_t)(c->net && c->net->enabled ? c->net->kprop : 0)};
            c->last_kernels = replay_graph(c, w, st, key, c->g_dev);
        } else {
            enqueue_estep(c, w, st, true, true);
            c->last_kernels = -1;
        }
        if (other) {
            T2B_CUDA(cudaEventRecord(c->handoff[1], st));
            T2B_CUDA(cudaStreamWaitEvent(c->stream, c->handoff[1], 0));
        }
        c->last_n = b->n;
    });
}

int t2b_autotune(t2b_ctx* c, const t2b_batch* b, t2b_tune_report* rep)
{
    return guarded([&] {
        T2B_REQUIRE(c && b && rep, T2B_ERR_ARG, "null argument");
        T2B_REQUIRE(c->configured, T2B_ERR_STATE, "t2b_configure must be called before t2b_autotune");
        T2B_REQUIRE(b->n >= 1 && b->n <= c->cfg.max_batch, T2B_ERR_ARG, "batch size out of range");
        T2B_REQUIRE(b->fimg && b->ctf && b->minvsigma2 && b->scalars, T2B_ERR_ARG, "missing batch inputs");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        c->quiesce();   // the tuning batches use slot 0's buffers
        cudaStream_t st = c->stream;
        Work w = c->wk;
        const int n = b->n, P = c->tb.P, K = c->tb.K;
        w.n = n;
        T2B_CUDA(cudaMemcpyAsync((void*)w.fimg, b->fimg, (size_t)n * P * sizeof(float2), cudaMemcpyHostToDevice, st));
        if (b->fimg_nomask)
            T2B_CUDA(cudaMemcpyAsync((void*)w.fimg_nm, b->fimg_nomask, (size_t)n * P * sizeof(float2),
                                     cudaMemcpyHostToDevice, st));
        else
            w.fimg_nm = w.fimg;
        T2B_CUDA(cudaMemcpyAsync((void*)w.ctf, b->ctf, (size_t)n * P * sizeof(float), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemcpyAsync((void*)w.minv, b->minvsigma2, (size_t)n * P * sizeof(float), cudaMemcpyHostToDevice, st));
        T2B_CUDA(cudaMemcpyAsync((void*)w.scal, b->scalars, (size_t)n * 8 * sizeof(double), cudaMemcpyHostToDevice, st));
        // the tuning batches backproject like real ones: keep the grids and put them back after
        std::vector<void*> saved;
        struct Restore {
            t2b_ctx* c;
            std::vector<void*>& saved;
            ~Restore()
            {
                for (size_t k = 0; k < saved.size() / 2; k++) {
                    const size_t nv = (size_t)c->gvol[k].xdim * c->gvol[k].ydim * c->gvol[k].zdim;
                    if (saved[2 * k]) cudaMemcpy(c->gdata[k], saved[2 * k], nv * sizeof(float2), cudaMemcpyDeviceToDevice);
                    if (saved[2 * k + 1])
                        cudaMemcpy(c->gweight[k], saved[2 * k + 1], nv * sizeof(float), cudaMemcpyDeviceToDevice);
                    cudaFree(saved[2 * k]);
                    cudaFree(saved[2 * k + 1]);
                }
            }
        } restore{c, saved};
        T2B_CUDA(cudaStreamSynchronize(st));
        for (int k = 0; k < K; k++) {
            const size_t nv = (size_t)c->gvol[k].xdim * c->gvol[k].ydim * c->gvol[k].zdim;
            void *d = nullptr, *wt = nullptr;
            saved.push_back(nullptr);
            saved.push_back(nullptr);
            T2B_CUDA(cudaMalloc(&d, nv * sizeof(float2)));
            saved[2 * k] = d;
            T2B_CUDA(cudaMalloc(&wt, nv * sizeof(float)));
            saved[2 * k + 1] = wt;
            T2B_CUDA(cudaMemcpy(d, c->gdata[k], nv * sizeof(float2), cudaMemcpyDeviceToDevice));
            T2B_CUDA(cudaMemcpy(wt, c->gweight[k], nv * sizeof(float), cudaMemcpyDeviceToDevice));
        }
        // one E-step of the batch with stage events; the faster of two runs (the first also warms)
        auto run = [&](int stage, int stage2) {
            float best = 1e30f;
            for (int rep_i = 0; rep_i < 2; rep_i++) {
                Work wr = w;
                wr.fine_ctas = c->wk.fine_ctas;
                wr.wsum_ctas = c->wk.wsum_ctas;
                enqueue_estep(c, wr, st, true, false);   // full coarse pass; the audit stream is not advanced
                T2B_CUDA(cudaStreamSynchronize(st));
                c->last_kernels = -1;
                collect_stage_ms(c);
                float t = c->stage_ms[stage];
                if (stage2 >= 0 && c->stage_ms[stage2] > 0.f) t += c->stage_ms[stage2];
                best = std::min(best, t);
            }
            return best;
        };
        *rep = t2b_tune_report{};
        // 1. contraction tile: N columns x raster group, timed on the full coarse pass (the
        // audit's full pass of the learned mode runs the same dense tiles with the same group)
        const bool tc = c->cfg.diff2_mode == T2B_DIFF2_SPLIT_BF16;
        const int tns[2] = {256, 128}, groups[4] = {4, 8, 16, 32};
        int best_i = -1;
        for (int i = 0; i < 8; i++) {
            if (!tc) { rep->diff2_ms[i] = -1.f; continue; }
            c->tc.dense_tn = tns[i / 4];
            c->tc.group_m = groups[i % 4];
            rep->diff2_ms[i] = run(2, -1);
            if (best_i < 0 || rep->diff2_ms[i] < rep->diff2_ms[best_i]) best_i = i;
        }
        if (tc) {
            c->tune.dense_tn = c->tc.dense_tn = tns[best_i / 4];
            c->tune.group_m = c->tc.group_m = groups[best_i % 4];
        }
        // 2. fine pass and 3. weighted sums + backprojection: CTAs per SM of the persistent kernels
        int bf = 0, bw = 0;
        for (int k = 1; k <= 4; k++) {
            c->wk.fine_ctas = k;
            rep->fine_ms[k - 1] = c->tb.ovs ? run(4, -1) : -1.f;
            if (c->tb.ovs && (bf == 0 || rep->fine_ms[k - 1] < rep->fine_ms[bf - 1])) bf = k;
        }
        c->tune.fine_ctas = c->wk.fine_ctas = bf ? bf : 4;
        for (int k = 1; k <= 4; k++) {
            c->wk.wsum_ctas = k;
            rep->wsum_ms[k - 1] = run(6, -1);
            if (bw == 0 || rep->wsum_ms[k - 1] < rep->wsum_ms[bw - 1]) bw = k;
        }
        c->tune.wsum_ctas = c->wk.wsum_ctas = bw;
        // 4. projection tile: pixels x orientations per CTA, on the first (up to 16384) rows of
        // the fine (else coarse) table of class 0, rewritten with identical values (chunked
        // configurations have no table: their projections go straight into the operands)
        if (c->tb.chunk) {
            for (int i = 0; i < 9; i++) rep->project_ms[i] = -1.f;
        } else {
            const bool fine = c->tb.ovs;
            const int rows = std::min(16384, fine ? c->tb.O * c->tb.R : c->tb.O);
            float2* out = const_cast<float2*>(fine ? c->tb.proj_f : c->tb.proj_c);
            const double* eul = fine ? c->tb.eul_f : c->tb.eul_c;
            const int pxs[3] = {128, 256, 512}, ors[3] = {1, 2, 4};
            cudaEvent_t e0, e1;
            T2B_CUDA(cudaEventCreate(&e0));
            T2B_CUDA(cudaEventCreate(&e1));
            int bp = -1;
            for (int i = 0; i < 9; i++) {
                float best = 1e30f;
                for (int r = 0; r < 2; r++) {
                    T2B_CUDA(cudaEventRecord(e0, st));
                    launch_project_table(c->mvol[0], c->mdl[0], eul, rows, c->tb.s, out, st, pxs[i / 3], ors[i % 3]);
                    T2B_CUDA(cudaEventRecord(e1, st));
                    T2B_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    T2B_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    best = std::min(best, ms);
                }
                rep->project_ms[i] = best;
                if (bp < 0 || best < rep->project_ms[bp]) bp = i;
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            c->tune.proj_px = pxs[bp / 3];
            c->tune.proj_orients = ors[bp % 3];
        }
        rep->diff2_tn = c->tune.dense_tn;
        rep->diff2_group = c->tune.group_m;
        rep->fine_ctas_per_sm = c->tune.fine_ctas;
        rep->wsum_ctas_per_sm = c->tune.wsum_ctas;
        rep->project_pixels = c->tune.proj_px;
        rep->project_orients = c->tune.proj_orients;
        c->drop_graphs();   // the next batch captures with the chosen shapes
    });
}

int t2b_tune_set(t2b_ctx* c, const t2b_tune_report* shapes)
{
    return guarded([&] {
        T2B_REQUIRE(c && shapes, T2B_ERR_ARG, "null argument");
        T2B_REQUIRE((shapes->diff2_tn == 256 || shapes->diff2_tn == 128) && shapes->diff2_group >= 1 &&
                        shapes->fine_ctas_per_sm >= 1 && shapes->fine_ctas_per_sm <= 4 &&
                        shapes->wsum_ctas_per_sm >= 1 && shapes->wsum_ctas_per_sm <= 4 &&
                        shapes->project_pixels >= 32 && shapes->project_pixels <= 1024 &&
                        shapes->project_pixels % 32 == 0 && shapes->project_orients >= 1 &&
                        shapes->project_orients <= 64,
                    T2B_ERR_ARG, "tile shapes out of range");
        std::lock_guard<std::mutex> lk(c->mu);
        c->tune.dense_tn = c->tc.dense_tn = shapes->diff2_tn;
        c->tune.group_m = c->tc.group_m = shapes->diff2_group;
        c->tune.fine_ctas = c->wk.fine_ctas = shapes->fine_ctas_per_sm;
        c->tune.wsum_ctas = c->wk.wsum_ctas = shapes->wsum_ctas_per_sm;
        c->tune.proj_px = shapes->project_pixels;
        c->tune.proj_orients = shapes->project_orients;
        c->drop_graphs();
    });
}

int t2b_stage_timing(t2b_ctx* c, int on)
{
    return guarded([&] {
        T2B_REQUIRE(c, T2B_ERR_ARG, "null context");
        std::lock_guard<std::mutex> lk(c->mu);
        c->stage_timing = on != 0;
    });
}

int t2b_last_launch_count(t2b_ctx* c, int* kernels)
{
    return guarded([&] {
        T2B_REQUIRE(c && kernels, T2B_ERR_ARG, "bad arguments");
        *kernels = c->last_kernels;
    });
}

int t2b_last_stage_ms(t2b_ctx* c, float* ms, int n)
{
    return guarded([&] {
        T2B_REQUIRE(c && ms && n >= 0 && n <= 9, T2B_ERR_ARG, "bad arguments");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        collect_stage_ms(c);
        for (int i = 0; i < n; i++) ms[i] = c->stage_ms[i];
    });
}

int t2b_debug_coarse_diff2(t2b_ctx* c, int b, float* out)
{
    return guarded([&] {
        T2B_REQUIRE(c && out && c->configured && b >= 0 && b < c->last_n, T2B_ERR_ARG, "bad particle index");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        const size_t n = (size_t)c->tb.K * c->tb.O * c->tb.T;
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        T2B_CUDA(cudaMemcpy(out, c->wk.d2c + (size_t)b * n, n * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

int t2b_debug_proposals(t2b_ctx* c, int b, int* prop, float* diff2, int* kprop)
{
    return guarded([&] {
        T2B_REQUIRE(c && kprop && c->configured && b >= 0 && b < c->last_n, T2B_ERR_ARG, "bad particle index");
        T2B_REQUIRE(c->net && c->net->enabled, T2B_ERR_STATE, "learned proposals are not enabled");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        const int k = c->net->kprop, T = c->tb.T;
        *kprop = k;
        if (prop)
            T2B_CUDA(cudaMemcpy(prop, c->net->prop + (size_t)b * k, k * sizeof(int), cudaMemcpyDeviceToHost));
        if (diff2)
            T2B_CUDA(cudaMemcpy(diff2, c->wk.d2c + (size_t)b * k * T, (size_t)k * T * sizeof(float),
                                cudaMemcpyDeviceToHost));
    });
}

int t2b_debug_fine(t2b_ctx* c, int b, long long* pairs, float* diff2, long long cap, long long* count)
{
    return guarded([&] {
        T2B_REQUIRE(c && count && c->configured && b >= 0 && b < c->last_n, T2B_ERR_ARG, "bad particle index");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        long long off[2];
        T2B_CUDA(cudaMemcpy(off, c->wk.pair_off + b, 2 * sizeof(long long), cudaMemcpyDeviceToHost));
        const long long np = off[1] - off[0];
        *count = np;
        const long long m = std::min(np, cap);
        const int rv = c->tb.ovs ? c->tb.R * c->tb.V : 1;
        if (pairs && m > 0)
            T2B_CUDA(cudaMemcpy(pairs, c->wk.pairs + off[0], m * sizeof(long long), cudaMemcpyDeviceToHost));
        if (diff2 && m > 0 && c->tb.ovs)
            T2B_CUDA(cudaMemcpy(diff2, c->wk.d2f + off[0] * rv, (size_t)m * rv * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

int t2b_debug_weights(t2b_ctx* c, int b, double* weights, long long cap, long long* count)
{
    return guarded([&] {
        T2B_REQUIRE(c && count && c->configured && b >= 0 && b < c->last_n, T2B_ERR_ARG, "bad particle index");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        long long off[2];
        T2B_CUDA(cudaMemcpy(off, c->wk.pair_off + b, 2 * sizeof(long long), cudaMemcpyDeviceToHost));
        const long long rv = c->tb.ovs ? (long long)c->tb.R * c->tb.V : 1;
        const long long nv = (off[1] - off[0]) * rv;
        *count = nv;
        const long long m = std::min(nv, cap);
        if (weights && m > 0)
            T2B_CUDA(cudaMemcpy(weights, c->wk.wf + off[0] * rv, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int t2b_debug_selection(t2b_ctx* c, int b, int* coarse_path, int* fine_path)
{
    return guarded([&] {
        T2B_REQUIRE(c && c->configured && b >= 0 && b < c->last_n, T2B_ERR_ARG, "bad particle index");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        T2B_CUDA(cudaStreamSynchronize(c->stream));
        SelState sc, sf;
        T2B_CUDA(cudaMemcpy(&sc, c->wk.sel_c + b, sizeof(SelState), cudaMemcpyDeviceToHost));
        T2B_CUDA(cudaMemcpy(&sf, c->wk.sel_f + b, sizeof(SelState), cudaMemcpyDeviceToHost));
        if (coarse_path) *coarse_path = sc.fast;
        if (fine_path) *fine_path = c->tb.ovs ? sf.fast : -1;
    });
}

int t2b_reconstruct_divide(t2b_ctx* c, int iclass, double* fconv)
{
    return guarded([&] {
        T2B_REQUIRE(c && fconv && iclass >= 0 && iclass < (int)c->gvol.size() && c->gdata[iclass], T2B_ERR_ARG,
                    "no such grid");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        const Volume& v = c->gvol[iclass];
        T2B_REQUIRE(v.ref_dim == 3, T2B_ERR_UNSUPPORTED, "reconstruction division is implemented for 3D grids");
        const int ps = v.ydim, fx = ps / 2 + 1;
        const size_t total = (size_t)ps * ps * fx;
        double2* fc = nullptr;
        double *fw = nullptr, *rad = nullptr;
        cudaStream_t st = c->stream;
        auto cleanup = [&] { cudaFree(fc); cudaFree(fw); cudaFree(rad); };
        if (cudaMalloc(&fc, total * sizeof(double2)) != cudaSuccess || cudaMalloc(&fw, total * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&rad, 2 * (size_t)v.r_max * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            cleanup();
            throw Error{T2B_ERR_NOMEM, "reconstruction buffers"};
        }
        try {
            launch_reconstruct(v, c->gdata[iclass], c->gweight[iclass], fc, fw, rad, rad + v.r_max, st);
            T2B_CUDA(cudaMemcpyAsync(fconv, fc, total * sizeof(double2), cudaMemcpyDeviceToHost, st));
            T2B_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
            cleanup();
            throw;
        }
        cleanup();
    });
}

int t2b_project(t2b_ctx* c, int iclass, const double* eulers, int n, int current_size, float* out)
{
    return guarded([&] {
        T2B_REQUIRE(c && eulers && out && n > 0 && current_size > 0 && current_size % 2 == 0, T2B_ERR_ARG, "bad arguments");
        T2B_REQUIRE(iclass >= 0 && iclass < (int)c->mvol.size() && c->mdl[iclass], T2B_ERR_ARG, "no such projector");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        const int P = current_size * (current_size / 2 + 1);
        double* de = nullptr;
        float2* dout = nullptr;
        cudaStream_t st = c->stream;
        if (cudaMalloc(&de, (size_t)n * 9 * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&dout, (size_t)n * P * sizeof(float2)) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(de);
            throw Error{T2B_ERR_NOMEM, "projection buffers"};
        }
        try {
            T2B_CUDA(cudaMemcpyAsync(de, eulers, (size_t)n * 9 * sizeof(double), cudaMemcpyHostToDevice, st));
            launch_project_table(c->mvol[iclass], c->mdl[iclass], de, n, current_size, dout, st, c->tune.proj_px,
                                 c->tune.proj_orients);
            T2B_CUDA(cudaMemcpyAsync(out, dout, (size_t)n * P * sizeof(float2), cudaMemcpyDeviceToHost, st));
            T2B_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
            cudaFree(de);
            cudaFree(dout);
            throw;
        }
        cudaFree(de);
        cudaFree(dout);
    });
}

}  // extern "C"
