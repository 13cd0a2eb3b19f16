// Internal declarations of libt2b (sm_100a E-step).  Not part of the ABI.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>
#include "../../include/t2b.h"

namespace t2b {

struct ProposalNet;
struct ImagePrep;

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);

struct Error {
    int code;
    std::string msg;
};

#define T2B_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            throw ::t2b::Error{T2B_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define T2B_REQUIRE(cond, code, msg)                                                         \
    do {                                                                                     \
        if (!(cond)) throw ::t2b::Error{(code), (msg)};                                      \
    } while (0)

// Run f, turning exceptions into status codes and the thread's error message.
template <typename F>
inline int guarded(F&& f)
{
    try {
        f();
        return T2B_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return T2B_ERR_NOMEM;
    } catch (const std::exception& e) {
        set_error(e.what());
        return T2B_ERR_ARG;
    }
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        T2B_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// ------------------------------------------------------------- geometry
struct Volume {           // projector model or backprojection grid
    int ref_dim = 0, xdim = 0, ydim = 0, zdim = 0, inity = 0, initz = 0, r_max = 0, pad = 0;
    size_t nvox() const { return (size_t)xdim * ydim * zdim; }
};

// Per-particle state of the radix significance search (FP64 weights).
struct SelState {
    double target;            // adaptive_fraction * sum of weights
    double cum_above;         // sum of the weights above the current prefix bin
    unsigned long long count_above;
    unsigned long long prefix;
    int shift;                // bits below the current prefix
    int phase;                // 0 searching, 1 gather, 2 done, 3 failed
    long long ncand;
    double thr;
    long long nr_sign;
    unsigned long long maxbits;
    long long argmax;
    int fast;                 // selected by the fast path
};

constexpr int HIST_BINS = 4096;  // 12-bit digits
constexpr int CAND_CAP = 4096;   // candidates sorted in shared memory
constexpr int FAST_CAP = 4096;   // weights gathered by the fast selection path

// Device views of the per-iteration tables.
struct Tables {
    int s, xh, P, ori_size;
    int K, n_dir, n_psi, O, T, R, V, ovs, ref_dim;
    int maxsig;               // maximum_significants of the coarse pass (<= 0: off)
    const float2* proj_c;     // K*O x P
    const float2* proj_f;     // K*O*R x P (ovs) else == proj_c
    const float2* ab_c;       // T x P phase factors
    const float2* ab_f;       // T*V x P
    const double* eul_c;      // O x 9 (A)
    const double* eul_f;      // O*R x 9
    const double* trans_c;    // T x 2 pixel shifts
    const double* trans_f;    // T*V x 2
    const double* trans_prior;// T x 2
    const double* pdf_o;      // K*n_dir, normalised
    const unsigned char* skip;// K*O: orientation not evaluated (pdf <= 0)
    const double* pdf_oc;     // K*O: normalised pdf_orientation of each orientation
    const int* mresol;        // P
    const int* kpix;          // nk: window pixels inside the projection radius (the only
    int nk;                   //     pixels whose projection, hence contraction term, can be non-zero)
    double sigma2_offset, pixel_size, adaptive_fraction;
    double lpo_min, lpo_max;  // extremes of log(pdf_o) over evaluated orientations
    const unsigned char* scl_ring; // K x (ori_size/2+1): ring enters the scale-correction sums
                                   // (data_vs_prior > 3), or nullptr: do_scale_correction off
    int chunk;                // > 0: coarse orientations in chunks of this many rows (proj_c holds one
                              // chunk, proj_f is null: fine and weighted-sum projections on the fly)
    const unsigned long long* mtex; // K: texture objects over the models' 3D arrays (on-the-fly
                                    // projection, project_pixel.cuh)
    const Volume* mvol;       // K: their geometry
};

// Device views of the batch workspace.
struct Work {
    int n;                    // particles in the batch
    const float2* fimg;       // n x P
    const float2* fimg_nm;    // n x P
    const float* ctf;         // n x P
    const float* minv;        // n x P
    const double* scal;       // n x 8
    float2* cvec;             // n x P  (M * s * ctf * X)
    float* w2;                // n x P  (0.5 * M * s^2 * ctf^2)
    float* c0;                // n      (Xi2/2 + sum 0.5 M |X|^2)
    float* norms;             // n x K*O
    float* d2c;               // n x K*O*T
    double* lbound;           // n x 2: min / max of log(pdf_o pdf_t)
    unsigned* minkey_c;       // n
    unsigned* minkey_f;       // n
    double* pdf_t;            // n x T
    double* sum_c;            // n
    double* sum_f;            // n
    SelState* sel_c;          // n
    SelState* sel_f;          // n
    unsigned* hist_cnt;       // n x HIST_BINS
    double* hist_sum;         // n x HIST_BINS
    double* cand;             // n x CAND_CAP
    double* fcand_w;          // n x FAST_CAP: fast-path candidates (weight, index)
    long long* fcand_i;
    double* flist_w;          // n x FAST_CAP: fast-path significant list, index order
    long long* flist_i;
    long long* pairs;         // pair_cap: coarse hidden index of significant pairs
    int* pair_b;              // pair_cap
    long long* pair_off;      // n+1
    long long pair_cap;
    int* chunk_cnt;           // n x max_chunks
    int max_chunks;
    float* d2f;               // pair_cap * R*V
    double* wf;               // pair_cap * R*V (final weights when ovs; coarse gathered otherwise)
    long long* groups;        // pair_cap: first pair of each orientation group
    long long* group_end;     // pair_cap: one past its last pair
    int* group_b;             // pair_cap
    long long* group_off;     // n+1
    unsigned long long* counters; // queue heads etc. (16)
    int* err;                 // device error flag of bounded waits (T2B_ERR_TIMEOUT)
    int* status;              // n
    // learned orientation proposals (gate == nullptr: every orientation is evaluated)
    const int* gate;          // device flag: != 0 while the coarse pass runs on the proposals only
    const int* prop;          // n x kprop: global orientation of each proposal (ranked)
    int kprop;
    int no_bp;                // 1: weighted sums only, the grids are not touched
    int fine_ctas, wsum_ctas; // CTAs per SM of the fine pass and of the weighted sums (0: 4; t2b_autotune)
    int* r_learned;           // n (optional): 1 if the particle's coarse pass used the proposals
    double* r_audit;          // n (optional): posterior mass in the proposals (audited), else -1
    // results (device)
    double *r_min, *r_sum, *r_sig, *r_csum, *r_csig, *r_pmax;
    long long *r_nsign, *r_ncsig;
    int* r_pose;
    double *r_norm, *r_sumw, *r_sig_off, *r_sigma2, *r_pdf_class, *r_pdf_dir;
    double *r_xa, *r_aa;      // n (optional): scale-correction sums XA, AA
};

// ------------------------------------------------------------- kernels
// projection tables (project.cu)
void launch_project_table(const Volume& v, const float2* mdl, const double* eul9, int n, int s,
                          float2* out, cudaStream_t st, int px = 256, int orients = 1);
void launch_phase_table(const double* shifts, int n, int s, int ori_size, float2* out, cudaStream_t st);
// neighbourhood copy of a model (32 bytes per voxel) for the on-the-fly projections
// a model as a 3D array of float2 texels and a point-sampled texture object over it
void make_model_texture(const Volume& v, const float2* mdl, cudaArray_t* arr, cudaTextureObject_t* tex,
                        cudaStream_t st);

// E-step stages (estep.cu)
void estep_init_attributes();
void tc_init_attributes();
void launch_prep(const Tables& tb, const Work& w, cudaStream_t st);
void launch_norms(const Tables& tb, const Work& w, cudaStream_t st);
void launch_diff2_simt(const Tables& tb, const Work& w, cudaStream_t st);
void launch_weights_coarse(const Tables& tb, const Work& w, int maxsig, cudaStream_t st);
void launch_fine(const Tables& tb, const Work& w, cudaStream_t st);
void launch_weights_fine(const Tables& tb, const Work& w, cudaStream_t st);
void launch_wsum_bp(const Tables& tb, const Work& w, const Volume& g, float2* const* grid_data,
                    float* const* grid_weight, cudaStream_t st);
void launch_reconstruct(const Volume& g, const float2* data, const float* weight, double2* fconv,
                        double* fw, double* rad, double* cnt, cudaStream_t st, const double* tau2 = nullptr,
                        double tscale = 1., int minres_map = 0);
// Projector::decenter of a grid with the MAP term (the first step of launch_reconstruct,
// without its division): the gridding iterations' input
void launch_decenter(const Volume& g, const float2* data, const float* weight, double2* fconv, double* fw,
                     double* rad, double* cnt, cudaStream_t st, const double* tau2, double tscale, int minres_map);

// tcgen05 split-BF16 coarse diff2 (diff2_tc.cu)
struct TcOperands {
    void* bh;                 // K*O_pad x Kdim bf16 (projections, hi)
    void* bl;                 // lo
    void* ah;                 // N_pad x Kdim bf16 (shifted images, hi)
    void* al;
    void* nh;                 // K*O_pad x Kn bf16 (|projection|^2, hi)
    void* nl;
    void* wh;                 // B_pad x Kn bf16 (0.5 M (scale CTF)^2, hi)
    void* wl;
    int m_pad, n_pad, kdim;   // padded sizes of the cross-term operands
    int kn, b_pad;            // padded sizes of the norm operands
    void* maps;               // TC_MAP_SLOTS CUtensorMap descriptors (128 B each) in device memory
    int dense_tn = 256;       // N columns of a dense coarse-pass tile (256 or 128; t2b_autotune)
    int group_m = 16;         // orientation tiles per raster group of the dense and audit tiles
    int chunk = 0;            // > 0: the projection operands hold one chunk of this many rows
};
// One chunk of the coarse orientations: rows [row0, row0 + rows) of the K*O layout.
struct RowChunk {
    int row0 = 0, rows = 0;   // rows == 0: every row (the resident operands)
};
constexpr int TC_MAP_SLOTS = 24;
size_t tc_kdim(int nk);
void tc_prepare_projections(const Tables& tb, TcOperands& op, cudaStream_t st);
// resident tables: split rows [0, rows) of tb.proj_c into the projection operands
void tc_split_chunk(const Tables& tb, TcOperands& op, int rows, cudaStream_t st);
// chunked: the projections of `rows` orientations (eul) of one model straight into the operands
void tc_project_split(const Tables& tb, TcOperands& op, cudaTextureObject_t mtex, const Volume& v, const double* eul,
                      int rows, cudaStream_t st);
void tc_split_images(const Tables& tb, const Work& w, TcOperands& op, cudaStream_t st, const int* gate);
void tc_launch_norms(const Tables& tb, const Work& w, TcOperands& op, cudaStream_t st, const int* gate = nullptr,
                     int gate_run = 0, RowChunk ch = RowChunk{}, bool split_w2 = true);
size_t tc_kn(int nk);
void tc_launch_diff2(const Tables& tb, const Work& w, TcOperands& op, cudaStream_t st, const int* gate = nullptr,
                     int gate_run = 0, RowChunk ch = RowChunk{});
bool tc_supported();
void tc_encode(void* ptr, int rows, int kdim, bool a_side, void* out128, int box_rows = 0);
void tc_set_map(TcOperands& op, int slot, void* ptr, int rows, int kdim, bool a_side);
int tc_slot_audit();
int tc_slot_rescore();
void tc_set_map_box(TcOperands& op, int slot, void* ptr, int rows, int kdim, int box_rows);
void tc_launch_rescore(int n, int k1, int T, int kr, TcOperands& op, const float* norms, const unsigned char* skip,
                       const int* cand, const double* pdf_t, const double* pdf_oc, float* score, int* err,
                       cudaStream_t st);
// Pre-swizzled K-blocked operand layout (proposal tiles): bf16 element (row, k) of a
// `rows`-row operand at this element offset; the rows [y, y + n) of k-block k / 64 (y a
// multiple of 8) are n * 128 contiguous bytes in the 128-byte-swizzled K-major layout of
// the tensor cores' shared-memory operand.
__host__ __device__ inline size_t swz_offset(size_t row, int k, size_t rows)
{
    return ((size_t)(k >> 6) * rows + row) * 64 + (size_t)((((k & 63) >> 3) ^ (int)(row & 7)) << 3) + (k & 7);
}
void tc_launch_prop(const Tables& tb, const Work& w, TcOperands& op, int kslot, int tn, const float* nprop,
                    const void* a_hi, const void* a_lo, int a_rows, const void* b_hi, const void* b_lo,
                    float* part, int* fix, int part_tiles, cudaStream_t st);
void tc_split_phases(const Tables& tb, const TcOperands& op, int rows, void* hi, void* lo, cudaStream_t st);
int tc_slot_audit_w2();
void tc_launch_audit_norms(const Tables& tb, TcOperands& op, int na_max, float* norma, int* err, cudaStream_t st);
int tc_audit_narrow_tn(int na_max, int T);
int tc_audit_tn(int na, int T);   // column-tile width of the audit's full variant
int tc_slot_audit_narrow();
void tc_launch_audit(const Tables& tb, TcOperands& op, int na_max, const int* na, const float* c0a,
                     const float* norma, float* d2a, unsigned* minkeya, int* err, cudaStream_t st);
int tc_gemm_raw(const void* maps, int ia, int ib, int M, int N, int K, float* out, int products, int* err,
                cudaStream_t st, int ksplit = 1, int tn = 256);

}  // namespace t2b

namespace t2b {
// Enqueue one E-step of the batch in `w` (api.cu); allow_prop = false forces the
// full coarse pass even while proposals are enabled.
void enqueue_estep(t2b_ctx* c, Work& w, cudaStream_t st, bool stage_events, bool allow_prop);
}

namespace t2b {
void imageprep_release(t2b_ctx* c);   // context destruction (imageprep.cu)
void noalloc_prepare_current_device(); // set-up of t2b_reconstruct_divide_noalloc (noalloc.cu)
}

struct t2b_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::vector<t2b::Volume> mvol;            // per class projector geometry
    std::vector<float2*> mdl;                 // per class device model
    // chunked configurations: the models as 3D arrays, read through the texture path
    std::vector<cudaArray_t> marr;
    std::vector<cudaTextureObject_t> mtex;
    std::vector<t2b::Volume> gvol;            // per class BP grid geometry
    std::vector<float2*> gdata;               // per class grid data
    std::vector<float*> gweight;              // per class grid weight
    void* sym_scratch = nullptr;              // symmetrisation sums of one grid (grown on demand)
    size_t sym_bytes = 0;
    bool configured = false;
    t2b_config cfg{};
    t2b::Tables tb{};
    t2b::Work wk{};
    t2b::TcOperands tc{};
    std::vector<void*> allocs;                // owned device allocations (tables + workspace)
    float2** gd_table = nullptr;              // device table of per-class grid data pointers
    float** gw_table = nullptr;               // device table of per-class grid weight pointers
    int last_n = 0;                           // particles of the last batch
    struct GraphSlot {                        // a captured batch and what it was captured for
        cudaGraphExec_t exec = nullptr;
        std::vector<const void*> key;         // shape / buffers / stream / proposal settings
        int kernels = -1;                     // its kernel nodes
    };
    GraphSlot g_dev;                          // device entry point
    // Host entry points: two staging slots, each with the batch inputs and results.  A
    // batch's inputs are copied into its slot on copy_stream while the previous batch
    // computes on `stream`, and its results leave the slot on d2h_stream while the next one
    // computes; slot 0 is the workspace's own buffers, slot 1 a second set.
    struct InSlot {
        float2* fimg = nullptr;
        float2* fimg_nm = nullptr;
        float* ctf = nullptr;
        float* minv = nullptr;
        double* scal = nullptr;
        double *r_min = nullptr, *r_sum = nullptr, *r_sig = nullptr, *r_csum = nullptr, *r_csig = nullptr,
               *r_pmax = nullptr, *r_norm = nullptr, *r_sumw = nullptr, *r_sig_off = nullptr, *r_sigma2 = nullptr,
               *r_pdf_class = nullptr, *r_pdf_dir = nullptr, *r_audit = nullptr, *r_xa = nullptr, *r_aa = nullptr;
        long long *r_nsign = nullptr, *r_ncsig = nullptr;
        int *r_pose = nullptr, *status = nullptr, *r_learned = nullptr;
        cudaEvent_t copied = nullptr;         // inputs in the slot (copy_stream)
        cudaEvent_t consumed = nullptr;       // the slot's batch has run (stream)
        cudaEvent_t done = nullptr;           // the slot's results are in host memory (d2h_stream)
        GraphSlot g;                          // the captured batch of this slot
    } in[2];
    cudaStream_t copy_stream = nullptr;
    cudaStream_t d2h_stream = nullptr;
    // second branch of a learned step: the audit's contraction beside the proposal inference
    // (fork: recorded after the image preparation; join: after the audit contraction)
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t fork[2]{};
    // Wait for every host batch in flight: its input copies, computation and result reads.
    void quiesce()
    {
        for (cudaStream_t s : {copy_stream, stream, aux_stream, d2h_stream})
            if (s) T2B_CUDA(cudaStreamSynchronize(s));
    }
    long long submitted = 0;                  // host batches submitted: the next ticket
    bool stage_timing = false;                // host batches run uncaptured with stage events
    void drop_graphs()
    {
        for (GraphSlot* g : {&g_dev, &in[0].g, &in[1].g}) {
            if (g->exec) cudaGraphExecDestroy(g->exec);
            g->exec = nullptr;
            g->key.clear();
        }
    }
    int last_kernels = -1;
    cudaEvent_t ev[12]{};                     // 8 stage boundaries + 2 pairs around the proposal-path GEMMs
    cudaEvent_t handoff[2]{};                 // orders a caller's stream after the context's and back
    float stage_ms[9]{};
    bool prop_events = false;                 // the last timed batch recorded ev[8..11]
    t2b::ProposalNet* net = nullptr;          // learned orientation proposals (proposal.cu)
    t2b::ImagePrep* prep = nullptr;           // image preparation state (imageprep.cu)
    struct Tune {                             // tile and launch shapes (t2b_autotune); kept across t2b_configure
        int dense_tn = 256, group_m = 16;     // dense contraction tile: N columns, raster group
        int fine_ctas = 4, wsum_ctas = 4;     // CTAs per SM: fine pass, weighted sums + backprojection
        int proj_px = 256, proj_orients = 1;  // projection tile: pixels x orientations per CTA
    } tune;
};
