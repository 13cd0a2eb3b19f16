/*
 * t2b.h - C ABI of the Blackwell (sm_100a) E-step library libt2b.so.
 *
 * The E-step hot path of RELION's MlOptimiser (as accelerated by T2-RELION):
 * Fourier-slice projection of the references, diff2 over every
 * (particle, orientation, translation), conversion to posterior weights with
 * the significance threshold, the adaptive-oversampling fine pass, the
 * weighted sums, backprojection into the padded reconstruction grid and the
 * skip-gridding division of backprojected data by backprojected weights.
 *
 * Conventions
 *  - every function returns T2B_OK (0) or a T2B_ERR_* code; t2b_last_error()
 *    gives the message of the calling thread's last failure.  No C++
 *    exception crosses this boundary.
 *  - the caller owns host buffers; the context owns device buffers.  Device
 *    pointers passed in (the *_device entry points) stay owned by the caller.
 *  - complex arrays are interleaved (re, im) float32.  2D Fourier images are
 *    the windowed FFTW half transform of a current_size x current_size image:
 *    current_size rows x (current_size/2 + 1) columns, pixel n = i*xh + j,
 *    ky = i for i < xh else i - current_size, kx = j.
 *  - 3D model grids use the centred half-complex layout of RELION's Projector:
 *    element (x, y, z) at ((z - initz) * ydim + (y - inity)) * xdim + x.
 *  - one context per device; calls on one context are serialised internally.
 */
#ifndef T2B_H
#define T2B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define T2B_OK 0
#define T2B_ERR_ARG 1        /* invalid argument / size                                  */
#define T2B_ERR_CUDA 2       /* CUDA runtime or driver failure                           */
#define T2B_ERR_NOSIGNIF 3   /* zero sum of weights / no significant sample (ERRNOSIGNIFS,
                                ERRSUMWEIGHTZERO of src/error.h:259-280)                   */
#define T2B_ERR_STATE 4      /* call order (e.g. E-step before t2b_configure)            */
#define T2B_ERR_NOMEM 5      /* device memory or workspace capacity exceeded             */
#define T2B_ERR_TIMEOUT 6    /* a bounded device-side wait ran out                       */
#define T2B_ERR_UNSUPPORTED 7

#define T2B_DIFF2_PLAIN_FP32 0   /* SIMT FP32 cross-term contraction                       */
#define T2B_DIFF2_SPLIT_BF16 1   /* tcgen05 BF16 hi/lo three-product contraction, FP32 acc */

typedef struct t2b_ctx t2b_ctx;

/* Context on CUDA device `device`.  Replaces MlDeviceBundle construction
 * (src/acc/cuda/cuda_ml_optimiser.h:17-72). */
int t2b_create(int device, t2b_ctx** ctx);
void t2b_destroy(t2b_ctx* ctx);
const char* t2b_last_error(void);
/* Library version string. */
const char* t2b_version(void);

/* Reference model of class `iclass` (AccProjector::setMdlDim + initMdl,
 * src/acc/acc_projector.h:69-78).  ref_dim 3: xdim = pad/2+1, ydim = zdim =
 * pad (the padded size of RELION's Projector, src/projector.cpp:55-80);
 * ref_dim 2: zdim = 1.  `mdl` is host memory, complex interleaved. */
int t2b_projector_set(t2b_ctx* ctx, int iclass, int ref_dim, int xdim, int ydim, int zdim,
                      int inity, int initz, int r_max, int padding_factor, const float* mdl);

/* Backprojection grid of class `iclass`, zeroed (AccBackprojector::setMdlDim
 * + initMdl, src/acc/acc_backprojector.h:51-79). */
int t2b_backprojector_init(t2b_ctx* ctx, int iclass, int ref_dim, int xdim, int ydim, int zdim,
                           int inity, int initz, int r_max, int padding_factor);
/* Zero the grid again (AccBackprojector::initMdl). */
int t2b_backprojector_clear(t2b_ctx* ctx, int iclass);
/* Copy grid to host (AccBackprojector::getMdlData, src/acc/acc_backprojector_impl.h:84-100).
 * real/imag/weight each hold xdim*ydim*zdim floats. */
int t2b_backprojector_get(t2b_ctx* ctx, int iclass, float* real, float* imag, float* weight);
/* Device pointers of the grid (AccBackprojector::getMdlDataPtrs): complex
 * interleaved data and weight; for an in-place NCCL reduction. */
int t2b_backprojector_device_ptrs(t2b_ctx* ctx, int iclass, float** data, float** weight);

/* Per-iteration sampling and E-step configuration.  Mirrors what
 * MlOptimiserCuda reads from MlOptimiser / HealpixSampling
 * (src/acc/acc_ml_optimiser_impl.h:2359-2560, src/healpix_sampling.cpp). */
typedef struct t2b_config {
    int ori_size;              /* full box size                                       */
    int current_size;          /* windowed size of both passes (even)                 */
    int ref_dim;               /* 3 (3D refs, 2D particles) or 2 (2D classification)  */
    int nr_classes;
    int n_dir, n_psi;          /* coarse orientations per class = n_dir * n_psi       */
    int n_trans;               /* coarse translations                                 */
    int adaptive_oversampling; /* 0: single pass; 1: coarse + fine pass               */
    int nover_rot, nover_trans;/* oversampling factors of the fine pass (1 if none)   */
    int maximum_significants;  /* > 0: cap of the coarse-pass significant samples (--maxsig) */
    int diff2_mode;            /* T2B_DIFF2_*                                         */
    int max_batch;             /* particles per t2b_estep_* call                      */
    int use_graph;             /* 1: t2b_estep_batch_device captures the batch into a CUDA
                                  graph on first use and replays it                     */
    const double* eul_coarse;  /* n_dir*n_psi x 9, Euler matrices (Euler_angles2matrix) */
    const double* eul_fine;    /* n_dir*n_psi*nover_rot x 9, or NULL                    */
    const double* trans_px;    /* n_trans x 2: coarse shifts in pixels                  */
    const double* trans_px_fine;/* n_trans*nover_trans x 2, or NULL                     */
    const double* trans_prior; /* n_trans x 2: HealpixSampling::translations_{x,y}      */
    const double* pdf_direction;/* nr_classes x n_dir                                   */
    const double* pdf_class;   /* nr_classes                                            */
    const int* mresol;         /* current_size*(current_size/2+1): ring index or -1     */
    double sigma2_offset;
    double pixel_size;
    double adaptive_fraction;
    size_t fine_capacity;      /* fine hypotheses per batch (0: default)                */
    const double* data_vs_prior;/* nr_classes x (ori_size/2+1): mymodel.data_vs_prior_class, or
                                  NULL.  Non-NULL turns on the scale-correction sums
                                  (do_scale_correction): a pixel of ring ires in class k adds to
                                  them when data_vs_prior[k][ires] > 3 (src/ml_optimiser.cpp:
                                  8477-8486)                                             */
    int orientation_chunk;     /* coarse orientations projected and contracted per chunk inside
                                  each batch.  0: automatic -- every projection table resident
                                  (built once here) when the coarse and fine tables and their
                                  split-BF16 operands fit in 60 % of the free device memory,
                                  else chunks of 16384; > 0: chunks of this many rows (at most
                                  nr_classes * n_dir * n_psi).  Chunked: split-BF16 contraction
                                  only, the fine pass and the weighted sums interpolate their
                                  projections from the models on the fly (the same FP64
                                  interpolation, so the same values), no learned proposals.
                                  The reference re-projects every orientation for every
                                  particle (orientation_matrix_handler.cuh:99-126)         */
    int _pad2;
} t2b_config;

/* Validate the configuration, build the projection tables of all coarse and
 * fine orientations and the phase tables, and size the workspace.  The
 * projectors of all classes must be set first. */
int t2b_configure(t2b_ctx* ctx, const t2b_config* cfg);

/* One batch of particles.  Host variant: pointers are host memory.  Device
 * variant: pointers are device memory (already resident). */
typedef struct t2b_batch {
    int n;                      /* particles in this batch (<= max_batch)               */
    int _pad;
    const float* fimg;          /* n x 2P, masked image (FFTW window), complex           */
    const float* fimg_nomask;   /* n x 2P or NULL (then fimg is used)                    */
    const float* ctf;           /* n x P                                                 */
    const float* minvsigma2;    /* n x P, 1/(fudge*sigma2_noise[ires]), 0 outside mask   */
    const double* scalars;      /* n x 8: minvsigma2_dc, highres_Xi2, old_offset x, y,
                                   prior x, y, scale_correction, unused                  */
} t2b_batch;

typedef struct t2b_result {
    double* min_diff2;          /* n: final pass (exp_min_diff2)                        */
    double* sum_weight;         /* n: final pass (exp_sum_weight)                       */
    double* sig_weight;         /* n: final pass (exp_significant_weight)               */
    double* coarse_sum_weight;  /* n                                                    */
    double* coarse_sig_weight;  /* n                                                    */
    long long* nr_sign;         /* n: METADATA_NR_SIGN                                  */
    long long* n_coarse_sig;    /* n: size of Mcoarse_significant                       */
    double* pmax;               /* n: METADATA_PMAX                                     */
    int* pose;                  /* n x 5: iclass, iorient, iover_rot, itrans, iover_trans */
    double* wsum_norm;          /* n: exp_wsum_norm_correction                          */
    double* sumw;               /* n: thr_sumw_group                                    */
    double* wsum_sigma2_offset; /* n                                                    */
    double* wsum_sigma2;        /* n x (ori_size/2+1)                                   */
    double* wsum_pdf_class;     /* n x nr_classes                                       */
    double* wsum_pdf_dir;       /* n x nr_classes*n_dir                                 */
    int* status;                /* n: T2B_OK or T2B_ERR_NOSIGNIF per particle           */
    /* learned proposals (optional, may be NULL; see t2b_proposal_enable) */
    double* audit_mass;         /* n: posterior mass of the full coarse pass held by the
                                   particle's proposals (audited particles), else -1     */
    int* learned;               /* n: 1 if the coarse pass ran on the proposals          */
    /* scale correction (optional, may be NULL; computed when t2b_config.data_vs_prior is set,
       else 0): exp_wsum_scale_correction_XA / _AA of src/ml_optimiser.cpp:8477-8486, 8859-8860
       = sum over significant hypotheses and pixels of w' Re(A conj(X_shift)) and w' |A|^2,
       A = scale CTF P, divided by scale_correction and its square                         */
    double* wsum_scale_xa;      /* n: thr_wsum_signal_product_spectra contribution          */
    double* wsum_scale_aa;      /* n: thr_wsum_reference_power_spectra contribution         */
} t2b_result;

/* E-step of one batch (MlOptimiserCuda::doThreadExpectationSomeParticles,
 * src/acc/cuda/cuda_ml_optimiser.cu:1345-1405, minus image preparation):
 * coarse pass, weights, fine pass, weights, weighted sums, backprojection into
 * the grids of t2b_backprojector_init.  The host variant copies the batch in,
 * runs, and copies the results out before returning.  The device variant only
 * enqueues on `stream` (cudaStream_t, NULL = the context's stream); result
 * pointers are device memory and valid after the stream completes.  Batches of
 * one context run in the order they were enqueued, on whichever entry point and
 * stream (the caller's stream waits for the context's earlier batches, and the
 * context's later batches for it). */
int t2b_estep_batch_host(t2b_ctx* ctx, const t2b_batch* batch, const t2b_result* out);
int t2b_estep_batch_device(t2b_ctx* ctx, const t2b_batch* batch, const t2b_result* out, void* stream);

/* Pipelined host batches (the reference overlaps batches by giving each host thread
 * its own CUDA stream, src/acc/cuda/cuda_ml_optimiser.cu:511-561): submit
 * enqueues what t2b_estep_batch_host does and returns at once with a ticket
 * (0, 1, 2, ... per context).  A batch's inputs are copied in on a copy stream while
 * the previous batch computes, and its results are read back on a third stream while
 * the next one computes; batches run and write their results in submission order.  The batch's host inputs and result arrays must stay valid and untouched
 * until t2b_estep_wait(ctx, ticket) (or a later ticket, or -1 = every batch) returns.
 * t2b_estep_batch_host is submit followed by wait.  The batch's input and result
 * arrays must be pinned host memory (cudaHostAlloc / cudaHostRegister) for batches to
 * overlap: copies from or into pageable memory make the call wait for them. */
int t2b_estep_submit_host(t2b_ctx* ctx, const t2b_batch* batch, const t2b_result* out, long long* ticket);
int t2b_estep_wait(t2b_ctx* ctx, long long ticket);

/* Skip-gridding reconstruction division in FP64 on the device
 * (BackProjector::reconstruct, src/backprojector.cpp:1463-1531).  Output is
 * the FFTW-ordered transform of a pad^3 volume, [pad][pad][pad/2+1] complex
 * double, host memory. */
int t2b_reconstruct_divide(t2b_ctx* ctx, int iclass, double* fconv);

/* M-step reconstruction of a grid on the device (BackProjector::reconstruct,
 * src/backprojector.cpp:1344-1530, on the reference's default skip-gridding
 * path, followed by windowToOridimRealSpace :2486-2620 and
 * Projector::griddingCorrect, src/projector.cpp:489-522): decenter, optional
 * MAP term 1 / (pad^3 tau2_fudge tau2[ires]) on the weights for shells >=
 * minres_map, FP64 division by max(weight, radial average / 1000), window to
 * pad * ori_size, inverse 3D FFT (FP32), real-space window to ori_size,
 * normalisation for 2D particles (pad^3 ori_size), soft mask (radius ori/2,
 * width 3, average background), sinc^2 gridding correction.  vol: host,
 * ori_size^3 doubles [z][y][x] (a 2D grid of 2D classification: ori_size^2,
 * normalisation pad^2), centre at ori_size/2.  pad * ori_size must be
 * a product of 2, 3, 5 and <= 512.  With gridding_iter > 0 (--dont_skip_gridding,
 * src/backprojector.cpp:1532-1655) the division is replaced by the iterative
 * gridding weights of Pipe & Menon: data and weight divided by normalise, weights
 * w = 1 inside ROUND(r_max pad)^2, each iteration convolving w * weight with the
 * blob (radius 3.8, alpha 15) through inverse and forward FFTs of the pad_size box
 * (FP32, shared-memory FFTs of any size) and dividing w by max(1e-6, |result|);
 * Fconv = data * w.  Expects the Hermitian-symmetrised grid
 * (t2b_backprojector_enforce_hermitian), as MlOptimiser::maximization provides it. */
typedef struct t2b_recon_config {
    int ori_size;               /* model box                                       */
    int do_map;                 /* add the inverse tau2 spectrum to the weights    */
    int minres_map;             /* first shell that gets the MAP term              */
    int gridding_iter;          /* 0: skip gridding (the default); > 0: that many
                                   iterations of the gridding weights
                                   (--dont_skip_gridding, gridding_nr_iter, 10 in
                                   the reference; src/backprojector.cpp:1532-1655) */
    double tau2_fudge;
    const double* tau2;         /* ori_size/2+1 (host); required with do_map       */
    double normalise;           /* gridding only: data and weight are divided by it
                                   first (the class's sum of weights, pdf_class;
                                   src/ml_optimiser.cpp:4861-4867)                 */
} t2b_recon_config;
int t2b_reconstruct(t2b_ctx* ctx, int iclass, const t2b_recon_config* cfg, double* vol);

/* Hermitian symmetry of the x = 0 plane of a grid, in place on the device
 * (BackProjector::enforceHermitianSymmetry, src/backprojector.cpp:2104-2121, which
 * MlOptimiser::maximization applies to every class before reconstructing,
 * src/ml_optimiser.cpp:4626): each Friedel pair (z, y, 0) <-> (-z, -y, 0) gets the sum
 * data(z, y) + conj(data(-z, -y)) (conjugated on the partner) and the sum of the two
 * weights.  Linear, so it may run before or after the reduction of the grids over GPUs, but
 * once.  Point-group symmetry follows it (t2b_backprojector_apply_symmetry). */
int t2b_backprojector_enforce_hermitian(t2b_ctx* ctx, int iclass);

/* The operators of a point group other than the identity, 3 x 3 row-major into
 * mats (capacity cap matrices; fewer are written when cap is smaller), their number
 * in *count, as SymList builds them (read_sym_file + compute_subgroup,
 * src/symmetries.cpp:133-191, 243-325, generators of fill_symmetry_class, :606-725): the
 * rotations k 360 / n about each generating axis, transposed; the reflections I - 2 u u^T of
 * mirror planes of normal u; the inversion -I; closed under products in the reference's
 * order, entries below 1e-6 zeroed, matrices equal within 1e-6 taken as one.  Groups, named
 * as the reference reads them (case-insensitive, n of one or two digits): C1, Cn, Ci, Cs, Cnv,
 * Cnh, Sn (n even; C(n/2) x Ci), Dn, Dnv, Dnh, T, Td, Th, O, Oh, I (= I2), I1, I3, I4, Ih
 * (= I2h), I1h, I3h, I4h.  Others (I5, I5h, which the reference does not implement either)
 * return T2B_ERR_UNSUPPORTED, an odd Sn T2B_ERR_ARG.  Orders: Cn n - 1, Dn 2n - 1, Cnv and
 * Cnh 2n - 1, Dnv and Dnh 4n - 1, T 11, Td, Th and O 23, Oh 47, I 59, Ih 119. */
int t2b_point_group(const char* group, double* mats, int cap, int* count);

/* Point-group symmetrisation of a 3D grid, in place on the device
 * (BackProjector::applyPointGroupSymmetry, src/backprojector.cpp:2279-2435, applied by
 * MlOptimiser::maximization after enforceHermitianSymmetry, src/ml_optimiser.cpp:4643):
 * each voxel with x^2 + y^2 + z^2 <= ROUND(r_max pad)^2 gains, for every operator R of the
 * group other than the identity, the grid read at R (x, y, z) by trilinear interpolation
 * (the complex conjugate of the Friedel partner where the rotated x < 0), data and weight
 * alike; not averaged.  Coordinates and sums in FP64, the grid in FP32; all reads come
 * from the grid as it was before the call.  C1 and 2D grids are left unchanged.  Expects
 * the Hermitian-symmetrised grid.  Linear, so it may run before or after the reduction of
 * the grids over GPUs, but once. */
int t2b_backprojector_apply_symmetry(t2b_ctx* ctx, int iclass, const char* group);

/* Helical symmetrisation of a 3D grid, in place on the device
 * (BackProjector::applyHelicalSymmetry, src/backprojector.cpp:2122-2277, applied by
 * MlOptimiser::maximization between enforceHermitianSymmetry and applyPointGroupSymmetry,
 * src/ml_optimiser.cpp:4630): for the asymmetric units hh = -n/2 .. n/2 - 1 (.. n/2 for odd
 * n = nr_asu) other than 0, each voxel inside ROUND(r_max pad)^2 gains the grid read at
 * Rz(-hh twist) (x, y, z) (twist in degrees; entries of the rotation below 1e-6 zeroed) by
 * trilinear interpolation (the conjugate where the rotated x < 0); the data term, when rise
 * (pixels: the reference passes helical_rise / pixel_size) is not 0, times
 * e^{2 pi i z hh rise / (-ori_size pad)}.  FP64 coordinates, phases and sums, FP32 grid; reads
 * from the grid as it was before the call.  nr_asu < 2 and 2D grids: unchanged. */
int t2b_backprojector_apply_helical(t2b_ctx* ctx, int iclass, int nr_asu, double twist, double rise, int ori_size);

/* Fourier shell correlation of two grids (two half-sets) after down-sampling to
 * the unpadded box (BackProjector::getDownsampledAverage +
 * calculateDownSampledFourierShellCorrelation, src/backprojector.cpp:933-1040);
 * fsc: host, ori_size/2+1 doubles, fsc[0] = 1. */
int t2b_fsc_halves(t2b_ctx* ctx, int grid_a, int grid_b, int ori_size, double* fsc);

/* BackProjector::updateSSNRarrays (src/backprojector.cpp:1041-1205) of a grid:
 * tau2 (in/out), sigma2, data_vs_prior and fourier_coverage, ori_size/2+1
 * doubles each (host). */
typedef struct t2b_ssnr_config {
    int ori_size;
    int update_tau2_with_fsc;
    int is_whole_instead_of_half;
    int correct_tau2_by_avgctf2;
    double tau2_fudge;
    const double* fsc;          /* ori_size/2+1, with update_tau2_with_fsc         */
    const double* avgctf2;      /* ori_size/2+1, with correct_tau2_by_avgctf2      */
} t2b_ssnr_config;
int t2b_update_ssnr(t2b_ctx* ctx, int iclass, const t2b_ssnr_config* cfg, double* tau2, double* sigma2,
                    double* data_vs_prior, double* fourier_coverage);

/* Maximum r_max of t2b_reconstruct_divide_noalloc. */
#define T2B_NOALLOC_MAX_RMAX 2048

/* No counterpart in the reference.  The skip-gridding division of
 * t2b_reconstruct_divide for callers that cannot allocate device memory: in a
 * RELION process the GPU arena allocator has already reserved most free device
 * memory, and cudaMalloc/cudaFree would synchronise the whole device under
 * work running on other streams.  Everything is caller-owned device memory:
 * `data` (complex interleaved) and `weight` are a centred 3D grid as returned
 * by t2b_backprojector_device_ptrs (3D only: zdim == ydim, xdim == ydim/2+1);
 * `fconv` receives [ydim][ydim][ydim/2+1] complex doubles in FFTW order, ydim
 * being the padded grid size (pad_size, e.g. 259), not the padding factor.  Enqueued on `stream` (cudaStream_t, NULL = legacy default
 * stream); no cudaMalloc, cudaFree or allocating library call.  Scratch (the
 * radial weight averages) is a fixed device array of 2 * T2B_NOALLOC_MAX_RMAX
 * doubles per device, shared by all calls and cleared by each: calls on one
 * device must not overlap on the GPU.  r_max > T2B_NOALLOC_MAX_RMAX returns
 * T2B_ERR_ARG.  Once per device the scratch address is resolved and the
 * division's kernels are loaded (lazy module loading: device memory for the code
 * and the array, possibly a context synchronisation): t2b_create does this for
 * its device; without a context, the first call on a device does it, so make that
 * call at set-up, before any stream capture and before an arena allocator
 * reserves the device's memory.  The grid must be complete: a context's grid is
 * written by batches on the context's own streams, so wait for them
 * (t2b_estep_wait(ctx, -1), or order `stream` after the context's work) first. */
int t2b_reconstruct_divide_noalloc(const float* data, const float* weight, int xdim, int ydim, int zdim,
                                   int inity, int initz, int r_max, int padding_factor, double* fconv,
                                   void* stream);

/* Projections of `n` orientations (host Euler matrices, n x 9) of class
 * `iclass` on the current_size window (AccProjectorKernel::project3Dmodel,
 * src/acc/acc_projectorkernel_impl.h:179-250); out: host, n x 2P. */
int t2b_project(t2b_ctx* ctx, int iclass, const double* eulers, int n, int current_size, float* out);

/* Inspection of the last batch (test support): coarse diff2 of particle b
 * (nr_classes*n_dir*n_psi*n_trans floats, orientation-major), and the fine
 * pass (pairs: coarse hidden index per significant pair; diff2: pairs x
 * nover_rot*nover_trans).  *count receives the number of pairs. */
int t2b_debug_coarse_diff2(t2b_ctx* ctx, int b, float* out);
int t2b_debug_fine(t2b_ctx* ctx, int b, long long* pairs, float* diff2, long long cap, long long* count);
/* Final-pass weights of particle b in the last batch (FP64, before the division
 * by sum_weight), in the order of t2b_debug_fine's pairs: pairs x
 * nover_rot*nover_trans values with adaptive oversampling, else one per pair
 * (the significant coarse pairs).  *count receives the number of values. */
int t2b_debug_weights(t2b_ctx* ctx, int b, double* weights, long long cap, long long* count);
/* Which significance search decided particle b's coarse and fine pass in the last batch:
 * 2 = one CTA per particle (<= 8192 hypotheses), 1 = the multi-kernel search whose
 * crossing-bin candidates were gathered by the fast path, 0 = the multi-kernel radix
 * search with its finer histogram levels.  fine_path is -1 without adaptive oversampling. */
int t2b_debug_selection(t2b_ctx* ctx, int b, int* coarse_path, int* fine_path);
/* Learned proposals of particle b in the last batch (valid where that batch's
 * `learned` result is 1): *kprop receives the proposals per particle; prop
 * (kprop ints, may be NULL) their orientation indices k*n_dir*n_psi + o, and
 * diff2 (kprop x n_trans floats, may be NULL) their coarse diff2. */
int t2b_debug_proposals(t2b_ctx* ctx, int b, int* prop, float* diff2, int* kprop);

/* Tile-shape autotuner (no counterpart in the reference; the reference's
 * kernels have fixed tile shapes).  Times candidate shapes on the caller's
 * batch (host buffers, as t2b_estep_batch_host) with CUDA events and keeps the
 * fastest of each for later batches and configurations:
 *   contraction tile of the dense coarse pass: N = 256 or 128 columns x raster
 *     groups of 4, 8, 16, 32 orientation tiles (diff2_ms[i]: N = 256 for i < 4);
 *   fine pass and weighted sums + backprojection: 1..4 persistent CTAs per SM;
 *   projection tile: 128, 256, 512 pixels x 1, 2, 4 orientations per CTA
 *     (project_ms[3 * ipx + ior]), on up to 16384 table rows.
 * None of the shapes changes a value the E-step computes (the backprojection's
 * FP32 atomics aside, whose order is never fixed).  The grids are restored
 * after the tuning batches; the learned proposals and their audit stream are
 * not used.  A few seconds at the box-128 workload.  t2b_tune_set installs
 * shapes directly (e.g. from an earlier run). */
typedef struct t2b_tune_report {
    int diff2_tn, diff2_group;              /* chosen shapes                                */
    int fine_ctas_per_sm, wsum_ctas_per_sm;
    int project_pixels, project_orients;
    float diff2_ms[8];                      /* coarse contraction per candidate (-1: n/a)   */
    float fine_ms[4], wsum_ms[4];           /* per CTAs-per-SM 1..4 (-1: no fine pass)      */
    float project_ms[9];
} t2b_tune_report;
int t2b_autotune(t2b_ctx* ctx, const t2b_batch* batch, t2b_tune_report* report);
int t2b_tune_set(t2b_ctx* ctx, const t2b_tune_report* shapes);

/* Kernel launches of the last batch: the kernel nodes of its CUDA graph that run
 * every time (the bodies of its conditional nodes, the multi-kernel selection that
 * runs only for particles with more hypotheses than one CTA selects, are not
 * counted); -1 when the last batch did not run as a graph.  With use_graph set,
 * both entry points replay a graph captured once per batch shape. */
int t2b_last_launch_count(t2b_ctx* ctx, int* kernels);
/* on != 0: host batches run uncaptured and record the per-stage events of
 * t2b_last_stage_ms (measurement support); 0 (default): graph replay. */
int t2b_stage_timing(t2b_ctx* ctx, int on);

/* Device time of the stages of the last batch, in ms (CUDA events on the
 * stream the stages ran on): [0] prep (+ proposal network), [1] tensor-core
 * operand split (+ proposal audit) + norms, [2] coarse diff2 contraction (on the
 * proposals when they are in use), [3] coarse weights + significance + compaction,
 * [4] fine pass, [5] fine weights, [6] weighted sums + backprojection; with
 * learned proposals also [7] the audit's full coarse contraction and [8] the
 * contraction on the proposals alone (-1 otherwise).  n <= 9.
 * A batch that ran as a CUDA graph reports -1 for every stage. */
int t2b_last_stage_ms(t2b_ctx* ctx, float* ms, int n);

/* ---------------------------------------------------------------------------
 * Learned orientation proposals (no counterpart in the reference).
 *
 * A network (8 lowest Fourier rings -> 16x16 image -> 2 conv + 3 dense layers,
 * BF16 weights, FP32 accumulation) ranks the nr_classes*n_dir*n_psi coarse
 * orientations of each particle (optionally followed by an exact
 * low-resolution rescoring of its best candidates); with proposals enabled the
 * coarse pass runs on the top-k of each particle only and every later stage is
 * unchanged.
 * Every `audit_every`-th particle also gets the full coarse pass; if the
 * proposals of an audited particle hold less than `audit_mass` of its coarse
 * posterior, the whole batch runs the full coarse pass instead (decided on the
 * device, inside the same launch sequence / CUDA graph).  Requires
 * diff2_mode T2B_DIFF2_SPLIT_BF16 and nr_classes*n_dir*n_psi <= 49152.
 * The network survives t2b_configure while nr_classes*n_dir*n_psi is
 * unchanged; enabling must be repeated after every t2b_configure.
 * ------------------------------------------------------------------------- */
typedef struct {
    int n_train;                /* synthetic training particles (e.g. 200000)              */
    int n_posterior;            /* of those, labelled with the plain E-step posterior too  */
    int n_val;                  /* held-out particles for the report                       */
    int epochs, batch;          /* Adam epochs, minibatch (8..1024)                        */
    float lr;                   /* Adam learning rate                                      */
    int topk;                   /* proposals per particle for the report                   */
    int rescore;                /* network candidates rescored at low resolution for the
                                   report's *_rescored figures (0: not measured)           */
    unsigned long long seed;
    double defocus_min, defocus_max, astig_max;   /* Angstrom                              */
    double voltage, cs, q0;     /* kV, mm, amplitude contrast                              */
    double max_shift;           /* pixels, uniform in [-max_shift, max_shift]^2            */
    double sigma_deg;           /* width of the geometric target around the true pose (8)  */
    float alpha;                /* logit scale of the matched-filter initialisation (3)    */
    const float* minvsigma2;    /* host, window (current_size x current_size/2+1): noise
                                   model of the synthetic particles (1/sigma^2 per complex
                                   component; 0 = no noise)                                */
} t2b_proposal_train_config;

typedef struct {
    double loss[64];            /* mean training loss per epoch (first 64 epochs)          */
    double val_mass_init;       /* mean posterior mass in the top-k of the initial network
                                   (the matched filter of the references) before training */
    double val_mass_trained;    /* ... after training                                      */
    double val_mass_min;        /* smallest after training                                 */
    double val_frac_999;        /* held-out particles with >= 0.999 of the mass in top-k   */
    double val_true_hit;        /* held-out particles whose true orientation is in top-k   */
    double val_mass_rescored;   /* mean mass in the top-k after low-resolution rescoring   */
    double val_mass_min_rescored;
    double val_frac_999_rescored;
    double val_frac_999_candidates; /* ... particles whose `rescore` network candidates hold >= 0.999 */
    double gen_ms, label_ms, train_ms;
    long long params;           /* network parameters                                      */
} t2b_proposal_report;

/* Generate the training set from the current references (projection, CTF,
 * shift, noise), label it (true orientation; plain E-step posterior for
 * n_posterior particles, which does not touch the backprojection grids),
 * train with Adam on the device, and report the held-out posterior mass the
 * top-k proposals hold before and after training.  Needs t2b_configure. */
int t2b_proposal_train(t2b_ctx* ctx, const t2b_proposal_train_config* cfg, t2b_proposal_report* report);
/* Enable (topk >= 1) or disable (topk = 0) proposals for the following batches.
 * rescore > 0: the network's top `rescore` orientations are rescored by the
 * exact low-resolution posterior (the coarse diff2 over the network's ring
 * pixels, with the particle's CTF, noise model and every translation) and the
 * best `topk` of them are the proposals; rescore = 0: the network's top-k. */
int t2b_proposal_enable(t2b_ctx* ctx, int topk, int rescore, int audit_every, double audit_mass);
/* Network parameters as one flat FP32 vector (count: its length, layout in
 * t2-relion_b200/proposal.py); get and/or set (NULL to skip); `set` also marks
 * the network as trained. */
int t2b_proposal_params(t2b_ctx* ctx, float* get, const float* set, long long* count);
/* Feature images (n x 256) of a host batch. */
int t2b_proposal_features(t2b_ctx* ctx, const t2b_batch* batch, float* imgs);
/* Logits (n x nr_classes*n_dir*n_psi, bias included) of host feature images
 * through the inference path (tensor-core dense layers). */
int t2b_proposal_logits(t2b_ctx* ctx, const float* imgs, int n, float* logits);
/* Loss (mean over the n samples) and its gradient with respect to every
 * parameter (count floats) through the training kernels; targets: n x 9
 * (orientation, weight) pairs, weights of a sample summing to 1, orientation
 * -1 = unused.  Parameters are not updated. */
int t2b_proposal_grad(t2b_ctx* ctx, const float* imgs, const int* tgt_oc, const float* tgt_w, int n, double* loss,
                      float* grad);

/* ---------------------------------------------------------------------------
 * Image preparation: real-space particles -> the t2b_batch inputs, on the device.
 *
 * MlOptimiser::getFourierTransformsAndCtfs (src/ml_optimiser.cpp:5689-6390;
 * accelerated counterpart src/acc/acc_ml_optimiser_impl.h:96-1030) for 2D
 * particle images, and the Minvsigma2 image of
 * precalculateShiftedImagesCtfsAndInvSigma2s (src/ml_optimiser.cpp:6680-6720):
 * norm correction, rounded old offset as an integer shift with zero fill,
 * the unmasked and the soft-masked image (average or noise background)
 * Fourier transformed (forward divided by N^2), windowed to current_size and
 * centred by sign, the masked image's power spectrum and highres_Xi2, the CTF
 * image (CTF::getFftwImage without padding) and Minvsigma2.  One optics group
 * per configuration; no helical, multi-body or subtomogram paths.
 * The noise background has the reference's spectrum but its own
 * counter-based generator (seed random_seed + part_id): the reference's
 * rand() / curand draws are not reproducible across thread schedules.
 * ------------------------------------------------------------------------- */
typedef struct t2b_prep_config {
    int image_size;             /* N: particle box (even, a product of 2, 3, 5; 8..512)   */
    int current_size;           /* s: window handed to the E-step (even, <= N)            */
    int max_batch;              /* particles per call                                     */
    int zero_mask;              /* 1: average background outside the mask (--zero_mask);
                                   0: noise background of spectrum sigma2_noise           */
    int random_seed;            /* noise of a particle: random_seed + its part_id         */
    int do_norm_correction;
    int do_ctf_correction;
    int ctf_premultiplied;      /* CTF image squared                                      */
    int ctf_phase_flipped;      /* |CTF| (do_abs)                                          */
    int only_flip_phases;       /* sign of the CTF                                        */
    int intact_ctf_first_peak;  /* 1 until the first peak                                 */
    int n_sigma2;               /* length of sigma2_noise (model ori_size/2 + 1)          */
    const double* sigma2_noise; /* mymodel.sigma2_noise[optics_group], host               */
    double pixel_size;          /* Angstrom per pixel of the particles                    */
    double mask_radius;         /* pixels: particle_diameter / (2 pixel_size)             */
    double width_mask_edge;     /* pixels                                                 */
    double avg_norm_correction;
    double sigma2_fudge;
    double remap_noise;         /* (image_size*pixel_size) / (ori_size*model pixel size)  */
    double remap_minv;          /* (ori_size*model pixel size) / (image_size*pixel_size)  */
    double voltage, cs, q0;     /* optics group: kV, mm, amplitude contrast               */
} t2b_prep_config;

/* Per-particle parameters, T2B_PREP_NPARAM doubles each: old offset x, y
 * (METADATA_XOFF/YOFF, pixels), offset prior x, y (999 = none), METADATA_NORM,
 * defocus U, V (Angstrom), defocus angle (deg), CTF B-factor, CTF scale
 * (k-factor), phase shift (deg), scale correction (mymodel.scale_correction). */
#define T2B_PREP_NPARAM 12

typedef struct t2b_prep_batch {
    int n;                      /* particles (<= max_batch)                               */
    int _pad;
    const float* images;        /* n x N x N real space, row-major, centre at (N/2, N/2)  */
    const double* params;       /* n x T2B_PREP_NPARAM                                    */
    const long long* part_id;   /* n (noise seeds; may be NULL with zero_mask)            */
} t2b_prep_batch;

typedef struct t2b_prep_out {   /* P = s*(s/2+1); layouts of t2b_batch                    */
    float* fimg;                /* n x 2P masked image                                    */
    float* fimg_nomask;         /* n x 2P unmasked image                                  */
    float* ctf;                 /* n x P                                                  */
    float* minvsigma2;          /* n x P                                                  */
    double* scalars;            /* n x 8: t2b_batch.scalars                               */
    double* power;              /* n x (N/2+1) power spectrum of the masked image
                                   (exp_power_img), or NULL                              */
} t2b_prep_out;

/* Upload the per-iteration state (noise spectrum, optics) and size the workspace. */
int t2b_prep_configure(t2b_ctx* ctx, const t2b_prep_config* cfg);
/* Host variant: host buffers in and out, returns when done.  Device variant:
 * device buffers, enqueued on `stream` (cudaStream_t, NULL = the context's). */
int t2b_prep_batch_host(t2b_ctx* ctx, const t2b_prep_batch* batch, const t2b_prep_out* out);
int t2b_prep_batch_device(t2b_ctx* ctx, const t2b_prep_batch* batch, const t2b_prep_out* out, void* stream);

/* ---------------------------------------------------------------------------
 * On-disk formats of real data (host code, no GPU).
 *
 * MRC image stacks (src/rwMRC.h): modes 0 (int8), 1 (int16), 2 (float32),
 * 6 (uint16), 12 (half); byte-swapped files are recognised as the reference
 * does; the pixel size is cella.x / mx.  t2b_mrc_read converts sections
 * [first, first + count) of a stack (nx * ny floats each) to float;
 * t2b_mrc_write writes mode 2.
 *
 * STAR metadata (MetaDataTable::read, src/metadata_table.cpp:959-1262): one
 * data block (the first, or data_<block>), a loop_ table or label-value pairs;
 * values are kept as text (t2b_star_value) or converted to numbers column by
 * column (t2b_star_column).  Labels are given without the leading '_'.
 * t2b_star_write writes a numeric loop_ block (append: after the file's blocks).
 * ------------------------------------------------------------------------- */
int t2b_mrc_info(const char* path, int* nx, int* ny, int* nz, int* mode, double* pixel_size);
int t2b_mrc_read(const char* path, long long first, long long count, float* out);
int t2b_mrc_write(const char* path, const float* data, int nx, int ny, int nz, double pixel_size);

typedef struct t2b_star t2b_star;
int t2b_star_open(const char* path, const char* block, t2b_star** table);
int t2b_star_shape(const t2b_star* table, long long* rows, int* cols);
int t2b_star_label(const t2b_star* table, int col, char* buf, int cap);
int t2b_star_column(const t2b_star* table, const char* label, double* out);
int t2b_star_value(const t2b_star* table, const char* label, long long row, char* buf, int cap);
void t2b_star_close(t2b_star* table);
int t2b_star_write(const char* path, const char* block, int ncols, const char* const* labels, long long nrows,
                   const double* values, int append);

/* Host sampling (HealpixSampling, src/healpix_sampling.cpp:534-640,
 * 1787-2040), C1 symmetry, no perturbation.  Fills Euler matrices of the
 * coarse orientations (idir*n_psi + ipsi), of the fine orientations
 * ((idir*n_psi + ipsi)*nover_rot + iover_rot), the coarse/fine translations
 * (pixels) and the prior translations (Angstrom).  Query sizes with NULL
 * outputs.  ref_dim 2 gives in-plane (psi-only) sampling. */
int t2b_sampling(int ref_dim, int healpix_order, double psi_step, int adaptive_oversampling,
                 double offset_range_px, double offset_step_px, double pixel_size,
                 int* n_dir, int* n_psi, int* n_trans, int* nover_rot, int* nover_trans,
                 double* eul_coarse, double* eul_fine, double* trans_px, double* trans_px_fine,
                 double* trans_prior, double* angles_coarse /* n_dir*n_psi x 3: rot tilt psi */);

#ifdef __cplusplus
}
#endif
#endif /* T2B_H */
