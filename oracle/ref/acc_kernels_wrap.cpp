// C wrapper over the reference's own CPU E-step kernels, compiled from the
// reference sources where they lie (oracle/Makefile, target `ref`) into
// oracle/_ref/.  Pins the FP64 oracle's coarse diff2 (projection, phase shift,
// weighted squared difference) to reference-owned code.  Test infrastructure.
//
//   CpuKernels::diff2_coarse<REF3D, !DATA3D>  src/acc/cpu/cpu_kernels/diff2.h:329-606
//   AccProjector / AccProjectorKernel (CPU)  src/acc/acc_projector_impl.h,
//                                            src/acc/acc_projectorkernel_impl.h:563-586
#include <complex>
#include <cstring>
#include <vector>
#include "src/acc/cpu/cpu_kernels/diff2.h"
#include "src/acc/acc_projector_impl.h"

int pin_alloc(void** ptr, size_t size)
{
    *ptr = std::malloc(size);
    return *ptr ? 0 : 1;
}
void pin_free(void* ptr) { std::free(ptr); }

// mdl: complex interleaved float (xdim*ydim*zdim); eulers_inv: O x 9 (A^-1,
// row-major, as generateEulerMatrices(inverse=true)); img_re/img_im: the image
// divided by the CTF; corr: Minvsigma2 * CTF^2; trans: -2 pi shift / ori_size;
// diff2: O x T, initialised here to xi2_half and accumulated by the kernel.
extern "C" int ref_coarse_diff2(const float* mdl, int xdim, int ydim, int zdim, int inity, int initz, int maxr,
                                int pad, const float* eulers_inv, int n_orient, const float* img_re,
                                const float* img_im, const float* corr, int img_x, int img_y,
                                const float* trans_x, const float* trans_y, int n_trans, float xi2_half,
                                float* diff2)
{
    const int epb = D2C_EULERS_PER_BLOCK_REF3D;
    if (n_orient % epb != 0) return 1;
    AccProjector p;
    p.setMdlDim(xdim, ydim, zdim, inity, initz, maxr, (XFLOAT)pad);
    const size_t nvox = (size_t)xdim * ydim * zdim;
    std::complex<XFLOAT>* data = new std::complex<XFLOAT>[nvox];
    for (size_t i = 0; i < nvox; i++) data[i] = std::complex<XFLOAT>(mdl[2 * i], mdl[2 * i + 1]);
    p.initMdl(data);  // shared, freed by the projector
    AccProjectorKernel k = AccProjectorKernel::makeKernel(p, img_x, img_y, 1, img_x - 1);
    std::vector<XFLOAT> e(eulers_inv, eulers_inv + 9 * (size_t)n_orient);
    std::vector<XFLOAT> tx(trans_x, trans_x + n_trans), ty(trans_y, trans_y + n_trans), tz(n_trans, 0.f);
    std::vector<XFLOAT> re(img_re, img_re + (size_t)img_x * img_y), im(img_im, img_im + (size_t)img_x * img_y);
    std::vector<XFLOAT> cr(corr, corr + (size_t)img_x * img_y);
    for (size_t i = 0; i < (size_t)n_orient * n_trans; i++) diff2[i] = xi2_half;
    CpuKernels::diff2_coarse<true, false, D2C_BLOCK_SIZE_REF3D, D2C_EULERS_PER_BLOCK_REF3D, 4>(
        n_orient / epb, e.data(), tx.data(), ty.data(), tz.data(), re.data(), im.data(), k, cr.data(), diff2,
        n_trans, (unsigned long)img_x * img_y);
    return 0;
}

// ---- fine pass, weighted sums, backprojection: the reference's other CPU E-step kernels
//   CpuKernels::diff2_fine_2D<REF3D>  src/acc/cpu/cpu_kernels/diff2.h:607-758
//   CpuKernels::wavg_ref3D<REFCTF, REF3D>  src/acc/cpu/cpu_kernels/wavg.h:22-204
//   CpuKernels::backprojectRef3D<CTF_PREMULTIPLIED>  src/acc/cpu/cpu_kernels/BP.h:504-760
#include "src/acc/cpu/cpu_kernels/wavg.h"
#include "src/acc/cpu/cpu_kernels/BP.h"

namespace {
struct RefModel {
    AccProjector p;
    RefModel(const float* mdl, int xdim, int ydim, int zdim, int inity, int initz, int maxr, int pad)
    {
        p.setMdlDim(xdim, ydim, zdim, inity, initz, maxr, (XFLOAT)pad);
        const size_t nvox = (size_t)xdim * ydim * zdim;
        std::complex<XFLOAT>* data = new std::complex<XFLOAT>[nvox];
        for (size_t i = 0; i < nvox; i++) data[i] = std::complex<XFLOAT>(mdl[2 * i], mdl[2 * i + 1]);
        p.initMdl(data);  // shared, freed by the projector
    }
};
}  // namespace

// Fine-pass diff2 of `n_jobs` jobs: job j evaluates rotation rot_idx[job_idx[j]] against the
// job_num[j] consecutive translations from trans_idx[job_idx[j]], writing
// diff2[job_idx[j] + i] (the reference's FinePassWeights layout).  Operands as ref_coarse_diff2
// (inverted Euler matrices, X / CTF, Minvsigma2 CTF^2, -2 pi shift / ori_size).
extern "C" int ref_fine_diff2(const float* mdl, int xdim, int ydim, int zdim, int inity, int initz, int maxr,
                              int pad, const float* eulers_inv, int n_rot, const float* img_re, const float* img_im,
                              const float* corr, int img_x, int img_y, const float* trans_x, const float* trans_y,
                              int n_trans, float xi2_half, int n_jobs, const unsigned long* rot_idx,
                              const unsigned long* trans_idx, const unsigned long* job_idx,
                              const unsigned long* job_num, long long n_out, float* diff2)
{
    RefModel m(mdl, xdim, ydim, zdim, inity, initz, maxr, pad);
    AccProjectorKernel k = AccProjectorKernel::makeKernel(m.p, img_x, img_y, 1, img_x - 1);
    std::vector<XFLOAT> e(eulers_inv, eulers_inv + 9 * (size_t)n_rot);
    std::vector<XFLOAT> tx(trans_x, trans_x + n_trans), ty(trans_y, trans_y + n_trans), tz(n_trans, 0.f);
    std::vector<XFLOAT> re(img_re, img_re + (size_t)img_x * img_y), im(img_im, img_im + (size_t)img_x * img_y);
    std::vector<XFLOAT> cr(corr, corr + (size_t)img_x * img_y);
    std::vector<unsigned long> ri(rot_idx, rot_idx + n_out), ti(trans_idx, trans_idx + n_out);
    std::vector<unsigned long> ji(job_idx, job_idx + n_jobs), jn(job_num, job_num + n_jobs);
    CpuKernels::diff2_fine_2D<true>(n_jobs, e.data(), re.data(), im.data(), tx.data(), ty.data(), tz.data(), k,
                                    cr.data(), diff2, (unsigned long)img_x * img_y, xi2_half, n_rot, n_trans,
                                    n_jobs, ri.data(), ti.data(), ji.data(), jn.data());
    return 0;
}

// Weighted sums of `n_orient` orientations (inverted Euler matrices) over `n_trans`
// translations: weights[o * n_trans + t] (those below sig_w skipped, the others divided by
// weight_norm); per pixel the sums of w |A - sX|^2, w Re(A conj sX), w |A|^2 with A = P CTF
// (REFCTF: ctf carries the scale), accumulated into parts / xa / aa (img_x * img_y each).
extern "C" int ref_wavg(const float* mdl, int xdim, int ydim, int zdim, int inity, int initz, int maxr, int pad,
                        const float* eulers_inv, int n_orient, const float* img_re, const float* img_im,
                        const float* ctf, int img_x, int img_y, const float* trans_x, const float* trans_y,
                        int n_trans, const float* weights, float weight_norm, float sig_w, float* parts, float* xa,
                        float* aa)
{
    RefModel m(mdl, xdim, ydim, zdim, inity, initz, maxr, pad);
    AccProjectorKernel k = AccProjectorKernel::makeKernel(m.p, img_x, img_y, 1, img_x - 1);
    std::vector<XFLOAT> e(eulers_inv, eulers_inv + 9 * (size_t)n_orient);
    std::vector<XFLOAT> tx(trans_x, trans_x + n_trans), ty(trans_y, trans_y + n_trans), tz(n_trans, 0.f);
    std::vector<XFLOAT> re(img_re, img_re + (size_t)img_x * img_y), im(img_im, img_im + (size_t)img_x * img_y);
    std::vector<XFLOAT> c(ctf, ctf + (size_t)img_x * img_y);
    std::vector<XFLOAT> w(weights, weights + (size_t)n_orient * n_trans);
    CpuKernels::wavg_ref3D<true, true>(e.data(), k, (unsigned long)img_x * img_y, n_orient, re.data(), im.data(),
                                      tx.data(), ty.data(), tz.data(), w.data(), c.data(), parts, aa, xa, n_trans,
                                      weight_norm, sig_w, 1.f);
    return 0;
}

// Backprojection of `n_img` orientations (inverted Euler matrices, as the reference builds them
// for this kernel: src/acc/acc_store_weight_sum.h:1041-1046) into the grid
// model_real / model_imag / model_weight (mdl_x x mdl_y x mdl_z, origin (0, inity, initz)):
// per pixel F = sum_t w' sX and Fw = sum_t w' CTF with w' = w / weight_norm * CTF * Minvsigma2
// over the translations with w >= sig_w, trilinear into the grid.
extern "C" int ref_backproject(const float* img_re, const float* img_im, int img_x, int img_y,
                               const float* trans_x, const float* trans_y, int n_trans, const float* weights,
                               const float* minvsigma2, const float* ctf, float sig_w, float weight_norm,
                               const float* eulers, int n_img, float* model_real, float* model_imag,
                               float* model_weight, int max_r, int pad, int mdl_x, int mdl_y, int mdl_z,
                               int mdl_inity, int mdl_initz)
{
    std::vector<XFLOAT> tx(trans_x, trans_x + n_trans), ty(trans_y, trans_y + n_trans);
    std::vector<XFLOAT> re(img_re, img_re + (size_t)img_x * img_y), im(img_im, img_im + (size_t)img_x * img_y);
    std::vector<XFLOAT> mv(minvsigma2, minvsigma2 + (size_t)img_x * img_y), c(ctf, ctf + (size_t)img_x * img_y);
    std::vector<XFLOAT> w(weights, weights + (size_t)n_img * n_trans), e(eulers, eulers + 9 * (size_t)n_img);
    std::vector<tbb::spin_mutex> mutexes((size_t)mdl_z * mdl_y);
    CpuKernels::backprojectRef3D<false>(n_img, re.data(), im.data(), tx.data(), ty.data(), w.data(), mv.data(),
                                        c.data(), n_trans, sig_w, weight_norm, e.data(), model_real, model_imag,
                                        model_weight, max_r, max_r * max_r, (XFLOAT)pad, img_x, img_y, 1,
                                        (size_t)img_x * img_y, mdl_x, mdl_y, mdl_inity, mdl_initz,
                                        mutexes.data());
    return 0;
}
