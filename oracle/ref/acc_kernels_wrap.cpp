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
