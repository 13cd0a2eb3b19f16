// Host sampling of libt2b: orientations and translations of the coarse and
// fine passes, as HealpixSampling produces them for C1 symmetry without
// random perturbation:
//   directions    HEALPix NEST pixel centres, rot = RAD2DEG(phi), tilt = ACOSD(z),
//                 checkDirection   (src/healpix_sampling.cpp:534-575, 1617-1649)
//   psi           nr_psi = CEIL(360/psi_step), psi = ipsi * 360/nr_psi
//                 (src/healpix_sampling.cpp:68-76, 577-585)
//   fine dirs     the 4 children at order+1 (xyf2nest over (i, j) of the parent's
//                 (x, y, face)), each with 2 oversampled psi
//                 (src/healpix_sampling.cpp:1914-2040)
//   translations  the disc |t|^2 < range^2 + 0.001 on a step grid, in Angstrom;
//                 fine: 2x2 sub-steps (src/healpix_sampling.cpp:291-440, 1800-1910)
//   matrices      Euler_angles2matrix (src/euler.cpp:52-91)
// The HEALPix pixel geometry restates Gorski et al. (2005) as implemented in
// src/Healpix_2.15a/healpix_base.cc:127-160, 460-527.
#include <cmath>
#include <cstring>
#include <vector>
#include "../../include/t2b.h"

namespace {

const double PI = 3.14159265358979323846;  // src/macros.h:102

int ROUNDi(double x) { return (x > 0) ? (int)(x + 0.5) : (int)(x - 0.5); }
int CEILi(double x) { return (x == (int)x) ? (int)x : ((x > 0) ? (int)(x + 1) : (int)x); }

void nest2xyf(int order, long pix, int& ix, int& iy, int& face)
{
    const long npface = 1L << (2 * order);
    face = (int)(pix >> (2 * order));
    const long p = pix & (npface - 1);
    ix = iy = 0;
    for (int b = 0; b < order; b++) {
        ix |= (int)(((p >> (2 * b)) & 1) << b);
        iy |= (int)(((p >> (2 * b + 1)) & 1) << b);
    }
}

long xyf2nest(int order, int ix, int iy, int face)
{
    long p = 0;
    for (int b = 0; b < order; b++) {
        p |= (long)((ix >> b) & 1) << (2 * b);
        p |= (long)((iy >> b) & 1) << (2 * b + 1);
    }
    return ((long)face << (2 * order)) + p;
}

void pix2zphi(int order, long pix, double& z, double& phi)
{
    static const int jrll[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
    static const int jpll[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};
    const long nside = 1L << order, npix = 12 * nside * nside;
    const double fact2 = 4. / npix, fact1 = (nside << 1) * fact2;
    int ix, iy, face;
    nest2xyf(order, pix, ix, iy, face);
    const long nl4 = 4 * nside;
    const long jr = ((long)jrll[face] << order) - ix - iy - 1;
    long nr, kshift;
    if (jr < nside) { nr = jr; z = 1 - nr * nr * fact2; kshift = 0; }
    else if (jr > 3 * nside) { nr = nl4 - jr; z = nr * nr * fact2 - 1; kshift = 0; }
    else { nr = nside; z = (2 * nside - jr) * fact1; kshift = (jr - nside) & 1; }
    long jp = (jpll[face] * nr + ix - iy + 1 + kshift) / 2;
    if (jp > nl4) jp -= nl4;
    if (jp < 1) jp += nl4;
    phi = (jp - (kshift + 1) * 0.5) * ((PI / 2) / nr);
}

void direction(int order, long pix, double& rot, double& tilt)
{
    double z, phi;
    pix2zphi(order, pix, z, phi);
    rot = phi * 180 / PI;            // RAD2DEG
    tilt = std::acos(z) * 180. / PI;  // ACOSD
    if (tilt < 0.) { tilt = -tilt; rot += 180.; }
    for (;;) {
        if (rot > 180.) rot -= 360.;
        else if (rot < -180.) rot += 360.;
        else break;
    }
}

void euler(double rot, double tilt, double psi, double* A)
{
    const double a = rot * PI / 180, b = tilt * PI / 180, g = psi * PI / 180;
    const double ca = std::cos(a), cb = std::cos(b), cg = std::cos(g);
    const double sa = std::sin(a), sb = std::sin(b), sg = std::sin(g);
    const double cc = cb * ca, cs = cb * sa, sc = sb * ca, ss = sb * sa;
    A[0] = cg * cc - sg * sa; A[1] = cg * cs + sg * ca; A[2] = -cg * sb;
    A[3] = -sg * cc - cg * sa; A[4] = -sg * cs + cg * ca; A[5] = sg * sb;
    A[6] = sc; A[7] = ss; A[8] = cb;
}

}  // namespace

extern "C" int t2b_sampling(int ref_dim, int order, double psi_step, int ovs, double range_px,
                            double step_px, double pixel_size, int* n_dir, int* n_psi, int* n_trans,
                            int* nover_rot, int* nover_trans, double* eul_coarse, double* eul_fine,
                            double* trans_px, double* trans_px_fine, double* trans_prior,
                            double* angles)
{
    if ((ref_dim != 2 && ref_dim != 3) || ovs < 0 || ovs > 1 || step_px <= 0. || range_px < 0. ||
        pixel_size <= 0. || (ref_dim == 3 && (order < 0 || order > 12)))
        return T2B_ERR_ARG;
    // directions
    std::vector<double> rots, tilts;
    std::vector<long> ipix;
    if (ref_dim == 3) {
        const long npix = 12L << (2 * order);
        for (long p = 0; p < npix; p++) {
            double r, t;
            direction(order, p, r, t);
            rots.push_back(r); tilts.push_back(t); ipix.push_back(p);
        }
        if (psi_step <= 0.) psi_step = 360. / (6 * ROUNDi(std::pow(2., order)));
    } else {
        rots.push_back(0.); tilts.push_back(0.); ipix.push_back(-1);
        if (psi_step <= 0.) psi_step = 10.;
    }
    const int npsi = CEILi(360. / psi_step);
    psi_step = 360. / (double)npsi;
    const int ndir = (int)rots.size();
    const int R = ovs ? (ref_dim == 3 ? 8 : 2) : 1;
    const int V = ovs ? 4 : 1;
    // translations (Angstrom)
    const double step = step_px * pixel_size, range = range_px * pixel_size;
    const int maxp = CEILi(range / step);
    std::vector<double> tx, ty;
    for (int ix = -maxp; ix <= maxp; ix++) {
        const double xoff = ix * step;
        for (int iy = -maxp; iy <= maxp; iy++) {
            const double yoff = iy * step;
            if (xoff * xoff + yoff * yoff < range * range + 0.001) { tx.push_back(xoff); ty.push_back(yoff); }
        }
    }
    const int T = (int)tx.size();
    if (n_dir) *n_dir = ndir;
    if (n_psi) *n_psi = npsi;
    if (n_trans) *n_trans = T;
    if (nover_rot) *nover_rot = R;
    if (nover_trans) *nover_trans = V;
    for (int d = 0; d < ndir; d++)
        for (int p = 0; p < npsi; p++) {
            const int o = d * npsi + p;
            const double psi = p * psi_step;
            if (eul_coarse) euler(rots[d], tilts[d], psi, eul_coarse + 9 * (size_t)o);
            if (angles) { angles[3 * o] = rots[d]; angles[3 * o + 1] = tilts[d]; angles[3 * o + 2] = psi; }
            if (eul_fine && ovs) {
                int r = 0;
                const double base_psi = p * psi_step;
                if (ref_dim == 3) {
                    int x, y, face;
                    nest2xyf(order, ipix[d], x, y, face);
                    for (int j = 2 * y; j < 2 * (y + 1); ++j)
                        for (int i = 2 * x; i < 2 * (x + 1); ++i) {
                            const long over = xyf2nest(order + 1, i, j, face);
                            double fr, ft;
                            direction(order + 1, over, fr, ft);
                            for (int po = 0; po < 2; po++) {
                                const double overpsi = base_psi - 0.5 * psi_step + (0.5 + po) * psi_step / 2;
                                euler(fr, ft, overpsi, eul_fine + 9 * ((size_t)o * R + r));
                                r++;
                            }
                        }
                } else {
                    for (int po = 0; po < 2; po++) {
                        double overpsi = base_psi - 0.5 * psi_step + (0.5 + po) * psi_step / 2;
                        if (overpsi > 180.) overpsi -= 360.;
                        euler(0., 0., overpsi, eul_fine + 9 * ((size_t)o * R + r));
                        r++;
                    }
                }
            }
        }
    for (int t = 0; t < T; t++) {
        if (trans_px) { trans_px[2 * t] = tx[t] / pixel_size; trans_px[2 * t + 1] = ty[t] / pixel_size; }
        if (trans_prior) { trans_prior[2 * t] = tx[t]; trans_prior[2 * t + 1] = ty[t]; }
        if (trans_px_fine && ovs) {
            int v = 0;
            for (int ox = 0; ox < 2; ox++) {
                const double over_x = tx[t] - 0.5 * step + (0.5 + ox) * step / 2;
                for (int oy = 0; oy < 2; oy++) {
                    const double over_y = ty[t] - 0.5 * step + (0.5 + oy) * step / 2;
                    trans_px_fine[2 * (t * V + v)] = over_x / pixel_size;
                    trans_px_fine[2 * (t * V + v) + 1] = over_y / pixel_size;
                    v++;
                }
            }
        }
    }
    return T2B_OK;
}
