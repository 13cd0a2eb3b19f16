// FP64 CPU oracle of the RELION / T2-RELION expectation-step hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// product: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
// leg may load it.  Nothing in the shipped library calls it.
//
// Every stage restates the reference CPU path (RFLOAT = double) in plain loops:
//   CTF                      src/ctf.h:181-238, src/ctf.cpp:206-256
//   Fourier-slice projection src/projector.cpp:524-650 (TRILINEAR branch)
//   2D in-plane rotation     src/projector.cpp:904-1016 (rotate2D, bilinear)
//   Fourier phase shift      src/fftw.cpp:842-918, src/ml_optimiser.cpp:3751-3830
//   diff2                    src/ml_optimiser.cpp:7113-7272
//   weights / significance   src/ml_optimiser.cpp:7510-8040
//   weighted sums            src/ml_optimiser.cpp:8043-8700
//   backprojection           src/backprojector.cpp:55-230 (backproject2Dto3D)
//   skip-gridding division   src/backprojector.cpp:1463-1531
//
// Two deliberate, documented deviations (both also taken by the CUDA path):
//  * the radius tests of projection and backprojection use the exact integer
//    criterion x*x+y*y <= r_max*r_max on the 2D pixel; the reference evaluates
//    the same quantity after rotation in floating point, so pixels lying exactly
//    on the circle are kept or dropped depending on rounding (and a dropped pixel
//    keeps a stale value from the previous orientation in Projector::project);
//  * A^{-1} of a rotation is taken as A^T.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <thread>

namespace {

const double PI = 3.14159265358979323846;
std::mutex g_bp_mutex;  // serialises grid accumulation across particle threads

inline double deg2rad(double d) { return d * PI / 180.0; }

// ------------------------------------------------------------------ CTF
struct CtfK { double K1, K2, K3, K4, K5, Axx, Axy, Ayy, scale; };

// params: defU, defV, defAngle(deg), kV, Cs(mm), Q0, Bfac, scale, phase_shift(deg)
// src/ctf.cpp:206-256 (CTF::initialise)
CtfK ctf_setup(const double* p)
{
    CtfK k;
    const double Cs = p[4] * 1e7, kV = p[3] * 1e3, Q0 = p[5];
    const double lambda = 12.2643247 / std::sqrt(kV * (1. + kV * 0.978466e-6));
    k.K1 = PI / 2 * 2 * lambda;
    k.K2 = PI / 2 * Cs * lambda * lambda * lambda;
    k.K3 = std::atan(Q0 / std::sqrt(1 - Q0 * Q0));
    k.K4 = -p[6] / 4.;
    k.K5 = deg2rad(p[8]);
    const double az = deg2rad(p[2]);
    const double c = std::cos(az), s = std::sin(az);
    const double dU = p[0], dV = p[1];
    // A = Q^T diag(-dU,-dV) Q with Q = [[c, s], [-s, c]]
    k.Axx = -dU * c * c - dV * s * s;
    k.Axy = (dV - dU) * c * s;
    k.Ayy = -dU * s * s - dV * c * c;
    k.scale = p[7];
    return k;
}

// src/ctf.h:181-238 (getCTF with damping, no abs / phase flip)
double ctf_eval(const CtfK& k, double X, double Y)
{
    const double u2 = X * X + Y * Y, u4 = u2 * u2;
    const double gamma = k.K1 * (k.Axx * X * X + 2.0 * k.Axy * X * Y + k.Ayy * Y * Y) + k.K2 * u4 - k.K5 - k.K3;
    double r = -std::sin(gamma);
    r *= std::exp(k.K4 * u2);
    r *= k.scale;
    if (std::fabs(r) < 1e-8) r = (r >= 0 ? 1.0 : -1.0) * 1e-8;
    return r;
}

// ------------------------------------------------------------ geometry
struct Map {
    const float* data;  // complex interleaved, [z][y][x]
    int xdim, ydim, zdim, inity, initz, r_max, pad;
};

inline void lerp2(double a, double lr, double li, double hr, double hi, double& r, double& i)
{
    r = lr + (hr - lr) * a;
    i = li + (hi - li) * a;
}

// One pixel of Projector::project (src/projector.cpp:566-650), TRILINEAR.
// Ainv is the already padded inverse rotation (row-major 3x3).
void project_pixel3d(const Map& m, const double* Ainv, int x, int y, double& re, double& im)
{
    re = im = 0.;
    if ((long)x * x + (long)y * y > (long)m.r_max * m.r_max) return;
    double xp = Ainv[0] * x + Ainv[1] * y;
    double yp = Ainv[3] * x + Ainv[4] * y;
    double zp = Ainv[6] * x + Ainv[7] * y;
    const bool neg = xp < 0;
    if (neg) { xp = -xp; yp = -yp; zp = -zp; }
    const int x0 = (int)std::floor(xp);
    const double fx = xp - x0;
    int y0 = (int)std::floor(yp);
    const double fy = yp - y0;
    y0 -= m.inity;
    int z0 = (int)std::floor(zp);
    const double fz = zp - z0;
    z0 -= m.initz;
    if (x0 < 0 || x0 + 1 >= m.xdim || y0 < 0 || y0 + 1 >= m.ydim || z0 < 0 || z0 + 1 >= m.zdim) return;
    auto at = [&](int z, int yy, int xx, double& r, double& i) {
        const size_t idx = ((size_t)z * m.ydim + yy) * m.xdim + xx;
        r = m.data[2 * idx]; i = m.data[2 * idx + 1];
    };
    double d000r, d000i, d001r, d001i, d010r, d010i, d011r, d011i;
    double d100r, d100i, d101r, d101i, d110r, d110i, d111r, d111i;
    at(z0, y0, x0, d000r, d000i);         at(z0, y0, x0 + 1, d001r, d001i);
    at(z0, y0 + 1, x0, d010r, d010i);     at(z0, y0 + 1, x0 + 1, d011r, d011i);
    at(z0 + 1, y0, x0, d100r, d100i);     at(z0 + 1, y0, x0 + 1, d101r, d101i);
    at(z0 + 1, y0 + 1, x0, d110r, d110i); at(z0 + 1, y0 + 1, x0 + 1, d111r, d111i);
    double x00r, x00i, x01r, x01i, x10r, x10i, x11r, x11i, y0r, y0i, y1r, y1i;
    lerp2(fx, d000r, d000i, d001r, d001i, x00r, x00i);
    lerp2(fx, d100r, d100i, d101r, d101i, x01r, x01i);
    lerp2(fx, d010r, d010i, d011r, d011i, x10r, x10i);
    lerp2(fx, d110r, d110i, d111r, d111i, x11r, x11i);
    lerp2(fy, x00r, x00i, x10r, x10i, y0r, y0i);
    lerp2(fy, x01r, x01i, x11r, x11i, y1r, y1i);
    lerp2(fz, y0r, y0i, y1r, y1i, re, im);
    if (neg) im = -im;
}

// Whole windowed image (s rows x s/2+1 cols, FFTW order) for rotation A.
void project_image3d(const Map& m, const double* A, int s, double* out /*2P*/)
{
    double Ainv[9];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) Ainv[3 * r + c] = A[3 * c + r] * m.pad;
    const int xh = s / 2 + 1;
    const int rmo = s / 2;
    std::memset(out, 0, sizeof(double) * 2 * s * xh);
    for (int i = 0; i < s; i++) {
        const int y = (i <= rmo) ? i : i - s;
        const int xmax = (int)std::floor(std::sqrt((double)(rmo * rmo - y * y)));
        for (int x = 0; x <= xmax && x < xh; x++)
            project_pixel3d(m, Ainv, x, y, out[2 * (i * xh + x)], out[2 * (i * xh + x) + 1]);
    }
}

// Projector::rotate2D (src/projector.cpp:904-1016): bilinear, 2D map
// [y][x] with inity, x from 0.
void project_image2d(const Map& m, const double* A, int s, double* out)
{
    // A is 3x3 (Euler with rot=tilt=0); the 2D rotation uses its top-left 2x2.
    double Ainv[4];
    Ainv[0] = A[0] * m.pad; Ainv[1] = A[3] * m.pad;
    Ainv[2] = A[1] * m.pad; Ainv[3] = A[4] * m.pad;
    const int xh = s / 2 + 1;
    const int rmo = s / 2;
    std::memset(out, 0, sizeof(double) * 2 * s * xh);
    for (int i = 0; i < s; i++) {
        const int y = (i <= rmo) ? i : i - s;
        const int xmax = (int)std::floor(std::sqrt((double)(rmo * rmo - y * y)));
        for (int x = 0; x <= xmax && x < xh; x++) {
            if ((long)x * x + (long)y * y > (long)m.r_max * m.r_max) continue;
            double xp = Ainv[0] * x + Ainv[1] * y;
            double yp = Ainv[2] * x + Ainv[3] * y;
            const bool neg = xp < 0;
            if (neg) { xp = -xp; yp = -yp; }
            const int x0 = (int)std::floor(xp);
            const double fx = xp - x0;
            int y0 = (int)std::floor(yp);
            const double fy = yp - y0;
            y0 -= m.inity;
            if (x0 < 0 || x0 + 1 >= m.xdim || y0 < 0 || y0 + 1 >= m.ydim) continue;
            auto at = [&](int yy, int xx, double& r, double& im) {
                const size_t idx = (size_t)yy * m.xdim + xx;
                r = m.data[2 * idx]; im = m.data[2 * idx + 1];
            };
            double d00r, d00i, d01r, d01i, d10r, d10i, d11r, d11i;
            at(y0, x0, d00r, d00i); at(y0, x0 + 1, d01r, d01i);
            at(y0 + 1, x0, d10r, d10i); at(y0 + 1, x0 + 1, d11r, d11i);
            double a0r, a0i, a1r, a1i, rr, ri;
            lerp2(fx, d00r, d00i, d01r, d01i, a0r, a0i);
            lerp2(fx, d10r, d10i, d11r, d11i, a1r, a1i);
            lerp2(fy, a0r, a0i, a1r, a1i, rr, ri);
            if (neg) ri = -ri;
            out[2 * (i * xh + x)] = rr;
            out[2 * (i * xh + x) + 1] = ri;
        }
    }
}

// Phase factors e^{-2 pi i (kx sx + ky sy)/N} of one shift (src/fftw.cpp:874-918).
void shift_table(int s, int ori, double sx, double sy, double* ab /*2P*/)
{
    const int xh = s / 2 + 1;
    const double xs = -sx / ori, ys = -sy / ori;
    for (int i = 0; i < s; i++) {
        const int y = (i < xh) ? i : i - s;
        for (int x = 0; x < xh; x++) {
            const double dotp = 2 * PI * (x * xs + y * ys);
            ab[2 * (i * xh + x)] = std::cos(dotp);
            ab[2 * (i * xh + x) + 1] = std::sin(dotp);
        }
    }
}

} // namespace

extern "C" {

// ------------------------------------------------------------- params
// Layout mirrored by ctypes in oracle/oracle.py.
struct OrcSetup {
    int ori_size;        // full box
    int s;               // current (windowed) size, even
    int ref_dim;         // 3: 3D refs + 2D particles, 2: 2D refs
    int nr_classes;
    int n_dir, n_psi;    // coarse orientations per class = n_dir * n_psi
    int n_trans;         // coarse translations
    int nover_rot, nover_trans;   // 1,1 when adaptive_oversampling == 0
    int adaptive_oversampling;    // 0 or 1
    int maximum_significants;     // <= 0: off
    // projector maps (nr_classes consecutive)
    const float* maps;
    int mxdim, mydim, mzdim, minity, minitz, mr_max, mpad;
    // sampling
    const double* eul_coarse;     // n_dir*n_psi x 9  (Euler matrices A, not inverted)
    const double* eul_fine;       // n_dir*n_psi*nover_rot x 9
    const double* trans_px;       // n_trans x 2, coarse shifts in pixels
    const double* trans_px_fine;  // n_trans*nover_trans x 2
    const double* trans_prior;    // n_trans x 2: sampling.translations_{x,y}
    const double* pdf_direction;  // nr_classes x n_dir
    const double* pdf_class;      // nr_classes
    double sigma2_offset, pixel_size, adaptive_fraction;
    // backprojection grids (nr_classes, double accumulators)
    double* bp_data;              // complex interleaved, nr_classes x grid
    double* bp_weight;            // nr_classes x grid
    int bxdim, bydim, bzdim, binity, binitz, br_max, bpad;
    // do_scale_correction: nr_classes x (ori_size/2+1) data_vs_prior_class, or nullptr (off)
    const double* data_vs_prior;
};

struct OrcParticle {
    const float* fimg;         // 2P complex interleaved (masked)
    const float* fimg_nomask;  // 2P (may equal fimg)
    const float* ctf;          // P
    const float* minvsigma2;   // P, 0 at DC / outside the resolution mask
    const int* mresol;         // P, ires or -1 (Mresol_fine)
    double minvsigma2_dc;      // 1/(fudge*sigma2_noise[0]) used in the weighted sums
    double highres_xi2;
    double old_offset[2];
    double prior[2];
    double scale;
};

struct OrcResult {
    double min_diff2;        // final pass
    double sum_weight;       // final pass
    double sig_weight;       // final pass significance threshold
    double coarse_min_diff2;
    double coarse_sum_weight;
    double coarse_sig_weight;
    long long nr_sign;       // significant coarse samples
    long long n_coarse_sig;  // size of the coarse significant mask
    double pmax;
    int pose[5];             // iclass, iorient, iover_rot, itrans, iover_trans
    double wsum_norm;
    double sumw;
    double wsum_sigma2_offset;
    double wsum_scale_xa;    // exp_wsum_scale_correction_XA / scale_correction
    double wsum_scale_aa;    // exp_wsum_scale_correction_AA / scale_correction^2
};

double orc_ctf_value(const double* params, double X, double Y)
{
    CtfK k = ctf_setup(params);
    return ctf_eval(k, X, Y);
}

// CTF image on the windowed grid (src/ctf.cpp:436-450 + windowFourierTransform).
void orc_ctf_image(const double* params, int ori_size, double angpix, int s, float* out)
{
    CtfK k = ctf_setup(params);
    const int xh = s / 2 + 1;
    const double xs = ori_size * angpix, ys = ori_size * angpix;
    for (int i = 0; i < s; i++) {
        const int ip = (i < xh) ? i : i - s;
        for (int j = 0; j < xh; j++) out[i * xh + j] = (float)ctf_eval(k, j / xs, ip / ys);
    }
}

static Map make_map(const OrcSetup* S, int iclass)
{
    Map m;
    const size_t nvox = (size_t)S->mxdim * S->mydim * S->mzdim;
    m.data = S->maps + 2 * nvox * iclass;
    m.xdim = S->mxdim; m.ydim = S->mydim; m.zdim = S->mzdim;
    m.inity = S->minity; m.initz = S->minitz; m.r_max = S->mr_max; m.pad = S->mpad;
    return m;
}

static void project(const OrcSetup* S, int iclass, const double* A, double* out)
{
    Map m = make_map(S, iclass);
    if (S->ref_dim == 3) project_image3d(m, A, S->s, out);
    else project_image2d(m, A, S->s, out);
}

void orc_project(const OrcSetup* S, int iclass, const double* A, double* out)
{
    project(S, iclass, A, out);
}

// diff2 of one (reference slice, shift table) pair: src/ml_optimiser.cpp:7251-7272
static double diff2_one(const OrcSetup* S, const OrcParticle* pt, const double* fref, const double* ab)
{
    const int P = S->s * (S->s / 2 + 1);
    double d = pt->highres_xi2 / 2.;
    for (int n = 0; n < P; n++) {
        const double c = pt->ctf[n] * pt->scale;
        const double rr = fref[2 * n] * c, ri = fref[2 * n + 1] * c;
        const double xr = pt->fimg[2 * n], xi = pt->fimg[2 * n + 1];
        const double sr = ab[2 * n] * xr - ab[2 * n + 1] * xi;
        const double si = ab[2 * n] * xi + ab[2 * n + 1] * xr;
        const double dr = rr - sr, di = ri - si;
        d += (dr * dr + di * di) * 0.5 * pt->minvsigma2[n];
    }
    return d;
}

// The same sum as diff2_one with its per-hypothesis factors hoisted: `rc` the
// reference times CTF and scale (per orientation), `sx` the shifted image (per
// translation), `nz` the pixels whose Minvsigma2 is non-zero (the others add an
// exact 0).  Every term is the same double expression, in the same order, so
// the result equals diff2_one's bit for bit.
static double diff2_pre(const OrcParticle* pt, const double* rc, const double* sx, const std::vector<int>& nz)
{
    double d = pt->highres_xi2 / 2.;
    for (const int n : nz) {
        const double dr = rc[2 * n] - sx[2 * n], di = rc[2 * n + 1] - sx[2 * n + 1];
        d += (dr * dr + di * di) * 0.5 * pt->minvsigma2[n];
    }
    return d;
}

static std::vector<int> nonzero_pixels(const OrcSetup* S, const OrcParticle* pt)
{
    const int P = S->s * (S->s / 2 + 1);
    std::vector<int> nz;
    for (int n = 0; n < P; n++)
        if (pt->minvsigma2[n] != 0.f) nz.push_back(n);
    return nz;
}

// Shifted images of `nt` shifts (src/ml_optimiser.cpp:7205-7245): nt x 2P.
static void shifted_images(const OrcSetup* S, const OrcParticle* pt, const double* shifts, int nt,
                           std::vector<double>& out)
{
    const int P = S->s * (S->s / 2 + 1);
    std::vector<double> ab((size_t)2 * P);
    out.resize((size_t)2 * P * nt);
    for (int t = 0; t < nt; t++) {
        shift_table(S->s, S->ori_size, shifts[2 * t], shifts[2 * t + 1], ab.data());
        double* o = &out[(size_t)2 * P * t];
        for (int n = 0; n < P; n++) {
            const double xr = pt->fimg[2 * n], xi = pt->fimg[2 * n + 1];
            o[2 * n] = ab[2 * n] * xr - ab[2 * n + 1] * xi;
            o[2 * n + 1] = ab[2 * n] * xi + ab[2 * n + 1] * xr;
        }
    }
}

// Frefctf = Fref * CTF * scale (src/ml_optimiser.cpp:7113-7140).
static void ref_ctf(const OrcSetup* S, const OrcParticle* pt, const double* fref, double* out)
{
    const int P = S->s * (S->s / 2 + 1);
    for (int n = 0; n < P; n++) {
        const double c = pt->ctf[n] * pt->scale;
        out[2 * n] = fref[2 * n] * c;
        out[2 * n + 1] = fref[2 * n + 1] * c;
    }
}

// diff2 of one hypothesis in the reference's literal per-pixel form (the check of
// diff2_pre's hoisting): class iclass, Euler matrix A, shift (sx, sy) in pixels.
double orc_diff2_literal(const OrcSetup* S, const OrcParticle* pt, int iclass, const double* A, double sx, double sy)
{
    const int P = S->s * (S->s / 2 + 1);
    std::vector<double> fref((size_t)2 * P), ab((size_t)2 * P);
    project(S, iclass, A, fref.data());
    shift_table(S->s, S->ori_size, sx, sy, ab.data());
    return diff2_one(S, pt, fref.data(), ab.data());
}

// Coarse pass diff2 over every (class, orientation, translation):
// out[(iclass*O + iorient)*T + itrans]; -999 where the orientation is skipped.
// Returns the minimum (src/ml_optimiser.cpp:6922-7300, exp_ipass == 0).
double orc_coarse_diff2(const OrcSetup* S, const OrcParticle* pt, double* out)
{
    const int P = S->s * (S->s / 2 + 1);
    const int O = S->n_dir * S->n_psi, T = S->n_trans;
    std::vector<double> fref(2 * P), rc(2 * P), sx;
    shifted_images(S, pt, S->trans_px, T, sx);
    const std::vector<int> nz = nonzero_pixels(S, pt);
    double mn = 1e300;
    for (int k = 0; k < S->nr_classes; k++) {
        for (int o = 0; o < O; o++) {
            double* dst = out + ((size_t)k * O + o) * T;
            const int idir = o / S->n_psi;
            if (!(S->pdf_class[k] > 0.) || !(S->pdf_direction[k * S->n_dir + idir] > 0.)) {
                for (int t = 0; t < T; t++) dst[t] = -999.;
                continue;
            }
            project(S, k, S->eul_coarse + 9 * o, fref.data());
            ref_ctf(S, pt, fref.data(), rc.data());
            for (int t = 0; t < T; t++) {
                dst[t] = diff2_pre(pt, rc.data(), &sx[(size_t)2 * P * t], nz);
                mn = std::min(mn, dst[t]);
            }
        }
    }
    return mn;
}

// pdf_orientation / pdf_offset exactly as src/ml_optimiser.cpp:7587-7716
// (NOPRIOR mode, 2D data, single image, no helix / bodies).
static void priors(const OrcSetup* S, const OrcParticle* pt, std::vector<double>& pdf_o /*K*n_dir*/, std::vector<double>& pdf_t /*T*/)
{
    const int K = S->nr_classes, T = S->n_trans;
    double om = 0, tm = 0;
    long oc = 0, tc = 0;
    auto tpdf = [&](int t) {
        const double ox = pt->old_offset[0] + S->trans_prior[2 * t];
        const double oy = pt->old_offset[1] + S->trans_prior[2 * t + 1];
        double td = (ox - pt->prior[0]) * (ox - pt->prior[0]) + (oy - pt->prior[1]) * (oy - pt->prior[1]);
        td *= S->pixel_size * S->pixel_size;
        if (S->sigma2_offset < 0.0001) return td > 0. ? 0. : 1.;
        return std::exp(td / (-2. * S->sigma2_offset)) / (2. * PI * S->sigma2_offset);
    };
    for (int k = 0; k < K; k++) {
        for (int d = 0; d < S->n_dir; d++)
            for (int p = 0; p < S->n_psi; p++) { om += S->pdf_direction[k * S->n_dir + d]; oc++; }
        for (int t = 0; t < T; t++) { tm += tpdf(t); tc++; }
    }
    om /= (double)oc;
    tm /= (double)tc;
    pdf_o.resize((size_t)K * S->n_dir);
    for (int k = 0; k < K; k++)
        for (int d = 0; d < S->n_dir; d++) {
            double v = S->pdf_direction[k * S->n_dir + d];
            if (om != 0.) v /= om;
            pdf_o[(size_t)k * S->n_dir + d] = v;
        }
    pdf_t.resize(T);
    for (int t = 0; t < T; t++) {
        double v = tpdf(t);
        if (tm > 0.) v /= tm;
        pdf_t[t] = v;
    }
}

// Convert diff2 -> weights, sum and the significance threshold
// (src/ml_optimiser.cpp:7770-7990).  Entries are addressed by coarse hidden
// index ihidden = iorientclass*T + itrans; `w` receives the weights.
// Returns 0 on success, 1 when the weights sum to zero / no significant sample.
static int to_weights(const OrcSetup* S, const OrcParticle* pt, int ipass,
                      const double* diff2, const long long* ihidden, long long n, double min_diff2,
                      double* w, double& sum_w, double& sig_w, long long& nr_sign)
{
    std::vector<double> pdf_o, pdf_t;
    priors(S, pt, pdf_o, pdf_t);
    const int T = S->n_trans, O = S->n_dir * S->n_psi;
    sum_w = 0.;
    for (long long i = 0; i < n; i++) {
        if (diff2[i] < 0.) { w[i] = 0.; continue; }
        const long long ih = ihidden[i];
        const int itrans = (int)(ih % T);
        const long long ioc = ih / T;
        const int k = (int)(ioc / O), iorient = (int)(ioc % O);
        const int idir = iorient / S->n_psi;
        double weight = pdf_o[(size_t)k * S->n_dir + idir] * pdf_t[itrans];
        const double d = diff2[i] - min_diff2;
        if (d > 700.) weight = 0.;
        else weight *= std::exp(-d);
        w[i] = weight;
        sum_w += weight;
    }
    if (sum_w == 0. || std::isnan(sum_w)) return 1;
    std::vector<double> sorted;
    sorted.reserve(n);
    for (long long i = 0; i < n; i++)
        if (w[i] > 0.) sorted.push_back(w[i]);
    std::sort(sorted.begin(), sorted.end());
    double frac = 0., sig = 0.;
    long long cnt = 0;
    for (long long i = (long long)sorted.size() - 1; i >= 0; i--) {
        if (S->maximum_significants > 0) {
            if (cnt < S->maximum_significants) {
                if (ipass == 0) cnt++;
                sig = sorted[i];
            }
        } else {
            if (ipass == 0) cnt++;
            sig = sorted[i];
        }
        frac += sorted[i];
        if (frac > S->adaptive_fraction * sum_w) break;
    }
    if (ipass == 0 && cnt == 0) return 1;
    sig_w = sig;
    nr_sign = cnt;
    return 0;
}

// Weights of an arbitrary list (used by the unit tests of the weights stage).
int orc_weights(const OrcSetup* S, const OrcParticle* pt, int ipass, const double* diff2,
                const long long* ihidden, long long n, double min_diff2, double* w,
                double* sum_w, double* sig_w, long long* nr_sign)
{
    return to_weights(S, pt, ipass, diff2, ihidden, n, min_diff2, w, *sum_w, *sig_w, *nr_sign);
}

// Fine pass over the coarse significant mask (src/ml_optimiser.cpp:7090-7272,
// exp_ipass == 1).  For every significant coarse pair (in ihidden order) writes
// nover_rot*nover_trans diff2 values in (iover_rot, iover_trans) order.
// Returns the number of pairs; *min receives the minimum.
long long orc_fine_diff2(const OrcSetup* S, const OrcParticle* pt, const unsigned char* mask,
                         long long* pairs, double* out, double* mn_out)
{
    const int P = S->s * (S->s / 2 + 1);
    const int O = S->n_dir * S->n_psi, T = S->n_trans;
    const int R = S->nover_rot, V = S->nover_trans;
    std::vector<double> fref((size_t)2 * P), rc((size_t)2 * P * R), sx;
    shifted_images(S, pt, S->trans_px_fine, T * V, sx);
    const std::vector<int> nz = nonzero_pixels(S, pt);
    long long np = 0;
    double mn = 1e300;
    for (int k = 0; k < S->nr_classes; k++)
        for (int o = 0; o < O; o++) {
            const long long base = ((long long)k * O + o) * T;
            bool any = false;
            for (int t = 0; t < T; t++) any |= mask[base + t] != 0;
            if (!any) continue;
            for (int r = 0; r < R; r++) {
                project(S, k, S->eul_fine + 9 * ((size_t)o * R + r), fref.data());
                ref_ctf(S, pt, fref.data(), &rc[(size_t)2 * P * r]);
            }
            for (int t = 0; t < T; t++) {
                if (!mask[base + t]) continue;
                pairs[np] = base + t;
                for (int r = 0; r < R; r++)
                    for (int v = 0; v < V; v++) {
                        const double d = diff2_pre(pt, &rc[(size_t)2 * P * r], &sx[(size_t)2 * P * (t * V + v)], nz);
                        out[np * R * V + r * V + v] = d;
                        mn = std::min(mn, d);
                    }
                np++;
            }
        }
    *mn_out = mn;
    return np;
}

// BackProjector::backproject2Dto3D (src/backprojector.cpp:55-230), trilinear,
// no magnification / Ewald sphere.
static void backproject3d(const OrcSetup* S, int iclass, const double* A, const double* fimg, const double* fweight)
{
    const int s = S->s, xh = s / 2 + 1;
    const size_t nvox = (size_t)S->bxdim * S->bydim * S->bzdim;
    double* data = S->bp_data + 2 * nvox * iclass;
    double* wgt = S->bp_weight + nvox * iclass;
    double Ainv[9];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) Ainv[3 * r + c] = A[3 * c + r] * S->bpad;
    const long rmax2 = (long)S->br_max * S->br_max;
    for (int i = 0; i < s; i++) {
        int y, first_x;
        if (i < xh) { y = i; first_x = 0; }
        else { y = i - s; first_x = 1; }
        for (int x = first_x; x < xh; x++) {
            if ((long)x * x + (long)y * y > rmax2) continue;
            const int n = i * xh + x;
            const double mw = fweight[n];
            if (mw <= 0.) continue;
            double vr = fimg[2 * n], vi = fimg[2 * n + 1];
            double xp = Ainv[0] * x + Ainv[1] * y;
            double yp = Ainv[3] * x + Ainv[4] * y;
            double zp = Ainv[6] * x + Ainv[7] * y;
            if (xp < 0) { xp = -xp; yp = -yp; zp = -zp; vi = -vi; }
            const int x0 = (int)std::floor(xp);
            const double fx = xp - x0;
            int y0 = (int)std::floor(yp);
            const double fy = yp - y0;
            y0 -= S->binity;
            int z0 = (int)std::floor(zp);
            const double fz = zp - z0;
            z0 -= S->binitz;
            if (x0 < 0 || x0 + 1 >= S->bxdim || y0 < 0 || y0 + 1 >= S->bydim || z0 < 0 || z0 + 1 >= S->bzdim) continue;
            const double mfx = 1. - fx, mfy = 1. - fy, mfz = 1. - fz;
            const double dd[8] = {mfz * mfy * mfx, mfz * mfy * fx, mfz * fy * mfx, mfz * fy * fx,
                                  fz * mfy * mfx, fz * mfy * fx, fz * fy * mfx, fz * fy * fx};
            for (int c = 0; c < 8; c++) {
                const int zz = z0 + (c >> 2), yy = y0 + ((c >> 1) & 1), xx = x0 + (c & 1);
                const size_t idx = ((size_t)zz * S->bydim + yy) * S->bxdim + xx;
                data[2 * idx] += dd[c] * vr;
                data[2 * idx + 1] += dd[c] * vi;
                wgt[idx] += dd[c] * mw;
            }
        }
    }
}

// BackProjector::backproject2Dto2D analogue for 2D references (bilinear).
static void backproject2d(const OrcSetup* S, int iclass, const double* A, const double* fimg, const double* fweight)
{
    const int s = S->s, xh = s / 2 + 1;
    const size_t nvox = (size_t)S->bxdim * S->bydim;
    double* data = S->bp_data + 2 * nvox * iclass;
    double* wgt = S->bp_weight + nvox * iclass;
    double Ainv[4];
    Ainv[0] = A[0] * S->bpad; Ainv[1] = A[3] * S->bpad;
    Ainv[2] = A[1] * S->bpad; Ainv[3] = A[4] * S->bpad;
    const long rmax2 = (long)S->br_max * S->br_max;
    for (int i = 0; i < s; i++) {
        int y, first_x;
        if (i < xh) { y = i; first_x = 0; }
        else { y = i - s; first_x = 1; }
        for (int x = first_x; x < xh; x++) {
            if ((long)x * x + (long)y * y > rmax2) continue;
            const int n = i * xh + x;
            const double mw = fweight[n];
            if (mw <= 0.) continue;
            double vr = fimg[2 * n], vi = fimg[2 * n + 1];
            double xp = Ainv[0] * x + Ainv[1] * y;
            double yp = Ainv[2] * x + Ainv[3] * y;
            if (xp < 0) { xp = -xp; yp = -yp; vi = -vi; }
            const int x0 = (int)std::floor(xp);
            const double fx = xp - x0;
            int y0 = (int)std::floor(yp);
            const double fy = yp - y0;
            y0 -= S->binity;
            if (x0 < 0 || x0 + 1 >= S->bxdim || y0 < 0 || y0 + 1 >= S->bydim) continue;
            const double mfx = 1. - fx, mfy = 1. - fy;
            const double dd[4] = {mfy * mfx, mfy * fx, fy * mfx, fy * fx};
            for (int c = 0; c < 4; c++) {
                const int yy = y0 + (c >> 1), xx = x0 + (c & 1);
                const size_t idx = (size_t)yy * S->bxdim + xx;
                data[2 * idx] += dd[c] * vr;
                data[2 * idx + 1] += dd[c] * vi;
                wgt[idx] += dd[c] * mw;
            }
        }
    }
}

void orc_backproject(const OrcSetup* S, int iclass, const double* A, const double* fimg, const double* fweight)
{
    if (S->ref_dim == 3) backproject3d(S, iclass, A, fimg, fweight);
    else backproject2d(S, iclass, A, fimg, fweight);
}

// Weighted sums and backprojection of one particle's final-pass hypotheses
// (src/ml_optimiser.cpp:8153-8700, storeWeightedSums): `pairs` are the
// significant coarse pairs (coarse hidden index, ascending), `wf` their
// npairs x R x V final weights (R = V = 1 without adaptive oversampling),
// `fsum` / `fsig` the final sum of weights and significance threshold.
static void wsum_stage(const OrcSetup* S, const OrcParticle* pt, const long long* pairs, long long npairs,
                       const double* wf, double fsum, double fsig, OrcResult* res, double* wsum_sigma2,
                       double* wsum_pdf_class, double* wsum_pdf_dir)
{
    const int P = S->s * (S->s / 2 + 1);
    const int O = S->n_dir * S->n_psi, T = S->n_trans;
    const int R = S->adaptive_oversampling ? S->nover_rot : 1;
    const int V = S->adaptive_oversampling ? S->nover_trans : 1;
    // ---- weighted sums (src/ml_optimiser.cpp:8153-8700), pairs grouped by orientation
    std::vector<double> fref((size_t)2 * P), fimg((size_t)2 * P), fw(P), ab((size_t)2 * P);
    const int half = S->ori_size / 2 + 1;
    res->pmax = -1.;
    res->wsum_norm = 0.; res->sumw = 0.; res->wsum_sigma2_offset = 0.;
    res->wsum_scale_xa = 0.; res->wsum_scale_aa = 0.;
    long long a = 0;
    while (a < npairs) {
        const long long ioc = pairs[a] / T;
        long long b = a;
        while (b < npairs && pairs[b] / T == ioc) b++;
        const int k = (int)(ioc / O), o = (int)(ioc % O);
        const int idir = o / S->n_psi;
        for (int r = 0; r < R; r++) {
            const double* A = S->adaptive_oversampling ? S->eul_fine + 9 * ((size_t)o * R + r) : S->eul_coarse + 9 * (size_t)o;
            project(S, k, A, fref.data());
            std::fill(fimg.begin(), fimg.end(), 0.);
            std::fill(fw.begin(), fw.end(), 0.);
            bool any = false;
            for (long long q = a; q < b; q++) {
                const int t = (int)(pairs[q] % T);
                for (int v = 0; v < V; v++) {
                    double weight = wf[(size_t)q * R * V + r * V + v];
                    if (!(weight >= fsig)) continue;
                    weight /= fsum;
                    any = true;
                    const double* sh = S->adaptive_oversampling ? &S->trans_px_fine[2 * (t * V + v)] : &S->trans_px[2 * t];
                    shift_table(S->s, S->ori_size, sh[0], sh[1], ab.data());
                    for (int n = 0; n < P; n++) {
                        const double c = pt->ctf[n] * pt->scale;
                        const double rr = fref[2 * n] * c, ri = fref[2 * n + 1] * c;
                        const double xr = pt->fimg[2 * n], xi = pt->fimg[2 * n + 1];
                        const double sr = ab[2 * n] * xr - ab[2 * n + 1] * xi;
                        const double si = ab[2 * n] * xi + ab[2 * n + 1] * xr;
                        const int ires = pt->mresol[n];
                        if (ires > -1) {
                            const double dr = rr - sr, di = ri - si;
                            const double wd = weight * (dr * dr + di * di);
                            wsum_sigma2[ires] += wd;
                            res->wsum_norm += wd;
                            // scale correction (src/ml_optimiser.cpp:8477-8486)
                            if (S->data_vs_prior && S->data_vs_prior[(size_t)k * half + ires] > 3.) {
                                res->wsum_scale_xa += weight * (rr * sr + ri * si);
                                res->wsum_scale_aa += weight * (rr * rr + ri * ri);
                            }
                        }
                        const double ur = pt->fimg_nomask[2 * n], ui = pt->fimg_nomask[2 * n + 1];
                        const double nr = ab[2 * n] * ur - ab[2 * n + 1] * ui;
                        const double ni = ab[2 * n] * ui + ab[2 * n + 1] * ur;
                        const double minv = (n == 0) ? pt->minvsigma2_dc : pt->minvsigma2[n];
                        const double wx = weight * c * minv;
                        fimg[2 * n] += nr * wx;
                        fimg[2 * n + 1] += ni * wx;
                        fw[n] += wx * c;
                    }
                    res->sumw += weight;
                    wsum_pdf_class[k] += weight;
                    const double dx = pt->prior[0] - pt->old_offset[0] - sh[0];
                    const double dy = pt->prior[1] - pt->old_offset[1] - sh[1];
                    res->wsum_sigma2_offset += weight * S->pixel_size * S->pixel_size * (dx * dx + dy * dy);
                    wsum_pdf_dir[(size_t)k * S->n_dir + idir] += weight;
                    if (weight > res->pmax) {
                        res->pmax = weight;
                        res->pose[0] = k; res->pose[1] = o; res->pose[2] = r; res->pose[3] = t; res->pose[4] = v;
                    }
                }
            }
            if (any) {
                std::lock_guard<std::mutex> lock(g_bp_mutex);
                orc_backproject(S, k, A, fimg.data(), fw.data());
            }
        }
        a = b;
    }
    // divided by scale_correction and its square: the scale entered Frefctf through the CTF
    // (src/ml_optimiser.cpp:8856-8861)
    res->wsum_scale_xa /= pt->scale;
    res->wsum_scale_aa /= pt->scale * pt->scale;
}

// Full E-step of one particle: coarse pass, weights, optional fine pass,
// weights, weighted sums and backprojection (src/ml_optimiser.cpp:4418-4560
// expectationOneParticle, single image, no bodies / helix / CC).
// wsum_sigma2: ori_size/2+1 values; wsum_pdf_class: K; wsum_pdf_dir: K*n_dir.
// Returns 0 on success, 1 when the weights sum to zero.
int orc_estep_particle(const OrcSetup* S, const OrcParticle* pt, OrcResult* res,
                       double* wsum_sigma2, double* wsum_pdf_class, double* wsum_pdf_dir,
                       double* coarse_diff2_out /* nullable, K*O*T */)
{
    const int P = S->s * (S->s / 2 + 1);
    const int O = S->n_dir * S->n_psi, T = S->n_trans, K = S->nr_classes;
    const long long NH = (long long)K * O * T;
    std::vector<double> d2(NH);
    const double mn = orc_coarse_diff2(S, pt, d2.data());
    if (coarse_diff2_out) std::copy(d2.begin(), d2.end(), coarse_diff2_out);
    std::vector<long long> ih(NH);
    for (long long i = 0; i < NH; i++) ih[i] = i;
    std::vector<double> w(NH);
    double sw, sig;
    long long nsig;
    if (to_weights(S, pt, 0, d2.data(), ih.data(), NH, mn, w.data(), sw, sig, nsig)) return 1;
    res->coarse_min_diff2 = mn;
    res->coarse_sum_weight = sw;
    res->coarse_sig_weight = sig;
    res->nr_sign = nsig;
    std::vector<unsigned char> mask(NH);
    long long nmask = 0;
    for (long long i = 0; i < NH; i++) { mask[i] = w[i] >= sig; nmask += mask[i]; }
    res->n_coarse_sig = nmask;

    const int R = S->adaptive_oversampling ? S->nover_rot : 1;
    const int V = S->adaptive_oversampling ? S->nover_trans : 1;
    // final-pass hypotheses: (pair, r, v) with weights wf
    std::vector<long long> pairs;
    std::vector<double> wf;
    double fmin, fsum, fsig;
    if (S->adaptive_oversampling) {
        pairs.resize(nmask);
        std::vector<double> fd((size_t)nmask * R * V);
        const long long np = orc_fine_diff2(S, pt, mask.data(), pairs.data(), fd.data(), &fmin);
        std::vector<long long> fih((size_t)np * R * V);
        for (long long i = 0; i < np; i++)
            for (int j = 0; j < R * V; j++) fih[i * R * V + j] = pairs[i];
        wf.resize(fd.size());
        long long dummy;
        if (to_weights(S, pt, 1, fd.data(), fih.data(), (long long)fd.size(), fmin, wf.data(), fsum, fsig, dummy)) return 1;
    } else {
        for (long long i = 0; i < NH; i++)
            if (mask[i]) { pairs.push_back(i); wf.push_back(w[i]); }
        fmin = mn; fsum = sw; fsig = sig;
    }
    res->min_diff2 = fmin;
    res->sum_weight = fsum;
    res->sig_weight = fsig;

    wsum_stage(S, pt, pairs.data(), (long long)pairs.size(), wf.data(), fsum, fsig, res, wsum_sigma2,
               wsum_pdf_class, wsum_pdf_dir);
    return 0;
}

// The weighted-sums stage alone on caller-supplied final weights (same-input
// checks of the device stage).  Grids accumulate into S->bp_data / bp_weight.
void orc_wsum_bp(const OrcSetup* S, const OrcParticle* pt, const long long* pairs, long long npairs,
                 const double* wf, double fsum, double fsig, OrcResult* res, double* wsum_sigma2,
                 double* wsum_pdf_class, double* wsum_pdf_dir)
{
    wsum_stage(S, pt, pairs, npairs, wf, fsum, fsig, res, wsum_sigma2, wsum_pdf_class, wsum_pdf_dir);
}

// Batch driver: particles spread over `nthreads` host threads (dynamic
// scheduling).  Per-particle wsum arrays are laid out [b][...].  Returns the
// number of particles that failed (zero weight sum).
int orc_estep(const OrcSetup* S, const OrcParticle* pts, int n, OrcResult* res,
              double* wsum_sigma2, double* wsum_pdf_class, double* wsum_pdf_dir, int nthreads)
{
    const int half = S->ori_size / 2 + 1;
    std::atomic<int> next(0), fails(0);
    auto work = [&]() {
        for (;;) {
            const int b = next.fetch_add(1);
            if (b >= n) break;
            fails += orc_estep_particle(S, &pts[b], &res[b], wsum_sigma2 + (size_t)b * half,
                                        wsum_pdf_class + (size_t)b * S->nr_classes,
                                        wsum_pdf_dir + (size_t)b * S->nr_classes * S->n_dir, nullptr);
        }
    };
    if (nthreads < 1) nthreads = 1;
    std::vector<std::thread> pool;
    for (int i = 1; i < nthreads; i++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    return fails.load();
}

// BackProjector::reconstruct, skip_gridding branch (src/backprojector.cpp:1463-1531)
// for a 3D grid.  The grid is the centred half-complex layout; output Fconv is
// the FFTW-ordered transform of a pad_size^3 volume: [pad][pad][pad/2+1].
// Pass tau2 == nullptr for do_map == false.
void orc_reconstruct_divide(const double* data, const double* weight, int xdim, int ydim, int zdim,
                            int inity, int initz, int r_max, int pad, double* fconv)
{
    const int ps = ydim;  // pad_size
    const int fx = ps / 2 + 1;
    const int max_r2 = (int)std::lround(r_max * (double)pad) * (int)std::lround(r_max * (double)pad);
    const int round_max_r2 = (int)std::lround(r_max * (double)pad * r_max * (double)pad);
    const size_t nF = (size_t)ps * ps * fx;
    std::vector<double> Fw(nF, 0.);
    std::fill(fconv, fconv + 2 * nF, 0.);
    // decenter (src/projector.h:242-253)
    for (int k = 0; k < ps; k++) {
        const int kp = (k < fx) ? k : k - ps;
        for (int i = 0; i < ps; i++) {
            const int ip = (i < fx) ? i : i - ps;
            for (int j = 0; j < fx; j++) {
                const int jp = j;
                if (kp * kp + ip * ip + jp * jp > max_r2) continue;
                const size_t src = ((size_t)(kp - initz) * ydim + (ip - inity)) * xdim + jp;
                const size_t dst = ((size_t)k * ps + i) * fx + j;
                Fw[dst] = weight[src];
                fconv[2 * dst] = data[2 * src];
                fconv[2 * dst + 1] = data[2 * src + 1];
            }
        }
    }
    std::vector<double> rad(r_max, 0.), cnt(r_max, 0.);
    for (int k = 0; k < ps; k++) {
        const int kp = (k < fx) ? k : k - ps;
        for (int i = 0; i < ps; i++) {
            const int ip = (i < fx) ? i : i - ps;
            for (int j = 0; j < fx; j++) {
                const int r2 = kp * kp + ip * ip + j * j;
                if (r2 < round_max_r2) {
                    const int ires = (int)std::floor(std::sqrt((double)r2) / pad);
                    rad[ires] += Fw[((size_t)k * ps + i) * fx + j];
                    cnt[ires] += 1.;
                }
            }
        }
    }
    for (int i = 0; i < r_max; i++)
        if (cnt[i] > 0. || rad[i] > 0.) rad[i] /= 1000. * cnt[i];
    for (int k = 0; k < ps; k++) {
        const int kp = (k < fx) ? k : k - ps;
        for (int i = 0; i < ps; i++) {
            const int ip = (i < fx) ? i : i - ps;
            for (int j = 0; j < fx; j++) {
                const int r2 = kp * kp + ip * ip + j * j;
                const int ires = (int)std::floor(std::sqrt((double)r2) / pad);
                const size_t n = ((size_t)k * ps + i) * fx + j;
                const double w = std::max(Fw[n], rad[(ires < r_max) ? ires : (r_max - 1)]);
                if (w != 0.) { fconv[2 * n] /= w; fconv[2 * n + 1] /= w; }
            }
        }
    }
}

// HEALPix nested pix2ang (z = cos(theta), phi), Gorski et al. 2005 as
// restated from src/Healpix_2.15a/healpix_base.cc:127-160,494-527.
void orc_healpix_nest_pix2zphi(int order, long long pix, double* z, double* phi)
{
    static const int jrll[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
    static const int jpll[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};
    const long long nside = 1LL << order, npface = nside * nside, npix = 12 * npface;
    const double fact2 = 4. / npix, fact1 = (nside << 1) * fact2;
    const int face = (int)(pix >> (2 * order));
    long long p = pix & (npface - 1);
    long long ix = 0, iy = 0;
    for (int b = 0; b < order; b++) {
        ix |= ((p >> (2 * b)) & 1) << b;
        iy |= ((p >> (2 * b + 1)) & 1) << b;
    }
    const long long nl4 = 4 * nside;
    const long long jr = ((long long)jrll[face] << order) - ix - iy - 1;
    long long nr, kshift;
    if (jr < nside) { nr = jr; *z = 1 - nr * nr * fact2; kshift = 0; }
    else if (jr > 3 * nside) { nr = nl4 - jr; *z = nr * nr * fact2 - 1; kshift = 0; }
    else { nr = nside; *z = (2 * nside - jr) * fact1; kshift = (jr - nside) & 1; }
    long long jp = (jpll[face] * nr + ix - iy + 1 + kshift) / 2;
    if (jp > nl4) jp -= nl4;
    if (jp < 1) jp += nl4;
    *phi = (jp - (kshift + 1) * 0.5) * ((PI / 2) / nr);
}

} // extern "C"
