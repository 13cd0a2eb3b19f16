"""FP64 oracle of the image preparation before the E-step (test infrastructure).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA image
preparation (t2-relion_b200/csrc/imageprep.cu).  The shipped library never uses it.

Restates, per particle, MlOptimiser::getFourierTransformsAndCtfs
(src/ml_optimiser.cpp:5689-6390) and the Minvsigma2 part of
precalculateShiftedImagesCtfsAndInvSigma2s (src/ml_optimiser.cpp:6680-6720) for
2D particle images of a 3D refinement or 2D classification:

  norm correction   img *= avg_norm_correction / norm          (:6014-6028)
  old offset        rounded (selfROUND), integer translation with zero fill:
                    selfTranslate(img, offset, DONT_WRAP)       (:6115-6116;
                    src/transformations.h:251-450, applyGeometry with an
                    integer shift reads in[y - ty][x - tx] exactly)
  unmasked image    FFT -> window(current_size) -> CenterFFTbySign (:6170-6180)
  soft mask         softMaskOutsideMap (src/mask.cpp:43-96): raised cosine
                    between radius and radius + width; outside it the average
                    background (zero_mask) or a noise image whose spectrum is
                    sigma2_fudge * sigma2_noise (:6187-6231)
  masked image      FFT -> power spectrum and highres_Xi2 over the full
                    transform (:6248-6275) -> window -> CenterFFTbySign (:6279-6282)
  CTF image         CTF::getFftwImage without padding (src/ctf.cpp:309-446,
                    src/ctf.h:180-238), squared when premultiplied (:6344-6350)
  Minvsigma2        1 / (sigma2_fudge * sigma2_noise[round(remap * ires)]) for
                    0 < ires < current_size/2 + 1 outside the redundant half of
                    the kx = 0 column, 0 elsewhere (:6706-6719, Mresol :5628-5660)
  scalars           1 / (sigma2_fudge * sigma2_noise[0]) (:8096), highres_Xi2,
                    rounded old offset, offset prior (999 -> 0, :5802-5807),
                    scale correction

FFT convention: RELION's FourierTransformer (src/fftw.cpp:333-365): forward
e^{-2 pi i k.x / N} divided by N^2, inverse unnormalised; numpy's FP64 FFT
computes the same sums.

Noise background.  The reference draws the noise spectrum from the process-wide
rand() stream (CPU path, src/funcs.cpp:570-620) or from curand (GPU path,
src/acc/utilities_impl.h:219-300), neither reproducible across thread
schedules.  The library and this oracle use one counter-based generator instead
(one SplitMix64 draw per half-transform element from the particle's key
random_seed + part_id and the element index; two 24-bit uniforms; Box-Muller,
FP32 on the device, FP64 here), so that the noise image is a function of the
particle alone; its spectrum is the reference's: N(0, sigma2_fudge * sigma2_noise[ires])
for the real and imaginary part of every half-transform element with
ires < N/2 + 1, zero elsewhere, transformed back unnormalised (c2r).
"""
import numpy as np

PI = 3.14159265358979323846

# per-particle parameters (t2b_prep_batch.params columns)
P_XOFF, P_YOFF, P_XPRIOR, P_YPRIOR, P_NORM, P_DEFU, P_DEFV, P_DEFANG, P_BFAC, P_KFAC, P_PHASE, P_SCALE = range(12)
NPARAM = 12


def relion_round(x):
    """ROUND (src/macros.h:195): half away from zero."""
    x = np.asarray(x, float)
    return np.where(x > 0, np.floor(x + 0.5), -np.floor(-x + 0.5)).astype(np.int64)


def window_index(s):
    """(ky, kx) of the s x (s/2+1) FFTW half transform (FOR_ALL_ELEMENTS_IN_FFTW_TRANSFORM)."""
    h = s // 2 + 1
    i = np.arange(s)[:, None]
    ky = np.where(i < h, i, i - s) * np.ones((1, h), np.int64)
    kx = np.arange(h)[None, :] * np.ones((s, 1), np.int64)
    return ky, kx


def ring_index(ky, kx):
    return relion_round(np.sqrt((ky * ky + kx * kx).astype(float)))


# ---------------------------------------------------------------- noise
M64 = (1 << 64) - 1


def splitmix64(z):
    """SplitMix64 finaliser on uint64 arrays (Steele, Lea, Flood 2014)."""
    z = (z + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(M64)
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(M64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(M64)
    return z ^ (z >> np.uint64(31))


def noise_spectrum(seed, N, sigma2_fudge, remapped):
    """N x (N/2+1) complex noise spectrum of one particle (see the module docstring)."""
    h = N // 2 + 1
    ky, kx = window_index(N)
    with np.errstate(over="ignore"):
        key = splitmix64(np.array([np.int64(seed)]).astype(np.uint64))[0]
        c = (ky % N * h + kx).astype(np.uint64)           # element index i * h + j
        x = splitmix64(key + c)
    u1 = ((x >> np.uint64(40)).astype(np.float64) + 1.0) * 2.0 ** -24                  # (0, 1]
    u2 = ((x >> np.uint64(8)) & np.uint64(0xFFFFFF)).astype(np.float64) * 2.0 ** -24    # [0, 1)
    rad = np.sqrt(-2.0 * np.log(u1))
    ires = ring_index(ky, kx)
    sig = np.zeros(ky.shape)
    ok = ires < h
    sig[ok] = np.sqrt(sigma2_fudge * remapped[ires[ok]])
    return rad * np.cos(2 * PI * u2) * sig + 1j * rad * np.sin(2 * PI * u2) * sig


def remap_noise(sigma2, N, remap):
    """remapped_sigma2_noise (src/ml_optimiser.cpp:6196-6205)."""
    out = np.zeros(N // 2 + 1)
    for i, v in enumerate(sigma2):
        ir = int(relion_round(remap * i))
        if ir < out.size:
            out[ir] = v
    return out


def noise_image(seed, N, sigma2_fudge, sigma2, remap):
    F = noise_spectrum(seed, N, sigma2_fudge, remap_noise(sigma2, N, remap))
    # unnormalised c2r: inverse over y, then the real inverse over x (imaginary
    # parts of the kx = 0 and kx = N/2 terms do not enter)
    return np.fft.irfft2(F, s=(N, N)) * (N * N)


# ---------------------------------------------------------------- steps
def translate_int(img, tx, ty):
    """out[y][x] = img[y - ty][x - tx], zero outside."""
    N = img.shape[0]
    out = np.zeros_like(img)
    ys, yd = (slice(0, N - ty), slice(ty, N)) if ty >= 0 else (slice(-ty, N), slice(0, N + ty))
    xs, xd = (slice(0, N - tx), slice(tx, N)) if tx >= 0 else (slice(-tx, N), slice(0, N + tx))
    if abs(tx) < N and abs(ty) < N:
        out[yd, xd] = img[ys, xs]
    return out


def soft_mask(img, radius, width, noise=None):
    N = img.shape[0]
    c = np.arange(N) - N // 2
    r = np.sqrt((c[:, None] ** 2 + c[None, :] ** 2).astype(float))
    rp = radius + width
    rc = 0.5 + 0.5 * np.cos(PI * (rp - r) / width)
    edge = (r >= radius) & (r <= rp)
    out_ = r > rp
    if noise is None:
        s = np.sum(out_) + np.sum(rc[edge])
        bg = (np.sum(img[out_]) + np.sum(rc[edge] * img[edge])) / s if s > 0 else 0.0
        fill = np.full_like(img, bg)
    else:
        fill = noise
    res = img.copy()
    res[out_] = fill[out_]
    res[edge] = (1 - rc[edge]) * img[edge] + rc[edge] * fill[edge]
    return res


def window_center(F, s):
    """windowFourierTransform to s (src/fftw.h:736-790) then CenterFFTbySign (:389-402)."""
    N = F.shape[0]
    ky, kx = window_index(s)
    W = F[ky % N, kx]
    sign = np.where(((np.arange(s)[:, None] ^ np.arange(s // 2 + 1)[None, :]) & 1) != 0, -1.0, 1.0)
    return W * sign


def ctf_window(par, cfg, s):
    """CTF::getFftwImage without padding, on the s window of an N box (src/ctf.cpp:438-446)."""
    defU, defV, ang, bfac, kfac, phase = (par[P_DEFU], par[P_DEFV], par[P_DEFANG], par[P_BFAC], par[P_KFAC],
                                          par[P_PHASE])
    kV = cfg["voltage"] * 1e3
    lam = 12.2643247 / np.sqrt(kV * (1. + kV * 0.978466e-6))
    K1 = PI / 2 * 2 * lam
    K2 = PI / 2 * cfg["cs"] * 1e7 * lam ** 3
    q0 = cfg["q0"]
    K3 = np.arctan(q0 / np.sqrt(1 - q0 * q0))
    K4 = -bfac / 4.
    K5 = phase * PI / 180.
    az = ang * PI / 180.
    c, sn = np.cos(az), np.sin(az)
    # A = Q^t D Q, D = diag(-defU, -defV)  (src/ctf.cpp:236-256)
    Axx = -defU * c * c - defV * sn * sn
    Axy = (defV - defU) * c * sn
    Ayy = -defU * sn * sn - defV * c * c
    ky, kx = window_index(s)
    xs = cfg["image_size"] * cfg["pixel_size"]
    X, Y = kx / xs, ky / xs
    u2 = X * X + Y * Y
    gamma = K1 * (Axx * X * X + 2.0 * Axy * X * Y + Ayy * Y * Y) + K2 * u2 * u2 - K5 - K3
    v = -np.sin(gamma)
    if cfg.get("intact_ctf_first_peak", 0):
        v = np.where(np.abs(gamma) < PI / 2, 1.0, v)
    v = v * np.exp(K4 * u2)
    if cfg.get("ctf_phase_flipped", 0):
        v = np.abs(v)
    elif cfg.get("only_flip_phases", 0):
        v = np.where(v < 0, -1.0, 1.0)
    v = v * kfac
    v = np.where(np.abs(v) < 1e-8, np.where(v >= 0, 1e-8, -1e-8), v)   # SGN (src/macros.h:141)
    if cfg.get("ctf_premultiplied", 0):
        v = v * v
    return v


def minvsigma2_window(cfg, s):
    ky, kx = window_index(s)
    ires = ring_index(ky, kx)
    h = s // 2 + 1
    valid = (ires < h) & ~((kx == 0) & (ky < 0)) & (ires > 0)
    sig = np.asarray(cfg["sigma2_noise"], float)
    irr = relion_round(cfg.get("remap_minv", 1.0) * ires)
    valid &= irr < sig.size
    out = np.zeros(ky.shape)
    out[valid] = 1.0 / (cfg["sigma2_fudge"] * sig[irr[valid]])
    return out


def prepare(images, params, part_id, cfg):
    """images (n, N, N); params (n, 12); part_id (n,) -> dict of E-step inputs (FP64).

    cfg keys: image_size, current_size, pixel_size, mask_radius, width_mask_edge,
    zero_mask, random_seed, do_norm_correction, avg_norm_correction, sigma2_fudge,
    sigma2_noise, remap_noise, remap_minv, do_ctf_correction, ctf_premultiplied,
    ctf_phase_flipped, only_flip_phases, intact_ctf_first_peak, voltage, cs, q0.
    """
    N, s = cfg["image_size"], cfg["current_size"]
    n = images.shape[0]
    h, hs = N // 2 + 1, s // 2 + 1
    P = s * hs
    out = dict(fimg=np.zeros((n, P), complex), fimg_nomask=np.zeros((n, P), complex), ctf=np.zeros((n, P)),
               minvsigma2=np.zeros((n, P)), scalars=np.zeros((n, 8)), power=np.zeros((n, h)))
    sig = np.asarray(cfg["sigma2_noise"], float)
    minv = minvsigma2_window(cfg, s)
    ky, kx = window_index(N)
    ires = ring_index(ky, kx)
    inspec = (ires > 0) & (ires < h) & ~((kx == 0) & (ky < 0))
    for p in range(n):
        par = params[p]
        img = images[p].astype(np.float64)
        if cfg.get("do_norm_correction", 0):
            img = img * (cfg["avg_norm_correction"] / par[P_NORM])
        tx, ty = int(relion_round(par[P_XOFF])), int(relion_round(par[P_YOFF]))
        img = translate_int(img, tx, ty)
        Fu = np.fft.rfft2(img) / (N * N)
        noise = None
        if not cfg.get("zero_mask", 0):
            noise = noise_image(int(cfg["random_seed"]) + int(part_id[p]), N, cfg["sigma2_fudge"], sig,
                                cfg.get("remap_noise", 1.0))
        m = soft_mask(img, cfg["mask_radius"], cfg["width_mask_edge"], noise)
        F = np.fft.rfft2(m) / (N * N)
        a2 = np.abs(F) ** 2
        out["power"][p] = np.bincount(ires[inspec], weights=a2[inspec], minlength=h)[:h]
        out["fimg"][p] = window_center(F, s).reshape(-1)
        out["fimg_nomask"][p] = window_center(Fu, s).reshape(-1)
        if cfg.get("do_ctf_correction", 1):
            out["ctf"][p] = ctf_window(par, cfg, s).reshape(-1)
        else:
            out["ctf"][p] = 1.0
        out["minvsigma2"][p] = minv.reshape(-1)
        sc = out["scalars"][p]
        sc[0] = 1.0 / (cfg["sigma2_fudge"] * sig[0]) if sig[0] > 0 else 0.0
        sc[1] = float(np.sum(a2[inspec & (ires >= hs)])) if s < N else 0.0
        sc[2], sc[3] = tx, ty
        px, py = par[P_XPRIOR], par[P_YPRIOR]
        sc[4] = 0.0 if 998.99 < px < 999.01 else px
        sc[5] = 0.0 if 998.99 < py < 999.01 else py
        sc[6] = par[P_SCALE]
    return out
