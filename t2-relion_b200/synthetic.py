"""Seeded synthetic E-step inputs (stand-in for the reference's AE datasets).

Follows the simulator of src/apps/project.cpp:254-282 in Fourier space:
reference map -> central slice at the true pose -> CTF -> phase shift -> white
complex Gaussian noise, on the windowed FFTW half-transform the E-step reads.
The reference map is a sum of seeded Gaussian blobs, zero padded by the
padding factor and Fourier transformed into the centred half-complex layout of
RELION's Projector (src/projector.cpp:55-80, 120-330; no gridding
pre-correction).  Everything is numpy / FP64 and deterministic for a seed.
"""
import numpy as np

PI = 3.14159265358979323846


def blob_volume(n, n_blobs=40, sigma=(2.0, 5.0), seed=0, ndim=3):
    """n^ndim real map of Gaussian blobs (centres within 0.3 n of the centre)."""
    rng = np.random.default_rng(seed)
    ax = np.arange(n) - n // 2
    grids = np.meshgrid(*([ax] * ndim), indexing="ij")
    vol = np.zeros((n,) * ndim)
    for _ in range(n_blobs):
        c = rng.uniform(-0.3 * n, 0.3 * n, ndim)
        s = rng.uniform(*sigma)
        a = rng.uniform(0.5, 1.5)
        r2 = sum((g - ci) ** 2 for g, ci in zip(grids, c))
        vol += a * np.exp(-r2 / (2 * s * s))
    return vol


def blob_class_volumes(n, n_classes, n_blobs=40, swap_frac=0.1, sigma=(2.0, 5.0), seed=0):
    """n^3 maps of `n_classes` classes that differ by a subset of their blobs: a seeded set of
    n_blobs Gaussian blobs, of which each class replaces its own swap_frac share (class k drops
    blobs [k m, k m + m), m = round(swap_frac n_blobs), and adds m blobs of its own).  Each blob
    is evaluated inside its own box of +-4 sigma (the rest is below 4e-4 of its peak)."""
    rng = np.random.default_rng(seed)
    m = int(round(swap_frac * n_blobs))

    def draw(k):
        return [(rng.uniform(-0.3 * n, 0.3 * n, 3), rng.uniform(*sigma), rng.uniform(0.5, 1.5)) for _ in range(k)]
    base = draw(n_blobs)
    extra = [draw(m) for _ in range(n_classes)]
    vols = []
    for k in range(n_classes):
        blobs = [b for i, b in enumerate(base) if not (k * m <= i < (k + 1) * m)] + extra[k]
        vol = np.zeros((n, n, n))
        for c, sg, a in blobs:
            ctr = c + n // 2
            lo = np.maximum(np.floor(ctr - 4 * sg).astype(int), 0)
            hi = np.minimum(np.ceil(ctr + 4 * sg).astype(int) + 1, n)
            ax = [np.arange(lo[d], hi[d]) - ctr[d] for d in range(3)]
            r2 = ax[0][:, None, None] ** 2 + ax[1][None, :, None] ** 2 + ax[2][None, None, :] ** 2
            vol[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] += a * np.exp(-r2 / (2 * sg * sg))
        vols.append(vol)
    return vols


def pad_size(r_max, padding_factor=2):
    """Projector::initialiseData (src/projector.cpp:56-84)."""
    return 2 * (int(np.floor(padding_factor * r_max + 0.5)) + 1) + 1


def fourier_map(vol, r_max, padding_factor=2):
    """Centred half-complex Fourier map (complex64) of a 3D or 2D volume.

    3D: shape (pad, pad, pad//2+1) indexed [z - initz][y - inity][x];
    2D: shape (pad, pad//2+1).  Frequencies beyond r_max*padding_factor are 0.
    """
    ndim = vol.ndim
    n = vol.shape[0]
    m = padding_factor * n
    big = np.zeros((m,) * ndim)
    sl = tuple(slice(m // 2 - n // 2, m // 2 - n // 2 + n) for _ in range(ndim))
    big[sl] = vol
    F = np.fft.rfftn(np.fft.ifftshift(big)) / float(n ** ndim)
    ps = pad_size(r_max, padding_factor)
    c = ps // 2
    xdim = ps // 2 + 1
    rp2 = (r_max * padding_factor) ** 2
    k = np.arange(-c, c + 1)
    x = np.arange(xdim)
    # a grid of r_max at Nyquist reaches one column past the transform's last (m/2): such
    # elements lie outside r_max * padding_factor and are zeroed, so their index is clipped
    xc = min(xdim, F.shape[-1]) - 1
    if ndim == 3:
        kz, ky, kx = np.meshgrid(k, k, x, indexing="ij")
        out = F[kz % m, ky % m, np.minimum(kx, xc)]
        out[kz * kz + ky * ky + kx * kx > rp2] = 0
    else:
        ky, kx = np.meshgrid(k, x, indexing="ij")
        out = F[ky % m, np.minimum(kx, xc)]
        out[ky * ky + kx * kx > rp2] = 0
    return np.ascontiguousarray(out.astype(np.complex64))


def window_coords(s):
    """(ky, kx) of every pixel of the s x (s/2+1) FFTW window."""
    xh = s // 2 + 1
    i = np.arange(s)[:, None]
    ky = np.where(i < xh, i, i - s) * np.ones((1, xh), int)
    kx = np.arange(xh)[None, :] * np.ones((s, 1), int)
    return ky.reshape(-1), kx.reshape(-1)


def euler_matrix(rot, tilt, psi):
    """Euler_angles2matrix (src/euler.cpp:52-91), angles in degrees; (..., 3, 3)."""
    a, b, g = (np.asarray(x, float) * PI / 180 for x in (rot, tilt, psi))
    ca, cb, cg, sa, sb, sg = np.cos(a), np.cos(b), np.cos(g), np.sin(a), np.sin(b), np.sin(g)
    cc, cs, sc, ss = cb * ca, cb * sa, sb * ca, sb * sa
    A = np.empty(np.shape(a) + (3, 3))
    A[..., 0, 0] = cg * cc - sg * sa
    A[..., 0, 1] = cg * cs + sg * ca
    A[..., 0, 2] = -cg * sb
    A[..., 1, 0] = -sg * cc - cg * sa
    A[..., 1, 1] = -sg * cs + cg * ca
    A[..., 1, 2] = sg * sb
    A[..., 2, 0] = sc
    A[..., 2, 1] = ss
    A[..., 2, 2] = cb
    return A


def project(fmap, A, s, r_max, padding_factor=2):
    """Trilinear (3D) / bilinear (2D) central slices for matrices A (B,3,3) -> (B, P) c128."""
    A = np.asarray(A, float).reshape(-1, 3, 3)
    ky, kx = window_coords(s)
    inside = (kx * kx + ky * ky <= (s // 2) ** 2) & (kx * kx + ky * ky <= r_max * r_max)
    c = fmap.shape[0] // 2
    out = np.zeros((A.shape[0], ky.size), np.complex128)
    F = fmap.astype(np.complex128)
    for b in range(A.shape[0]):
        At = A[b].T * padding_factor
        xp = At[0, 0] * kx + At[0, 1] * ky
        yp = At[1, 0] * kx + At[1, 1] * ky
        zp = At[2, 0] * kx + At[2, 1] * ky
        neg = xp < 0
        xp, yp, zp = np.where(neg, -xp, xp), np.where(neg, -yp, yp), np.where(neg, -zp, zp)
        x0 = np.floor(xp).astype(int)
        y0 = np.floor(yp).astype(int)
        fx, fy = xp - x0, yp - y0
        y0 = y0 + c
        if fmap.ndim == 3:
            z0 = np.floor(zp).astype(int)
            fz = zp - z0
            z0 = z0 + c
            ok = inside & (x0 >= 0) & (x0 + 1 < fmap.shape[2]) & (y0 >= 0) & (y0 + 1 < fmap.shape[1]) \
                & (z0 >= 0) & (z0 + 1 < fmap.shape[0])
            x0, y0, z0 = np.where(ok, x0, 0), np.where(ok, y0, 0), np.where(ok, z0, 0)

            def at(dz, dy, dx):
                return F[z0 + dz, y0 + dy, x0 + dx]
            x00 = at(0, 0, 0) + (at(0, 0, 1) - at(0, 0, 0)) * fx
            x01 = at(1, 0, 0) + (at(1, 0, 1) - at(1, 0, 0)) * fx
            x10 = at(0, 1, 0) + (at(0, 1, 1) - at(0, 1, 0)) * fx
            x11 = at(1, 1, 0) + (at(1, 1, 1) - at(1, 1, 0)) * fx
            y0v = x00 + (x10 - x00) * fy
            y1v = x01 + (x11 - x01) * fy
            v = y0v + (y1v - y0v) * fz
        else:
            ok = inside & (x0 >= 0) & (x0 + 1 < fmap.shape[1]) & (y0 >= 0) & (y0 + 1 < fmap.shape[0])
            x0, y0 = np.where(ok, x0, 0), np.where(ok, y0, 0)
            a0 = F[y0, x0] + (F[y0, x0 + 1] - F[y0, x0]) * fx
            a1 = F[y0 + 1, x0] + (F[y0 + 1, x0 + 1] - F[y0 + 1, x0]) * fx
            v = a0 + (a1 - a0) * fy
        v = np.where(neg, np.conj(v), v)
        out[b] = np.where(ok, v, 0)
    return out


def ctf_image(params, ori_size, angpix, s):
    """CTF::getCTF on the window (src/ctf.h:181-238, src/ctf.cpp:206-256).

    params: defU, defV, defAngle, kV, Cs, Q0, Bfac, scale, phase_shift.
    """
    defU, defV, ang, kV, Cs, Q0, Bfac, scale, phase = params
    lam = 12.2643247 / np.sqrt(kV * 1e3 * (1. + kV * 1e3 * 0.978466e-6))
    K1 = PI / 2 * 2 * lam
    K2 = PI / 2 * Cs * 1e7 * lam ** 3
    K3 = np.arctan(Q0 / np.sqrt(1 - Q0 * Q0))
    K4 = -Bfac / 4.
    K5 = phase * PI / 180
    az = ang * PI / 180
    c, sn = np.cos(az), np.sin(az)
    Axx = -defU * c * c - defV * sn * sn
    Axy = (defV - defU) * c * sn
    Ayy = -defU * sn * sn - defV * c * c
    ky, kx = window_coords(s)
    X = kx / (ori_size * angpix)
    Y = ky / (ori_size * angpix)
    u2 = X * X + Y * Y
    gamma = K1 * (Axx * X * X + 2.0 * Axy * X * Y + Ayy * Y * Y) + K2 * u2 * u2 - K5 - K3
    r = -np.sin(gamma) * np.exp(K4 * u2) * scale
    r = np.where(np.abs(r) < 1e-8, np.where(r >= 0, 1.0, -1.0) * 1e-8, r)
    return r.astype(np.float32)


def mresol(s):
    ky, kx = window_coords(s)
    ires = np.rint(np.sqrt(ky * ky + kx * kx)).astype(int)
    xh = s // 2 + 1
    return np.where((ires < xh) & ~((kx == 0) & (ky < 0)), ires, -1)


def make_particles(fmap, n, *, ori_size, s, r_max, angpix, snr, seed, max_shift=3.0,
                   padding_factor=2, ref_dim=3, defocus=(10000., 30000.), astig=1000.,
                   sigma2=None, classes=None, class_maps=None):
    """n particles on the s-window.  Returns a dict of E-step inputs and truth.

    The image of a particle with true shift t is CTF * P(A) * e^{+2 pi i k.t/N}, so
    the E-step's best translation (shift applied as e^{-2 pi i k.t/N}) is t.
    Noise: each component N(0, sigma2); sigma2 is set so that the mean
    |CTF P|^2 / (2 sigma2) over the resolution mask equals snr.
    """
    rng = np.random.default_rng(seed)
    if ref_dim == 3:
        rot = rng.uniform(-180, 180, n)
        tilt = np.degrees(np.arccos(rng.uniform(-1, 1, n)))
        psi = rng.uniform(0, 360, n)
    else:
        rot = np.zeros(n)
        tilt = np.zeros(n)
        psi = rng.uniform(0, 360, n)
    shifts = rng.uniform(-max_shift, max_shift, (n, 2))
    defU = rng.uniform(*defocus, n)
    defV = defU - rng.uniform(0, astig, n)
    dang = rng.uniform(0, 180, n)
    A = euler_matrix(rot, tilt, psi)
    cls = np.zeros(n, int) if classes is None else classes
    if class_maps is None:
        proj = project(fmap, A, s, r_max, padding_factor)
    else:
        proj = np.zeros((n, s * (s // 2 + 1)), np.complex128)
        for k in np.unique(cls):
            sel = np.nonzero(cls == k)[0]
            proj[sel] = project(class_maps[k], A[sel], s, r_max, padding_factor)
    ky, kx = window_coords(s)
    ctf = np.stack([ctf_image((defU[i], defV[i], dang[i], 300., 2.7, 0.1, 0., 1., 0.), ori_size, angpix, s)
                    for i in range(n)])
    sig = ctf * proj
    phase = 2 * PI * (kx[None, :] * shifts[:, :1] + ky[None, :] * shifts[:, 1:2]) / ori_size
    sig = sig * np.exp(1j * phase)
    mr = mresol(s)
    mask = mr > 0
    if sigma2 is None:
        sigma2 = float(np.mean(np.abs(sig[:, mask]) ** 2) / (2 * snr))
    noise = rng.normal(0, np.sqrt(sigma2), (n, ky.size, 2))
    fimg = (sig + noise[..., 0] + 1j * noise[..., 1]).astype(np.complex64)
    minv = np.where(mask, 1.0 / sigma2, 0.0).astype(np.float32)
    minv = np.broadcast_to(minv, (n, ky.size)).copy()
    # noise power between the window and Nyquist of the full box (highres_Xi2)
    nf = ori_size
    full_i = np.arange(nf)[:, None]
    fy = np.where(full_i < nf // 2 + 1, full_i, full_i - nf)
    fx = np.arange(nf // 2 + 1)[None, :]
    ir = np.rint(np.sqrt(fy * fy + fx * fx))
    nhr = int(np.sum((ir >= s // 2 + 1) & (ir < nf // 2 + 1) & ~((fx == 0) & (fy < 0))))
    xi2 = rng.chisquare(2 * nhr, n) * sigma2 if nhr > 0 else np.zeros(n)
    scal = np.zeros((n, 8))
    scal[:, 0] = 1.0 / sigma2
    scal[:, 1] = xi2
    scal[:, 6] = 1.0
    return dict(fimg=fimg, ctf=ctf, minv=minv, scalars=scal, sigma2=sigma2,
                rot=rot, tilt=tilt, psi=psi, shifts=shifts, A=A, classes=cls, defU=defU, defV=defV, dang=dang)


# Named workloads: the 3D refinements at box 64 and box 128.  Sizes only; seeds are per call.
CONFIGS = {
    # 3D refine, CPU-runnable: 64^3, 2 A/px, order 2, psi 7.5, range 3 step 1, r 16
    "refine3d_box64": dict(ori_size=64, angpix=2.0, n_blobs=40, healpix_order=2, psi_step=7.5,
                           offset_range=3, offset_step=1, r_max=16, snr=0.05, ovs=0,
                           bp_r_max=16, max_shift=3.0),
    # box 128, order 3 + adaptive oversampling 1, range 5 step 1, r 40, BP grid r_max 64
    "refine3d_box128": dict(ori_size=128, angpix=1.3, n_blobs=40, healpix_order=3, psi_step=7.5,
                            offset_range=5, offset_step=1, r_max=40, snr=0.03, ovs=1,
                            bp_r_max=64, max_shift=5.0),
}
