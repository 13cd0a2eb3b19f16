"""HealpixSampling restated in numpy (test infrastructure).

TEST INFRASTRUCTURE ONLY: used by tests/ (as the checker of the library's sampler) and by
bench.py's reference arm and CPU-baseline leg (which must not load the library).  The shipped
library never uses it.

C1 symmetry, no random perturbation (src/healpix_sampling.cpp):
  directions    HEALPix NEST pixel centres (the oracle's pix2zphi, Gorski et al. 2005 as in
                src/Healpix_2.15a/healpix_base.cc), rot = RAD2DEG(phi), tilt = ACOSD(z),
                rot wrapped into [-180, 180]            (:534-575, 1617-1649)
  psi           nr_psi = CEIL(360 / psi_step), psi = ipsi * 360 / nr_psi      (:68-76, 577-585)
  fine          the 4 children at order + 1 (xyf2nest over (i, j) of the parent's
                (x, y, face)), each with psi - step/2 + (0.5 + k) step/2, k = 0, 1 (:1914-2040)
  translations  the disc x^2 + y^2 < range^2 + 0.001 on the step grid in Angstrom, x-major;
                fine: the 2 x 2 sub-steps of half a step                    (:291-440, 1800-1910)
  matrices      Euler_angles2matrix (src/euler.cpp:52-91)
"""
import math

import numpy as np

import oracle as _orc


def _nest2xyf(order, pix):
    npface = 1 << (2 * order)
    face = pix >> (2 * order)
    p = pix & (npface - 1)
    ix = iy = 0
    for b in range(order):
        ix |= ((p >> (2 * b)) & 1) << b
        iy |= ((p >> (2 * b + 1)) & 1) << b
    return ix, iy, face


def _xyf2nest(order, ix, iy, face):
    p = 0
    for b in range(order):
        p |= ((ix >> b) & 1) << (2 * b)
        p |= ((iy >> b) & 1) << (2 * b + 1)
    return (face << (2 * order)) + p


def _direction(order, pix):
    z, phi = _orc.healpix_pix2zphi(order, pix)
    rot = phi * 180 / math.pi
    tilt = math.acos(z) * 180. / math.pi
    while rot > 180. or rot < -180.:
        rot += -360. if rot > 180. else 360.
    return rot, tilt


def euler(rot, tilt, psi):
    """Euler_angles2matrix, row-major 9 values."""
    a, b, g = (x * math.pi / 180 for x in (rot, tilt, psi))
    ca, cb, cg, sa, sb, sg = math.cos(a), math.cos(b), math.cos(g), math.sin(a), math.sin(b), math.sin(g)
    cc, cs, sc, ss = cb * ca, cb * sa, sb * ca, sb * sa
    return [cg * cc - sg * sa, cg * cs + sg * ca, -cg * sb,
            -sg * cc - cg * sa, -sg * cs + cg * ca, sg * sb,
            sc, ss, cb]


def sampling(order, psi_step, ovs, range_px, step_px, pixel_size):
    """3D sampling lists in the library's layout (see t2b_sampling): eul_coarse (O x 9, direction-
    major, psi minor), eul_fine (O*8 x 9), trans_px (T x 2), trans_px_fine (T*4 x 2), trans_prior
    (T x 2, Angstrom) and the counts."""
    npix = 12 << (2 * order)
    dirs = [_direction(order, p) for p in range(npix)]
    npsi = math.ceil(360. / psi_step)
    step_psi = 360. / npsi
    coarse, fine = [], []
    for d in range(npix):
        for p in range(npsi):
            coarse.append(euler(dirs[d][0], dirs[d][1], p * step_psi))
            if ovs:
                x, y, face = _nest2xyf(order, d)
                for j in range(2 * y, 2 * (y + 1)):
                    for i in range(2 * x, 2 * (x + 1)):
                        fr, ft = _direction(order + 1, _xyf2nest(order + 1, i, j, face))
                        for po in range(2):
                            fine.append(euler(fr, ft, p * step_psi - 0.5 * step_psi + (0.5 + po) * step_psi / 2))
    step, rng = step_px * pixel_size, range_px * pixel_size
    maxp = math.ceil(rng / step)
    tr = [(ix * step, iy * step) for ix in range(-maxp, maxp + 1) for iy in range(-maxp, maxp + 1)
          if (ix * step) ** 2 + (iy * step) ** 2 < rng * rng + 0.001]
    tf = []
    for tx, ty in tr:
        for ox in range(2):
            for oy in range(2):
                tf.append((tx - 0.5 * step + (0.5 + ox) * step / 2, ty - 0.5 * step + (0.5 + oy) * step / 2))
    tr, tf = np.array(tr), np.array(tf).reshape(-1, 2)
    return dict(n_dir=npix, n_psi=npsi, n_trans=len(tr), nover_rot=8 if ovs else 1, nover_trans=4 if ovs else 1,
                eul_coarse=np.array(coarse), eul_fine=np.array(fine).reshape(-1, 9),
                trans_px=tr / pixel_size, trans_px_fine=tf / pixel_size, trans_prior=tr)


def sampling2d(psi_step, ovs, range_px, step_px, pixel_size):
    """2D classification (one direction, in-plane psi): the library's layout; fine psi are the
    2 halves of each psi step, wrapped above 180 deg (src/healpix_sampling.cpp:1914-2040)."""
    npsi = math.ceil(360. / psi_step)
    step_psi = 360. / npsi
    coarse, fine = [], []
    for p in range(npsi):
        coarse.append(euler(0., 0., p * step_psi))
        if ovs:
            for po in range(2):
                over = p * step_psi - 0.5 * step_psi + (0.5 + po) * step_psi / 2
                fine.append(euler(0., 0., over - 360. if over > 180. else over))
    s3 = sampling(0, 360., ovs, range_px, step_px, pixel_size)   # translations only
    return dict(n_dir=1, n_psi=npsi, n_trans=s3["n_trans"], nover_rot=2 if ovs else 1, nover_trans=s3["nover_trans"],
                eul_coarse=np.array(coarse), eul_fine=np.array(fine).reshape(-1, 9), trans_px=s3["trans_px"],
                trans_px_fine=s3["trans_px_fine"], trans_prior=s3["trans_prior"])
