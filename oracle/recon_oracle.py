"""FP64 oracle of the M-step reconstruction on the device (test infrastructure).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of
t2-relion_b200/csrc/recon.cu.  The shipped library never uses it.

Restates in numpy, on a centred half-complex backprojection grid (data
complex, weight real; z, y centred at -initz, -inity; x from 0; 3D grids of
3D refinements or 2D grids of 2D classes):

  reconstruct_map   BackProjector::reconstruct (src/backprojector.cpp:1344-1530),
                    the skip-gridding path (the reference's default:
                    skip_gridding = !--dont_skip_gridding, src/ml_optimiser.cpp:525):
                    Projector::decenter to the FFTW layout of the pad_size box
                    (r^2 <= ROUND(r_max pad)^2), the MAP term
                    1 / (pad^3 tau2_fudge tau2[ROUND(r / pad)]) added to the
                    weight for r^2 < max_r2 and shells >= minres_map (:1412-1455),
                    the division by max(weight, radial average / 1000) (:1463-1531);
                    then windowToOridimRealSpace (:2486-2620): window the transform
                    to pad * ori_size (src/fftw.h:736-790), CenterFFTbySign, unnormalised inverse FFT,
                    real-space window to ori_size, divide by pad^3 ori_size (2D
                    particles), softMaskOutsideMap (src/mask.cpp:43-96; radius
                    ori_size / 2, cosine width 3, average background); and
                    Projector::griddingCorrect (src/projector.cpp:489-522:
                    divide by sinc^2 of r / (ori_size pad), trilinear)
                    With gridding_iter > 0 (--dont_skip_gridding, :1532-1655), the
                    division is replaced by the iterative weights of Pipe & Menon
                    (1999): data and weight divided by `normalise`; weights w_n = 1
                    inside r^2 < max_r2; each iteration convolves w_n * weight with the
                    blob (inverse FFT, multiply by the blob's tabulated Fourier
                    transform over its value at 0, forward FFT:
                    BackProjector::convoluteBlobRealSpace, :2439-2480) and divides w_n
                    by max(1e-6, |result|) inside max_r2; then Fconv = data * w_n.
  ftblob_table      TabFtBlob (src/tabfuncs.cpp:95-121): the Fourier transform of the
                    order-0 Kaiser-Bessel blob of radius 3.8 and alpha 15 in 3D
                    (Lewitt 1990), 10,000 samples over [0, 0.5), looked up at
                    floor(|r| / 5e-5), 0 beyond
  enforce_hermitian_symmetry
                    BackProjector::enforceHermitianSymmetry (src/backprojector.cpp:2104-2121),
                    applied by MlOptimiser::maximization before reconstruct
                    (src/ml_optimiser.cpp:4626)
  point_group       SymList::read_sym_file + compute_subgroup (src/symmetries.cpp:133-191,
                    243-325), with the generators of SymList::fill_symmetry_class
                    (:606-725): rotations k 360 / n about each axis, transposed, entries
                    below 1e-6 zeroed; mirror planes I - 2 u u^T; the inversion -I; closed
                    under products in the reference's order, equality within 1e-6, the
                    identity left out
  apply_point_group_symmetry
                    BackProjector::applyPointGroupSymmetry (src/backprojector.cpp:2279-2435):
                    the sum over the operators of the trilinear read at R (x, y, z)
                    (conjugated where the rotated x < 0), inside ROUND(r_max pad)^2
  helical_operators BackProjector::applyHelicalSymmetry (:2122-2277): the rotations about z
                    and the z phase shifts of the helical units, summed by
                    apply_point_group_symmetry(..., zshift)
  downsampled_fsc   getDownsampledAverage + calculateDownSampledFourierShellCorrelation
                    (src/backprojector.cpp:933-1040)
  update_ssnr       BackProjector::updateSSNRarrays (src/backprojector.cpp:1041-1205)
"""
import numpy as np

PI = 3.14159265358979323846


def relion_round(x):
    x = np.asarray(x, float)
    return np.where(x > 0, np.floor(x + 0.5), -np.floor(-x + 0.5)).astype(np.int64)


def _logical(shape, initz, inity):
    zd, yd, xd = shape
    k = np.arange(zd)[:, None, None] + initz
    i = np.arange(yd)[None, :, None] + inity
    j = np.arange(xd)[None, None, :]
    return k, i, j


def enforce_hermitian_symmetry(data, weight):
    """The reference's loop over the x = 0 plane, element by element in its order: for z from
    STARTINGZ to FINISHINGZ, y from (z < 0 ? 0 : 1) to FINISHINGY, the pair (z, y) / (-z, -y)
    gets fsum = data(z, y) + conj(data(-z, -y)) and conj(fsum), and both weights their sum.
    Returns new arrays (3D [z][y][x] or 2D [y][x] centred grids)."""
    d = np.array(data, copy=True)
    w = np.array(weight, copy=True)
    two_d = w.ndim == 2
    if two_d:
        d, w = d[None], w[None]
    zd, yd = w.shape[0], w.shape[1]
    initz, inity = -(zd // 2), -(yd // 2)
    for z in range(initz, initz + zd):
        for y in range(0 if z < 0 else 1, inity + yd):
            a = (z - initz, y - inity, 0)
            b = (-z - initz, -y - inity, 0)
            f = d[a] + np.conj(d[b])
            d[a] = f
            d[b] = np.conj(f)
            ws = w[a] + w[b]
            w[a] = ws
            w[b] = ws
    return (d[0], w[0]) if two_d else (d, w)


# generators of the point groups (src/symmetries.cpp:606-725): ("rot", fold, axis),
# ("mirror", normal) or ("inv",)
_T = [("rot", 3, (0., 0., 1.)), ("rot", 2, (0., 0.816496, 0.577350))]
_O = [("rot", 3, (.5773502, .5773502, .5773502)), ("rot", 4, (0., 0., 1.))]
_I2 = [("rot", 2, (0., 0., 1.)), ("rot", 5, (0.525731114, 0., 0.850650807)),
       ("rot", 3, (0., 0.356822076, 0.934172364))]
_I1 = [("rot", 2, (1., 0., 0.)), ("rot", 5, (0.85065080702670, 0., -0.5257311142635)),
       ("rot", 3, (0.9341723640, 0.3568220765, 0.))]
_I3 = [("rot", 2, (-0.5257311143, 0., 0.8506508070)), ("rot", 5, (0., 0., 1.)),
       ("rot", 3, (-0.4911234778630044, 0.3568220764705179, 0.7946544753759428))]
_I4 = [("rot", 2, (0.5257311143, 0., 0.8506508070)), ("rot", 5, (0.8944271932547096, 0., 0.4472135909903704)),
       ("rot", 3, (0.4911234778630044, 0.3568220764705179, 0.7946544753759428))]
_PG_FIXED = {
    "CI": [("inv",)], "CS": [("mirror", (0., 0., 1.))],
    "T": _T, "TD": _T + [("mirror", (1.4142136, 2.4494897, 0.0000000))],
    "TH": [("rot", 3, (0., 0., 1.)), ("rot", 2, (0., -0.816496, -0.577350)), ("inv",)],
    "O": _O, "OH": _O + [("mirror", (0., 1., 1.))],
    "I": _I2, "I2": _I2, "I1": _I1, "I3": _I3, "I4": _I4,
    "IH": _I2 + [("mirror", (1., 0., 0.))], "I2H": _I2 + [("mirror", (1., 0., 0.))],
    "I1H": _I1 + [("mirror", (0., 0., -1.))], "I3H": _I3 + [("mirror", (0.850650807, 0., 0.525731114))],
    "I4H": _I4 + [("mirror", (0.850650807, 0., -0.525731114))],
}


def _pg_generators(name):
    """Generators of a group named as SymList::isSymmetryGroup reads it (src/symmetries.cpp:331-600)."""
    g = name.upper().replace(" ", "")
    if g in ("", "C1"):
        return []
    if g in _PG_FIXED:
        return _PG_FIXED[g]
    suffix = g[-1] if g[-1:] in ("V", "H") else ""
    digits = g[1:len(g) - len(suffix)]
    if g[:1] in ("C", "D", "S") and 1 <= len(digits) <= 2 and digits.isdigit() and int(digits) >= 1:
        n = int(digits)
        z = ("rot", n, (0., 0., 1.))
        if g[0] == "S" and not suffix:
            if n % 2:
                raise ValueError("the order of an Sn group must be even")
            return [("rot", n // 2, (0., 0., 1.)), ("inv",)]
        if g[0] == "C":
            return {"": [z], "V": [z, ("mirror", (0., 1., 0.))], "H": [z, ("mirror", (0., 0., 1.))]}[suffix]
        if g[0] == "D":
            dn = ([z] if n > 1 else []) + [("rot", 2, (1., 0., 0.))]
            return {"": dn, "V": dn + [("mirror", (1., 0., 0.))], "H": dn + [("mirror", (0., 0., 1.))]}[suffix]
    raise ValueError(f"point group {name!r} is not one of C1, Cn, Ci, Cs, Cnv, Cnh, Sn, Dn, Dnv, Dnh, "
                     "T, Td, Th, O, Oh, I, I1-I4, Ih, I1h-I4h")


def point_group(name):
    """The group's operators other than the identity, (n, 3, 3), built as SymList builds them.
    A rotation axis contributes the transposes of its rotations by k 360 / fold (axis-angle matrix
    cos I + sin [a]x + (1 - cos) a a^T, zeroed below 1e-6); a mirror plane of unit normal u the
    reflection I - 2 u u^T; an inversion -I.  Each operator carries the reference's second matrix
    L = diag(1, 1, lz): lz = -1 for the inversion, 1 otherwise.  The list is then closed under
    products (R_i R_j, lz_i lz_j) in the order of found_not_tried (src/symmetries.cpp:243-270:
    for n = 0, 1, ..., the pairs (0..n, n), then (n, n-1..0)), appending each product that is
    neither the identity nor present (lz equal and every entry within 1e-6), zeroed below 1e-6."""
    zero = lambda m: np.where(np.abs(m) < 1e-6, 0.0, m)
    ops = []
    for gen in _pg_generators(name):
        if gen[0] == "inv":
            ops.append((-np.eye(3), -1))
            continue
        a = np.asarray(gen[-1], float) / np.linalg.norm(gen[-1])
        if gen[0] == "mirror":
            ops.append((np.eye(3) - 2.0 * np.outer(a, a), 1))
            continue
        fold = gen[1]
        cross = np.array([[0., -a[2], a[1]], [a[2], 0., -a[0]], [-a[1], a[0], 0.]])
        for k in range(1, fold):
            t = k * 2.0 * PI / fold
            rot = np.cos(t) * np.eye(3) + np.sin(t) * cross + (1.0 - np.cos(t)) * np.outer(a, a)
            ops.append((zero(rot.T), 1))
    R = np.zeros((1001, 3, 3))
    L = np.zeros(1001, np.int64)
    R[0], L[0] = np.eye(3), 1            # slot 0: the identity, never part of the result
    for m, (r, lz) in enumerate(ops, 1):
        R[m], L[m] = r, lz
    m = len(ops) + 1
    n = 1
    while n < m:
        for i, j in [(i, n) for i in range(1, n + 1)] + [(n, j) for j in range(n - 1, 0, -1)]:
            p, plz = R[i] @ R[j], L[i] * L[j]
            if np.any(np.all(np.abs(R[:m] - p) <= 1e-6, axis=(1, 2)) & (L[:m] == plz)):
                continue
            if m == 1001:
                raise ValueError("point group does not close")
            R[m], L[m] = zero(p), plz
            m += 1
        n += 1
    return R[1:m].copy()


def helical_operators(nr_asu, twist, rise, ori_size, pad):
    """The operators and z shifts of BackProjector::applyHelicalSymmetry (src/backprojector.cpp:
    2122-2277): for hh = -n/2 .. n/2 - 1 (+1 for odd n) other than 0, rotation3DMatrix(-hh twist,
    'Z') = [[c, -s, 0], [s, c, 0], [0, 0, 1]] zeroed below 1e-6, and zshift = hh rise /
    (-ori_size pad) (0 when rise is 0)."""
    mats, zsh = [], []
    if nr_asu < 2:
        return np.zeros((0, 3, 3)), np.zeros(0)
    h_min = -(nr_asu // 2)
    for hh in range(h_min, -h_min + nr_asu % 2):
        if hh == 0:
            continue
        ang = (hh * -twist) * PI / 180.0
        r = np.array([[np.cos(ang), -np.sin(ang), 0.], [np.sin(ang), np.cos(ang), 0.], [0., 0., 1.]])
        mats.append(np.where(np.abs(r) < 1e-6, 0.0, r))
        zsh.append((hh * rise) / (-ori_size * float(pad)) if abs(rise) > 0 else 0.0)
    return np.array(mats), np.array(zsh)


def apply_point_group_symmetry(data, weight, mats, r_max, pad, zshift=None):
    """Sum over the operators R of the grid read at R (x, y, z), added to the grid itself, for
    r^2 <= ROUND(r_max pad)^2 (FP64 coordinates and sums; the reads come from the input
    grid).  With zshift (helical symmetry), operator s's data read is also multiplied by
    e^{2 pi i z zshift[s]}, z the voxel's own, formed as (ac - bd, (a + b)(c + d) - ac - bd).
    3D centred half-complex grids; returns new complex128 / float64 arrays."""
    d = np.asarray(data, np.complex128)
    w = np.asarray(weight, np.float64)
    zd, yd, xd = w.shape
    initz, inity = -(zd // 2), -(yd // 2)
    k, i, j = _logical(w.shape, initz, inity)
    x, y, z = [np.broadcast_to(a, w.shape).astype(np.float64).ravel() for a in (j, i, k)]
    rp = int(relion_round(r_max * pad))
    inside = x * x + y * y + z * z <= rp * rp
    x, y, z = x[inside], y[inside], z[inside]
    sd = d.ravel().copy()
    sw = w.ravel().copy()
    acc_d = np.zeros(x.size, np.complex128)
    acc_w = np.zeros(x.size)
    for s_, m in enumerate(mats):
        xp = x * m[0, 0] + y * m[0, 1] + z * m[0, 2]
        yp = x * m[1, 0] + y * m[1, 1] + z * m[1, 2]
        zp = x * m[2, 0] + y * m[2, 1] + z * m[2, 2]
        neg = xp < 0
        xp, yp, zp = np.where(neg, -xp, xp), np.where(neg, -yp, yp), np.where(neg, -zp, zp)
        x0, y0, z0 = np.floor(xp).astype(np.int64), np.floor(yp).astype(np.int64), np.floor(zp).astype(np.int64)
        fx, fy, fz = xp - x0, yp - y0, zp - z0
        y0, z0 = y0 - inity, z0 - initz
        ok = (x0 >= 0) & (x0 + 1 < xd) & (y0 >= 0) & (y0 + 1 < yd) & (z0 >= 0) & (z0 + 1 < zd)
        x0, y0, z0 = np.where(ok, x0, 0), np.where(ok, y0, 0), np.where(ok, z0, 0)

        def tri(a):
            c = lambda dz, dy, dx: a[z0 + dz, y0 + dy, x0 + dx]
            x00 = c(0, 0, 0) + (c(0, 0, 1) - c(0, 0, 0)) * fx
            x01 = c(1, 0, 0) + (c(1, 0, 1) - c(1, 0, 0)) * fx
            x10 = c(0, 1, 0) + (c(0, 1, 1) - c(0, 1, 0)) * fx
            x11 = c(1, 1, 0) + (c(1, 1, 1) - c(1, 1, 0)) * fx
            y0v = x00 + (x10 - x00) * fy
            y1v = x01 + (x11 - x01) * fy
            return y0v + (y1v - y0v) * fz

        vd = tri(d)
        vd = np.where(neg, np.conj(vd), vd)
        if zshift is not None and zshift[s_] != 0:
            dotp = 2 * PI * (z * zshift[s_])
            a, b = np.cos(dotp), np.sin(dotp)
            c, dd = vd.real, vd.imag
            ac, bd = a * c, b * dd
            vd = (ac - bd) + 1j * ((a + b) * (c + dd) - ac - bd)
        acc_d += np.where(ok, vd, 0)
        acc_w += np.where(ok, tri(w), 0.0)
    sd[inside] += acc_d
    sw[inside] += acc_w
    return sd.reshape(d.shape), sw.reshape(w.shape)


def ftblob_table(radius=3.8, alpha=15.0, nr=10000):
    """The blob's Fourier transform sampled at w = i * 0.5 / nr (TabFtBlob::fillTable): for the
    order-0 Kaiser-Bessel blob in 3D, (2 pi)^(3/2) a^3 I_{3/2}(s) / (I_0(alpha) s^(3/2)) with
    s = sqrt(alpha^2 - (2 pi a w)^2), and J_{3/2} of sqrt((2 pi a w)^2 - alpha^2) where
    2 pi a w > alpha; the half-integer Bessel functions in closed form."""
    w = np.arange(nr) * (0.5 / nr)
    u = 2.0 * PI * radius * w
    s = np.sqrt(np.abs(alpha * alpha - u * u))
    i32 = np.sqrt(2.0 / (PI * s)) * (np.cosh(s) - np.sinh(s) / s)
    j32 = np.sqrt(2.0 / (PI * s)) * (np.sin(s) / s - np.cos(s))
    bes = np.where(u > alpha, j32, i32)
    return (2.0 * PI) ** 1.5 * radius ** 3 * bes / (np.i0(alpha) * s ** 1.5)


def _fftw_coords(ps, two_d):
    fx = ps // 2 + 1
    k = np.arange(ps)
    kp = np.where(k < fx, k, k - ps)
    kz = np.zeros(1, np.int64) if two_d else kp
    return np.meshgrid(kz, kp, np.arange(fx), indexing="ij")


def gridding_weights(W, ps, ori_size, pad, max_r2, niter, two_d=False):
    """The iterative weights (FFTW layout of W, FP64) of BackProjector::reconstruct's gridding
    branch, W already divided by `normalise`."""
    KP, IP, JP = _fftw_coords(ps, two_d)
    inside = (KP * KP + IP * IP + JP * JP) < max_r2
    FN = inside.astype(float)
    tab = ftblob_table()
    ph = ps // 2
    k = np.arange(ps)
    kc = np.where(k < ph, k, k - ps)
    if two_d:
        r2 = kc[:, None] ** 2 + kc[None, :] ** 2
    else:
        r2 = kc[:, None, None] ** 2 + kc[None, :, None] ** 2 + kc[None, None, :] ** 2
    rval = np.sqrt(r2.astype(float)) / (ori_size * pad)
    idx = (np.abs(rval) / (0.5 / 10000)).astype(np.int64)
    B = np.where(idx < tab.size, tab[np.minimum(idx, tab.size - 1)], 0.0) / tab[0]
    axes = (0, 1) if two_d else (0, 1, 2)
    shape = (ps, ps) if two_d else (ps, ps, ps)
    for _ in range(niter):
        G = FN * W
        G = G[0] if two_d else G
        real = np.fft.irfftn(G, s=shape, axes=axes)
        conv = np.fft.rfftn(real * B, axes=axes)
        conv = conv[None] if two_d else conv
        w = np.maximum(1e-6, np.abs(conv))
        FN = np.where(inside, FN / w, FN)
    return FN


def decenter(data, weight, r_max, pad, tau2=None, tau2_fudge=1.0, minres_map=0):
    """Projector::decenter of data and weight to the FFTW layout of the pad_size box
    (r^2 <= ROUND(r_max pad)^2), the MAP term added to the weight; FP64, 3D layout (a 2D
    grid as one plane).  Returns F, W, r2, max_r2."""
    two_d = weight.ndim == 2
    if two_d:
        data, weight = data[None], weight[None]
    zd, yd, xd = weight.shape
    ps = yd
    fx = ps // 2 + 1
    initz, inity = -(zd // 2), -(yd // 2)
    rp = int(relion_round(r_max * pad))
    max_r2 = rp * rp
    k = np.arange(ps)
    kp = np.where(k < fx, k, k - ps)
    kz = np.zeros(1, np.int64) if two_d else kp
    KP, IP, JP = np.meshgrid(kz, kp, np.arange(fx), indexing="ij")
    r2 = KP * KP + IP * IP + JP * JP
    inside = r2 <= max_r2
    zs, ys = KP - initz, IP - inity
    F = np.zeros(KP.shape, complex)
    W = np.zeros(KP.shape)
    F[inside] = data[zs[inside], ys[inside], JP[inside]]
    W[inside] = weight[zs[inside], ys[inside], JP[inside]]
    oc = float(pad) ** (2 if two_d else 3)
    if tau2 is not None:
        m = r2 < max_r2
        ires = relion_round(np.sqrt(r2[m].astype(float)) / pad)
        t = np.asarray(tau2, float)[ires]
        invw = W[m]
        invtau2 = np.where(t > 0, 1.0 / (oc * tau2_fudge * np.where(t > 0, t, 1.0)),
                           np.where(invw > 1e-20, 1.0 / (0.001 * np.where(invw > 1e-20, invw, 1.0)), 0.0))
        W[m] = np.where(ires >= minres_map, invw + invtau2, invw)
    return F, W, r2, max_r2


def decenter_divide(data, weight, r_max, pad, tau2=None, tau2_fudge=1.0, minres_map=0, gridding_iter=0,
                    normalise=1.0, ori_size=None):
    """Fconv of the pad_size box (FFTW layout [ps][ps][ps/2+1], 2D: [ps][ps/2+1]) after the MAP
    term and the skip-gridding division (gridding_iter 0), or the gridding iterations, FP64."""
    two_d = weight.ndim == 2
    F, W, r2, max_r2 = decenter(data, weight, r_max, pad, tau2, tau2_fudge, minres_map)
    if gridding_iter > 0:
        ps = W.shape[1]
        FN = gridding_weights(W / normalise, ps, ori_size, pad, max_r2, gridding_iter, two_d)
        out = F / normalise * FN
        return out[0] if two_d else out
    # radial averages below ROUND((r_max pad)^2)
    rr2 = int(relion_round(r_max * pad * r_max * pad))
    m = r2 < rr2
    ires = np.floor(np.sqrt(r2[m].astype(float)) / pad).astype(int)
    rad = np.bincount(ires, W[m], r_max)[:r_max]
    cnt = np.bincount(ires, minlength=r_max)[:r_max]
    rad = np.where((cnt > 0) | (rad > 0), rad / (1000. * np.maximum(cnt, 1)), rad)
    iall = np.floor(np.sqrt(r2.astype(float)) / pad).astype(int)
    wfin = np.maximum(W, rad[np.minimum(iall, r_max - 1)])
    out = np.where(wfin != 0, F / np.where(wfin != 0, wfin, 1.0), F)
    return out[0] if two_d else out


def _radius(n, nd):
    c = np.arange(n) - n // 2
    if nd == 2:
        return np.sqrt(c[:, None] ** 2 + c[None, :] ** 2)
    return np.sqrt(c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2)


def soft_mask_bg(vol, radius, width):
    r = _radius(vol.shape[0], vol.ndim)
    rp = radius + width
    rc = 0.5 + 0.5 * np.cos(PI * (rp - r) / width)
    edge = (r >= radius) & (r <= rp)
    out_ = r > rp
    s = np.sum(out_) + np.sum(rc[edge])
    bg = (np.sum(vol[out_]) + np.sum(rc[edge] * vol[edge])) / s if s > 0 else 0.0
    res = vol.copy()
    res[out_] = bg
    res[edge] = (1 - rc[edge]) * vol[edge] + rc[edge] * bg
    return res


def reconstruct_map(data, weight, r_max, pad, ori_size, tau2=None, tau2_fudge=1.0, minres_map=0, gridding_iter=0,
                    normalise=1.0):
    """Real-space map (ori_size^3, or ori_size^2 for a 2D grid; FP64) of the reconstruction (2D
    particles): skip-gridding, or gridding_iter iterations of the gridding weights."""
    nd = weight.ndim
    F = decenter_divide(data, weight, r_max, pad, tau2, tau2_fudge, minres_map, gridding_iter, normalise, ori_size)
    if nd == 2:
        F = F[None]
    ps = F.shape[1]
    N = int(relion_round(pad * ori_size))
    N += N % 2
    h = N // 2 + 1
    k = np.arange(N)
    kp = np.where(k < h, k, k - N)
    half = ps // 2
    # windowFourierTransform (src/fftw.h:736-790): shrinking copies every output element;
    # enlarging copies the input elements with r^2 <= (XSIZE(in) - 1)^2 and zeros the rest
    ok = (kp >= -half) & (kp <= half)
    src = np.where(kp < 0, kp + ps, kp)
    jj = np.arange(h)
    kz, okz, srcz = (np.zeros(1, np.int64), np.ones(1, bool), np.zeros(1, np.int64)) if nd == 2 else (kp, ok, src)
    sel = okz[:, None, None] & ok[None, :, None] & (jj <= half)[None, None, :]
    if N > ps:
        sel &= (kz[:, None, None] ** 2 + kp[None, :, None] ** 2 + jj[None, None, :] ** 2) <= half * half
    Z, Y, X = np.broadcast_arrays(srcz[:, None, None], src[None, :, None], np.minimum(jj, half)[None, None, :])
    G = np.zeros(sel.shape, complex)
    G[sel] = F[Z[sel], Y[sel], X[sel]]
    kk = np.arange(G.shape[0])
    sign = np.where(((kk[:, None, None] ^ k[None, :, None] ^ jj[None, None, :]) & 1) != 0, -1.0, 1.0)
    G = G * sign
    o0 = N // 2 - ori_size // 2
    if nd == 3:
        big = np.fft.irfftn(G, s=(N, N, N), axes=(0, 1, 2)) * float(N) ** 3
        vol = big[o0:o0 + ori_size, o0:o0 + ori_size, o0:o0 + ori_size] / (float(pad) ** 3 * ori_size)
    else:
        big = np.fft.irfftn(G[0], s=(N, N), axes=(0, 1)) * float(N) ** 2
        vol = big[o0:o0 + ori_size, o0:o0 + ori_size] / float(pad) ** 2
    vol = soft_mask_bg(vol, ori_size / 2.0, 3.0)
    r = _radius(ori_size, nd)
    rval = r / (ori_size * pad)
    with np.errstate(invalid="ignore", divide="ignore"):
        sinc = np.where(r > 0, np.sin(PI * rval) / (PI * np.where(r > 0, rval, 1.0)), 1.0)
    return vol / (sinc * sinc)


def downsampled_average(data, weight, r_max, pad):
    two_d = weight.ndim == 2
    if two_d:
        data, weight = data[None], weight[None]
    zd, yd, xd = weight.shape
    K, I, J = _logical(weight.shape, -(zd // 2), -(yd // 2))
    K, I, J = np.broadcast_arrays(K, I, J)
    ds = 2 * (r_max + 1) + 1
    dh = ds // 2
    nzb = 1 if two_d else ds
    kp = np.zeros_like(K) if two_d else relion_round(K / pad) + dh
    ip = relion_round(I / pad) + dh
    jp = relion_round(J / pad)
    idx = (kp * ds + ip) * (dh + 1) + jp
    n = nzb * ds * (dh + 1)
    ar = np.bincount(idx.ravel(), data.real.ravel(), n)
    ai = np.bincount(idx.ravel(), data.imag.ravel(), n)
    w = np.bincount(idx.ravel(), weight.ravel(), n)
    avg = np.where(w > 0, (ar + 1j * ai) / np.where(w > 0, w, 1.0), 0.0)
    return avg.reshape(nzb, ds, dh + 1)


def downsampled_fsc(data1, w1, data2, w2, r_max, pad, ori_size):
    a1 = downsampled_average(data1, w1, r_max, pad)
    a2 = downsampled_average(data2, w2, r_max, pad)
    ds = a1.shape[1]
    dh = ds // 2
    c = np.arange(ds) - dh
    kz = np.zeros(1) if a1.shape[0] == 1 else c
    R = np.sqrt(kz[:, None, None] ** 2 + c[None, :, None] ** 2 + np.arange(dh + 1)[None, None, :] ** 2)
    m = R <= r_max
    idx = relion_round(R[m])
    nb = ori_size // 2 + 1
    num = np.bincount(idx, (a1[m] * np.conj(a2[m])).real, nb)
    d1 = np.bincount(idx, np.abs(a1[m]) ** 2, nb)
    d2 = np.bincount(idx, np.abs(a2[m]) ** 2, nb)
    fsc = np.where(d1 * d2 > 0, num / np.sqrt(np.where(d1 * d2 > 0, d1 * d2, 1.0)), 0.0)
    fsc[0] = 1.0
    return fsc


def update_ssnr(weight, r_max, pad, ori_size, tau2_fudge, tau2, fsc, avgctf2=None, update_tau2_with_fsc=True,
                is_whole_instead_of_half=False, correct_tau2_by_avgctf2=False):
    """Returns tau2, sigma2, data_vs_prior, fourier_coverage (FP64)."""
    two_d = weight.ndim == 2
    w3 = weight[None] if two_d else weight
    zd, yd, xd = w3.shape
    K, I, J = np.broadcast_arrays(*_logical(w3.shape, -(zd // 2), -(yd // 2)))
    r2 = K * K + I * I + J * J
    rp = int(relion_round(r_max * pad))
    m = r2 < rp * rp
    ires = relion_round(np.sqrt(r2[m].astype(float)) / pad)
    nb = ori_size // 2 + 1
    oc = float(pad) ** (2 if two_d else 3)
    wv = w3[m]
    s2 = np.bincount(ires, oc * wv, nb)
    cnt = np.bincount(ires, minlength=nb).astype(float)
    sigma2 = np.where(s2 > 1e-10, cnt / np.where(s2 > 1e-10, s2, 1.0), 0.0)
    tau2 = np.array(tau2, float).copy()
    dvp = np.zeros(nb)
    if update_tau2_with_fsc:
        myfsc = np.maximum(0.001, np.asarray(fsc, float))
        if is_whole_instead_of_half:
            myfsc = np.sqrt(2. * myfsc / (myfsc + 1.))
        myfsc = np.minimum(0.999, myfsc)
        ssnr = myfsc / (1. - myfsc) * tau2_fudge
        tau2 = ssnr * sigma2
        dvp = ssnr.copy()
    t = tau2[ires]
    with np.errstate(divide="ignore"):
        invtau2 = np.where(t > 0, 1.0 / (oc * tau2_fudge * np.where(t > 0, t, 1.0)), 1.0 / (0.001 * wv))
    if correct_tau2_by_avgctf2 and avgctf2 is not None:
        a = np.asarray(avgctf2, float)[ires]
        invtau2 = np.where((t > 0) & (a > 0), invtau2 / np.where(a > 0, a, 1.0), invtau2)
    ratio = wv / invtau2
    if not update_tau2_with_fsc:
        dvp = np.bincount(ires, ratio, nb)
    cov = np.bincount(ires, (ratio >= 1.).astype(float), nb)
    cnt2 = np.bincount(ires, minlength=nb).astype(float)
    if not update_tau2_with_fsc:
        i = np.arange(nb)
        dvp = np.where(i > r_max, 0.0, np.where(cnt2 < 0.001, 999., dvp / np.maximum(cnt2, 1e-300)))
    cov = np.where(cnt2 > 0, cov / np.maximum(cnt2, 1e-300), cov)
    return tau2, sigma2, dvp, cov
