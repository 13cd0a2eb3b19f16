"""The FP64 reconstruction oracle (oracle/recon_oracle.py) on the CPU: its
skip-gridding division against the C++ E-step oracle's, its real-space chain
(window, CenterFFTbySign, inverse FFT, normalisation, gridding correction) on
the Fourier map of a known volume, and the FSC / SSNR arrays against direct
sums."""
import numpy as np
import pytest

import recon_oracle as ro


def _grid(rng, r_max, pad=2):
    ps = 2 * (r_max * pad + 1) + 1
    data = (rng.standard_normal((ps, ps, ps // 2 + 1)) + 1j * rng.standard_normal((ps, ps, ps // 2 + 1)))
    weight = rng.uniform(0.5, 2.0, (ps, ps, ps // 2 + 1))
    return data.astype(np.complex64).astype(np.complex128), weight.astype(np.float32).astype(np.float64)


def test_division_matches_cpp_oracle(oracle):
    rng = np.random.default_rng(1)
    data, weight = _grid(rng, 8)
    got = ro.decenter_divide(data, weight, 8, 2)
    ref = oracle.reconstruct_divide(data, weight, 8, 2)
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_map_term_raises_the_weights():
    rng = np.random.default_rng(2)
    data, weight = _grid(rng, 8)
    tau2 = np.full(17, 0.5)
    plain = ro.decenter_divide(data, weight, 8, 2)
    reg = ro.decenter_divide(data, weight, 8, 2, tau2=tau2, tau2_fudge=1.0, minres_map=0)
    # inside the sphere the weight grows by 1/(pad^3 tau2) = 0.25: |F| shrinks
    m = np.abs(plain) > 0
    assert np.all(np.abs(reg[m]) <= np.abs(plain[m]) * (1 + 1e-12))
    assert np.any(np.abs(reg[m]) < 0.9 * np.abs(plain[m]))


@pytest.mark.parametrize("ori,r_max", [(32, 16), (32, 8)], ids=["shrink", "enlarge"])
def test_reconstruction_of_a_known_volume(synth, ori, r_max):
    """Grid = the padded Fourier map of a band-limited volume V with weight 1: the map is
    V / ori (normalisation of 2D particles) over sinc^2 (gridding correction), low-passed
    at r_max."""
    vol = synth.blob_volume(ori, 8, sigma=(2.5, 4.0), seed=3)
    # the map a projector holds: centred half-complex of the 2x padded volume (weights 1),
    # on the pad_size box 2 (2 r_max + 1) + 1 (which exceeds the padded box when r_max = ori/2)
    m = 2 * ori
    big0 = np.zeros((m,) * 3)
    big0[ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori] = vol
    F0 = np.fft.rfftn(np.fft.ifftshift(big0)) / float(ori) ** 3
    ps = 2 * (2 * r_max + 1) + 1
    kk = np.arange(ps) - ps // 2
    KZ, KY, KX = np.meshgrid(kk, kk, np.arange(ps // 2 + 1), indexing="ij")
    keep = KZ * KZ + KY * KY + KX * KX <= (2 * r_max) ** 2
    fmap = np.where(keep, F0[KZ % m, KY % m, np.minimum(KX, m // 2)], 0)
    weight = np.ones(fmap.shape)
    got = ro.reconstruct_map(fmap, weight, r_max, 2, ori)
    c = np.arange(ori) - ori // 2
    r = np.sqrt(c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2)
    rv = r / (2 * ori)
    sinc = np.where(r > 0, np.sin(np.pi * rv) / (np.pi * np.where(r > 0, rv, 1)), 1.0)
    # the same low-pass applied to V directly
    N = 2 * ori
    big = np.zeros((N,) * 3)
    big[ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori] = vol
    F = np.fft.rfftn(np.fft.ifftshift(big))
    k = np.fft.fftfreq(N) * N
    kx = np.arange(N // 2 + 1)
    r2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kx[None, None, :] ** 2
    F[r2 > (2 * r_max) ** 2] = 0
    lp = np.fft.fftshift(np.fft.irfftn(F, s=(N,) * 3, axes=(0, 1, 2)))[ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori,
                                                        ori // 2:ori // 2 + ori]
    want = ro.soft_mask_bg(lp / ori, ori / 2.0, 3.0) / (sinc * sinc)
    assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))


def test_fsc_of_identical_and_independent_halves():
    rng = np.random.default_rng(4)
    d1, w1 = _grid(rng, 8)
    f_same = ro.downsampled_fsc(d1, w1, d1, w1, 8, 2, 32)
    assert np.allclose(f_same[:9], 1.0, atol=1e-12) and np.all(f_same[9:] == 0)
    d2, w2 = _grid(rng, 8)
    f_ind = ro.downsampled_fsc(d1, w1, d2, w2, 8, 2, 32)
    assert f_ind[0] == 1.0 and np.all(np.abs(f_ind[2:9]) < 0.3)


def test_ssnr_arrays_against_direct_sums():
    rng = np.random.default_rng(5)
    _, w = _grid(rng, 8)
    ori, nb = 32, 17
    tau2 = rng.uniform(0.1, 1.0, nb)
    fsc = np.clip(1.0 - np.linspace(0, 1.2, nb), -0.1, 1.0)
    t, s2, dvp, cov = ro.update_ssnr(w, 8, 2, ori, 1.5, tau2, fsc)
    # direct: shell of every voxel with r^2 < (r_max pad)^2, ires = ROUND(r / pad)
    ps = w.shape[0]
    k = np.arange(ps) - ps // 2
    K, I, J = np.meshgrid(k, k, np.arange(w.shape[2]), indexing="ij")
    r2 = K * K + I * I + J * J
    m = r2 < 16 * 16
    ires = np.floor(np.sqrt(r2[m]) / 2 + 0.5).astype(int)
    s = np.bincount(ires, 8 * w[m], nb)
    n = np.bincount(ires, minlength=nb)
    assert np.allclose(s2[n > 0], n[n > 0] / s[n > 0], rtol=1e-12)
    f = np.minimum(0.999, np.maximum(0.001, fsc))
    assert np.allclose(dvp, f / (1 - f) * 1.5, rtol=1e-12)
    assert np.allclose(t, f / (1 - f) * 1.5 * s2, rtol=1e-12)
    assert np.all((cov >= 0) & (cov <= 1))


@pytest.mark.parametrize("ori,r_max", [(32, 16), (32, 8)], ids=["shrink", "enlarge"])
def test_reconstruction_of_a_known_image_2d(synth, ori, r_max):
    """2D classes: the padded Fourier map of a band-limited image with weight 1 gives the
    image itself (normalisation pad^2 of 2D maps from 2D particles) over sinc^2, low-passed
    at r_max."""
    img = synth.blob_volume(ori, 6, sigma=(2.5, 4.0), seed=5, ndim=2)
    m = 2 * ori
    big0 = np.zeros((m, m))
    big0[ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori] = img
    F0 = np.fft.rfft2(np.fft.ifftshift(big0)) / float(ori) ** 2
    ps = 2 * (2 * r_max + 1) + 1
    kk = np.arange(ps) - ps // 2
    KY, KX = np.meshgrid(kk, np.arange(ps // 2 + 1), indexing="ij")
    keep = KY * KY + KX * KX <= (2 * r_max) ** 2
    fmap = np.where(keep, F0[KY % m, np.minimum(KX, m // 2)], 0)
    got = ro.reconstruct_map(fmap, np.ones(fmap.shape), r_max, 2, ori)
    assert got.shape == (ori, ori)
    big = np.zeros((m, m))
    big[ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori] = img
    F = np.fft.rfft2(np.fft.ifftshift(big))
    k = np.fft.fftfreq(m) * m
    r2 = k[:, None] ** 2 + np.arange(m // 2 + 1)[None, :] ** 2
    F[r2 > (2 * r_max) ** 2] = 0
    lp = np.fft.fftshift(np.fft.irfft2(F, s=(m, m)))[ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori]
    c = np.arange(ori) - ori // 2
    r = np.sqrt(c[:, None] ** 2 + c[None, :] ** 2)
    rv = r / (2 * ori)
    sinc = np.where(r > 0, np.sin(np.pi * rv) / (np.pi * np.where(r > 0, rv, 1)), 1.0)
    want = ro.soft_mask_bg(lp, ori / 2.0, 3.0) / (sinc * sinc)
    assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))


@pytest.mark.parametrize("shape", [(9, 9, 5), (9, 5)], ids=["3d", "2d"])
def test_hermitian_symmetry_restatement(shape):
    """enforceHermitianSymmetry (src/backprojector.cpp:2104-2121) on a grid whose Friedel
    partners of the x = 0 plane differ: each pair holds old(z, y) + conj(old(-z, -y)) and
    its conjugate, weights the pair's sum; the origin and every x > 0 element stay."""
    rng = np.random.default_rng(4)
    d = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    w = rng.uniform(0, 1, shape)
    sd, sw = ro.enforce_hermitian_symmetry(d, w)
    d3, w3, s3, t3 = (a[None] if len(shape) == 2 else a for a in (d, w, sd, sw))
    zd, yd = w3.shape[0], w3.shape[1]
    cz, cy = zd // 2, yd // 2
    for z in range(-cz, cz + 1):
        for y in range(-cy, cy + 1):
            a, b = (z + cz, y + cy, 0), (-z + cz, -y + cy, 0)
            if z == 0 and y == 0:
                assert s3[a] == d3[a] and t3[a] == w3[a]
                continue
            assert s3[a] == np.conj(s3[b])
            assert t3[a] == t3[b] == w3[a] + w3[b]
            assert np.isclose(s3[a], d3[a] + np.conj(d3[b]), rtol=1e-15)
    assert np.array_equal(s3[..., 1:], d3[..., 1:]) and np.array_equal(t3[..., 1:], w3[..., 1:])


def test_blob_fourier_table_against_a_direct_transform():
    """TabFtBlob's values (the order-0 Kaiser-Bessel blob, radius 3.8, alpha 15, in 3D): the
    closed form of the oracle against the radial Fourier integral of the blob profile
    I_0(alpha sqrt(1 - (r/a)^2)) / I_0(alpha), 4 pi int r^2 b(r) sinc(2 w r) dr."""
    from scipy import integrate, special
    a, al = 3.8, 15.0
    tab = ro.ftblob_table()

    def direct(w):
        f = lambda r: special.i0(al * np.sqrt(max(0.0, 1 - (r / a) ** 2))) / special.i0(al) * r * r * np.sinc(2 * w * r)
        return 4 * np.pi * integrate.quad(f, 0, a, limit=400, epsabs=1e-14, epsrel=1e-13)[0]

    for i in (0, 1000, 3000, 5000, 8000, 9999):
        assert abs(tab[i] - direct(i * 0.5 / 10000)) <= 1e-12 * tab[0], i


@pytest.mark.parametrize("two_d", [False, True], ids=["3d", "2d"])
def test_gridding_weights_on_uniform_sampling(synth, two_d):
    """With weight 1 everywhere the gridding iterations keep the weights near 1 (the blob
    kernel sums to 1), so the map is the skip-gridding map up to the edge of the sphere."""
    ori, r_max = 32, 16
    m = 2 * ori
    if two_d:
        img = synth.blob_volume(ori, 6, sigma=(2.5, 4.0), seed=5, ndim=2)
        big0 = np.zeros((m, m))
        big0[ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori] = img
        F0 = np.fft.rfft2(np.fft.ifftshift(big0)) / float(ori) ** 2
        ps = 2 * (2 * r_max + 1) + 1
        kk = np.arange(ps) - ps // 2
        KY, KX = np.meshgrid(kk, np.arange(ps // 2 + 1), indexing="ij")
        keep = KY * KY + KX * KX <= (2 * r_max) ** 2
        fmap = np.where(keep, F0[KY % m, np.minimum(KX, m // 2)], 0)
    else:
        vol = synth.blob_volume(ori, 8, sigma=(2.5, 4.0), seed=3)
        big0 = np.zeros((m,) * 3)
        big0[ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori, ori // 2:ori // 2 + ori] = vol
        F0 = np.fft.rfftn(np.fft.ifftshift(big0)) / float(ori) ** 3
        ps = 2 * (2 * r_max + 1) + 1
        kk = np.arange(ps) - ps // 2
        KZ, KY, KX = np.meshgrid(kk, kk, np.arange(ps // 2 + 1), indexing="ij")
        keep = KZ * KZ + KY * KY + KX * KX <= (2 * r_max) ** 2
        fmap = np.where(keep, F0[KZ % m, KY % m, np.minimum(KX, m // 2)], 0)
    w = np.ones(fmap.shape)
    skip = ro.reconstruct_map(fmap, w, r_max, 2, ori)
    grid = ro.reconstruct_map(fmap, w, r_max, 2, ori, gridding_iter=10, normalise=3.7)
    assert np.corrcoef(skip.ravel(), grid.ravel())[0, 1] >= 0.9999
    assert np.max(np.abs(skip - grid)) <= 1e-2 * np.max(np.abs(skip))
