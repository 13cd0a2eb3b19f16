"""The FP64 image-preparation oracle (oracle/imageprep_oracle.py) on the CPU:
the reference's CTF known answer, the FFT / window / CenterFFTbySign
conventions against the E-step's own synthetic Fourier-space particles, the
translation direction, the noise background's spectrum, and the power spectrum.
"""
import numpy as np
import pytest

import imageprep_oracle as ipo


def base_cfg(N, s, **kw):
    cfg = dict(image_size=N, current_size=s, pixel_size=2.0, mask_radius=N, width_mask_edge=5.0, zero_mask=1,
               random_seed=11, do_norm_correction=0, avg_norm_correction=1.0, sigma2_fudge=1.0,
               sigma2_noise=np.full(N // 2 + 1, 0.5), remap_noise=1.0, remap_minv=1.0, do_ctf_correction=1,
               ctf_premultiplied=0, ctf_phase_flipped=0, only_flip_phases=0, intact_ctf_first_peak=0,
               voltage=300.0, cs=2.7, q0=0.1)
    cfg.update(kw)
    return cfg


def params(n, rng, offset=0.0):
    par = np.zeros((n, ipo.NPARAM))
    par[:, ipo.P_XOFF] = rng.uniform(-offset, offset, n)
    par[:, ipo.P_YOFF] = rng.uniform(-offset, offset, n)
    par[:, ipo.P_XPRIOR] = 999.
    par[:, ipo.P_YPRIOR] = 999.
    par[:, ipo.P_NORM] = 1.0
    par[:, ipo.P_DEFU] = rng.uniform(10000, 30000, n)
    par[:, ipo.P_DEFV] = par[:, ipo.P_DEFU] - rng.uniform(0, 1000, n)
    par[:, ipo.P_DEFANG] = rng.uniform(0, 180, n)
    par[:, ipo.P_KFAC] = 1.0
    par[:, ipo.P_SCALE] = 1.0
    return par


def real_space_from_window(win, N):
    """Real-space image whose prepared (FFT, window, CenterFFTbySign) transform is
    the Hermitian part of the centred full window `win` (N x (N/2+1))."""
    sign = np.where(((np.arange(N)[:, None] ^ np.arange(N // 2 + 1)[None, :]) & 1) != 0, -1.0, 1.0)
    return np.fft.irfft2(win.reshape(N, N // 2 + 1) * sign, s=(N, N)) * (N * N)


def test_ctf_golden_value():
    # tests/ctf.cpp:5-9 of the reference: setValues(10000, 12000, 90, 300, 2.7, 0.1, 0, 1, 0),
    # getCTF(10, 10); a 2-pixel box of 0.05 A/px puts window pixel (1, 1) at X = Y = 10 / A
    cfg = base_cfg(2, 2, pixel_size=0.05)
    par = np.zeros(ipo.NPARAM)
    par[[ipo.P_DEFU, ipo.P_DEFV, ipo.P_DEFANG, ipo.P_KFAC]] = 10000.0, 12000.0, 90.0, 1.0
    v = ipo.ctf_window(par, cfg, 2)
    assert v[1, 1] == pytest.approx(0.59154, abs=5e-6)


def test_ctf_matches_estep_oracle_ctf(oracle):
    p = [15000.0, 14500.0, 33.0, 300.0, 2.7, 0.1, 0.0, 1.0, 0.0]
    cfg = base_cfg(128, 80, pixel_size=1.3)
    par = np.zeros(ipo.NPARAM)
    par[[ipo.P_DEFU, ipo.P_DEFV, ipo.P_DEFANG, ipo.P_KFAC]] = 15000.0, 14500.0, 33.0, 1.0
    a = ipo.ctf_window(par, cfg, 80).reshape(-1)
    b = oracle.ctf_image(p, 128, 1.3, 80)
    assert np.max(np.abs(a - b)) < 1e-6


def test_window_and_sign_recover_synthetic_particles(synth):
    """Fourier-space particles of the E-step generator, taken to real space and
    prepared (no mask, no offset), come back as the same window."""
    N, r, s = 32, 8, 16
    fmap = synth.fourier_map(synth.blob_volume(N, 10, seed=5), r)
    parts = synth.make_particles(fmap, 3, ori_size=N, s=N, r_max=r, angpix=2.0, snr=0.5, seed=4)
    imgs = np.stack([real_space_from_window(parts["fimg"][b].astype(np.complex128), N) for b in range(3)])
    cfg = base_cfg(N, s, mask_radius=2 * N)
    out = ipo.prepare(imgs, params(3, np.random.default_rng(0)), np.arange(3), cfg)
    # the Hermitian part of the full window, windowed to s
    ky, kx = ipo.window_index(s)
    for b in range(3):
        full = parts["fimg"][b].reshape(N, N // 2 + 1).astype(np.complex128)
        herm = np.fft.rfft2(real_space_from_window(full, N)) / (N * N)
        sign = np.where(((np.arange(N)[:, None] ^ np.arange(N // 2 + 1)[None, :]) & 1) != 0, -1.0, 1.0)
        herm = herm * sign
        want = herm[ky % N, kx].reshape(-1)
        assert np.max(np.abs(out["fimg"][b] - want)) < 1e-12 * np.max(np.abs(want))
        assert np.array_equal(out["fimg"][b], out["fimg_nomask"][b])
        # interior pixels (not in the kx = 0 column) are the generator's own values
        inner = (kx.reshape(-1) > 0) & (kx.reshape(-1) < s // 2)
        gen = full[ky % N, kx].reshape(-1)
        assert np.max(np.abs(out["fimg"][b][inner] - gen[inner])) < 1e-5 * np.max(np.abs(gen))


def test_translation_direction():
    """selfTranslate by the rounded old offset: out[y][x] = in[y - ty][x - tx]."""
    rng = np.random.default_rng(2)
    N = 24
    img = np.zeros((1, N, N))
    img[0, 8:16, 8:16] = rng.standard_normal((8, 8))
    par = params(1, rng)
    par[0, ipo.P_XOFF], par[0, ipo.P_YOFF] = 2.5, -1.5       # ROUND: 3, -2 (half away from zero)
    cfg = base_cfg(N, N, mask_radius=2 * N)
    out = ipo.prepare(img, par, np.zeros(1, np.int64), cfg)
    moved = np.zeros_like(img)
    moved[0, 6:14, 11:19] = img[0, 8:16, 8:16]
    par2 = par.copy()
    par2[0, ipo.P_XOFF] = par2[0, ipo.P_YOFF] = 0.
    ref = ipo.prepare(moved, par2, np.zeros(1, np.int64), cfg)
    assert np.allclose(out["fimg"], ref["fimg"], atol=1e-15)
    assert tuple(out["scalars"][0, 2:4]) == (3.0, -2.0)


def test_noise_background_spectrum():
    """Noise image: E|F|^2 = 2 sigma2_fudge sigma2_noise[ring] on the interior pixels."""
    N = 64
    h = N // 2 + 1
    sig = 0.2 + np.linspace(1.0, 0.1, h) ** 2
    fudge = 1.5
    ky, kx = ipo.window_index(N)
    ires = ipo.ring_index(ky, kx)
    acc = np.zeros(h)
    cnt = np.zeros(h)
    for seed in range(40):
        img = ipo.noise_image(1000 + seed, N, fudge, sig, 1.0)
        F = np.fft.rfft2(img) / (N * N)
        inner = (kx > 0) & (kx < N // 2) & (ires < h)
        acc += np.bincount(ires[inner], np.abs(F[inner]) ** 2, h)
        cnt += np.bincount(ires[inner], minlength=h)
    ok = cnt > 200
    ratio = acc[ok] / cnt[ok] / (2 * fudge * sig[ok])
    assert np.all(np.abs(ratio - 1) < 0.1), ratio
    # a function of the seed alone
    assert np.array_equal(ipo.noise_image(5, N, fudge, sig, 1.0), ipo.noise_image(5, N, fudge, sig, 1.0))
    assert not np.array_equal(ipo.noise_image(5, N, fudge, sig, 1.0), ipo.noise_image(6, N, fudge, sig, 1.0))


def test_power_spectrum_and_highres_xi2():
    rng = np.random.default_rng(3)
    N, s = 48, 24
    imgs = rng.standard_normal((2, N, N))
    cfg = base_cfg(N, s, mask_radius=15.0, zero_mask=1)
    out = ipo.prepare(imgs, params(2, rng), np.arange(2), cfg)
    h, hs = N // 2 + 1, s // 2 + 1
    assert out["power"][:, 0].tolist() == [0.0, 0.0]
    assert np.allclose(out["scalars"][:, 1], out["power"][:, hs:].sum(1), rtol=1e-12)
    # all rings together: the half-plane power of the masked image below Nyquist
    ky, kx = ipo.window_index(N)
    ires = ipo.ring_index(ky, kx)
    m = ipo.soft_mask(imgs[0], 15.0, 5.0)
    F = np.fft.rfft2(m) / (N * N)
    sel = (ires > 0) & (ires < h) & ~((kx == 0) & (ky < 0))
    assert out["power"][0].sum() == pytest.approx(np.sum(np.abs(F[sel]) ** 2), rel=1e-12)


def test_minvsigma2_and_scalars():
    rng = np.random.default_rng(4)
    N, s = 32, 20
    sig = rng.uniform(0.5, 2.0, N // 2 + 1)
    cfg = base_cfg(N, s, sigma2_noise=sig, sigma2_fudge=2.0)
    par = params(1, rng)
    par[0, ipo.P_XPRIOR], par[0, ipo.P_YPRIOR], par[0, ipo.P_SCALE] = 1.25, 999.0, 0.8
    out = ipo.prepare(rng.standard_normal((1, N, N)), par, np.zeros(1, np.int64), cfg)
    ky, kx = ipo.window_index(s)
    ires = ipo.ring_index(ky, kx).reshape(-1)
    mv = out["minvsigma2"][0]
    hs = s // 2 + 1
    for q in range(mv.size):
        if ires[q] == 0 or ires[q] >= hs or (kx.reshape(-1)[q] == 0 and ky.reshape(-1)[q] < 0):
            assert mv[q] == 0
        else:
            assert mv[q] == pytest.approx(1.0 / (2.0 * sig[ires[q]]), rel=1e-15)
    sc = out["scalars"][0]
    assert sc[0] == pytest.approx(1.0 / (2.0 * sig[0]))
    assert (sc[4], sc[5], sc[6]) == (1.25, 0.0, 0.8)
