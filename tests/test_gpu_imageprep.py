"""Image preparation on the GPU (t2b_prep_batch_*) against the FP64 oracle
(oracle/imageprep_oracle.py), and the device-resident particle path: real-space
particles -> GPU preparation -> GPU E-step, against the E-step on the oracle's
preparation.

Tolerances: the transforms are FP32 (the reference's accelerated path runs them
in XFLOAT = float through cuFFT): the windowed images within 2e-5 of the
largest coefficient; the CTF within 1e-6 (FP64 evaluation rounded to float);
Minvsigma2 to float rounding; the ring powers and highres_Xi2 within 1e-4
relative; offsets, priors and scale exactly.
"""
import ctypes

import numpy as np
import pytest

import imageprep_oracle as ipo
import problems
from test_imageprep_oracle import base_cfg, params, real_space_from_window

pytestmark = pytest.mark.gpu

CASES = {
    # N, s, options
    "n128_s80_zeromask": (128, 80, dict(zero_mask=1, mask_radius=50.0)),
    "n128_s80_noise": (128, 80, dict(zero_mask=0, mask_radius=50.0, sigma2_fudge=1.3)),
    "n96_full_norm_premult": (96, 96, dict(zero_mask=1, mask_radius=40.0, do_norm_correction=1,
                                           avg_norm_correction=0.9, ctf_premultiplied=1, ctf_phase_flipped=1)),
    "n100_s64_noise_intact": (100, 64, dict(zero_mask=0, mask_radius=38.0, intact_ctf_first_peak=1,
                                            remap_noise=1.0, remap_minv=1.0)),
    "n60_s32_flip_noctf_edge": (60, 32, dict(zero_mask=1, mask_radius=20.0, only_flip_phases=1,
                                             width_mask_edge=3.0)),
    "n64_s64_noctf": (64, 64, dict(zero_mask=0, mask_radius=24.0, do_ctf_correction=0, random_seed=-3)),
    # boxes whose two half spectra exceed shared memory take the two-pass kernels
    "n192_s120_noise_twopass": (192, 120, dict(zero_mask=0, mask_radius=80.0)),
    "n160_s96_zeromask_twopass": (160, 96, dict(zero_mask=1, mask_radius=60.0)),
}


def _images(N, n, rng):
    """Centred blobs plus white noise, as float32 real-space particles."""
    c = np.arange(N) - N // 2
    y, x = np.meshgrid(c, c, indexing="ij")
    imgs = np.zeros((n, N, N))
    for b in range(n):
        for _ in range(6):
            cx, cy = rng.uniform(-0.25 * N, 0.25 * N, 2)
            s = rng.uniform(2, 6)
            imgs[b] += rng.uniform(0.5, 2) * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * s * s))
    return (imgs + rng.standard_normal((n, N, N)) * 0.7).astype(np.float32)


def _check(got, ref, N, s, cfg):
    for k in ("fimg", "fimg_nomask"):
        err = np.max(np.abs(got[k] - ref[k])) / np.max(np.abs(ref[k]))
        assert err <= 2e-5, (k, err)
    assert np.max(np.abs(got["ctf"] - ref["ctf"])) <= 1e-6
    assert np.allclose(got["minvsigma2"], ref["minvsigma2"], rtol=2e-7, atol=0)
    assert np.allclose(got["scalars"][:, 0], ref["scalars"][:, 0], rtol=1e-15)
    assert np.allclose(got["scalars"][:, 1], ref["scalars"][:, 1], rtol=1e-4, atol=1e-12)
    assert np.array_equal(got["scalars"][:, 2:8], ref["scalars"][:, 2:8])
    pw, rpw = got["power"], ref["power"]
    assert np.allclose(pw, rpw, rtol=1e-4, atol=1e-7 * rpw.max())


@pytest.fixture(scope="module")
def ctx(t2b):
    es = t2b.EStep(0)
    yield es
    es.close()


@pytest.mark.parametrize("case", list(CASES))
def test_prep_matches_oracle(ctx, case):
    N, s, opts = CASES[case]
    rng = np.random.default_rng(100 + list(CASES).index(case))
    n = 7
    sig = 0.3 + np.linspace(1.0, 0.05, N // 2 + 1) ** 2
    cfg = base_cfg(N, s, sigma2_noise=sig, **opts)
    imgs = _images(N, n, rng)
    par = params(n, rng, offset=4.6)
    par[:, ipo.P_NORM] = rng.uniform(0.8, 1.2, n)
    par[:, ipo.P_BFAC] = rng.uniform(0, 80, n)
    par[:, ipo.P_KFAC] = rng.uniform(0.9, 1.1, n)
    par[:, ipo.P_PHASE] = rng.uniform(0, 20, n)
    par[0, ipo.P_XOFF], par[0, ipo.P_YOFF] = -2.5, 2.5          # ROUND half away from zero
    par[1, ipo.P_XOFF], par[1, ipo.P_YOFF] = 1.5 * N, 0.0      # shifted out of the box
    par[2, ipo.P_XPRIOR], par[2, ipo.P_YPRIOR] = -1.75, 3.0
    pid = np.arange(n, dtype=np.int64) * 37 + 5
    ctx.configure_prep(max_batch=8, **cfg)
    got = ctx.prepare_images(imgs, par, pid)
    ref = ipo.prepare(imgs.astype(np.float64), par, pid, cfg)
    _check(got, ref, N, s, cfg)


def test_device_variant_equals_host_variant(ctx):
    import torch
    N, s = 128, 80
    rng = np.random.default_rng(1)
    n = 5
    cfg = base_cfg(N, s, sigma2_noise=np.linspace(1.0, 0.2, N // 2 + 1), zero_mask=0, mask_radius=50.0)
    imgs = _images(N, n, rng)
    par = params(n, rng, offset=3.0)
    pid = np.arange(n, dtype=np.int64)
    ctx.configure_prep(max_batch=n, **cfg)
    host = ctx.prepare_images(imgs, par, pid)
    dev = torch.device("cuda")
    ti = torch.from_numpy(imgs).to(dev)
    tp = torch.from_numpy(par).to(dev)
    tq = torch.from_numpy(pid).to(dev)
    P = s * (s // 2 + 1)
    out = dict(fimg=torch.zeros(n, 2 * P, device=dev), fimg_nomask=torch.zeros(n, 2 * P, device=dev),
               ctf=torch.zeros(n, P, device=dev), minvsigma2=torch.zeros(n, P, device=dev),
               scalars=torch.zeros(n, 8, dtype=torch.float64, device=dev),
               power=torch.zeros(n, N // 2 + 1, dtype=torch.float64, device=dev))
    st = torch.cuda.Stream()
    ctx.prepare_images_device(n, ctypes.c_void_p(ti.data_ptr()), ctypes.c_void_p(tp.data_ptr()),
                              ctypes.c_void_p(tq.data_ptr()),
                              {k: ctypes.c_void_p(v.data_ptr()) for k, v in out.items()}, stream=st.cuda_stream)
    st.synchronize()
    got = {k: v.cpu().numpy() for k, v in out.items()}
    assert np.array_equal(got["fimg"].view(np.complex64), host["fimg"])
    assert np.array_equal(got["fimg_nomask"].view(np.complex64), host["fimg_nomask"])
    for k in ("ctf", "minvsigma2", "scalars", "power"):
        assert np.array_equal(got[k], host[k]), k


def test_bad_arguments_are_rejected(ctx, t2b):
    with pytest.raises(t2b.T2BError):
        ctx.configure_prep(image_size=98, current_size=64, max_batch=2, sigma2_noise=np.ones(50),
                           pixel_size=1.0, mask_radius=30.0)           # 98 = 2 * 7^2
    with pytest.raises(t2b.T2BError):
        ctx.configure_prep(image_size=64, current_size=80, max_batch=2, sigma2_noise=np.ones(33),
                           pixel_size=1.0, mask_radius=30.0)
    ctx.configure_prep(image_size=32, current_size=16, max_batch=2, sigma2_noise=np.ones(17), pixel_size=1.0,
                       mask_radius=12.0)
    with pytest.raises(t2b.T2BError):
        ctx.prepare_images(np.zeros((3, 32, 32), np.float32), np.ones((3, 12)), np.arange(3))


def test_device_particle_path_matches_oracle_preparation():
    """Real-space particles -> GPU preparation -> GPU E-step, against the E-step
    on the oracle's preparation of the same images: the same poses."""
    pb = problems.build("refine_o2", n_particles=24, seed=13)
    sy, N, s, r = pb["sy"], pb["N"], pb["s"], pb["r"]
    full = sy.make_particles(pb["maps"][0], 24, ori_size=N, s=N, r_max=r, angpix=2.0, snr=0.05, seed=13,
                             max_shift=3.0)
    imgs = np.stack([real_space_from_window(full["fimg"][b].astype(np.complex128), N) for b in range(24)])
    rng = np.random.default_rng(5)
    par = params(24, rng)
    # the particles' own CTFs
    defU, defV, dang = full["defU"], full["defV"], full["dang"]
    par[:, ipo.P_DEFU], par[:, ipo.P_DEFV], par[:, ipo.P_DEFANG] = defU, defV, dang
    cfg = base_cfg(N, s, sigma2_noise=np.full(N // 2 + 1, full["sigma2"]), pixel_size=2.0, mask_radius=28.0,
                   zero_mask=1)
    es = pb["product"]()
    es.configure_prep(max_batch=24, **cfg)
    got = es.prepare_images(imgs.astype(np.float32), par, np.arange(24))
    ref = ipo.prepare(imgs.astype(np.float32).astype(np.float64), par, np.arange(24), cfg)
    # the CTF the generator applied is the CTF the preparation computes
    want_ctf = np.stack([sy.ctf_image((defU[b], defV[b], dang[b], 300., 2.7, 0.1, 0., 1., 0.), N, 2.0, s)
                         for b in range(24)])
    assert np.max(np.abs(got["ctf"] - want_ctf)) <= 1e-6
    a = es.expectation(got["fimg"], got["ctf"], got["minvsigma2"], got["scalars"], fimg_nomask=got["fimg_nomask"])
    b = es.expectation(ref["fimg"].astype(np.complex64), ref["ctf"].astype(np.float32),
                       ref["minvsigma2"].astype(np.float32), ref["scalars"],
                       fimg_nomask=ref["fimg_nomask"].astype(np.complex64))
    es.close()
    assert np.all(a["status"] == 0) and np.all(b["status"] == 0)
    same = np.all(a["pose"] == b["pose"], axis=1)
    assert same.mean() >= 0.95, same.mean()
    assert np.allclose(a["min_diff2"], b["min_diff2"], rtol=1e-4)


def test_particles_from_star_and_mrc_files(tmp_path):
    """The real-data path: a STAR particles block and an MRC stack on disk -> the library's
    readers -> device preparation -> E-step; the same poses as the in-memory batch."""
    pb = problems.build("refine_o2", n_particles=16, seed=31)
    t2b, sy, N, s, r = pb["t2b"], pb["sy"], pb["N"], pb["s"], pb["r"]
    full = sy.make_particles(pb["maps"][0], 16, ori_size=N, s=N, r_max=r, angpix=2.0, snr=0.05, seed=31,
                             max_shift=3.0)
    imgs = np.stack([real_space_from_window(full["fimg"][b].astype(np.complex128), N)
                     for b in range(16)]).astype(np.float32)
    stack = tmp_path / "particles.mrcs"
    t2b.write_mrc(str(stack), imgs, 2.0)
    star = tmp_path / "particles.star"
    t2b.write_star(str(star), "particles", {"rlnDefocusU": full["defU"], "rlnDefocusV": full["defV"],
                                            "rlnDefocusAngle": full["dang"], "rlnOriginXAngst": np.zeros(16),
                                            "rlnOriginYAngst": np.zeros(16)})
    tab = t2b.StarTable(str(star), "particles")
    par = t2b.prep_params_from_star(tab, 2.0)
    nx, ny, nz, mode, px = t2b.mrc_info(str(stack))
    assert (nx, ny, nz, mode) == (N, N, 16, 2) and px == pytest.approx(2.0)
    disk = t2b.read_mrc(str(stack))
    assert np.array_equal(disk, imgs)
    cfg = base_cfg(N, s, sigma2_noise=np.full(N // 2 + 1, full["sigma2"]), pixel_size=px, mask_radius=28.0,
                   zero_mask=0, random_seed=5)
    es = pb["product"]()
    es.configure_prep(max_batch=16, **cfg)
    a_in = es.prepare_images(disk, par, np.arange(16))
    direct_par = params(16, np.random.default_rng(0))
    direct_par[:, ipo.P_DEFU], direct_par[:, ipo.P_DEFV], direct_par[:, ipo.P_DEFANG] = full["defU"], full["defV"], \
        full["dang"]
    direct_par[:, ipo.P_XPRIOR] = direct_par[:, ipo.P_YPRIOR] = 999.0
    b_in = es.prepare_images(imgs, direct_par, np.arange(16))
    for k in ("fimg", "fimg_nomask", "ctf", "minvsigma2", "scalars"):
        assert np.array_equal(a_in[k], b_in[k]), k
    a = es.expectation(a_in["fimg"], a_in["ctf"], a_in["minvsigma2"], a_in["scalars"], fimg_nomask=a_in["fimg_nomask"])
    es.close()
    assert np.all(a["status"] == 0)
