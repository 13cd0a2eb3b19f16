"""The FP64 oracle of the proposal network, pinned on the CPU.

Its analytic gradient (which the CUDA training kernels are checked against on
the GPU) is checked here against central finite differences of its own loss,
and its feature transform against a direct inverse DFT of the full Hermitian
plane.
"""
import numpy as np
import pytest

import proposal_oracle as po


def _problem(KO=64, n=3, seed=0):
    rng = np.random.default_rng(seed)
    L = po.layout(KO)
    th = po.bf16(rng.standard_normal(L["total"]) * 0.05)
    imgs = rng.standard_normal((n, 256))
    to = np.full((n, 9), -1)
    tw = np.zeros((n, 9))
    to[0, :2], tw[0, :2] = [5, 7], [0.6, 0.4]
    to[1, :3], tw[1, :3] = [1, 2, 9], [0.2, 0.3, 0.5]
    to[2, 0], tw[2, 0] = 0, 1.0
    skip = np.zeros(KO, bool)
    skip[3] = True
    return L, th, imgs, to, tw, skip


def test_gradient_matches_finite_differences():
    KO = 64
    L, th, imgs, to, tw, skip = _problem(KO)
    _, g = po.loss_grad(th, imgs, to, tw, skip, KO, round_bf16=False)
    rng = np.random.default_rng(1)
    idx = []
    for name, size in (("wc1", 144), ("bc1", 16), ("wc2", 4608), ("bc2", 32), ("w1", 1024 * 2048), ("b1", 1024),
                       ("w2", 1024 * 1024), ("b2", 1024), ("w3", KO * 1024), ("b3", KO)):
        # parameters whose gradient is not exactly zero (inactive ReLUs give zero)
        cand = L[name] + rng.choice(size, min(size, 400), replace=False)
        nz = cand[np.abs(g[cand]) > 1e-6][:4]
        idx.extend(nz.tolist())
    assert len(idx) >= 25
    h = 1e-5
    for i in idx:
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        lp, _ = po.loss_grad(tp, imgs, to, tw, skip, KO, round_bf16=False)
        lm, _ = po.loss_grad(tm, imgs, to, tw, skip, KO, round_bf16=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (i, fd, g[i])


def test_skipped_orientations_have_no_gradient():
    KO = 64
    L, th, imgs, to, tw, skip = _problem(KO)
    _, g = po.loss_grad(th, imgs, to, tw, skip, KO)
    assert g[L["b3"] + 3] == 0.0
    assert np.all(g[L["w3"] + 3 * 1024:L["w3"] + 4 * 1024] == 0.0)


def test_features_equal_full_plane_inverse_dft(synth):
    """The half-plane sum with weights 1 / 2 is the real inverse DFT of the Hermitian
    plane restricted to the ring, sampled on 16 x 16 points."""
    s = 32
    rng = np.random.default_rng(3)
    ky, kx = synth.window_coords(s)
    P = ky.size
    # a real 16x16 image's low frequencies, placed on the window (Hermitian column kx = 0)
    img = rng.standard_normal((16, 16))
    F16 = np.fft.fft2(img) / 256.0
    fimg = np.zeros((1, P), np.complex128)
    for n in range(P):
        if kx[n] * kx[n] + ky[n] * ky[n] <= 64 and abs(ky[n]) < 8 and kx[n] < 8:
            fimg[0, n] = F16[ky[n] % 16, kx[n]]
    ones = np.ones((1, P))
    got = po.features(fimg, ones, ones, s)[0]
    # the same coefficients over the full plane (Hermitian completion), inverse DFT
    full = np.zeros((16, 16), np.complex128)
    for n in range(P):
        if fimg[0, n] != 0:
            full[ky[n] % 16, kx[n]] = fimg[0, n]
            full[(-ky[n]) % 16, (-kx[n]) % 16] = np.conj(fimg[0, n])
    ref = np.real(np.fft.ifft2(full) * 256.0).reshape(-1)
    ref = ref / np.sqrt((ref ** 2).mean())
    assert np.allclose(got, ref, atol=1e-9)


def test_layout_is_aligned():
    L = po.layout(36864)
    for k in ("wc1", "bc1", "wc2", "bc2", "b1", "b2", "b3", "w1", "w2", "w3"):
        assert L[k] % 64 == 0
    assert L["total"] == L["w3"] + 36864 * 1024
