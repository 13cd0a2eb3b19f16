"""FP64 oracle of the learned orientation-proposal network (test infrastructure).

Restates, in numpy, what t2-relion_b200/csrc/proposal.cu computes, so that the
CUDA forward, backward (gradient) and feature kernels can be checked:
  features  16 x 16 real image of X * CTF * sqrt(Minvsigma2) over the window
            pixels with kx^2 + ky^2 <= min(8, current_size/2)^2 (inverse DFT of
            the half plane: weight 1 on the kx = 0 column, 2 elsewhere), divided
            by its RMS
  conv1     3x3, pad 1, 1 -> 16, ReLU;  conv2 3x3, stride 2, pad 1, 16 -> 32, ReLU
  fc1, fc2  2048 -> 1024 -> 1024, ReLU;  fc3 1024 -> K*O
  loss      softmax cross-entropy (orientations with zero prior excluded)
            against sparse soft targets, mean over the batch
Every weight is used as its BF16 rounding (round to nearest even), exactly as
the CUDA kernels read them; the gradient is with respect to those values.
The network has no counterpart in the reference; its gradient is pinned by
finite differences in tests/test_proposal_oracle.py.
"""
import numpy as np

C1, C2, H0, H1, H2, NPIX = 16, 32, 2048, 1024, 1024, 256


def layout(KO):
    """Offsets of the flat parameter vector (same order and 64-element alignment as the library)."""
    al = lambda x: (x + 63) // 64 * 64
    L, o = {}, 0
    for name, size in (("wc1", C1 * 9), ("bc1", C1), ("wc2", C2 * C1 * 9), ("bc2", C2), ("b1", H1), ("b2", H2),
                       ("b3", KO), ("w1", H1 * H0), ("w2", H2 * H1)):
        L[name] = o
        o = al(o + size)
    L["w3"] = o
    L["total"] = o + KO * H2
    L["KO"] = KO
    return L


def bf16(x):
    """Round float values to BF16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def params(theta, KO, round_bf16=True):
    L = layout(KO)
    t = bf16(theta) if round_bf16 else np.asarray(theta, np.float64)
    g = lambda n, shape: t[L[n]:L[n] + int(np.prod(shape))].reshape(shape)
    return dict(wc1=g("wc1", (C1, 1, 3, 3)), bc1=g("bc1", (C1,)), wc2=g("wc2", (C2, C1, 3, 3)), bc2=g("bc2", (C2,)),
                w1=g("w1", (H1, H0)), b1=g("b1", (H1,)), w2=g("w2", (H2, H1)), b2=g("b2", (H2,)),
                w3=g("w3", (KO, H2)), b3=g("b3", (KO,)))


def ring_pixels(s):
    xh = s // 2 + 1
    R = min(8, s // 2)
    n = np.arange(s * xh)
    i, x = n // xh, n % xh
    y = np.where(i < xh, i, i - s)
    m = x * x + y * y <= R * R
    return n[m], x[m], y[m]


def features(fimg, ctf, minv, s):
    """n x 256 feature images of windowed particles (n x P complex, n x P, n x P)."""
    n_, kx, ky = ring_pixels(s)
    F = fimg[:, n_].astype(np.complex128) * ctf[:, n_] * np.sqrt(np.maximum(minv[:, n_], 0))
    F = F * np.where(kx == 0, 1.0, 2.0)
    u = np.arange(16)
    ph = 2 * np.pi * ((ky[:, None, None] * u[None, :, None] + kx[:, None, None] * u[None, None, :]) % 16) / 16
    img = np.einsum("nk,kab->nab", F.real, np.cos(ph)) - np.einsum("nk,kab->nab", F.imag, np.sin(ph))
    img = img.reshape(len(img), NPIX)
    ms = (img ** 2).mean(axis=1, keepdims=True)
    return np.where(ms > 0, img / np.sqrt(np.where(ms > 0, ms, 1)), 0.0)


def _conv(x, w, b, stride):
    """x: n x Cin x H x W, w: Cout x Cin x 3 x 3, pad 1."""
    n, cin, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    Ho, Wo = (H - 1) // stride + 1, (W - 1) // stride + 1
    cols = np.zeros((n, cin, 3, 3, Ho, Wo))
    for dy in range(3):
        for dx in range(3):
            cols[:, :, dy, dx] = xp[:, :, dy:dy + stride * Ho:stride, dx:dx + stride * Wo:stride]
    return np.einsum("ncdeyx,ocde->noyx", cols, w) + b[None, :, None, None], cols


def forward(theta, imgs, KO, round_bf16=True):
    p = params(theta, KO, round_bf16)
    x = np.asarray(imgs, np.float64).reshape(-1, 1, 16, 16)
    z1, cols1 = _conv(x, p["wc1"], p["bc1"], 1)
    a1 = np.maximum(z1, 0)
    z2, cols2 = _conv(a1, p["wc2"], p["bc2"], 2)
    a2 = np.maximum(z2, 0)
    x0 = a2.reshape(len(x), H0)
    h1 = np.maximum(x0 @ p["w1"].T + p["b1"], 0)
    h2 = np.maximum(h1 @ p["w2"].T + p["b2"], 0)
    y = h2 @ p["w3"].T + p["b3"]
    return y, dict(p=p, x=x, cols1=cols1, a1=a1, cols2=cols2, a2=a2, x0=x0, h1=h1, h2=h2)


def loss_grad(theta, imgs, tgt_oc, tgt_w, skip, KO, round_bf16=True):
    """Mean cross-entropy and its gradient (flat, library layout)."""
    y, c = forward(theta, imgs, KO, round_bf16)
    n = len(y)
    yy = np.where(skip[None, :], -np.inf, y)
    mx = yy.max(axis=1, keepdims=True)
    e = np.exp(yy - mx)
    lse = np.log(e.sum(axis=1, keepdims=True))
    sm = e / e.sum(axis=1, keepdims=True)
    q = np.zeros_like(y)
    for b in range(n):
        for oc, w in zip(tgt_oc[b], tgt_w[b]):
            if oc >= 0 and w > 0 and not skip[oc]:
                q[b, oc] += w
    z = np.where(skip[None, :], 0.0, yy - mx)
    loss = float((q * (lse - z)).sum() / n)
    dy = np.where(skip[None, :], 0.0, sm - q) / n
    p, L = c["p"], layout(KO)
    g = np.zeros(L["total"])
    put = lambda name, arr: g.__setitem__(slice(L[name], L[name] + arr.size), arr.reshape(-1))
    put("w3", dy.T @ c["h2"])
    put("b3", dy.sum(0))
    dh2 = (dy @ p["w3"]) * (c["h2"] > 0)
    put("w2", dh2.T @ c["h1"])
    put("b2", dh2.sum(0))
    dh1 = (dh2 @ p["w2"]) * (c["h1"] > 0)
    put("w1", dh1.T @ c["x0"])
    put("b1", dh1.sum(0))
    dx0 = (dh1 @ p["w1"]).reshape(c["a2"].shape) * (c["a2"] > 0)
    put("wc2", np.einsum("noyx,ncdeyx->ocde", dx0, c["cols2"]))
    put("bc2", dx0.sum(axis=(0, 2, 3)))
    # back through conv2 (stride 2) to a1
    da1p = np.zeros((n, C1, 18, 18))
    for dy_ in range(3):
        for dx_ in range(3):
            da1p[:, :, dy_:dy_ + 16:2, dx_:dx_ + 16:2] += np.einsum("noyx,oc->ncyx", dx0, p["wc2"][:, :, dy_, dx_])
    da1 = da1p[:, :, 1:17, 1:17] * (c["a1"] > 0)
    put("wc1", np.einsum("noyx,ncdeyx->ocde", da1, c["cols1"]))
    put("bc1", da1.sum(axis=(0, 2, 3)))
    return loss, g
