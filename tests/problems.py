"""Small seeded E-step problems shared by the parity tests."""
import numpy as np

from conftest import load_package


def build(name, n_particles=16, seed=7, nr_classes=1, diff2_mode=0, max_batch=None, ref_dim=3, maxsig=-1,
          scale_correction=False):
    """scale_correction: per-particle scale_correction in U(0.8, 1.2) and a data_vs_prior per
    class and ring spread around the threshold 3, so both kinds of ring occur."""
    t2b = load_package()
    import t2relion_b200.synthetic as sy
    import oracle as orc
    presets = {
        # box 64, order 2 (9216 orientations), 29 shifts, r 16: the CPU-runnable refine
        "refine_o2": dict(N=64, angpix=2.0, order=2, psi=7.5, rng=3, r=16, snr=0.05, ovs=0),
        # box 64, order 1 + adaptive oversampling (fine pass), 29 shifts
        "refine_o1_ovs": dict(N=64, angpix=2.0, order=1, psi=15.0, rng=3, r=16, snr=0.05, ovs=1),
        # box 64, order 2 + adaptive oversampling, high SNR: a sharp posterior, the regime in
        # which the learned proposals hold the posterior (the box-128 benchmark's regime)
        "learn_o2": dict(N=64, angpix=2.0, order=2, psi=7.5, rng=3, r=16, snr=0.5, ovs=1),
        # the same at SNR 0.03 (the box-128 benchmark's noise level): broad posteriors at box 64,
        # where 64 proposals miss posterior mass and the audit must send batches to the full pass
        "learn_o2_lowsnr": dict(N=64, angpix=2.0, order=2, psi=7.5, rng=3, r=16, snr=0.03, ovs=1),
        # 2D classification: 2D references, psi 6 deg, oversampling 1
        "class2d": dict(N=48, angpix=2.0, order=0, psi=6.0, rng=3, r=12, snr=0.2, ovs=1),
    }
    p = presets[name]
    N, r, s = p["N"], p["r"], 2 * p["r"]
    ref_dim = 2 if name == "class2d" else 3
    maps = []
    for k in range(nr_classes):
        vol = sy.blob_volume(N, 40 if ref_dim == 3 else 12, seed=seed + 101 * k, ndim=ref_dim)
        maps.append(sy.fourier_map(vol, r))
    samp = t2b.sampling(ref_dim, p["order"], p["psi"], p["ovs"], p["rng"], 1, p["angpix"])
    cls = np.arange(n_particles) % nr_classes
    parts = sy.make_particles(maps[0], n_particles, ori_size=N, s=s, r_max=r, angpix=p["angpix"],
                              snr=p["snr"], seed=seed, max_shift=p["rng"], ref_dim=ref_dim,
                              classes=cls, class_maps=maps)
    dvp = None
    if scale_correction:
        srng = np.random.default_rng(seed + 977)
        parts["scalars"][:, 6] = srng.uniform(0.8, 1.2, n_particles)
        dvp = srng.uniform(0.0, 8.0, (nr_classes, N // 2 + 1))
    sigma2_offset = (p["rng"] * p["angpix"]) ** 2
    pdf_dir = np.ones((nr_classes, samp["n_dir"])) / (samp["n_dir"] * nr_classes)
    pdf_cls = np.ones(nr_classes) / nr_classes
    ps = sy.pad_size(r)
    prob = orc.Problem(ori_size=N, s=s, ref_dim=ref_dim, maps=maps, r_max=r, pad=2, samp=samp,
                       pdf_direction=pdf_dir, pdf_class=pdf_cls, sigma2_offset=sigma2_offset,
                       pixel_size=p["angpix"], adaptive_fraction=0.999, ovs=p["ovs"], bp_pad_size=ps,
                       bp_r_max=r, maximum_significants=maxsig, data_vs_prior=dvp)
    mres = sy.mresol(s)
    oparts = prob.particles(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"], mres)

    def product(use_graph=1, orientation_chunk=0):
        es = t2b.EStep(0)
        for k in range(nr_classes):
            es.set_projector(k, maps[k], ref_dim, r, 2)
            es.init_backprojector(k, ref_dim, ps, r, 2)
        es.configure(ori_size=N, current_size=s, ref_dim=ref_dim, nr_classes=nr_classes, samp=samp,
                     pdf_direction=pdf_dir, pdf_class=pdf_cls, sigma2_offset=sigma2_offset,
                     pixel_size=p["angpix"], adaptive_oversampling=p["ovs"], diff2_mode=diff2_mode,
                     max_batch=max_batch or n_particles, maximum_significants=maxsig, data_vs_prior=dvp,
                     use_graph=use_graph, orientation_chunk=orientation_chunk)
        return es

    def oracle_problem():
        """A second oracle Problem of the same setup (own grids) for same-input stage checks;
        `oparts` can be passed to it."""
        return orc.Problem(ori_size=N, s=s, ref_dim=ref_dim, maps=maps, r_max=r, pad=2, samp=samp,
                           pdf_direction=pdf_dir, pdf_class=pdf_cls, sigma2_offset=sigma2_offset,
                           pixel_size=p["angpix"], adaptive_fraction=0.999, ovs=p["ovs"], bp_pad_size=ps,
                           bp_r_max=r, maximum_significants=maxsig, data_vs_prior=dvp)

    return dict(t2b=t2b, sy=sy, maps=maps, samp=samp, parts=parts, prob=prob, oparts=oparts,
                product=product, oracle_problem=oracle_problem, N=N, s=s, r=r, pad_size=ps, ovs=p["ovs"],
                K=nr_classes, ref_dim=ref_dim, data_vs_prior=dvp)


def fsc(a, b, shells, nshell):
    """Fourier shell correlation of two centred half-complex grids."""
    num = np.bincount(shells, (a * np.conj(b)).real, nshell)
    da = np.bincount(shells, np.abs(a) ** 2, nshell)
    db = np.bincount(shells, np.abs(b) ** 2, nshell)
    with np.errstate(invalid="ignore", divide="ignore"):
        return num / np.sqrt(da * db)


def shells_of(shape):
    if len(shape) == 3:
        z, y, x = shape
        kz = np.arange(z)[:, None, None] - z // 2
        ky = np.arange(y)[None, :, None] - y // 2
        kx = np.arange(x)[None, None, :]
        r = np.sqrt(kz * kz + ky * ky + kx * kx)
    else:
        y, x = shape
        ky = np.arange(y)[:, None] - y // 2
        kx = np.arange(x)[None, :]
        r = np.sqrt(ky * ky + kx * kx)
    return np.rint(r).astype(int).reshape(-1)


# The benchmarked workload: box 128, 1.3 A/px, 40-blob map (seed 11), HEALPix order 3 x psi
# 7.5 deg, adaptive oversampling 1, translations range 5 step 1, Fourier radius 40, 2x padded
# backprojection grid of r_max 64, white noise at SNR 0.03.
BOX128 = dict(ori_size=128, angpix=1.3, n_blobs=40, map_seed=11, order=3, psi_step=7.5, offset_range=5,
              offset_step=1, r_max=40, bp_r_max=64, snr=0.03)


def box128(n_particles, seed, data_vs_prior=None):
    """Inputs, sampling and an oracle Problem of the box-128 workload (n particles, seed)."""
    t2b = load_package()
    import t2relion_b200.synthetic as sy
    import oracle as orc
    w = BOX128
    N, r = w["ori_size"], w["r_max"]
    s = 2 * r
    fmap = sy.fourier_map(sy.blob_volume(N, w["n_blobs"], seed=w["map_seed"]), r)
    samp = t2b.sampling(3, w["order"], w["psi_step"], 1, w["offset_range"], w["offset_step"], w["angpix"])
    parts = sy.make_particles(fmap, n_particles, ori_size=N, s=s, r_max=r, angpix=w["angpix"], snr=w["snr"],
                              seed=seed, max_shift=w["offset_range"])
    pdf_dir = np.full((1, samp["n_dir"]), 1.0 / samp["n_dir"])
    sigma2_offset = (w["offset_range"] * w["angpix"]) ** 2
    ps = sy.pad_size(w["bp_r_max"])
    prob = orc.Problem(ori_size=N, s=s, ref_dim=3, maps=[fmap], r_max=r, pad=2, samp=samp, pdf_direction=pdf_dir,
                       pdf_class=np.ones(1), sigma2_offset=sigma2_offset, pixel_size=w["angpix"],
                       adaptive_fraction=0.999, ovs=1, bp_pad_size=ps, bp_r_max=w["bp_r_max"],
                       data_vs_prior=data_vs_prior)
    oparts = prob.particles(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"], sy.mresol(s))

    def product(diff2_mode, max_batch=None, use_graph=1):
        es = t2b.EStep(0)
        es.set_projector(0, fmap, 3, r, 2)
        es.init_backprojector(0, 3, ps, w["bp_r_max"], 2)
        es.configure(ori_size=N, current_size=s, ref_dim=3, nr_classes=1, samp=samp, pdf_direction=pdf_dir,
                     pdf_class=np.ones(1), sigma2_offset=sigma2_offset, pixel_size=w["angpix"],
                     adaptive_oversampling=1, diff2_mode=diff2_mode, max_batch=max_batch or n_particles,
                     use_graph=use_graph, data_vs_prior=data_vs_prior)
        return es

    return dict(t2b=t2b, sy=sy, fmap=fmap, samp=samp, parts=parts, prob=prob, oparts=oparts, product=product,
                pad_size=ps)


def input_digest(parts):
    """SHA-256 of the E-step inputs (detects a change of the generator)."""
    import hashlib
    h = hashlib.sha256()
    for k in ("fimg", "ctf", "minv", "scalars"):
        h.update(np.ascontiguousarray(parts[k]).tobytes())
    return h.hexdigest()


# 2D classification at its stated size: K = 50 references of 100 x 100 (seeded blob images),
# particles from those classes with random in-plane rotation and shifts U(-5, 5) px, SNR
# 0.05; psi step 6 deg (60), translations range 5 step 1 (81), adaptive oversampling 1 (2 psi
# x 4 shifts per significant pair), the window to Nyquist (r 50: 100 x 51 pixels).
CLASS2D = dict(ori_size=100, angpix=2.0, n_blobs=12, n_classes=50, map_seed=31, psi_step=6.0, offset_range=5,
               offset_step=1, r_max=50, snr=0.05)


def class2d_k50(n_particles, seed, n_classes=None):
    """Inputs, sampling and an oracle Problem of the 2D-classification workload."""
    t2b = load_package()
    import t2relion_b200.synthetic as sy
    import oracle as orc
    w = CLASS2D
    K = n_classes or w["n_classes"]
    N, r = w["ori_size"], w["r_max"]
    s = 2 * r
    maps = [sy.fourier_map(sy.blob_volume(N, w["n_blobs"], seed=w["map_seed"] + 101 * k, ndim=2), r)
            for k in range(K)]
    samp = t2b.sampling(2, 0, w["psi_step"], 1, w["offset_range"], w["offset_step"], w["angpix"])
    cls = np.random.default_rng(seed + 7).integers(0, K, n_particles)
    parts = sy.make_particles(maps[0], n_particles, ori_size=N, s=s, r_max=r, angpix=w["angpix"], snr=w["snr"],
                              seed=seed, max_shift=w["offset_range"], ref_dim=2, classes=cls, class_maps=maps)
    pdf_dir = np.ones((K, 1))
    pdf_cls = np.full(K, 1.0 / K)
    sigma2_offset = (w["offset_range"] * w["angpix"]) ** 2
    ps = sy.pad_size(r)
    prob = orc.Problem(ori_size=N, s=s, ref_dim=2, maps=maps, r_max=r, pad=2, samp=samp, pdf_direction=pdf_dir,
                       pdf_class=pdf_cls, sigma2_offset=sigma2_offset, pixel_size=w["angpix"],
                       adaptive_fraction=0.999, ovs=1, bp_pad_size=ps, bp_r_max=r)
    oparts = prob.particles(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"], sy.mresol(s))

    def product(diff2_mode, max_batch=None, use_graph=1):
        es = t2b.EStep(0)
        for k in range(K):
            es.set_projector(k, maps[k], 2, r, 2)
            es.init_backprojector(k, 2, ps, r, 2)
        es.configure(ori_size=N, current_size=s, ref_dim=2, nr_classes=K, samp=samp, pdf_direction=pdf_dir,
                     pdf_class=pdf_cls, sigma2_offset=sigma2_offset, pixel_size=w["angpix"],
                     adaptive_oversampling=1, diff2_mode=diff2_mode, max_batch=max_batch or n_particles,
                     use_graph=use_graph)
        return es

    return dict(t2b=t2b, sy=sy, maps=maps, samp=samp, parts=parts, prob=prob, oparts=oparts, product=product,
                pad_size=ps, K=K, classes=cls)


# Large 3D classification: K = 4 maps of 256^3 at 0.85 A/px that differ by 10 % of their blobs,
# particles 256 x 256 at SNR 0.02, defocus U(0.8, 2.5) um; HEALPix order 4 x psi 3.75 deg
# (294,912 orientations per class), adaptive oversampling 1, translations range 4 step 1 (49),
# Fourier radius 100 (200 x 101 pixels), 2x padded grids of r_max 128 (515 x 515 x 258).
LARGE3D = dict(ori_size=256, angpix=0.85, n_blobs=40, n_classes=4, map_seed=5, order=4, psi_step=3.75,
               offset_range=4, offset_step=1, r_max=100, bp_r_max=128, snr=0.02, defocus=(8000., 25000.))


def large3d(n_particles, seed, with_grids=True):
    """Inputs and sampling of the large 3D classification, and an oracle Problem for literal
    per-hypothesis diff2 checks (its own grids are tiny: the full pass is out of the oracle's
    reach at this size)."""
    t2b = load_package()
    import t2relion_b200.synthetic as sy
    import oracle as orc
    w = LARGE3D
    K, N, r = w["n_classes"], w["ori_size"], w["r_max"]
    s = 2 * r
    maps = [sy.fourier_map(v, r) for v in sy.blob_class_volumes(N, K, w["n_blobs"], seed=w["map_seed"])]
    samp = t2b.sampling(3, w["order"], w["psi_step"], 1, w["offset_range"], w["offset_step"], w["angpix"])
    cls = np.arange(n_particles) % K
    parts = sy.make_particles(maps[0], n_particles, ori_size=N, s=s, r_max=r, angpix=w["angpix"], snr=w["snr"],
                              seed=seed, max_shift=w["offset_range"], defocus=w["defocus"], classes=cls,
                              class_maps=maps)
    pdf_dir = np.full((K, samp["n_dir"]), 1.0 / samp["n_dir"])
    pdf_cls = np.full(K, 1.0 / K)
    sigma2_offset = (w["offset_range"] * w["angpix"]) ** 2
    ps = sy.pad_size(w["bp_r_max"])
    prob = orc.Problem(ori_size=N, s=s, ref_dim=3, maps=maps, r_max=r, pad=2, samp=samp, pdf_direction=pdf_dir,
                       pdf_class=pdf_cls, sigma2_offset=sigma2_offset, pixel_size=w["angpix"],
                       adaptive_fraction=0.999, ovs=1, bp_pad_size=sy.pad_size(1), bp_r_max=1)
    oparts = prob.particles(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"], sy.mresol(s))

    def product(max_batch=None, use_graph=1, orientation_chunk=0):
        es = t2b.EStep(0)
        for k in range(K):
            es.set_projector(k, maps[k], 3, r, 2)
            if with_grids:
                es.init_backprojector(k, 3, ps, w["bp_r_max"], 2)
        es.configure(ori_size=N, current_size=s, ref_dim=3, nr_classes=K, samp=samp, pdf_direction=pdf_dir,
                     pdf_class=pdf_cls, sigma2_offset=sigma2_offset, pixel_size=w["angpix"],
                     adaptive_oversampling=1, diff2_mode=1, max_batch=max_batch or n_particles,
                     use_graph=use_graph, orientation_chunk=orientation_chunk)
        return es

    return dict(t2b=t2b, sy=sy, maps=maps, samp=samp, parts=parts, prob=prob, oparts=oparts, product=product,
                pad_size=ps, K=K, classes=cls)


def angle_between(A, B):
    """Rotation angle (degrees) between rotation matrices A and B (3 x 3)."""
    c = (np.trace(np.asarray(A).reshape(3, 3) @ np.asarray(B).reshape(3, 3).T) - 1) / 2
    return float(np.degrees(np.arccos(np.clip(c, -1.0, 1.0))))
