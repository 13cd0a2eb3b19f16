"""E-step throughput benchmark (particles/s) on the box-128 refinement workload.

Workload (the headline configuration): 128^3 map of 40 seeded Gaussian blobs at
1.3 A/px; particles 128x128 with CTF (300 kV, Cs 2.7, Q0 0.1, defocus U(1,3) um,
astigmatism <= 0.1 um) and white noise at SNR 0.03; HEALPix order 3 x 48 psi =
36,864 coarse orientations, adaptive oversampling 1 (fine pass at order 4, 8
rotations x 4 shifts per significant coarse pair); translations range 5 step 1
(81); Fourier radius 40 px (80 x 41 = 3,280 pixels); backprojection into the
2x padded 259 x 259 x 130 grid.  A step is one E-step over one batch of
`--batch` particles: coarse diff2, FP64 weights and significance, fine pass,
FP64 weights, weighted sums and backprojection.

value: particles/s with inputs resident in HBM (device entry point, CUDA events
on the launching stream, max over ranks).  e2e: the same metric through the
host entry points with pinned host buffers (H2D of the batch and D2H of the
results inside the timed region, host wall clock): the pipelined pair
t2b_estep_submit_host / t2b_estep_wait, step i's inputs copying while step i-1
computes (`synchronous_value`: t2b_estep_batch_host, one blocking call per step).  `--impl reference` times the reference's CPU
E-step on the host cores instead: the reference's own CPU diff2 kernel compiled
from its sources (oracle/_ref) when built, else the FP64 port in oracle/.
"""
import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))


def load_package():
    name = "t2relion_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = os.path.join(ROOT, "t2-relion_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


WORKLOAD = dict(name="refine3d_box128_order3_ovs1", ori_size=128, angpix=1.3, n_blobs=40, order=3,
                psi_step=7.5, offset_range=5, offset_step=1, r_max=40, bp_r_max=64, snr=0.03, seed=11)
# reduced case for ncu captures (device memory of a few GB): HEALPix order 2, otherwise identical
PROFILE_WORKLOAD = dict(WORKLOAD, name="refine3d_box128_order2_ovs1_profile", order=2)
METRIC = "E-step particles/s box128: learned+split-BF16 vs plain FP32 GPU; roofline %"
# learned proposals: network top-1024 rescored at low resolution, best 64 to the coarse
# pass; every 50th particle (2 %) audited by the full coarse pass (>= 0.999 of its mass)
PROP = dict(topk=64, rescore=1024, audit_every=50, audit_mass=0.999)
# end-to-end timing: at least this many steps per timed run
E2E_STEPS = 30
# DRAM bytes (read + write) of k_diff2_tc per step from one ncu capture, stamped with the
# SHA-256 (first 16 hex digits) of the kernel's source at capture time; a line whose kernel
# source differs reports traffic null rather than a stale figure.
#   learned, 512 particles: the audit + proposal launches; captured on the reduced case (HEALPix
#   order 2), the audit's operand and output scaled x 4 to the 36,864 orientations (audit 267.5 MB
#   read + 16.8 MB written, proposal pass 675.5 + 6.3 MB, which does not depend on them)
TRAFFIC = {"kernel_sha": "84303c0f85bebd48", "learned_batch": 512,
           "learned": 4 * (267.5e6 + 16.8e6) + 675.5e6 + 6.3e6}
# particles of the learned-vs-plain quality check (not the timed batch)
QUALITY_PARTICLES = 2048
# timed steps of the plain FP32 comparator (1,154 particles/s: about 0.11 s per 128-particle step)
PLAIN_STEPS = 5


def kernel_sha():
    import hashlib
    with open(os.path.join(ROOT, "t2-relion_b200", "csrc", "diff2_tc.cu"), "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()[:16]


def build_problem(t2b, sy, n_particles, seed):
    w = WORKLOAD
    N, r = w["ori_size"], w["r_max"]
    s = 2 * r
    vol = sy.blob_volume(N, w["n_blobs"], seed=w["seed"])
    fmap = sy.fourier_map(vol, r)
    samp = t2b.sampling(3, w["order"], w["psi_step"], 1, w["offset_range"], w["offset_step"], w["angpix"])
    parts = sy.make_particles(fmap, n_particles, ori_size=N, s=s, r_max=r, angpix=w["angpix"], snr=w["snr"],
                              seed=seed, max_shift=w["offset_range"])
    return fmap, samp, parts


def setup_context(t2b, sy, fmap, samp, mode, batch, device=0, use_graph=1):
    w = WORKLOAD
    es = t2b.EStep(device)
    es.set_projector(0, fmap, 3, w["r_max"], 2)
    es.init_backprojector(0, 3, sy.pad_size(w["bp_r_max"]), w["bp_r_max"], 2)
    es.configure(ori_size=w["ori_size"], current_size=2 * w["r_max"], ref_dim=3, nr_classes=1, samp=samp,
                 pdf_direction=np.full((1, samp["n_dir"]), 1.0 / samp["n_dir"]), pdf_class=np.ones(1),
                 sigma2_offset=(w["offset_range"] * w["angpix"]) ** 2, pixel_size=w["angpix"],
                 adaptive_oversampling=1, diff2_mode=mode, max_batch=batch, use_graph=use_graph)
    return es


class ClockSampler:
    """SM clock / throttle-reason sampling during the timed region.

    NVML (pynvml) polled every 10 ms from a thread, on the device whose UUID
    torch reports for `gpu`; nvidia-smi at 200 ms when pynvml is missing.
    """
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.thread = None
        self.samples = []   # (sm_mhz, reason bits)
        self.max_mhz = None
        self.lines = []

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid if not uuid.startswith("GPU-") else uuid)
        except pynvml.NVMLError:
            if pynvml.nvmlDeviceGetCount() == 1:
                return pynvml, pynvml.nvmlDeviceGetHandleByIndex(0)
            raise

    def _poll(self, nv, h):
        while not self.stop.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except nv.NVMLError:
                pass
            self.stop.wait(0.01)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], self.max_mhz, set()
        for mhz, bits in self.samples:
            sm.append(float(mhz))
            for n, b in self.REASONS:
                if bits & b:
                    reasons.add(n)
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for (n, _), v in zip(self.REASONS, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.samples else ("nvidia-smi" if self.lines else None)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d, "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def load_synthetic():
    """The particle generator, t2-relion_b200/synthetic.py (numpy only), loaded by its path
    without the package: the reference arm and the CPU baseline must not load the library."""
    name = "t2b_synthetic_standalone"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "t2-relion_b200", "synthetic.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules[name] = mod
    return sys.modules[name]


def workload_config():
    """`config` of the JSON line: the workload alone, identical in both arms."""
    w = WORKLOAD
    s = 2 * w["r_max"]
    return {"workload": w["name"], "box": w["ori_size"], "healpix_order": w["order"], "psi_step": w["psi_step"],
            "orientations": 12 * 4 ** w["order"] * int(np.ceil(360 / w["psi_step"])),
            "translations": 81 if w["offset_range"] == 5 else None, "pixels": s * (s // 2 + 1),
            "adaptive_oversampling": 1, "fine_hypotheses_per_pair": 32, "snr": w["snr"],
            "grid": [259, 259, 130]}


class CpuEStep:
    """The reference's CPU E-step of the workload on the host cores, one particle per thread.

    Coarse pass: the reference's own CPU kernel, CpuKernels::diff2_coarse
    (src/acc/cpu/cpu_kernels/diff2.h:329-606, compiled from the reference sources into
    oracle/_ref/libacc_ref.so), over every orientation and translation; where that library is
    absent, the FP64 oracle's coarse pass.  The rest -- weights and significance, fine pass,
    weights, weighted sums, backprojection -- by the FP64 oracle port (oracle/), which is
    more than 95 % cheaper than the coarse pass at this workload.  Nothing of the library is
    loaded: sampling from oracle/sampling_oracle.py, particles from synthetic.py by path.
    """

    def __init__(self, n_particles, seed):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        import sampling_oracle as so
        w = WORKLOAD
        self.sy = sy = load_synthetic()
        N, r = w["ori_size"], w["r_max"]
        self.s = s = 2 * r
        self.fmap = fmap = sy.fourier_map(sy.blob_volume(N, w["n_blobs"], seed=w["seed"]), r)
        self.samp = samp = so.sampling(w["order"], w["psi_step"], 1, w["offset_range"], w["offset_step"], w["angpix"])
        self.parts = parts = sy.make_particles(fmap, n_particles, ori_size=N, s=s, r_max=r, angpix=w["angpix"],
                                               snr=w["snr"], seed=seed, max_shift=w["offset_range"])
        self.prob = orc.Problem(ori_size=N, s=s, ref_dim=3, maps=[fmap], r_max=r, pad=2, samp=samp,
                                pdf_direction=np.full((1, samp["n_dir"]), 1.0 / samp["n_dir"]), pdf_class=np.ones(1),
                                sigma2_offset=(w["offset_range"] * w["angpix"]) ** 2, pixel_size=w["angpix"],
                                adaptive_fraction=0.999, ovs=1, bp_pad_size=sy.pad_size(w["bp_r_max"]),
                                bp_r_max=w["bp_r_max"])
        self.op = self.prob.particles(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"], sy.mresol(s))
        self.O, self.T = samp["n_dir"] * samp["n_psi"], samp["n_trans"]
        lib_path = os.path.join(ROOT, "oracle", "_ref", "libacc_ref.so")
        self.kind = "reference" if os.path.exists(lib_path) else "port"
        if self.kind == "reference":
            self.lib = ctypes.CDLL(lib_path)
            self.lib.ref_coarse_diff2.restype = ctypes.c_int
            self.fm = np.ascontiguousarray(fmap.view(np.float32))
            eul = samp["eul_coarse"].reshape(-1, 3, 3)
            self.einv = np.ascontiguousarray(np.transpose(eul, (0, 2, 1)).reshape(-1, 9), np.float32)
            self.tx = np.ascontiguousarray(-2 * np.pi * samp["trans_px"][:, 0] / N, np.float32)
            self.ty = np.ascontiguousarray(-2 * np.pi * samp["trans_px"][:, 1] / N, np.float32)
            # the reference kernel's operands (refs_are_ctf_corrected): X / CTF and Minvsigma2 CTF^2
            self.ops = []
            for b in range(n_particles):
                ctf = parts["ctf"][b].astype(np.float64)
                X = parts["fimg"][b].astype(np.complex128) / ctf
                self.ops.append((np.ascontiguousarray(X.real, np.float32), np.ascontiguousarray(X.imag, np.float32),
                                 np.ascontiguousarray(parts["minv"][b] * ctf * ctf, np.float32),
                                 float(parts["scalars"][b, 1] / 2)))

    def coarse(self, b, n_orient=None):
        no = self.O if n_orient is None else n_orient
        if self.kind != "reference":
            d2, _ = self.prob.coarse_diff2(self.op, b)
            return d2
        w, mz, my, mx = WORKLOAD, *self.fmap.shape
        out = np.empty((no, self.T), np.float32)
        re, im, corr, xi2 = self.ops[b]
        rc = self.lib.ref_coarse_diff2(
            ctypes.c_void_p(self.fm.ctypes.data), mx, my, mz, -(my // 2), -(mz // 2), w["r_max"], 2,
            ctypes.c_void_p(self.einv.ctypes.data), no, ctypes.c_void_p(re.ctypes.data),
            ctypes.c_void_p(im.ctypes.data), ctypes.c_void_p(corr.ctypes.data), self.s // 2 + 1, self.s,
            ctypes.c_void_p(self.tx.ctypes.data), ctypes.c_void_p(self.ty.ctypes.data), self.T, ctypes.c_float(xi2),
            ctypes.c_void_p(out.ctypes.data))
        if rc != 0:
            raise RuntimeError("reference coarse kernel refused the orientation count")
        return out.reshape(-1)

    def particle(self, b):
        """The whole E-step of particle b (its backprojection into the oracle's grid)."""
        prob, op = self.prob, self.op
        d2 = self.coarse(b).astype(np.float64)
        rc, w, sw, sig, _ = prob.weights(op, b, 0, d2, np.arange(d2.size), d2.min())
        if rc != 0:
            raise RuntimeError("no significant coarse sample")
        pairs, fd, fmn = prob.fine_diff2(op, b, (w >= sig).astype(np.uint8))
        rc, wf, fsum, fsig, _ = prob.weights(op, b, 1, fd.reshape(-1), np.repeat(pairs, prob.RV), fmn)
        prob.wsum_bp(op, b, pairs, wf, fsum, fsig)

    def run(self, particles, warm=False):
        """Seconds for `particles`, one host thread each (warm: one direction's coarse pass only)."""
        fn = (lambda b: self.coarse(b, self.samp["n_psi"])) if warm else self.particle
        t0 = time.perf_counter()
        ths = [threading.Thread(target=fn, args=(b,)) for b in particles]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        return time.perf_counter() - t0

    def sample_text(self, n):
        src = ("the reference's CpuKernels::diff2_coarse, compiled from its sources" if self.kind == "reference"
               else "the FP64 oracle port")
        return (f"{n} particles per step, one per host thread, each through the whole E-step: coarse pass over "
                f"all {self.O} orientations x {self.T} translations by {src}; FP64 weights and significance, fine "
                f"pass, weighted sums and backprojection by the FP64 oracle port")


def cpu_baseline(cores=None):
    """The reference's CPU E-step on the host cores, bounded sample: one step of CpuEStep
    (a particle per host thread through the whole E-step, about 12-20 s)."""
    n = cores or os.cpu_count() or 1
    cpu = CpuEStep(n, WORKLOAD["seed"] + 1)
    cpu.run(range(n), warm=True)
    t = cpu.run(range(n))
    return {"value": n / t, "unit": "particles/s", "cores": n, "kind": cpu.kind, "sample": cpu.sample_text(n) +
            f"; {t:.1f} s"}


def _fsc_min(a, b, r_max_pad):
    """Smallest Fourier shell correlation of two FFTW-ordered half transforms
    [n][n][n/2+1] over the shells 1 .. r_max_pad."""
    n = a.shape[0]
    f = np.fft.fftfreq(n) * n
    kz, ky = np.meshgrid(f, f, indexing="ij")
    kx = np.arange(a.shape[2])
    r = np.rint(np.sqrt(kz[..., None] ** 2 + ky[..., None] ** 2 + kx[None, None, :] ** 2)).astype(int).ravel()
    num = np.bincount(r, (a * np.conj(b)).real.ravel())
    da = np.bincount(r, (np.abs(a) ** 2).ravel())
    db = np.bincount(r, (np.abs(b) ** 2).ravel())
    sh = np.arange(1, min(r_max_pad, len(num) - 1) + 1)
    fsc = num[sh] / np.sqrt(np.maximum(da[sh] * db[sh], 1e-300))
    return float(fsc.min())


def quality_vs_plain(es, es_plain, sy, fmap, n_check, batch, seed):
    """The learned E-step against the plain FP32 path on `n_check` particles that are not the
    timed batch (host entry points, outside the timed region): pose agreement, and the FSC of
    the two reconstructions (FP64 skip-gridding division of the backprojected grids) after
    Hermitian symmetrisation, as the M-step sees them."""
    w = WORKLOAD
    parts = sy.make_particles(fmap, n_check, ori_size=w["ori_size"], s=2 * w["r_max"], r_max=w["r_max"],
                              angpix=w["angpix"], snr=w["snr"], seed=seed, max_shift=w["offset_range"])
    es.clear_backprojector(0)
    es_plain.clear_backprojector(0)
    same, learned, audited = 0, 0, 0
    for a in range(0, n_check, batch):
        args = [parts[k][a:a + batch] for k in ("fimg", "ctf", "minv", "scalars")]
        got = es.expectation(*args)
        ref = es_plain.expectation(*args)
        same += int(np.all(got["pose"] == ref["pose"], axis=1).sum())
        learned += int(got["learned"].sum())
        audited += int((got["audit_mass"] >= 0).sum())
    for e in (es, es_plain):
        e.enforce_hermitian_symmetry(0)
    rp = w["r_max"] * 2   # padded-grid radius reached by the r_max window (padding factor 2)
    fsc = _fsc_min(es.reconstruct_divide(0), es_plain.reconstruct_divide(0), rp)
    return {"particles": n_check, "pose_agreement_vs_plain": same / n_check, "map_fsc_min_vs_plain": fsc,
            "learned_fraction": learned / n_check, "audited_particles": audited}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, world, rank):
    """The reference's CPU E-step (CpuEStep) on the host cores: every step one particle per host
    thread through the whole E-step; warm-up steps run one direction's coarse pass per thread.
    Rank 0 alone runs and prints; other ranks exit without work."""
    if rank != 0:
        return
    n = os.cpu_count() or 1
    cpu = CpuEStep(n, WORKLOAD["seed"] + 1)
    for _ in range(args.warmup):
        cpu.run(range(n), warm=True)
    times = [cpu.run(range(n)) for _ in range(args.steps)]
    total = float(np.sum(times))
    v = n * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "particles/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (coarse kernel) / f64 (rest)" if cpu.kind == "reference" else "f64",
            "data": "synthetic", "config": workload_config(), "particles_per_step": n,
            "cpu_baseline": {"value": v, "unit": "particles/s", "cores": n, "kind": cpu.kind,
                             "sample": cpu.sample_text(n)},
            "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


PREP_WORKLOAD = dict(name="prep_box128_s80_noise_background", image_size=128, current_size=80, pixel_size=1.3,
                     mask_radius=50.0, width_mask_edge=5.0, zero_mask=0, random_seed=11, sigma2_fudge=1.0,
                     voltage=300.0, cs=2.7, q0=0.1)


def run_prep(args):
    """Image preparation (t2b_prep_batch_*) of box-128 real-space particles to the
    80-pixel E-step window with the noise background: particles/s."""
    import torch
    t2b = load_package()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    W = PREP_WORKLOAD
    N, s, B = W["image_size"], W["current_size"], args.prep_batch
    rng = np.random.default_rng(W["random_seed"])
    imgs = rng.standard_normal((B, N, N)).astype(np.float32)
    par = np.zeros((B, t2b.PREP_NPARAM))
    par[:, 0:2] = rng.uniform(-5, 5, (B, 2))
    par[:, 2:4] = 999.
    par[:, 4] = 1.0
    par[:, 5] = rng.uniform(10000, 30000, B)
    par[:, 6] = par[:, 5] - rng.uniform(0, 1000, B)
    par[:, 7] = rng.uniform(0, 180, B)
    par[:, 9] = par[:, 11] = 1.0
    pid = np.arange(B, dtype=np.int64)
    sig = 0.2 + np.linspace(1.0, 0.05, N // 2 + 1) ** 2
    es = t2b.EStep(0)
    cfg = {k: v for k, v in W.items() if k != "name"}
    es.configure_prep(max_batch=B, sigma2_noise=sig, **cfg)
    dev = torch.device("cuda", 0)
    P, h = s * (s // 2 + 1), N // 2 + 1
    ti, tp, tq = (torch.from_numpy(a).to(dev) for a in (imgs, par, pid))
    out = dict(fimg=torch.zeros(B, 2 * P, device=dev), fimg_nomask=torch.zeros(B, 2 * P, device=dev),
               ctf=torch.zeros(B, P, device=dev), minvsigma2=torch.zeros(B, P, device=dev),
               scalars=torch.zeros(B, 8, dtype=torch.float64, device=dev),
               power=torch.zeros(B, h, dtype=torch.float64, device=dev))
    optr = {k: ctypes.c_void_p(v.data_ptr()) for k, v in out.items()}
    stream = torch.cuda.Stream(dev)

    def step():
        es.prepare_images_device(B, ctypes.c_void_p(ti.data_ptr()), ctypes.c_void_p(tp.data_ptr()),
                                 ctypes.c_void_p(tq.data_ptr()), optr, stream=stream.cuda_stream)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        torch.cuda.nvtx.range_push("timed_steps")
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = ev0.elapsed_time(ev1) / args.steps
    value = B / (ms / 1000.0)
    # end to end through the host entry point (host images in, host E-step inputs out)
    pin_img = torch.from_numpy(imgs).pin_memory()
    pin_par = torch.from_numpy(par).pin_memory()
    pin_pid = torch.from_numpy(pid).pin_memory()
    hout = {k: torch.zeros(v.shape, dtype=v.dtype).pin_memory() for k, v in out.items()}
    b = t2b.PrepBatch(B, 0, ctypes.c_void_p(pin_img.data_ptr()), ctypes.c_void_p(pin_par.data_ptr()),
                      ctypes.c_void_p(pin_pid.data_ptr()))
    o = t2b.PrepOut(*[ctypes.c_void_p(hout[k].data_ptr()) for k, _ in t2b.PrepOut._fields_])
    for _ in range(2):
        t2b._check(t2b.lib.t2b_prep_batch_host(es._h, ctypes.byref(b), ctypes.byref(o)))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        t2b._check(t2b.lib.t2b_prep_batch_host(es._h, ctypes.byref(b), ctypes.byref(o)))
    e2e_s = (time.perf_counter() - t0) / args.steps
    h2d = pin_img.numel() * 4 + pin_par.numel() * 8 + pin_pid.numel() * 8
    d2h = sum(v.numel() * v.element_size() for v in hout.values())
    # algorithmic bytes per particle: the image and its parameters in, the E-step inputs out
    per = N * N * 4 + t2b.PREP_NPARAM * 8 + 8 + 2 * (2 * P * 4) + 2 * (P * 4) + 8 * 8 + h * 8
    peaks, src = measured_peaks()
    achieved = per * B / (ms / 1000.0) / 1e9
    peak = peaks.get("hbm_gbs", 6650.0)
    line = {"metric": "image preparation particles/s box128 -> 80-pixel window, noise background",
            "value": value, "unit": "particles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FFT) / f64 (sums, noise, CTF)", "data": "synthetic",
            "config": {"workload": W["name"], "particles_per_step": B,
                       "l2": "inputs (%.0f MB) larger than L2" % (B * N * N * 4 / 1e6)},
            "e2e": {"value": B / e2e_s, "unit": "particles/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            # the box-128 workload takes the fused path: k_noise_fused + k_prep_fused per call
            "gpu_launches": 2 * args.steps, "clocks": clk.summary(),
            "roofline": {"bound": "hbm", "kernel": "the preparation pass (k_noise_fused, k_prep_fused)",
                         "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": src, "traffic": None,
                         "bytes_per_particle": per}}
    if not args.no_cpu_baseline:
        import imageprep_oracle as ipo
        ocfg = dict(cfg, sigma2_noise=sig, do_norm_correction=0, avg_norm_correction=1.0, remap_noise=1.0,
                    remap_minv=1.0, do_ctf_correction=1, ctf_premultiplied=0, ctf_phase_flipped=0,
                    only_flip_phases=0, intact_ctf_first_peak=0)
        t0, k = time.perf_counter(), 0
        while time.perf_counter() - t0 < min(args.ref_seconds, 10.0):
            ipo.prepare(imgs[k:k + 8].astype(np.float64), par[k:k + 8], pid[k:k + 8], ocfg)
            k += 8
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": k / dt, "unit": "particles/s", "cores": 1, "kind": "port",
                                "sample": f"{k} particles through the FP64 numpy oracle"}
    print(json.dumps(line), flush=True)
    es.close()


def run_recon(args):
    """M-step reconstruction of the box-128 workload's backprojection grid (pad_size 259,
    r_max 64, pad 2): t2b_reconstruct (skip-gridding division with the MAP term, 256^3
    inverse FFT, window, mask, gridding correction), the half-map FSC and the SSNR arrays.
    A step is one map; the grid is filled by one E-step of 128 particles first."""
    import torch
    t2b = load_package()
    import t2relion_b200.synthetic as sy
    B = args.batch
    fmap, samp, parts = build_problem(t2b, sy, B, WORKLOAD["seed"])
    es = setup_context(t2b, sy, fmap, samp, t2b.DIFF2_SPLIT_BF16, B, device=0)
    es.expectation(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"])
    ori = WORKLOAD["ori_size"]
    nb = ori // 2 + 1
    _, w = es.get_backprojector(0)
    tau2 = np.full(nb, float(np.mean(w)))
    for _ in range(max(args.warmup, 3)):
        es.reconstruct(0, ori, tau2=tau2, tau2_fudge=1.0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vol = es.reconstruct(0, ori, tau2=tau2, tau2_fudge=1.0)
    rec_s = (time.perf_counter() - t0) / args.steps
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fsc = es.fsc_halves(0, 0, ori)        # same cost as two half-set grids
        es.update_ssnr(0, ori, tau2, tau2_fudge=1.0, fsc=fsc)
    ssnr_s = (time.perf_counter() - t0) / args.steps

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(n):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t) / n * 1e3

    # the gridding iterations (--dont_skip_gridding, 10 iterations as the reference's default)
    grid_ms = timed(lambda: es.reconstruct(0, ori, tau2=tau2, tau2_fudge=1.0, gridding_iter=10), args.steps)
    # symmetrisation, in place (the sums grow with every call; timed last, few calls)
    sym_ms = {"hermitian": timed(lambda: es.enforce_hermitian_symmetry(0), 3),
              "helical_5_units": timed(lambda: es.apply_helical_symmetry(0, 5, -35.3, 4.7, ori), 3),
              "point_group_D7": timed(lambda: es.apply_point_group_symmetry(0, "D7"), 3),
              "point_group_I": timed(lambda: es.apply_point_group_symmetry(0, "I"), 3)}
    line = {"metric": "M-step reconstruction maps/s box128 (pad_size 259 -> 256^3 inverse FFT -> 128^3 map)",
            "value": 1.0 / rec_s, "unit": "maps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": rec_s * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (division, sums) / f32 (inverse FFT)", "data": "synthetic",
            "config": {"workload": "recon_box128_rmax64_pad2", "grid": [259, 259, 130],
                       "fsc_plus_ssnr_ms": ssnr_s * 1e3,
                       "gridding_10_iterations_ms": grid_ms,
                       "symmetrise_ms": sym_ms,
                       "timing": "host wall clock around the host entry point (the grid stays on the device; "
                                 "the 16.8 MB map is copied out; symmetrisation allocates and frees its "
                                 "104 MB of scratch per call)"},
            "map_rms": float(np.sqrt(np.mean(vol ** 2)))}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import recon_oracle as ro
        data, w = es.get_backprojector(0)
        t0 = time.perf_counter()
        ro.reconstruct_map(data.astype(np.complex128), w.astype(np.float64), WORKLOAD["bp_r_max"], 2, ori,
                           tau2=tau2, tau2_fudge=1.0)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "maps/s", "cores": 1, "kind": "port",
                                "sample": "one map through the FP64 numpy oracle"}
        t0 = time.perf_counter()
        ro.apply_point_group_symmetry(data, w, ro.point_group("C2"), WORKLOAD["bp_r_max"], 2)
        line["cpu_baseline"]["symmetrise_ms_per_operator"] = (time.perf_counter() - t0) * 1e3
    print(json.dumps(line), flush=True)
    es.close()


# 2D classification: K = 50 seeded blob references of 100 x 100 at 2 A/px, 20,000 particles drawn
# from them (in-plane rotation, shifts U(-5, 5) px, SNR 0.05); psi step 6 deg, translations range
# 5 step 1, adaptive oversampling 1 (2 psi x 4 shifts per significant pair), window to Nyquist
CLASS2D = dict(name="class2d_k50_box100_psi6_ovs1", ori_size=100, angpix=2.0, n_blobs=12, n_classes=50,
               map_seed=31, psi_step=6.0, offset_range=5, offset_step=1, r_max=50, snr=0.05, seed=57,
               n_particles=20000, batch=500)
METRIC_CLASS2D = "E-step particles/s 2D classification K=50 box100: split-BF16 vs plain FP32 GPU; roofline %"


def class2d_inputs(sy, samp_fn, n, seed, chunk=2000):
    """References, sampling and n particles of the 2D-classification workload (numpy; particles
    generated in chunks with one noise variance)."""
    w = CLASS2D
    N, r, K = w["ori_size"], w["r_max"], w["n_classes"]
    maps = [sy.fourier_map(sy.blob_volume(N, w["n_blobs"], seed=w["map_seed"] + 101 * k, ndim=2), r)
            for k in range(K)]
    samp = samp_fn()
    cls = np.random.default_rng(seed + 7).integers(0, K, n)
    out, sigma2 = [], None
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        p = sy.make_particles(maps[0], b - a, ori_size=N, s=2 * r, r_max=r, angpix=w["angpix"], snr=w["snr"],
                              seed=seed + a, max_shift=w["offset_range"], ref_dim=2, classes=cls[a:b],
                              class_maps=maps, sigma2=sigma2)
        sigma2 = p["sigma2"]
        out.append(p)
    parts = {k: np.concatenate([p[k] for p in out]) for k in ("fimg", "ctf", "minv", "scalars")}
    return maps, samp, parts, cls


def class2d_config():
    w = CLASS2D
    s = 2 * w["r_max"]
    return {"workload": w["name"], "box": w["ori_size"], "classes": w["n_classes"], "psi_step": w["psi_step"],
            "orientations_per_class": int(np.ceil(360 / w["psi_step"])), "translations": 81,
            "pixels": s * (s // 2 + 1), "adaptive_oversampling": 1, "fine_hypotheses_per_pair": 8,
            "snr": w["snr"], "particles": w["n_particles"]}


def class2d_cpu(maps, samp, parts, n, sy):
    """The FP64 oracle port's whole E-step on n particles, one per host thread: (seconds, text)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    w = CLASS2D
    K, r, s = w["n_classes"], w["r_max"], 2 * w["r_max"]
    prob = orc.Problem(ori_size=w["ori_size"], s=s, ref_dim=2, maps=maps, r_max=r, pad=2, samp=samp,
                       pdf_direction=np.ones((K, 1)), pdf_class=np.full(K, 1.0 / K),
                       sigma2_offset=(w["offset_range"] * w["angpix"]) ** 2, pixel_size=w["angpix"],
                       adaptive_fraction=0.999, ovs=1, bp_pad_size=sy.pad_size(r), bp_r_max=r)
    op = prob.particles(parts["fimg"][:n], parts["ctf"][:n], parts["minv"][:n], parts["scalars"][:n], sy.mresol(s))
    t0 = time.perf_counter()
    prob.estep(op, nthreads=n)
    t = time.perf_counter() - t0
    return t, (f"{n} particles, one per host thread, through the whole E-step of the FP64 oracle port (2D "
               f"references: the reference's CPU kernels are compiled here for 3D references only)")


def run_class2d(args, world, rank):
    w = CLASS2D
    K, N, r = w["n_classes"], w["ori_size"], w["r_max"]
    s = 2 * r
    if args.impl == "reference":
        if rank != 0:
            return
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import sampling_oracle as so
        sy = load_synthetic()
        n = os.cpu_count() or 1
        maps, samp, parts, _ = class2d_inputs(
            sy, lambda: so.sampling2d(w["psi_step"], 1, w["offset_range"], w["offset_step"], w["angpix"]), n,
            w["seed"] + 1)
        class2d_cpu(maps, samp, parts, 1, sy)
        times = [class2d_cpu(maps, samp, parts, n, sy)[0] for _ in range(args.steps)]
        v = n * args.steps / float(np.sum(times))
        text = class2d_cpu(maps, samp, parts, 1, sy)[1].replace("1 particles", f"{n} particles")
        print(json.dumps({"impl": "reference", "metric": METRIC_CLASS2D, "value": v, "unit": "particles/s",
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1000.0 * float(np.mean(times)), "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": class2d_config(), "particles_per_step": n,
                          "cpu_baseline": {"value": v, "unit": "particles/s", "cores": n, "kind": "port",
                                           "sample": text},
                          "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    t2b = load_package()
    import t2relion_b200.synthetic as sy
    torch.cuda.set_device(local_rank())
    dev = torch.device("cuda", local_rank())
    B = w["batch"]
    n_all = w["n_particles"]
    maps, samp, parts, cls = class2d_inputs(
        sy, lambda: t2b.sampling(2, 0, w["psi_step"], 1, w["offset_range"], w["offset_step"], w["angpix"]), n_all,
        w["seed"] + 1000 * rank)
    ps = sy.pad_size(r)

    def context(mode):
        es = t2b.EStep(local_rank())
        for k in range(K):
            es.set_projector(k, maps[k], 2, r, 2)
            es.init_backprojector(k, 2, ps, r, 2)
        es.configure(ori_size=N, current_size=s, ref_dim=2, nr_classes=K, samp=samp, pdf_direction=np.ones((K, 1)),
                     pdf_class=np.full(K, 1.0 / K), sigma2_offset=(w["offset_range"] * w["angpix"]) ** 2,
                     pixel_size=w["angpix"], adaptive_oversampling=1, diff2_mode=mode, max_batch=B)
        return es

    es = context(t2b.DIFF2_SPLIT_BF16)
    first = {k: v[:B] for k, v in parts.items()}
    t0 = time.perf_counter()
    rep = es.autotune(first["fimg"], first["ctf"], first["minv"], first["scalars"])
    tuned = {k: rep[k] for k in ("diff2_tn", "diff2_group", "fine_ctas_per_sm", "wsum_ctas_per_sm",
                                 "project_pixels", "project_orients")}
    tune_s = time.perf_counter() - t0
    # the whole dataset resident in HBM; each step copies its batch into the entry point's
    # fixed input buffers (device to device) and runs the E-step on them
    alld = {"fimg": torch.from_numpy(parts["fimg"].view(np.float32)).to(dev),
            "ctf": torch.from_numpy(parts["ctf"]).to(dev), "minv": torch.from_numpy(parts["minv"]).to(dev),
            "scal": torch.from_numpy(parts["scalars"]).to(dev)}
    stage = {k: v[:B].clone() for k, v in alld.items()}
    half = N // 2 + 1

    def device_pass(e, steps):
        res = result_tensors(B, K, 1, dev, half)
        rptr = {k: ctypes.c_void_p(v.data_ptr()) for k, v in res.items()}
        stream = torch.cuda.Stream(dev)
        poses = []

        def step(i):
            a = (i * B) % n_all
            with torch.cuda.stream(stream):
                for k in stage:
                    stage[k].copy_(alld[k][a:a + B], non_blocking=True)
            e.expectation_device(B, ctypes.c_void_p(stage["fimg"].data_ptr()), ctypes.c_void_p(stage["ctf"].data_ptr()),
                                 ctypes.c_void_p(stage["minv"].data_ptr()), ctypes.c_void_p(stage["scal"].data_ptr()),
                                 rptr, stream=stream.cuda_stream)
        for i in range(3):
            step(i)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local_rank()) as clk:
            ev0.record(stream)
            for i in range(steps):
                step(i)
            ev1.record(stream)
            torch.cuda.synchronize()
        if int(res["status"].ne(0).sum()) != 0:
            raise RuntimeError("E-step status errors")
        ms = ev0.elapsed_time(ev1)
        return B * steps / (ms / 1000.0), ms / steps, clk.summary(), e.launch_count()

    steps = n_all // B
    value, ms_step, clocks, launches = device_pass(es, steps)
    # per-stage device times of host-path steps (coarse contraction = stage 2)
    es.stage_timing(True)
    st = []
    for i in range(3):
        a = i * B
        es.expectation(*[parts[k][a:a + B] for k in ("fimg", "ctf", "minv", "scalars")])
        st.append(es.stage_ms())
    es.stage_timing(False)
    stages = np.mean(np.array(st), axis=0)
    # end to end: host entry points over the dataset's batches (pinned)
    pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in
           [("fimg", parts["fimg"].view(np.float32)), ("ctf", parts["ctf"]), ("minv", parts["minv"]),
            ("scal", parts["scalars"])]}
    hres = [{k: v.pin_memory() for k, v in result_tensors(B, K, 1, "cpu", half).items()} for _ in range(2)]
    P = s * (s // 2 + 1)

    def host_batch(i):
        a = (i * B) % n_all
        b = t2b.Batch(B, 0, ctypes.c_void_p(pin["fimg"][a:a + B].data_ptr()), None,
                      ctypes.c_void_p(pin["ctf"][a:a + B].data_ptr()), ctypes.c_void_p(pin["minv"][a:a + B].data_ptr()),
                      ctypes.c_void_p(pin["scal"][a:a + B].data_ptr()))
        h = hres[i & 1]
        res = t2b.Result(*[ctypes.c_void_p(h[n].data_ptr()) if n in h else None for n, _ in t2b.Result._fields_])
        return b, res
    ticket = ctypes.c_longlong(-1)
    keep = []
    t0 = time.perf_counter()
    prev = None
    for i in range(steps):
        b, res = host_batch(i)
        keep.append((b, res))
        t2b._check(t2b.lib.t2b_estep_submit_host(es._h, ctypes.byref(b), ctypes.byref(res), ctypes.byref(ticket)))
        if prev is not None:
            t2b._check(t2b.lib.t2b_estep_wait(es._h, prev))
        prev = ticket.value
    t2b._check(t2b.lib.t2b_estep_wait(es._h, prev))
    e2e_s = time.perf_counter() - t0
    h2d = B * (P * 8 + P * 4 + P * 4 + 8 * 8)
    d2h = sum(v.numel() * v.element_size() for v in hres[0].values())
    # the plain FP32 comparator on the first PLAIN_STEPS batches, and the poses of both passes there
    es_p = context(t2b.DIFF2_PLAIN_FP32)
    es_p.tune_set(**tuned)
    pv, pms, pclk, _ = device_pass(es_p, PLAIN_STEPS)
    same, n_cmp = 0, 0
    for i in range(PLAIN_STEPS):
        a = i * B
        args_ = [parts[k][a:a + B] for k in ("fimg", "ctf", "minv", "scalars")]
        ra, rb = es.expectation(*args_), es_p.expectation(*args_)
        same += int(np.all(ra["pose"] == rb["pose"], axis=1).sum())
        n_cmp += B
        if i == 0:
            nsig = ra["nr_sign"]
            cls_ok = float(np.mean(ra["pose"][:, 0] == cls[a:a + B]))
    es_p.close()
    peaks, src = measured_peaks()
    at_max = bool(clocks.get("sm_mhz") and clocks.get("sm_max_mhz") and clocks["sm_mhz"] >= 0.97 * clocks["sm_max_mhz"]
                  and "sw_power_cap" not in clocks["reasons"])
    peak = peaks.get("bf16_tflops", 1590.0) if at_max else peaks.get("bf16_tflops_sustained", 1400.0)
    O, T = samp["n_psi"], samp["n_trans"]
    flops = 8.0 * K * O * T * P * B
    achieved = flops / (float(stages[2]) / 1000.0) / 1e12
    line = {"metric": METRIC_CLASS2D, "value": value, "unit": "particles/s", "n_gpus": world,
            "steps": steps, "warmup": 3, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / pv,
            "vs_baseline_definition": "value / plain.value: the plain FP32 GPU path timed in this run",
            "dtype": "f32+bf16x3/f64", "data": "synthetic (seeded blob references, CTF, white noise)",
            "config": class2d_config(), "particles_per_step": B,
            "run": {"diff2": "splitbf16", "tile_shapes": dict(tuned, tune_s=tune_s),
                    "l2": "inputs: 20,000 distinct particles (1.6 GB) resident, one pass"},
            "e2e": {"value": B * steps / e2e_s, "unit": "particles/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "api": "t2b_estep_submit_host + t2b_estep_wait over the dataset"},
            "gpu_launches": launches * steps if launches > 0 else None, "clocks": clocks,
            "plain": {"value": pv, "ms_per_step": pms, "steps": PLAIN_STEPS, "clocks": pclk},
            "quality_vs_plain": {"particles": n_cmp, "pose_agreement": same / n_cmp,
                                 "true_class_fraction": cls_ok},
            "nr_sign": {"min": int(nsig.min()), "median": float(np.median(nsig)), "max": int(nsig.max())},
            "roofline": {"bound": "tensor", "kernel": "k_diff2_tc", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "peak_source": src, "traffic": None,
                         "flops_per_launch": flops},
            "stage_ms": {n: float(v) for n, v in zip(
                ["prep_network", "operands_audit_norms", "coarse_diff2", "coarse_weights", "fine", "fine_weights",
                 "wsum_bp", "audit_contraction", "proposal_contraction"], stages)}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n = os.cpu_count() or 1
        t, text = class2d_cpu(maps, samp, parts, n, sy)
        line["cpu_baseline"] = {"value": n / t, "unit": "particles/s", "cores": n, "kind": "port", "sample": text}
    if rank == 0:
        print(json.dumps(line), flush=True)
    es.close()


# Large 3D classification: K = 4 maps of 256^3 at 0.85 A/px differing by 10 % of their blobs,
# particles 256 x 256 at SNR 0.02, defocus U(0.8, 2.5) um; HEALPix order 4 x psi 3.75 deg,
# adaptive oversampling 1, translations range 4 step 1, Fourier radius 100, 515^3 grids.
LARGE3D = dict(name="class3d_k4_box256_order4_ovs1", ori_size=256, angpix=0.85, n_blobs=40, n_classes=4,
               map_seed=5, order=4, psi_step=3.75, offset_range=4, offset_step=1, r_max=100, bp_r_max=128,
               snr=0.02, defocus=(8000., 25000.), seed=73, batch=256)
METRIC_LARGE3D = "E-step particles/s 3D classification K=4 box256 order4 (chunked split-BF16); roofline %"


def large3d_inputs(sy, samp_fn, n, seed):
    w = LARGE3D
    K, N, r = w["n_classes"], w["ori_size"], w["r_max"]
    maps = [sy.fourier_map(v, r) for v in sy.blob_class_volumes(N, K, w["n_blobs"], seed=w["map_seed"])]
    samp = samp_fn()
    cls = np.arange(n) % K
    parts = sy.make_particles(maps[0], n, ori_size=N, s=2 * r, r_max=r, angpix=w["angpix"], snr=w["snr"], seed=seed,
                              max_shift=w["offset_range"], defocus=w["defocus"], classes=cls, class_maps=maps)
    return maps, samp, parts, cls


def large3d_config():
    w = LARGE3D
    s = 2 * w["r_max"]
    return {"workload": w["name"], "box": w["ori_size"], "classes": w["n_classes"], "healpix_order": w["order"],
            "psi_step": w["psi_step"], "orientations": w["n_classes"] * 12 * 4 ** w["order"] * int(360 / w["psi_step"]),
            "translations": 49, "pixels": s * (s // 2 + 1), "adaptive_oversampling": 1, "fine_hypotheses_per_pair": 32,
            "snr": w["snr"], "grid": [515, 515, 258]}


def large3d_cpu(maps, samp, parts, n, n_dir_slice=16):
    """The reference's CPU coarse kernel (CpuKernels::diff2_coarse, oracle/_ref) on a bounded
    sample: one particle per host thread over the first n_dir_slice directions x all psi of
    class 0, extrapolated to every class and orientation (the coarse pass is > 95 % of the
    CPU E-step).  Returns (particles/s, text) or None without the library."""
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libacc_ref.so")
    if not os.path.exists(lib_path):
        return None
    w = LARGE3D
    lib = ctypes.CDLL(lib_path)
    lib.ref_coarse_diff2.restype = ctypes.c_int
    N, r, s, K = w["ori_size"], w["r_max"], 2 * w["r_max"], w["n_classes"]
    fm = np.ascontiguousarray(maps[0].view(np.float32))
    mz, my, mx = maps[0].shape
    no = n_dir_slice * samp["n_psi"]
    eul = samp["eul_coarse"][:no].reshape(-1, 3, 3)
    einv = np.ascontiguousarray(np.transpose(eul, (0, 2, 1)).reshape(-1, 9), np.float32)
    tx = np.ascontiguousarray(-2 * np.pi * samp["trans_px"][:, 0] / N, np.float32)
    ty = np.ascontiguousarray(-2 * np.pi * samp["trans_px"][:, 1] / N, np.float32)
    T = len(tx)

    def one(b):
        ctf = parts["ctf"][b].astype(np.float64)
        X = parts["fimg"][b].astype(np.complex128) / ctf
        re, im = np.ascontiguousarray(X.real, np.float32), np.ascontiguousarray(X.imag, np.float32)
        corr = np.ascontiguousarray(parts["minv"][b] * ctf * ctf, np.float32)
        out = np.empty((no, T), np.float32)
        lib.ref_coarse_diff2(ctypes.c_void_p(fm.ctypes.data), mx, my, mz, -(my // 2), -(mz // 2), r, 2,
                             ctypes.c_void_p(einv.ctypes.data), no, ctypes.c_void_p(re.ctypes.data),
                             ctypes.c_void_p(im.ctypes.data), ctypes.c_void_p(corr.ctypes.data), s // 2 + 1, s,
                             ctypes.c_void_p(tx.ctypes.data), ctypes.c_void_p(ty.ctypes.data), T,
                             ctypes.c_float(parts["scalars"][b, 1] / 2), ctypes.c_void_p(out.ctypes.data))
    t0 = time.perf_counter()
    ths = [threading.Thread(target=one, args=(b,)) for b in range(n)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    t = time.perf_counter() - t0
    total = K * samp["n_dir"] * samp["n_psi"]
    return n * (no / total) / t, (f"{n} particles, one per host thread, through the reference's "
                                  f"CpuKernels::diff2_coarse over {no} of {total} class-orientations x {T} "
                                  f"translations ({t:.1f} s), extrapolated to all of them")


def run_large3d(args, world, rank):
    w = LARGE3D
    K = w["n_classes"]
    if args.impl == "reference":
        if rank != 0:
            return
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import sampling_oracle as so
        sy = load_synthetic()
        n = os.cpu_count() or 1
        maps, samp, parts, _ = large3d_inputs(
            sy, lambda: so.sampling(w["order"], w["psi_step"], 0, w["offset_range"], w["offset_step"], w["angpix"]),
            n, w["seed"] + 1)
        vals = [large3d_cpu(maps, samp, parts, n) for _ in range(args.steps)]
        v = float(np.median([x[0] for x in vals]))
        print(json.dumps({"impl": "reference", "metric": METRIC_LARGE3D, "value": v, "unit": "particles/s",
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1000.0 * n / v, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": large3d_config(),
                          "particles_per_step": n,
                          "cpu_baseline": {"value": v, "unit": "particles/s", "cores": n, "kind": "reference",
                                           "sample": vals[-1][1]},
                          "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    t2b = load_package()
    import t2relion_b200.synthetic as sy
    torch.cuda.set_device(local_rank())
    dev = torch.device("cuda", local_rank())
    if args.profile_case:
        # reduced case for ncu captures: HEALPix order 2 (73,728 class-orientations, 5 chunks),
        # 8 particles per step; not a bench number
        w = dict(LARGE3D, name=LARGE3D["name"] + "_profile_order2", order=2, batch=8)
        LARGE3D.update(w)
    B = args.batch if args.batch_given else w["batch"]
    steps = args.steps if args.steps_given else 4
    n_all = B * steps
    t0 = time.perf_counter()
    maps, samp, parts, cls = large3d_inputs(
        sy, lambda: t2b.sampling(3, w["order"], w["psi_step"], 1, w["offset_range"], w["offset_step"], w["angpix"]),
        n_all, w["seed"] + 1000 * rank)
    gen_s = time.perf_counter() - t0
    N, r, s = w["ori_size"], w["r_max"], 2 * w["r_max"]
    ps = sy.pad_size(w["bp_r_max"])
    es = t2b.EStep(local_rank())
    for k in range(K):
        es.set_projector(k, maps[k], 3, r, 2)
        es.init_backprojector(k, 3, ps, w["bp_r_max"], 2)
    t0 = time.perf_counter()
    es.configure(ori_size=N, current_size=s, ref_dim=3, nr_classes=K, samp=samp,
                 pdf_direction=np.full((K, samp["n_dir"]), 1.0 / samp["n_dir"]), pdf_class=np.full(K, 1.0 / K),
                 sigma2_offset=(w["offset_range"] * w["angpix"]) ** 2, pixel_size=w["angpix"],
                 adaptive_oversampling=1, diff2_mode=t2b.DIFF2_SPLIT_BF16, max_batch=B,
                 use_graph=0 if args.no_graph else 1)
    conf_s = time.perf_counter() - t0
    alld = {"fimg": torch.from_numpy(parts["fimg"].view(np.float32)).to(dev),
            "ctf": torch.from_numpy(parts["ctf"]).to(dev), "minv": torch.from_numpy(parts["minv"]).to(dev),
            "scal": torch.from_numpy(parts["scalars"]).to(dev)}
    stage = {k: v[:B].clone() for k, v in alld.items()}
    res = result_tensors(B, K, samp["n_dir"], dev, N // 2 + 1)
    rptr = {k: ctypes.c_void_p(v.data_ptr()) for k, v in res.items()}
    stream = torch.cuda.Stream(dev)
    poses = []

    def step(i):
        a = (i % steps) * B
        with torch.cuda.stream(stream):
            for k in stage:
                stage[k].copy_(alld[k][a:a + B], non_blocking=True)
        es.expectation_device(B, ctypes.c_void_p(stage["fimg"].data_ptr()), ctypes.c_void_p(stage["ctf"].data_ptr()),
                              ctypes.c_void_p(stage["minv"].data_ptr()), ctypes.c_void_p(stage["scal"].data_ptr()),
                              rptr, stream=stream.cuda_stream)
    for i in range(max(args.warmup, 3)):
        step(i)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank()) as clk:
        torch.cuda.nvtx.range_push("timed_steps")   # lets a profiler select the timed launches
        ev0.record(stream)
        for i in range(steps):
            step(i)
        ev1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = ev0.elapsed_time(ev1)
    if int(res["status"].ne(0).sum()) != 0:
        raise RuntimeError("E-step status errors")
    value = B * steps / (ms / 1000.0)
    # poses of every particle against the simulated truth (host entry point, outside the timed region)
    R = samp["nover_rot"]
    O = samp["n_dir"] * samp["n_psi"]
    good_cls, errs = 0, []
    es.stage_timing(True)
    st = []
    for i in range(steps):
        a = i * B
        got = es.expectation(*[parts[k][a:a + B] for k in ("fimg", "ctf", "minv", "scalars")])
        st.append(es.stage_ms())
        for j in range(B):
            k, o, rr = got["pose"][j][:3]
            good_cls += int(k == cls[a + j])
            Af = samp["eul_fine"][o * R + rr].reshape(3, 3)
            c = (np.trace(Af @ parts["A"][a + j].T) - 1) / 2
            errs.append(float(np.degrees(np.arccos(np.clip(c, -1, 1)))))
    es.stage_timing(False)
    stages = np.mean(np.array(st), axis=0)
    peaks, src = measured_peaks()
    at_max = bool(clk.summary().get("sm_mhz") and clk.summary()["sm_mhz"] >= 0.97 * (clk.summary()["sm_max_mhz"] or 1e9)
                  and "sw_power_cap" not in clk.summary()["reasons"])
    peak = peaks.get("bf16_tflops", 1590.0) if at_max else peaks.get("bf16_tflops_sustained", 1400.0)
    P = s * (s // 2 + 1)
    T = samp["n_trans"]
    flops = 8.0 * K * O * T * P * B
    achieved = flops / (float(stages[2]) / 1000.0) / 1e12
    line = {"metric": METRIC_LARGE3D, "value": value, "unit": "particles/s", "n_gpus": world, "steps": steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+bf16x3/f64",
            "data": "synthetic (seeded blob maps, CTF, white noise; stands in for the reference's datasets)",
            "config": large3d_config(), "particles_per_step": B,
            "run": {"diff2": "splitbf16, chunked coarse pass (projection tables would need 190 GB coarse + "
                             "1.5 TB fine)", "input_gen_s": gen_s, "configure_s": conf_s,
                    "l2": "inputs and model larger than L2; %d distinct particles" % n_all},
            "gpu_launches": es.launch_count() * steps if es.launch_count() > 0 else None,
            "clocks": clk.summary(),
            "quality_vs_truth": {"particles": len(errs), "class_fraction": good_cls / len(errs),
                                 "orientation_error_deg_median": float(np.median(errs)),
                                 "within_5deg_fraction": float(np.mean(np.array(errs) < 5.0))},
            "roofline": {"bound": "tensor", "kernel": "k_diff2_tc (chunked, with the per-chunk projection)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": src, "traffic": None, "flops_per_launch": flops},
            "stage_ms": {n: float(v) for n, v in zip(
                ["prep_network", "operands_audit_norms", "coarse_diff2", "coarse_weights", "fine", "fine_weights",
                 "wsum_bp", "audit_contraction", "proposal_contraction"], stages)}}
    # end to end through the host entry point, the same steps
    t0 = time.perf_counter()
    for i in range(steps):
        a = i * B
        es.expectation(*[parts[k][a:a + B] for k in ("fimg", "ctf", "minv", "scalars")])
    e2e_s = time.perf_counter() - t0
    P8 = P * 16 + 64
    line["e2e"] = {"value": B * steps / e2e_s, "unit": "particles/s", "h2d_bytes_per_step": B * P8,
                   "d2h_bytes_per_step": sum(v.numel() * v.element_size() for v in res.values()),
                   "api": "t2b_estep_batch_host (blocking), host arrays"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = large3d_cpu(maps, samp, parts, min(os.cpu_count() or 1, n_all))
        if cb:
            line["cpu_baseline"] = {"value": cb[0], "unit": "particles/s", "cores": min(os.cpu_count() or 1, n_all),
                                    "kind": "reference", "sample": cb[1]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    es.close()


def local_rank():
    return int(os.environ.get("LOCAL_RANK", "0"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # 25 steps of 512 particles are whole periods of the audit pattern (every 50th particle:
    # 256 audited in 12,800), so the timed steps hold the average mix of 10- and 11-particle audits
    ap.add_argument("--steps", type=int, default=25)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="learned", choices=["learned", "splitbf16", "plain"],
                    help="learned: proposal network + split-BF16 tensor-core contraction (the headline); "
                         "splitbf16: full coarse pass on tcgen05; plain: full coarse pass, FP32 SIMT")
    ap.add_argument("--topk", type=int, default=PROP["topk"], help="learned: proposals per particle")
    ap.add_argument("--rescore", type=int, default=PROP["rescore"], help="learned: network candidates rescored")
    ap.add_argument("--train-particles", type=int, default=200000)
    ap.add_argument("--train-epochs", type=int, default=8)
    # particles per step: the audit streams the whole projection operand once per step, so a
    # larger batch spreads it over more audited particles (128: 110.6k, 256: 93.6k with one
    # fallback step, 512: 150.6k, 768: 158.0k, 1024: 108.4k with one fallback step, particles/s
    # on one box); 512 keeps a fallback step -- the whole batch re-run on the full coarse
    # pass when an audited particle's proposals miss posterior mass -- affordable
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP32 comparator and quality check")
    ap.add_argument("--ref-seconds", type=float, default=15.0)
    ap.add_argument("--profile-case", action="store_true",
                    help="HEALPix order 2 instead of 3 (for ncu captures; not a bench number)")
    ap.add_argument("--stage", default="estep", choices=["estep", "prep", "recon"],
                    help="estep: the E-step (the headline); prep: the image preparation before it "
                         "(real-space particles -> E-step inputs), its own JSON line")
    ap.add_argument("--prep-batch", type=int, default=1024, help="prep: particles per call")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default tile shapes")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch each step's kernels one by one instead of replaying its CUDA graph (ncu cannot "
                         "profile the kernel nodes of a graph with conditional nodes; not a bench number)")
    ap.add_argument("--workload", default="box128", choices=["box128", "class2d", "class3d_large"],
                    help="box128: the 3D refinement headline; class2d: 2D classification, K = 50 references of "
                         "100 x 100, 20,000 particles (its own JSON line)")
    args = ap.parse_args()
    args.steps_given = any(a == "--steps" or a.startswith("--steps=") for a in sys.argv[1:])
    args.batch_given = any(a == "--batch" or a.startswith("--batch=") for a in sys.argv[1:])
    if args.workload == "class3d_large":
        world, rank, _ = dist_init()
        run_large3d(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "class2d":
        world, rank, _ = dist_init()
        run_class2d(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.stage == "prep":
        run_prep(args)
        return
    if args.stage == "recon":
        run_recon(args)
        return
    if args.profile_case:
        WORKLOAD.update(PROFILE_WORKLOAD)
    PROP.update(topk=args.topk, rescore=args.rescore)
    world, rank, local = dist_init()
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    t2b = load_package()
    import t2relion_b200.synthetic as sy
    torch.cuda.set_device(local)
    B = args.batch
    fmap, samp, parts = build_problem(t2b, sy, B, WORKLOAD["seed"] + 1000 * rank)
    mode = t2b.DIFF2_PLAIN_FP32 if args.mode == "plain" else t2b.DIFF2_SPLIT_BF16
    es = setup_context(t2b, sy, fmap, samp, mode, B, device=local, use_graph=0 if args.no_graph else 1)
    tuned = None
    if not args.no_autotune:
        # once per configuration, before the timed region: the library's tile-shape autotuner
        # times its candidate shapes on this batch and keeps the fastest (no value changes)
        t0 = time.perf_counter()
        rep = es.autotune(parts["fimg"], parts["ctf"], parts["minv"], parts["scalars"])
        tuned = {k: rep[k] for k in ("diff2_tn", "diff2_group", "fine_ctas_per_sm", "wsum_ctas_per_sm",
                                     "project_pixels", "project_orients")}
        tuned["tune_s"] = time.perf_counter() - t0
        tuned["coarse_diff2_ms"] = rep["diff2_ms"]
        tuned["fine_ms"] = rep["fine_ms"]     # per CTAs-per-SM build, 1..4
        tuned["wsum_ms"] = rep["wsum_ms"]
    learned = None
    if args.mode == "learned":
        # once per iteration, before the E-step: train the proposal network on particles
        # generated from the current reference (outside the timed region; reported)
        t0 = time.perf_counter()
        rep = es.train_proposals(parts["minv"][0], n_train=args.train_particles, n_posterior=8192, n_val=1024,
                                 epochs=args.train_epochs, batch=256, lr=3e-4, topk=PROP["topk"],
                                 rescore=PROP["rescore"], seed=WORKLOAD["seed"], max_shift=WORKLOAD["offset_range"],
                                 sigma_deg=5.0)
        learned = {"train_s": time.perf_counter() - t0, "train_particles": args.train_particles,
                   "train_epochs": args.train_epochs, "val_mass_init": rep["val_mass_init"],
                   "val_mass_network": rep["val_mass_trained"], "val_mass_rescored": rep["val_mass_rescored"],
                   "val_frac_999_rescored": rep["val_frac_999_rescored"],
                   "val_frac_999_candidates": rep["val_frac_999_candidates"], "final_loss": rep["loss"][-1],
                   **PROP}
        es.enable_proposals(topk=PROP["topk"], rescore=PROP["rescore"], audit_every=PROP["audit_every"],
                            audit_mass=PROP["audit_mass"])
    timing = time_device(es, parts, B, args.steps, args.warmup, local, world, t2b)
    e2e, pin, hres = time_e2e(es, parts, B, args.steps, world, t2b)
    # per-stage device times (CUDA events around each stage) of separately synchronised
    # host-path steps; not part of `value`
    # (one period of the audit pattern when learned: each step's audited count is kept)
    lib = t2b.lib
    batch = t2b.Batch(B, 0, ctypes.c_void_p(pin["fimg"].data_ptr()), None, ctypes.c_void_p(pin["ctf"].data_ptr()),
                      ctypes.c_void_p(pin["minv"].data_ptr()), ctypes.c_void_p(pin["scal"].data_ptr()))
    result = t2b.Result(*[ctypes.c_void_p(hres[n].data_ptr()) if n in hres else None for n, _ in t2b.Result._fields_])
    stage_steps, audited = [], []
    es.stage_timing(True)
    for _ in range(min(25, args.steps)):
        t2b._check(lib.t2b_estep_batch_host(es._h, ctypes.byref(batch), ctypes.byref(result)))
        stage_steps.append(es.stage_ms())
        audited.append(int((hres["audit_mass"].numpy() >= 0).sum()))
    es.stage_timing(False)
    stage_steps = np.array(stage_steps)
    stages = np.mean(stage_steps, axis=0)
    clocks = timing["clocks"]
    value = timing["value"]

    # roofline of the dominant kernel (the tcgen05 contraction k_diff2_tc)
    O, T = samp["n_dir"] * samp["n_psi"], samp["n_trans"]
    P = parts["fimg"].shape[1]
    s = 2 * WORKLOAD["r_max"]
    K = 1
    peaks, src = measured_peaks()
    # the burst tensor peak when the timed region ran at the maximum SM clock (no power cap
    # bit it), the sustained one otherwise
    at_max = bool(clocks.get("sm_mhz") and clocks.get("sm_max_mhz")
                  and clocks["sm_mhz"] >= 0.97 * clocks["sm_max_mhz"] and "sw_power_cap" not in clocks["reasons"])
    tensor_peak = peaks.get("bf16_tflops", 1590.0) if at_max else peaks.get("bf16_tflops_sustained", 1400.0)
    peak_kind = "burst (timed region at the maximum SM clock)" if at_max else "sustained"
    traffic_ok = kernel_sha() == TRAFFIC["kernel_sha"] and not args.profile_case
    # the contraction runs over the nk window pixels inside the projection radius only
    # (projections are zero outside); "executed" counts what the tensor cores did
    nk = int(sum(1 for n in range(P) if (lambda i, x: x * x + (i if i < s // 2 + 1 else i - s) ** 2)(n // (s // 2 + 1), n % (s // 2 + 1)) <= (s // 2) ** 2))
    kdim = (2 * nk + 63) // 64 * 64
    if learned is None:
        flops = 8.0 * K * O * T * P * B
        gemm = float(stages[2])
        if mode == t2b.DIFF2_SPLIT_BF16:
            peak = tensor_peak
            bound = "tensor"
        else:
            peak = 148 * 128 * 2 * 1.965e-3  # FP32 SIMT nominal TFLOP/s (no measured figure)
            bound = "fp32_simt"
            src, peak_kind = "nominal", "FP32 FMA nominal"
        achieved = flops / (gemm / 1000.0) / 1e12
        executed = (12.0 if mode == t2b.DIFF2_SPLIT_BF16 else 4.0) * K * O * T * nk * B / (gemm / 1000.0) / 1e12
        traffic = None   # no capture of the dense pass of this kernel source
        roof = {"bound": bound, "kernel": "k_diff2_tc" if mode else "k_diff2_simt", "achieved": achieved,
                "executed_tflops": executed, "contraction_pixels": nk,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "peak_source": src, "peak_kind": peak_kind,
                "traffic": traffic, "flops_per_launch": flops}
    else:
        # learned: the audit's full coarse contraction (audited particles x every orientation)
        # and the contraction on the proposals (every particle x its top-k), each one launch of
        # k_diff2_tc per step, timed by the library's CUDA events around exactly those launches
        # over the stage-timed steps, each with its own audited count
        t_audit, t_prop = float(stages[7]), float(stages[8])
        t_sum = float(np.sum(stage_steps[:, 7] + stage_steps[:, 8])) / 1000.0
        f_prop = 8.0 * PROP["topk"] * T * P * B
        f_sum = sum(8.0 * K * O * T * P * na + f_prop for na in audited)
        # audit launch: 128-row tiles over every orientation; na_max slots of T columns in the
        # fewest 256-wide column tiles, each narrowed to a multiple of 32, or the (na_max - 1)-slot
        # variant when fewer were audited and its tiles cover fewer columns
        na_max = int(np.ceil(B / PROP["audit_every"]))

        def audit_shape(cols):
            nt = (cols + 255) // 256
            return nt, ((cols + nt - 1) // nt + 31) // 32 * 32
        full = audit_shape(na_max * T)
        narrow = audit_shape((na_max - 1) * T) if na_max > 1 else full
        tile_flops = 128 * kdim * 2 * 3.0

        def audit_tiles(na):
            if na == 0:
                return 0.0
            nt, tn = narrow if (na < na_max and narrow[0] * narrow[1] < full[0] * full[1]) else full
            return ((K * O + 127) // 128) * nt * tn
        # proposal tiles: 128 rows of 128 / kslot particles x T phase rows padded to 32 columns
        ppt = 2 if PROP["topk"] <= 64 else 1
        prop_exec = ((B + ppt - 1) // ppt) * 128 * ((T + 31) // 32 * 32) * kdim * 2 * 3.0
        executed = sum(audit_tiles(na) * tile_flops + prop_exec for na in audited) / t_sum / 1e12
        achieved = f_sum / t_sum / 1e12
        na = float(np.mean(audited))
        roof = {"bound": "tensor", "kernel": "k_diff2_tc (audit + proposal launches)", "achieved": achieved,
                "executed_tflops": executed, "contraction_pixels": nk, "peak": tensor_peak, "unit": "TFLOP/s",
                "frac": achieved / tensor_peak, "peak_source": src, "peak_kind": peak_kind,
                "traffic": TRAFFIC["learned"] if (traffic_ok and B == TRAFFIC["learned_batch"]) else None,
                "flops_per_launch": f_sum / (2.0 * len(audited)), "audit_ms": t_audit, "proposal_ms": t_prop,
                "audited_particles": na}
    roof["traffic_capture"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of this kernel source (sha256 "
                               f"{TRAFFIC['kernel_sha']})" if roof["traffic"] is not None else
                               "no capture of this kernel source")
    line = {"metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": timing["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16x3/f64" if mode else "f32/f64",
            "data": "synthetic (seeded blob map, CTF, white noise; stands in for the reference's datasets)",
            "config": workload_config(), "particles_per_step": B,
            "run": {"diff2": args.mode, "l2": "working set > L2 (bf16 hi/lo projection operands 0.97 GB per step)"},
            "e2e": e2e, "gpu_launches": timing["gpu_launches"], "clocks": clocks, "roofline": roof,
            "stage_ms": {n: float(v) for n, v in zip(
                ["prep_network", "operands_audit_norms", "coarse_diff2", "coarse_weights", "fine", "fine_weights",
                 "wsum_bp", "audit_contraction", "proposal_contraction"], stages)},
            "nr_sign_mean": float(timing["res"]["nr_sign"].double().mean()),
            "n_coarse_sig_mean": float(timing["res"]["n_coarse_sig"].double().mean())}
    if tuned is not None:
        line["run"]["tile_shapes"] = tuned
    if learned is not None:
        learned["learned_fraction"] = float(hres["learned"].double().mean())
        line["run"]["learned"] = learned
    if args.mode != "plain" and not args.no_plain:
        # the metric's comparator, in the same run: the plain FP32 SIMT coarse pass on the same
        # batch, timed the same way (device and end to end), then the learned path's quality
        # against it on QUALITY_PARTICLES other particles
        es_plain = setup_context(t2b, sy, fmap, samp, t2b.DIFF2_PLAIN_FP32, B, device=local)
        if tuned is not None:
            es_plain.tune_set(**{k: tuned[k] for k in ("diff2_tn", "diff2_group", "fine_ctas_per_sm",
                                                        "wsum_ctas_per_sm", "project_pixels", "project_orients")})
        pt = time_device(es_plain, parts, B, PLAIN_STEPS, 3, local, world, t2b)
        pe, _, _ = time_e2e(es_plain, parts, B, PLAIN_STEPS, world, t2b, min_steps=PLAIN_STEPS)
        line["plain"] = {"value": pt["value"], "ms_per_step": pt["ms_per_step"], "steps": PLAIN_STEPS,
                         "e2e": {"value": pe["value"], "synchronous_value": pe["synchronous_value"]},
                         "clocks": pt["clocks"]}
        line["vs_baseline"] = value / pt["value"]
        line["vs_baseline_definition"] = ("value / plain.value: the plain FP32 GPU path timed in this run "
                                          "(no published number exists for this metric)")
        line["vs_plain_e2e"] = e2e["value"] / pe["value"]
        if rank == 0 and learned is not None:
            line["quality_vs_plain"] = quality_vs_plain(es, es_plain, sy, fmap, QUALITY_PARTICLES, B,
                                                        WORKLOAD["seed"] + 5000 + 1000 * rank)
        es_plain.close()
    if world > 1:
        line["exchange"] = exchange_once(es, world, t2b)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    es.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def result_tensors(B, K, nd, dev, half=None):
    import torch
    half = half or WORKLOAD["ori_size"] // 2 + 1
    return {k: torch.zeros(shape, dtype=dt, device=dev) for k, shape, dt in [
        ("min_diff2", B, torch.float64), ("sum_weight", B, torch.float64), ("sig_weight", B, torch.float64),
        ("coarse_sum_weight", B, torch.float64), ("coarse_sig_weight", B, torch.float64),
        ("nr_sign", B, torch.int64), ("n_coarse_sig", B, torch.int64), ("pmax", B, torch.float64),
        ("pose", (B, 5), torch.int32), ("wsum_norm", B, torch.float64), ("sumw", B, torch.float64),
        ("wsum_sigma2_offset", B, torch.float64), ("wsum_sigma2", (B, half), torch.float64),
        ("wsum_pdf_class", (B, K), torch.float64), ("wsum_pdf_dir", (B, K * nd), torch.float64),
        ("status", B, torch.int32), ("audit_mass", B, torch.float64), ("learned", B, torch.int32)]}


def time_device(es, parts, B, steps, warmup, local, world, t2b):
    """`steps` E-steps of the batch through the device entry point (inputs resident in HBM),
    CUDA events on the launching stream, barrier + synchronize on both sides, max over ranks."""
    import torch
    dev = torch.device("cuda", local)
    fimg = torch.from_numpy(parts["fimg"].view(np.float32)).to(dev)
    ctf = torch.from_numpy(parts["ctf"]).to(dev)
    minv = torch.from_numpy(parts["minv"]).to(dev)
    scal = torch.from_numpy(parts["scalars"]).to(dev)
    res = result_tensors(B, es.cfg["nr_classes"], es.cfg["n_dir"], dev, es.cfg["ori_size"] // 2 + 1)
    rptr = {k: ctypes.c_void_p(v.data_ptr()) for k, v in res.items()}
    # an explicit stream: the library runs a NULL stream argument on its own stream
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def step():
        es.expectation_device(B, ctypes.c_void_p(fimg.data_ptr()), ctypes.c_void_p(ctf.data_ptr()),
                              ctypes.c_void_p(minv.data_ptr()), ctypes.c_void_p(scal.data_ptr()), rptr,
                              stream=stream.cuda_stream)

    for _ in range(max(warmup, 3)):
        step()
    torch.cuda.synchronize()
    assert stream.cuda_stream != 0
    if int(res["status"].ne(0).sum()) != 0:
        raise RuntimeError(f"E-step status errors: {res['status'].cpu().numpy()}")
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed_steps")   # lets a profiler select the timed launches
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    # kernel nodes of the captured step graph, times the timed steps
    gpu_launches = es.launch_count() * steps if es.launch_count() > 0 else None
    total_ms = ev0.elapsed_time(ev1)
    if world > 1:
        torch.distributed.barrier()
    total_ms = max_over_ranks(total_ms, world)
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    return {"value": B * steps * world / (total_ms / 1000.0), "ms_per_step": total_ms / steps,
            "gpu_launches": gpu_launches, "clocks": clk.summary(), "res": res}


def time_e2e(es, parts, B, steps, world, t2b, min_steps=E2E_STEPS):
    """The same metric end to end through the host entry points with pinned host buffers:
    H2D of each step's batch and D2H of its results inside the timed region, host wall clock,
    median of 3 runs.  Returns (e2e dict, pinned inputs, pinned results)."""
    import torch
    pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in
           [("fimg", parts["fimg"].view(np.float32)), ("ctf", parts["ctf"]), ("minv", parts["minv"]),
            ("scal", parts["scalars"])]}
    hres = {k: v.pin_memory() for k, v in result_tensors(B, es.cfg["nr_classes"], es.cfg["n_dir"], "cpu",
                                                          es.cfg["ori_size"] // 2 + 1).items()}
    lib = t2b.lib
    batch = t2b.Batch(B, 0, ctypes.c_void_p(pin["fimg"].data_ptr()), None, ctypes.c_void_p(pin["ctf"].data_ptr()),
                      ctypes.c_void_p(pin["minv"].data_ptr()), ctypes.c_void_p(pin["scal"].data_ptr()))
    result = t2b.Result(*[ctypes.c_void_p(hres[n].data_ptr()) if n in hres else None for n, _ in t2b.Result._fields_])
    ticket = ctypes.c_longlong(-1)

    def e2e_step():
        t2b._check(lib.t2b_estep_batch_host(es._h, ctypes.byref(batch), ctypes.byref(result)))

    def e2e_submit():
        t2b._check(lib.t2b_estep_submit_host(es._h, ctypes.byref(batch), ctypes.byref(result), ctypes.byref(ticket)))
        return ticket.value

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    n_e2e = max(steps, min_steps)

    def timed(loop):
        runs = []
        for _ in range(3):
            if world > 1:
                torch.distributed.barrier()
            t0 = time.perf_counter()
            loop()
            runs.append(max_over_ranks(time.perf_counter() - t0, world))
        return float(np.median(runs))

    def sync_loop():
        # one call per step, each waiting for its own results
        for _ in range(n_e2e):
            e2e_step()

    def pipelined_loop():
        # step i is submitted (its inputs copy in while step i-1 computes), then the host
        # waits for the results of step i-1; after the loop, for the last step's
        prev = None
        for _ in range(n_e2e):
            cur = e2e_submit()
            if prev is not None:
                t2b._check(lib.t2b_estep_wait(es._h, prev))
            prev = cur
        t2b._check(lib.t2b_estep_wait(es._h, prev))

    sync_s = timed(sync_loop)
    e2e_s = timed(pipelined_loop)
    h2d = sum(v.numel() * v.element_size() for v in pin.values())
    d2h = sum(v.numel() * v.element_size() for v in hres.values())
    return ({"value": B * n_e2e * world / e2e_s, "unit": "particles/s", "h2d_bytes_per_step": h2d,
             "d2h_bytes_per_step": d2h, "api": "t2b_estep_submit_host + t2b_estep_wait (one step in flight)",
             "steps": n_e2e, "timing": "host wall clock, median of 3 runs",
             "synchronous_value": B * n_e2e * world / sync_s}, pin, hres)


def exchange_once(es, world, t2b):
    """The iteration's one exchange, after the timed region: the backprojection grids summed
    over each gold-standard half in place (NCCL all-reduce on the library's device grids)."""
    import torch
    import t2relion_b200.parallel as par
    halves = par.gold_standard_groups(world)
    torch.cuda.synchronize()
    torch.distributed.barrier()
    t0 = time.perf_counter()
    par.allreduce_grids_(es, es.cfg["nr_classes"], group=halves.mine)
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, world)
    nvox = int(np.prod(es._grid_shape))
    return {"what": "in-place all-reduce of the grids (data + weight) within each gold-standard half",
            "bytes_per_rank": 12 * nvox * es.cfg["nr_classes"], "ms": dt * 1e3, "halves": halves.sizes}

if __name__ == "__main__":
    main()
