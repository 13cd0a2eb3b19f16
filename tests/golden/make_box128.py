"""Golden fixtures of the box-128 HEALPix-order-3 refinement E-step (the benchmarked
workload) from the FP64 oracle, computed on the host cores.

Test infrastructure: the FP64 oracle (oracle/estep_oracle.cpp, a restatement of the
reference CPU E-step) runs the whole E-step -- coarse pass over 36,864 orientations x 81
translations, FP64 weights and significance, fine pass (8 rotations x 4 shifts per
significant pair), weighted sums with the scale-correction sums, backprojection into the
259 x 259 x 130 grid -- on 256 seeded particles, and this script stores what the GPU
test (tests/test_gpu_box128.py) compares against:

  per particle   pose, pmax, min_diff2, sum / significance weights of both passes,
                 nr_sign, the size of the coarse significant mask, wsum_norm, sumw,
                 sigma2_offset, scale-correction XA / AA, sigma2 rings, pdf_direction sums
  coarse diff2   for 8 particles: the 2,048 smallest values and 2,048 random ones (index,
                 FP64 value) out of 2,985,984
  grid           the down-sampled average of the backprojected grid (getDownsampledAverage,
                 src/backprojector.cpp:933-1000: the FSC input) inside radius 41 of the
                 128-pixel box, and the weight summed per padded shell

The particles are regenerated on the GPU box from the seed (numpy, deterministic); the
SHA-256 of the inputs is stored with the fixtures and checked there.

Run:  python tests/golden/make_box128.py   (about 10 minutes on 8 host cores)
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))

import problems  # noqa: E402
import recon_oracle as ro  # noqa: E402

N_PARTICLES = 256
SEED = 4242
N_DIFF2 = 8
OUT = os.path.join(HERE, "box128_order3.npz")
AVG_RADIUS = 41


def data_vs_prior():
    """A data_vs_prior_class per ring: above 3 up to ring 24, below from there on."""
    dvp = np.full((1, problems.BOX128["ori_size"] // 2 + 1), 1.0)
    dvp[0, :25] = 6.0
    return dvp


def _arg(name, default, kind=int):
    return kind(sys.argv[sys.argv.index(name) + 1]) if name in sys.argv else default


def main():
    threads = _arg("--threads", os.cpu_count())
    n = _arg("--n", N_PARTICLES)            # fewer particles: a quick run of the recipe only
    out = _arg("--out", OUT, str)
    pb = problems.box128(n, SEED, data_vs_prior=data_vs_prior())
    prob, op = pb["prob"], pb["oparts"]
    t0 = time.time()
    ores = prob.estep(op, nthreads=threads)
    t_estep = time.time() - t0
    assert ores["fails"] == 0
    data, weight = prob.grids()
    avg = ro.downsampled_average(data[0], weight[0], problems.BOX128["bp_r_max"], 2)
    ds = avg.shape[1]
    c = np.arange(ds) - ds // 2
    R = np.sqrt(c[:, None, None] ** 2 + c[None, :, None] ** 2 + np.arange(avg.shape[2])[None, None, :] ** 2)
    mask = R <= AVG_RADIUS
    zd, yd, xd = weight[0].shape
    K, I, J = np.meshgrid(np.arange(zd) - zd // 2, np.arange(yd) - yd // 2, np.arange(xd), indexing="ij")
    shell = ro.relion_round(np.sqrt(K * K + I * I + J * J))
    shell_w = np.bincount(shell.ravel(), weight[0].ravel())
    # coarse diff2 samples of the first N_DIFF2 particles
    rng = np.random.default_rng(SEED + 1)
    nd = min(N_DIFF2, n)
    rnd = [rng.choice(prob.O * prob.T, 2048, replace=False) for _ in range(nd)]
    t0 = time.time()
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=threads) as ex:     # the oracle call releases the GIL
        rows = list(ex.map(lambda b: prob.coarse_diff2(op, b)[0], range(nd)))
    d2_idx, d2_val = [], []
    for b, d2 in enumerate(rows):
        low = np.argsort(d2, kind="stable")[:2048]
        idx = np.concatenate([low, rnd[b]]).astype(np.int32)
        d2_idx.append(idx)
        d2_val.append(d2[idx])
    t_d2 = time.time() - t0
    meta = dict(workload=problems.BOX128, n_particles=n, seed=SEED, avg_radius=AVG_RADIUS,
                input_sha256=problems.input_digest(pb["parts"]), oracle_threads=threads,
                oracle_estep_s=round(t_estep, 1), oracle_diff2_s=round(t_d2, 1))
    keys = ("pose", "pmax", "min_diff2", "sum_weight", "sig_weight", "coarse_min_diff2", "coarse_sum_weight",
            "coarse_sig_weight", "nr_sign", "n_coarse_sig", "wsum_norm", "sumw", "wsum_sigma2_offset",
            "wsum_scale_xa", "wsum_scale_aa", "wsum_sigma2", "wsum_pdf_dir", "wsum_pdf_class")
    np.savez_compressed(out, meta=json.dumps(meta), data_vs_prior=data_vs_prior(),
                        **{k: ores[k] for k in keys},
                        d2_index=np.stack(d2_idx), d2_value=np.stack(d2_val),
                        grid_avg=avg[mask].astype(np.complex64), grid_shell_weight=shell_w)
    print(json.dumps(meta), f"-> {out} ({os.path.getsize(out) / 1e6:.2f} MB)")


if __name__ == "__main__":
    main()
