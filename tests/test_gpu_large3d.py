"""The large 3D classification on one B200: K = 4 maps of 256^3, HEALPix order 4 x 96 psi
(1,179,648 class-orientations) x 49 translations, window 200 x 101, 515^3 grids.

Its projection tables would take 190 GB (coarse) and 1.5 TB (fine), so the context runs the
chunked coarse pass (chosen automatically) with on-the-fly fine and weighted-sum projections.
The full FP64 E-step of one such particle is out of the oracle's reach, so parity is checked
per hypothesis on 4 particles: the device's coarse diff2 at 128 random hypotheses and at its
own minimum, and the fine diff2 of 16 significant pairs (all 32 fine hypotheses each),
against the oracle's literal per-pixel diff2 of the same hypothesis (relative error <= 1e-5).
The poses are checked against the simulated truth: the right class, and the max-weight
orientation within 5 degrees of the true one, for every particle.
"""
import numpy as np
import pytest

import problems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def large():
    pb = problems.large3d(4, seed=71)
    es = pb["product"]()
    P = pb["parts"]
    pb["res"] = es.expectation(P["fimg"], P["ctf"], P["minv"], P["scalars"])
    pb["d2"] = [es.coarse_diff2(b) for b in range(4)]
    pb["fine"] = [es.fine(b) for b in range(4)]
    es.close()
    return pb


def test_status_and_truth(large):
    res, P, samp = large["res"], large["parts"], large["samp"]
    assert np.all(res["status"] == 0)
    O, R = samp["n_dir"] * samp["n_psi"], samp["nover_rot"]
    for b in range(4):
        k, o, r = res["pose"][b][:3]
        assert k == large["classes"][b], (b, res["pose"][b])
        err = problems.angle_between(samp["eul_fine"][o * R + r], P["A"][b])
        assert err < 5.0, (b, err)


def test_coarse_diff2_against_literal_oracle(large):
    prob, op, samp = large["prob"], large["oparts"], large["samp"]
    O, T = samp["n_dir"] * samp["n_psi"], samp["n_trans"]
    rng = np.random.default_rng(5)
    worst = 0.
    for b in range(4):
        d2 = large["d2"][b]
        assert d2.size == 4 * O * T
        idx = list(rng.integers(0, d2.size, 128)) + [int(np.argmin(np.where(d2 >= 0, d2, np.inf)))]
        for i in idx:
            oc, t = divmod(int(i), T)
            k, o = divmod(oc, O)
            ref = prob.diff2_literal(op, b, k, samp["eul_coarse"][o], samp["trans_px"][t])
            worst = max(worst, abs(float(d2[i]) - ref) / abs(ref))
    assert worst <= 1e-5, worst


def test_fine_diff2_against_literal_oracle(large):
    prob, op, samp = large["prob"], large["oparts"], large["samp"]
    O, T, R, V = samp["n_dir"] * samp["n_psi"], samp["n_trans"], samp["nover_rot"], samp["nover_trans"]
    worst = 0.
    for b in range(4):
        pairs, d2f = large["fine"][b]
        assert len(pairs) >= 1
        for q in np.linspace(0, len(pairs) - 1, min(16, len(pairs))).astype(int):
            oc, t = divmod(int(pairs[q]), T)
            k, o = divmod(oc, O)
            for r in range(R):
                for v in range(V):
                    ref = prob.diff2_literal(op, b, k, samp["eul_fine"][o * R + r], samp["trans_px_fine"][t * V + v])
                    worst = max(worst, abs(float(d2f[q, r * V + v]) - ref) / abs(ref))
    assert worst <= 1e-5, worst
