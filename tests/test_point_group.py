"""Point-group symmetry on the host: the library's group generator (t2b_point_group) against
the oracle's restatement of SymList (oracle/recon_oracle.py), both pinned by facts of the
groups themselves (orders, improper counts, angle classes, the exact matrices of C4, D2, O,
Oh, Cs, C2v and S4, the inversion groups as rotations x Ci), and the
oracle's symmetrisation of a grid against a direct loop for the 4-fold group, whose rotated
coordinates are integers.  No GPU."""
import itertools

import numpy as np
import pytest

import recon_oracle as ro

ORDERS = {"C1": 0, "c2": 1, "C4": 3, "C12": 11, "D1": 1, "D2": 3, "d7": 13, "T": 11, "O": 23,
          "I": 59, "I1": 59, "I2": 59, "I3": 59, "I4": 59,
          # with mirror planes or an inversion (Sn is C(n/2) x Ci in the reference)
          "Ci": 1, "Cs": 1, "C3v": 5, "c4h": 7, "S4": 3, "S10": 9, "D1h": 3, "D3v": 11, "D2h": 7, "D12h": 47,
          "Td": 23, "Th": 23, "Oh": 47, "Ih": 119, "I1h": 119, "I2h": 119, "I3h": 119, "I4h": 119}
IMPROPER = {"Ci": 1, "Cs": 1, "C3v": 3, "c4h": 4, "S4": 2, "S10": 5, "D1h": 2, "D3v": 6, "D2h": 4, "D12h": 24,
            "Td": 12, "Th": 12, "Oh": 24, "Ih": 60, "I1h": 60, "I2h": 60, "I3h": 60, "I4h": 60}


@pytest.mark.parametrize("group", list(ORDERS))
def test_library_group_equals_oracle(t2b, group):
    got = t2b.point_group(group)
    ref = ro.point_group(group)
    assert len(got) == len(ref) == ORDERS[group]
    if len(ref):
        assert np.max(np.abs(got - ref)) <= 1e-12


@pytest.mark.parametrize("group", ["C12", "D7", "T", "O", "I", "I1", "I3", "I4", "C3v", "S10", "D12h", "Td", "Th",
                                   "Oh", "Ih", "I3h"])
def test_group_is_closed_and_orthogonal(group):
    ops = ro.point_group(group)
    eye = np.eye(3)
    dets = []
    for m in ops:
        assert np.max(np.abs(m @ m.T - eye)) <= 1e-6
        dets.append(np.linalg.det(m))
        assert abs(abs(dets[-1]) - 1.0) <= 1e-6
    assert int(np.sum(np.array(dets) < 0)) == IMPROPER.get(group, 0)
    members = np.concatenate([ops, eye[None]])
    prods = np.einsum("aij,bjk->abik", members, members).reshape(-1, 1, 3, 3)
    dist = np.max(np.abs(prods - members[None]), axis=(2, 3)).min(axis=1)
    assert np.all(dist <= 1e-5)


def _angles(ops):
    return np.round(np.degrees(np.arccos(np.clip((np.trace(ops, axis1=1, axis2=2) - 1) / 2, -1, 1)))).astype(int)


@pytest.mark.parametrize("group", ["I", "I1", "I3", "I4"])
def test_icosahedral_angle_classes(group):
    """15 two-fold, 20 three-fold and 24 five-fold rotations (12 by 72 and 12 by 144 degrees)."""
    a = _angles(ro.point_group(group))
    assert {v: int(np.sum(a == v)) for v in (72, 120, 144, 180)} == {72: 12, 120: 20, 144: 12, 180: 15}


def test_octahedral_group_is_the_signed_permutations():
    ops = ro.point_group("O")
    want = []
    for perm in itertools.permutations(range(3)):
        for signs in itertools.product((1, -1), repeat=3):
            m = np.zeros((3, 3))
            m[range(3), perm] = signs
            if round(np.linalg.det(m)) == 1 and not np.array_equal(m, np.eye(3)):
                want.append(m)
    assert len(want) == 23
    for w in want:
        assert min(np.max(np.abs(w - m)) for m in ops) <= 1e-12


def test_octahedral_with_mirrors_is_every_signed_permutation():
    ops = ro.point_group("Oh")
    want = []
    for perm in itertools.permutations(range(3)):
        for signs in itertools.product((1, -1), repeat=3):
            m = np.zeros((3, 3))
            m[range(3), perm] = signs
            if not np.array_equal(m, np.eye(3)):
                want.append(m)
    assert len(want) == len(ops) == 47
    for w in want:
        assert min(np.max(np.abs(w - m)) for m in ops) <= 1e-12


@pytest.mark.parametrize("proper,full", [("I", "Ih"), ("I1", "I1h"), ("I3", "I3h"), ("I4", "I4h"), ("T", "Th"),
                                         ("D6", "D6h"), ("C4", "C4h")])
def test_groups_with_a_centre_of_inversion(proper, full):
    """Each of these holds the inversion, so its improper operators are minus its rotations: the
    rotations of the proper group (Th is generated about the negated 2-fold axis, the same group)."""
    rot = list(ro.point_group(proper)) + [np.eye(3)]
    ops = ro.point_group(full)
    assert len(ops) == 2 * len(rot) - 1
    for m in ops:
        cand = m if np.linalg.det(m) > 0 else -m
        assert min(np.max(np.abs(cand - r)) for r in rot) <= 1e-6


def test_mirror_generators():
    """Cs: the mirror z -> -z; C2v: the two vertical mirrors (normals x and y) and the 2-fold;
    S4 (the reference's C2 x Ci): the 2-fold about z, the inversion and the mirror z -> -z."""
    assert np.array_equal(ro.point_group("Cs")[0], np.diag([1., 1., -1.]))
    for ops, want in ((ro.point_group("C2v"), [np.diag([-1., -1., 1.]), np.diag([1., -1., 1.]), np.diag([-1., 1., 1.])]),
                      (ro.point_group("S4"), [np.diag([-1., -1., 1.]), -np.eye(3), np.diag([1., 1., -1.])])):
        assert len(ops) == 3
        for w in want:
            assert min(np.max(np.abs(w - m)) for m in ops) <= 1e-12


def test_dihedral_and_cyclic_matrices():
    d2 = ro.point_group("D2")
    for diag in ((1, -1, -1), (-1, 1, -1), (-1, -1, 1)):
        assert min(np.max(np.abs(np.diag(diag) - m)) for m in d2) == 0
    c4 = ro.point_group("C4")
    for k in (1, 2, 3):
        t = np.radians(90 * k)
        rz = np.array([[np.cos(t), -np.sin(t), 0], [np.sin(t), np.cos(t), 0], [0, 0, 1]])
        assert min(np.max(np.abs(np.where(np.abs(rz) < 1e-6, 0, rz) - m)) for m in c4) == 0
    # the icosahedral orientations: a 2-fold about z for I (= I2), about x for I1
    for g, two in (("I", np.diag([-1., -1., 1.])), ("I1", np.diag([1., -1., -1.]))):
        assert min(np.max(np.abs(two - m)) for m in ro.point_group(g)) <= 1e-9


@pytest.mark.parametrize("bad", ["I5", "I5h", "C0", "C123", "D2x", "Tv", "X", "S3"])
def test_unknown_groups_are_refused(t2b, bad):
    """I5 / I5h are not implemented by the reference either; an Sn group needs an even n."""
    with pytest.raises(t2b.T2BError) as e:
        t2b.point_group(bad)
    assert e.value.code == (t2b.T2B_ERR_ARG if bad == "S3" else t2b.T2B_ERR_UNSUPPORTED)
    with pytest.raises(ValueError):
        ro.point_group(bad)


def _grid(rp, seed):
    rng = np.random.default_rng(seed)
    n = 2 * (rp + 1) + 1
    d = (rng.normal(size=(n, n, rp + 2)) + 1j * rng.normal(size=(n, n, rp + 2)))
    w = rng.uniform(0.5, 2.0, size=(n, n, rp + 2))
    return d, w


def test_symmetrisation_by_four_fold_matches_a_direct_loop():
    """C4 maps integer points to integer points: the trilinear reads are the grid's own values,
    conjugated where the rotated x is negative (then read at the negated point)."""
    rp = 5
    d, w = _grid(rp, 3)
    ops = ro.point_group("C4")
    sd, sw = ro.apply_point_group_symmetry(d, w, ops, rp, 1)
    c = rp + 1
    for z, y, x in itertools.product(range(-c, c + 1), range(-c, c + 1), range(0, c + 1)):
        ed, ew = d[z + c, y + c, x], w[z + c, y + c, x]
        if x * x + y * y + z * z <= rp * rp:
            for m in ops:
                p = np.rint(m @ np.array([x, y, z], float)).astype(int)
                neg = p[0] < 0
                if neg:
                    p = -p
                v = d[p[2] + c, p[1] + c, p[0]]
                ed += np.conj(v) if neg else v
                ew += w[p[2] + c, p[1] + c, p[0]]
        assert abs(sd[z + c, y + c, x] - ed) <= 1e-12 and abs(sw[z + c, y + c, x] - ew) <= 1e-12


def test_symmetrisation_of_an_invariant_weight():
    """A weight that depends on the radius alone, summed over O (signed permutations, so every
    read lands on a grid point): 24 times itself inside the sphere, itself outside."""
    rp = 6
    c = rp + 1
    z, y, x = np.meshgrid(np.arange(-c, c + 1), np.arange(-c, c + 1), np.arange(0, c + 1), indexing="ij")
    r2 = (x * x + y * y + z * z).astype(float)
    w = 1.0 + r2
    d = np.zeros(w.shape, complex)
    _, sw = ro.apply_point_group_symmetry(d, w, ro.point_group("O"), rp, 1)
    inside = r2 <= rp * rp
    assert np.allclose(sw[inside], 24 * w[inside], rtol=1e-9)
    assert np.array_equal(sw[~inside], w[~inside])


def test_helical_operators_follow_the_unit_range():
    """n units hh = -n/2 .. n/2 - 1 (+1 for odd n), hh = 0 left out; rotations by -hh twist."""
    for n, hs in ((2, [-1]), (3, [-1, 1]), (4, [-2, -1, 1]), (5, [-2, -1, 1, 2])):
        mats, zsh = ro.helical_operators(n, 30.0, 2.5, 64, 2)
        assert len(mats) == len(hs)
        for m, z, hh in zip(mats, zsh, hs):
            t = np.radians(-hh * 30.0)
            assert np.allclose(m, [[np.cos(t), -np.sin(t), 0], [np.sin(t), np.cos(t), 0], [0, 0, 1]], atol=1e-6)
            assert z == hh * 2.5 / (-64 * 2.0)
    assert len(ro.helical_operators(1, 30.0, 2.5, 64, 2)[0]) == 0
    assert np.all(ro.helical_operators(3, 30.0, 0.0, 64, 2)[1] == 0)


def test_helical_rise_alone_is_a_phase_sum():
    """Twist 0: every unit reads the voxel itself, so the data become data x sum_hh
    e^{2 pi i z hh rise / (-ori pad)} (hh = 0 included) and the weights n x weight."""
    rp, n, rise, ori, pad = 5, 4, 3.7, 10, 1
    d, w = _grid(rp, 5)
    mats, zsh = ro.helical_operators(n, 0.0, rise, ori, pad)
    sd, sw = ro.apply_point_group_symmetry(d, w, mats, rp, pad, zshift=zsh)
    c = rp + 1
    z, y, x = np.meshgrid(np.arange(-c, c + 1), np.arange(-c, c + 1), np.arange(0, c + 1), indexing="ij")
    inside = x * x + y * y + z * z <= rp * rp
    hh = np.array([-2, -1, 0, 1])
    phase = np.exp(2j * np.pi * z[..., None] * hh * rise / (-ori * pad)).sum(-1)
    assert np.allclose(sd[inside], d[inside] * phase[inside], rtol=1e-12, atol=1e-12)
    assert np.allclose(sw[inside], n * w[inside], rtol=1e-12)
    assert np.array_equal(sd[~inside], d[~inside])


def test_helical_quarter_twist_matches_a_direct_loop():
    """Twist 90 degrees, three units: integer rotations about z, so the reads are grid values."""
    rp, rise, ori, pad = 5, 1.5, 12, 1
    d, w = _grid(rp, 7)
    mats, zsh = ro.helical_operators(3, 90.0, rise, ori, pad)
    sd, sw = ro.apply_point_group_symmetry(d, w, mats, rp, pad, zshift=zsh)
    c = rp + 1
    for z, y, x in itertools.product(range(-c, c + 1), range(-c, c + 1), range(0, c + 1)):
        ed, ew = d[z + c, y + c, x], w[z + c, y + c, x]
        if x * x + y * y + z * z <= rp * rp:
            for hh in (-1, 1):
                t = np.radians(-hh * 90.0)
                p = np.rint(np.array([[np.cos(t), -np.sin(t), 0], [np.sin(t), np.cos(t), 0], [0, 0, 1]])
                            @ np.array([x, y, z], float)).astype(int)
                neg = p[0] < 0
                if neg:
                    p = -p
                v = d[p[2] + c, p[1] + c, p[0]]
                v = np.conj(v) if neg else v
                ed += v * np.exp(2j * np.pi * z * hh * rise / (-ori * pad))
                ew += w[p[2] + c, p[1] + c, p[0]]
        assert abs(sd[z + c, y + c, x] - ed) <= 1e-12 and abs(sw[z + c, y + c, x] - ew) <= 1e-12


def test_point_group_abi_contract(t2b):
    """t2b_point_group fills at most cap matrices and always reports the count; a null count is
    refused.  The grid entry points refuse a null context before touching a device."""
    import ctypes
    lib = t2b.lib
    n = ctypes.c_int(-1)
    assert lib.t2b_point_group(b"O", None, 0, ctypes.byref(n)) == t2b.T2B_OK and n.value == 23
    buf = np.full((30, 3, 3), 7.0)
    assert lib.t2b_point_group(b"O", buf.ctypes.data_as(ctypes.c_void_p), 5, ctypes.byref(n)) == t2b.T2B_OK
    assert n.value == 23
    assert np.array_equal(buf[:5], t2b.point_group("O")[:5]) and np.all(buf[5:] == 7.0)
    assert lib.t2b_point_group(b"O", None, 0, None) == t2b.T2B_ERR_ARG
    assert lib.t2b_point_group(b"O", None, 4, ctypes.byref(n)) == t2b.T2B_ERR_ARG
    assert lib.t2b_point_group(None, None, 0, ctypes.byref(n)) == t2b.T2B_OK and n.value == 0   # C1
    assert lib.t2b_backprojector_apply_symmetry(None, 0, b"C2") == t2b.T2B_ERR_ARG
    assert lib.t2b_backprojector_apply_helical(None, 0, 3, 10.0, 2.0, 64) == t2b.T2B_ERR_ARG
