"""Point-group symmetry on the host: the library's group generator (t2b_point_group) against
the oracle's restatement of SymList (oracle/recon_oracle.py), both pinned by facts of the
groups themselves (orders, angle classes, the exact matrices of C4, D2 and O), and the
oracle's symmetrisation of a grid against a direct loop for the 4-fold group, whose rotated
coordinates are integers.  No GPU."""
import itertools

import numpy as np
import pytest

import recon_oracle as ro

ORDERS = {"C1": 0, "c2": 1, "C4": 3, "C12": 11, "D1": 1, "D2": 3, "d7": 13, "T": 11, "O": 23,
          "I": 59, "I1": 59, "I2": 59, "I3": 59, "I4": 59}


@pytest.mark.parametrize("group", list(ORDERS))
def test_library_group_equals_oracle(t2b, group):
    got = t2b.point_group(group)
    ref = ro.point_group(group)
    assert len(got) == len(ref) == ORDERS[group]
    if len(ref):
        assert np.max(np.abs(got - ref)) <= 1e-12


@pytest.mark.parametrize("group", ["C12", "D7", "T", "O", "I", "I1", "I3", "I4"])
def test_group_is_closed_rotations(group):
    ops = ro.point_group(group)
    eye = np.eye(3)
    for m in ops:
        assert np.max(np.abs(m @ m.T - eye)) <= 1e-6
        assert abs(np.linalg.det(m) - 1.0) <= 1e-6
    members = list(ops) + [eye]
    for a, b in itertools.product(members, members):
        p = a @ b
        assert min(np.max(np.abs(p - m)) for m in members) <= 1e-5


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


@pytest.mark.parametrize("bad", ["C2v", "D2h", "Ci", "Cs", "S4", "Td", "Oh", "Ih", "I5", "C123", "X"])
def test_groups_with_mirrors_or_unknown_are_refused(t2b, bad):
    with pytest.raises(t2b.T2BError) as e:
        t2b.point_group(bad)
    assert e.value.code == t2b.T2B_ERR_UNSUPPORTED
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
