"""CPU: the host's flag-driven remesh (the refine_fine stand-in the GPU
remesh tests drive): refined regions shrink from their finest level, octs
that survive keep their igrids, freed igrids are reused, and the new tree
satisfies the nesting rule (every oct's father cell exists one level up)."""
import numpy as np

from ramses_b200 import mesh


def _tree():
    return mesh.build_tree(3, 5, mesh.sphere_refine((0.5, 0.5, 0.5), 0.2), spare=4000)


def _check_nesting(t):
    for l in range(2, t.nlevelmax + 1):
        for g in t.active[l]:
            f = int(t.father[g - 1])
            assert t.son[f - 1] == g


def test_no_flags_removes_the_finest_level():
    t = _tree()
    assert t.noct(5) > 0
    new = mesh.refine_from_flags(t, np.zeros(t.ncell + 1, np.int32))
    assert new.noct(5) == 0 and new.noct(4) > 0
    # octs at a position the old tree had keep its igrid
    old = {tuple(c): g for c, g in zip(t.coords[4].tolist(), t.active[4].tolist())}
    kept = [(old[tuple(c)], g) for c, g in zip(new.coords[4].tolist(), new.active[4].tolist()) if tuple(c) in old]
    assert kept and all(a == b for a, b in kept)
    _check_nesting(new)


def test_flags_grow_the_tree_and_reuse_igrids():
    t = _tree()
    f = np.zeros(t.ncell + 1, np.int32)
    # flag every cell of every level-4 oct
    cells4 = t.ncoarse + np.arange(8)[:, None] * t.ngridmax + t.active[4][None, :]
    f[cells4.ravel()] = 1
    new = mesh.refine_from_flags(t, f)
    assert new.noct(5) >= t.noct(5)
    kept = set(t.active[5].tolist()) & set(new.active[5].tolist())
    assert kept, "surviving level-5 octs keep their igrids"
    used = np.concatenate([new.active[l] for l in range(1, 6) if new.noct(l)])
    assert len(np.unique(used)) == len(used) and used.max() <= new.ngridmax
    _check_nesting(new)


def test_sorted_set_helpers_match_numpy():
    """The sort-based set helpers of the tree builder (the hashing np.unique is
    slow on large int64 key arrays) give numpy's answers."""
    rng = np.random.default_rng(11)
    for n in (0, 1, 5, 1000, 50000):
        a = rng.integers(0, 4000, n)
        b = rng.integers(0, 4000, max(n // 3, 1))
        np.testing.assert_array_equal(mesh._unique(a), np.unique(a))
        np.testing.assert_array_equal(mesh._isin(a, b), np.isin(a, b))
    assert mesh._isin(np.arange(5), np.zeros(0, np.int64)).sum() == 0


def test_separable_dilation_equals_the_27_point_neighbourhood():
    """Three one-axis dilations give the periodic 26-neighbourhood of a cell
    set, as the 27-point expansion does."""
    rng = np.random.default_rng(5)
    for n in (4, 16, 64):
        cells = rng.integers(0, n, (200, 3))
        want = np.unique(mesh._keys(mesh._neighbourhood(cells) % n, n))
        np.testing.assert_array_equal(mesh._dilated_keys(cells, n), want)
