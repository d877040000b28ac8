"""The oracle's restatement of the merge step (Merger.merge_catalog, Exclusion,
finalize_eulerian), pinned on the reference's own test cases (test/test_merger.jl)."""
import math

import numpy as np
import pytest

from oracle import catalog as oc


def mk(x, y, z, R, vx=0.0, vy=0.0, vz=0.0, od=0.0):
    return [x, y, z, vx, vy, vz, R, 0.0, 0.0, 0.0, od]


def test_sphere_overlap_cases():
    """test_merger.jl:8-45."""
    assert oc.sphere_overlap(10.0, 2.0, 3.0) == (0.0, 0.0)      # apart
    assert oc.sphere_overlap(5.0, 2.0, 3.0) == (0.0, 0.0)       # touching
    assert oc.sphere_overlap(0.5, 3.0, 1.0) == (0.0, 0.0)       # one inside the other
    assert oc.sphere_overlap(0.0, 2.0, 2.0) == (0.0, 0.0)
    r = 2.0
    v1, v2 = oc.sphere_overlap(r, r, r)
    h = r / 2
    assert v1 == pytest.approx(v2) and v1 == pytest.approx(math.pi / 3 * h * h * (3 * r - h))
    assert 0 < v1 + v2 < 4 * math.pi / 3 * r ** 3
    v1, v2 = oc.sphere_overlap(3.0, 3.0, 1.0)
    assert 0 < v1 < v2


def test_synthetic_catalog():
    """test_merger.jl:195-222: the small halo inside the large one goes, the overlapping and
    the isolated ones keep their radii (no volume reduction by default)."""
    h = np.array([mk(0, 0, 0, 5, od=1), mk(1, 1, 1, 1, od=.5), mk(7, 0, 0, 3, od=.8),
                  mk(50, 50, 50, 2, od=.3)], np.float32)
    m = oc.merge_catalog(h)
    assert m.shape[0] == 3 and not any((r[:3] == 1).all() for r in m)
    assert np.array_equal(m[:, 6], np.float32([5, 3, 2]))


def test_exclusion_cases():
    """test_merger.jl:103-138: basic and equal-radius exclusion."""
    m = oc.merge_catalog(np.array([mk(0, 0, 0, 2), mk(.3, .3, .3, .5), mk(10, 10, 10, 1)], np.float32))
    assert m.shape[0] == 2 and m[0, 6] == 2 and m[1, 6] == 1
    m = oc.merge_catalog(np.array([mk(0, 0, 0, 2), mk(.5, 0, 0, 2)], np.float32))
    assert m.shape[0] == 1 and m[0, 0] == 0.0         # the first of two equal radii survives
    # chain (test_merger.jl:236-245): every smaller halo sits inside a larger one
    chain = np.array([mk(0, 0, 0, 10)] + [mk(k, 0, 0, 10 - k) for k in range(1, 6)], np.float32)
    m = oc.merge_catalog(chain)
    assert m.shape[0] == 1 and m[0, 6] == 10


def test_volume_reduction_cases():
    """test_merger.jl:47-78 and 140-193: a pair loses its own caps, the shared reduction
    equals the brute-force all-pairs sum on a random set, fortran_ties doubles an equal pair."""
    h = np.array([mk(50, 50, 50, 3), mk(54, 50, 50, 2)], np.float32)
    v1, v2 = oc.sphere_overlap(4.0, 3.0, 2.0)
    assert np.array_equal(oc.merge_catalog(h)[:, 6], np.float32([3, 2]))
    got = np.sort(oc.merge_catalog(h, volume_reduction=True)[:, 6])[::-1]
    want = [math.cbrt(27 - 3 * v1 / (4 * math.pi)), math.cbrt(8 - 3 * v2 / (4 * math.pi))]
    assert np.allclose(got, want, rtol=1e-5)
    rng = np.random.default_rng(7)
    hs = np.array([mk(*(100 * rng.random(3)), 1 + 4 * rng.random()) for _ in range(600)], np.float32)
    ex = oc.merge_catalog(hs)
    red = oc.merge_catalog(hs, volume_reduction=True)
    dV = np.zeros(len(ex))
    pos = ex[:, :3].astype(np.float64)
    for a in range(len(ex)):
        for b in range(a + 1, len(ex)):
            d = float(np.sqrt(((pos[a] - pos[b]) ** 2).sum()))
            if d < ex[a, 6] + ex[b, 6]:
                va, vb = oc.sphere_overlap(d, float(ex[a, 6]), float(ex[b, 6]))
                dV[a] += va
                dV[b] += vb
    want = {tuple(e[:3]): math.cbrt(float(e[6]) ** 3 - 3 * dV[k] / (4 * math.pi))
            for k, e in enumerate(ex) if float(e[6]) ** 3 > 3 * dV[k] / (4 * math.pi)}
    assert len(red) == len(want) and (dV > 0).sum() > 50
    assert all(math.isclose(float(e[6]), want[tuple(e[:3])], rel_tol=1e-5) for e in red)
    ht = np.array([mk(50, 50, 50, 2), mk(53, 50, 50, 2)], np.float32)
    v1t, _ = oc.sphere_overlap(3.0, 2.0, 2.0)
    assert np.allclose(oc.merge_catalog(ht, volume_reduction=True)[:, 6],
                       math.cbrt(8 - 3 * v1t / (4 * math.pi)))
    assert np.allclose(oc.merge_catalog(ht, volume_reduction=True, fortran_ties=True)[:, 6],
                       math.cbrt(8 - 6 * v1t / (4 * math.pi)))


def test_deterministic_under_input_order():
    """test_merger.jl:278-290: the surviving set does not depend on the input order."""
    rng = np.random.default_rng(1)
    hs = np.array([mk(*(60 * rng.random(3)), 1 + 3 * rng.random()) for _ in range(400)], np.float32)
    key = lambda m: sorted(map(tuple, m[:, [0, 1, 2, 6]].tolist()))
    ref = key(oc.merge_catalog(hs))
    assert len(ref) < len(hs)
    for s in range(3):
        assert key(oc.merge_catalog(hs[np.random.default_rng(s).permutation(len(hs))])) == ref


def test_finalize_eulerian_formulas(ht):
    """Merger.jl:114-146 at a snapshot: x = q + d1 + d2, v = a 100 E f (d1 + 2 d2)."""
    cat = ht.catalog
    cp = cat.CosmologyParams()
    g = cat.dlinear_tables(cp)
    chi2z = cat.build_chi_to_z(cp, z_max=10.0, npts=200)
    rec = np.array([mk(10, 20, 30, 2, 1.0, -2.0, 0.5)], np.float32)
    rec[0, 7:10] = [0.1, 0.2, -0.3]
    out = oc.finalize_eulerian(rec, g, cp.Om, cp.OL, (0, 0, 0), chi2z.chis, chi2z.zs,
                               chi2z.z_max, ievol=0, z_out=0.0)
    f = oc.growth_f(g, 1.0)
    assert 0.48 < f < 0.58                            # test_cosmology.jl:46's bounds at z = 0
    assert np.allclose(out[0, :3], [11.1, 18.2, 30.2], rtol=1e-6)
    vfac = 100.0 * math.sqrt(cp.Om + cp.OL) * f
    assert np.allclose(out[0, 3:6], vfac * np.array([1.2, -1.6, -0.1]), rtol=1e-6)
    assert (out[0, 7:10] == 0).all() and out[0, 6] == 2
