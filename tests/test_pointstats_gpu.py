"""Device overlap checks and number-variance window counts against the oracle: the same index sets,
and window moments equal to the last bit (the counts are integers; the centres come from the same
std::mt19937_64 stream; the moments are updated in the same order)."""
import pickle

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pattern(ndim, n, seed, spread=1.0, shift=0.0):
    rng = np.random.default_rng(seed)
    L = np.array([1.0, 1.2, 0.9])[:ndim]
    x = (rng.random((n, ndim)) * L * spread + shift).ravel()
    return rng, L, x


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("density", [0.3, 1.0])
def test_overlap_matches_oracle(ndim, periodic, density):
    from fresco_b200.distances import CheckOverlap, Distance

    n = {1: 500, 2: 4000, 3: 6000}[ndim]
    rng, L, x = _pattern(ndim, n, 30 + ndim, spread=1.3, shift=-0.1)  # points outside the box too
    rad = rng.uniform(0.2, 1.0, n) * density * 0.5 * float(np.prod(L) / n) ** (1.0 / ndim)
    method = Distance.PERIODIC if periodic else Distance.CARTESIAN
    chk = CheckOverlap(rad, L, method=method)
    got = chk.get_overlapping_particles(x)
    want = O.overlapping_particles(x, rad, L, periodic=periodic)
    assert got.dtype == np.uint64 and 0 < len(want) < n
    assert np.array_equal(got, want)
    changed = rng.choice(n, 40, replace=False)
    got = chk.get_overlapping_particles_ca(x, changed)
    assert np.array_equal(got, O.overlapping_particles(x, rad, L, periodic=periodic, changed=changed))


def test_overlap_edge_cases():
    from fresco_b200.distances import CheckOverlap, Distance

    # large radii against a small box: one or two cells per axis, every image considered
    rng, L, x = _pattern(2, 60, 5)
    rad = np.full(60, 0.3)
    got = CheckOverlap(rad, L).get_overlapping_particles(x)
    assert np.array_equal(got, O.overlapping_particles(x, rad, L, periodic=True))
    rad = np.full(60, 0.04)
    got = CheckOverlap(rad, L).get_overlapping_particles(x)
    assert np.array_equal(got, O.overlapping_particles(x, rad, L, periodic=True))
    # one particle, zero radii, touching pairs (strict <)
    assert len(CheckOverlap([0.5], [1.0, 1.0]).get_overlapping_particles([0.1, 0.1])) == 0
    assert len(CheckOverlap(np.zeros(60), L).get_overlapping_particles(x)) == 0
    two = np.array([0.0, 0.0, 0.5, 0.0])
    assert len(CheckOverlap([0.25, 0.25], [4.0, 4.0]).get_overlapping_particles(two)) == 0
    assert list(CheckOverlap([0.25, 0.2500001], [4.0, 4.0]).get_overlapping_particles(two)) == [0, 1]
    # the pair through the periodic boundary, and not in the Cartesian metric
    edge = np.array([0.02, 0.5, 0.98, 0.5])
    assert list(CheckOverlap([0.03, 0.03], [1.0, 1.0]).get_overlapping_particles(edge)) == [0, 1]
    assert len(CheckOverlap([0.03, 0.03], [1.0, 1.0], method=Distance.CARTESIAN)
               .get_overlapping_particles(edge)) == 0
    # the reference's argument errors
    with pytest.raises(RuntimeError, match="illegal input"):
        CheckOverlap(np.full(60, 0.01), L).get_overlapping_particles(x[:-1])
    with pytest.raises(RuntimeError, match="illegal input"):
        CheckOverlap(np.full(60, 0.01), L).get_overlapping_particles(x[:-2])
    with pytest.raises(RuntimeError, match="illegal input: radii"):
        CheckOverlap(np.zeros(0), L)
    with pytest.raises(RuntimeError, match="more than 1 dimension"):
        CheckOverlap([0.1], [1.0], use_cell_lists=True)
    # with cell lists the reference checks every pair in get_overlapping_particles_ca
    rad = rng.uniform(0.01, 0.05, 60)
    full = O.overlapping_particles(x, rad, L, periodic=True)
    assert np.array_equal(CheckOverlap(rad, L, use_cell_lists=True).get_overlapping_particles_ca(x, [0]), full)
    chk = pickle.loads(pickle.dumps(CheckOverlap(rad, L)))
    assert np.array_equal(chk.get_overlapping_particles(x), full)


def test_overlap_large_pattern():
    """2^20 points in 2D at the jammed-packing radius of the repulsion benchmark; the oracle checks the
    changed-atom pairs and a sample of the full set."""
    from fresco_b200.distances import CheckOverlap

    n = 1 << 20
    rng = np.random.default_rng(2)
    L = np.array([2 * np.pi, 2 * np.pi])
    x = (rng.random((n, 2)) * L).ravel()
    rad = np.full(n, 0.25 / np.sqrt(n) * 2 * np.pi)
    chk = CheckOverlap(rad, L)
    got = chk.get_overlapping_particles(x)
    changed = rng.choice(n, 300, replace=False)
    want_ca = O.overlapping_particles(x, rad, L, periodic=True, changed=changed)
    assert np.array_equal(chk.get_overlapping_particles_ca(x, changed), want_ca)
    # every changed atom is in the full set exactly when the oracle finds it overlapping
    assert np.array_equal(np.isin(changed, got), np.isin(changed, want_ca))
    assert 0.2 * n < len(got) < 0.9 * n


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("radius", [0.01, 0.08, 0.3, 0.7])
def test_window_moments_match_oracle(ndim, radius):
    from fresco_b200.utils import PointPatternStatistics

    n = {1: 3000, 2: 20000, 3: 30000}[ndim]
    _, L, x = _pattern(ndim, n, 40 + ndim, spread=1.0, shift=-0.25)
    s = PointPatternStatistics(x, L, radius, 99 + ndim)
    o = O.BatchPPS(x, L, [radius], 99 + ndim)
    s.run(150)
    o.run(150)
    assert s.get_count() == 150
    assert s.get_mean() == o.mean()[0] and s.get_variance() == o.variance()[0]
    s.run(50)  # continues the same stream
    o.run(50)
    assert s.mean_var == (o.mean()[0], o.variance()[0]) and s.count == 200
    s.set_generator_seed(5)
    o.gen.seed(5)
    s.run(40)
    o.run(40)
    assert s.get_seed() == 5 and s.mean == o.mean()[0] and s.var == o.variance()[0]


def test_batch_windows_match_oracle():
    from fresco_b200.utils import BatchPPS

    _, L, x = _pattern(2, 50000, 8)
    radii = np.array([0.002, 0.01, 0.03, 0.05, 0.1, 0.2, 0.35, 0.45, 0.55])
    b = BatchPPS(x, L, radii, 2024)
    o = O.BatchPPS(x, L, radii, 2024)
    b.run(200)
    o.run(200)
    assert np.array_equal(b.get_mean(), o.mean()) and np.array_equal(b.get_variance(), o.variance())
    assert list(b.get_count()) == [200] * len(radii)
    b2 = pickle.loads(pickle.dumps(BatchPPS(x, L, radii, 2024)))
    b2.run(200)
    assert np.array_equal(b2.mean, b.mean)
    with pytest.raises(ValueError, match="ascending"):
        BatchPPS(x, L, radii[::-1], 1)


def test_windows_in_chunks_and_empty_pattern():
    """More windows than one launch holds (65536), run in pieces; a pattern with no points."""
    from fresco_b200.utils import PointPatternStatistics

    _, L, x = _pattern(2, 3000, 9)
    a = PointPatternStatistics(x, L, 0.1, 3)
    a.run(70000)
    b = PointPatternStatistics(x, L, 0.1, 3)
    for _ in range(7):
        b.run(10000)
    assert a.count == b.count == 70000 and a.mean == b.mean and a.var == b.var
    o = O.BatchPPS(x, L, [0.1], 3)
    o.run(70000)
    assert a.mean == o.mean()[0] and a.var == o.variance()[0]
    e = PointPatternStatistics(np.zeros(0), L, 0.1, 3)
    e.run(10)
    assert e.mean == 0.0 and e.var == 0.0 and e.count == 10
