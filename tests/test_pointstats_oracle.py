"""Oracle for the point-pattern statistics and overlap checks (CPU only): the restated
std::mt19937_64 against the C++ standard's known answer, and the restated window counts, moments and
overlap sets against the reference's own point_pattern_statistics.hpp / check_overlap*.hpp built
serially in oracle/_ref."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import refimpl as R

needs_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")


def test_mt19937_64_known_answer():
    # [rand.predef]: the 10000th consecutive output of a default-constructed mt19937_64
    g = O.MT19937_64()
    for _ in range(9999):
        g()
    assert g() == 9981545732273789042


def test_batch_radii_equal_single_radius_runs():
    rng = np.random.default_rng(1)
    L = np.array([1.0, 2.0])
    x = (rng.random((500, 2)) * L).ravel()
    radii = [0.02, 0.1, 0.3, 0.7]
    b = O.BatchPPS(x, L, radii, 9)
    b.run(50)
    for i, r in enumerate(radii):
        s = O.BatchPPS(x, L, [r], 9)
        s.run(50)
        assert s.mean()[0] == b.mean()[i] and s.variance()[0] == b.variance()[i]


@needs_ref
@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("radius", [0.03, 0.2, 0.7])
def test_window_moments_equal_reference(ndim, radius):
    rng = np.random.default_rng(ndim)
    L = np.array([1.0, 1.3, 0.8])[:ndim]
    n = {1: 400, 2: 1500, 3: 3000}[ndim]
    x = (rng.random((n, ndim)) * L - 0.3).ravel()  # some points outside the box
    ref = R.PointPatternStatistics(x, L, radius, 1234 + ndim)
    ref.run(120)
    o = O.BatchPPS(x, L, [radius], 1234 + ndim)
    o.run(120)
    m, v, c = ref.mean_var_count()
    assert c == 120 and m == o.mean()[0] and v == o.variance()[0]
    # reseeding restarts the stream
    ref.set_generator_seed(77)
    ref.run(30)
    o.gen.seed(77)
    o.run(30)
    m, v, c = ref.mean_var_count()
    assert c == 150 and m == o.mean()[0] and v == o.variance()[0]


@needs_ref
@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_overlap_sets_equal_reference(ndim):
    rng = np.random.default_rng(10 + ndim)
    L = np.array([1.0, 1.2, 0.9])[:ndim]
    n = {1: 300, 2: 2000, 3: 3000}[ndim]
    x = (rng.random((n, ndim)) * L).ravel()
    rad = rng.uniform(0.2, 1.0, n) * 0.5 * float(np.prod(L) / n) ** (1.0 / ndim)
    changed = rng.choice(n, 25, replace=False)
    for periodic, cells in [(True, False), (True, True), (False, False)]:
        if cells and ndim == 1:  # the reference's cell lists refuse one dimension (cell_lists.hpp:837-839)
            with pytest.raises(RuntimeError, match="more than 1 dimension"):
                R.overlapping_particles(rad, L, x, periodic=periodic, cell_lists=cells)
            continue
        a = R.overlapping_particles(rad, L, x, periodic=periodic, cell_lists=cells)
        b = O.overlapping_particles(x, rad, L, periodic=periodic)
        assert 0 < len(b) < n and np.array_equal(a, b), (periodic, cells)
        a = R.overlapping_particles(rad, L, x, periodic=periodic, cell_lists=cells, changed=changed)
        # with cell lists the reference passes no old coordinates, so it checks every pair
        # (check_overlap_cell_lists.hpp:128, 145-149)
        b = O.overlapping_particles(x, rad, L, periodic=periodic, changed=None if cells else changed)
        assert np.array_equal(a, b), (periodic, cells, "changed")
