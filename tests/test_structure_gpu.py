"""export_structure on the device against the oracle (exact type-1 sums, numpy FFT and radial profiles)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) <= tol * max(np.max(np.abs(b)), 1.0)


@pytest.mark.parametrize("ndim,N,Nk,radii,shift", [(2, 3000, 101, False, False), (2, 2000, 64, True, True),
                                                    (3, 600, 21, False, False), (3, 400, 16, True, False)])
def test_export_structure_matches_oracle(ndim, N, Nk, radii, shift):
    from fresco_b200.utils import export_structure

    rng = np.random.default_rng(ndim * 100 + Nk)
    L = 1.0 + rng.random(ndim) * 2.0
    x = rng.random((N, ndim)) * L
    if shift:  # coordinates beyond the box trigger the reference's -1/2 shift
        x[0, 0] = 1.2 * L[0]
    rad = 0.5 + rng.random(N) if radii else None
    got = export_structure(x.ravel(), L, Nk=Nk, radii=rad, tol=1e-12)
    ref = O.export_structure(x.ravel(), L, Nk=Nk, radii=rad)
    q, S, Sk, r, g, gr = got
    q0, S0, Sk0, r0, g0, gr0 = ref
    assert Sk.shape == Sk0.shape and gr.shape == gr0.shape
    np.testing.assert_array_equal(q, q0)
    np.testing.assert_allclose(r, r0)
    assert _close(Sk, Sk0, 1e-9)
    assert _close(gr, gr0, 1e-9)
    assert _close(S, S0, 1e-9)
    assert _close(g, g0, 1e-9)


def test_export_structure_alias_and_errors():
    import fresco_b200

    fresco_b200.install_alias()
    from fresco.utils import export_structure

    with pytest.raises(ValueError):
        export_structure(np.zeros(10), [1.0], Nk=8)
    x = np.full((5, 2), np.nan)
    with pytest.raises(ValueError):
        export_structure(x.ravel(), [1.0, 1.0], Nk=8)
