"""One NUwU pattern split over shards (fresco_b200.ShardedNUwU) against the oracle's exact sums.

One process drives every shard and sums their rho arrays itself, which is what the all-reduce does
across ranks: each shard sorts, spreads and transforms only its own points, and finishes with the
pattern's rho.  The energy must equal the whole pattern's on every shard and the shards' gradients,
concatenated, the whole pattern's gradient.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

PRECISIONS = [("fp64", 1e-12, 1e-10), ("fp32", 1e-6, 1e-5)]


def _pattern(ndim, N, K, seed):
    x, _, Sk, V, L = O.stealthy_nuwu_inputs(N, K, K - 1, ndim=ndim, seed=seed)
    rng = np.random.default_rng(seed + 7)
    radii = 0.5 + rng.random(N)
    V = V * (0.5 + rng.random(V.shape))
    Sk = np.where(rng.random(Sk.shape) < 0.3, 0.5 + rng.random(Sk.shape), 0.0)
    return x, radii, Sk, V, L


def _shards(x, radii, ndim, cuts):
    pts = x.reshape(-1, ndim)
    out = []
    for a, b in zip([0] + cuts, cuts + [len(radii)]):
        out.append((pts[a:b].ravel(), radii[a:b]))
    return out


@pytest.mark.parametrize("prec,eps,tol", PRECISIONS)
@pytest.mark.parametrize("ndim,N,K,cuts", [(2, 2000, 12, [700, 1500]), (3, 600, 4, [0, 250]), (1, 300, 20, [100])])
def test_shards_sum_to_the_pattern(prec, eps, tol, ndim, N, K, cuts):
    import torch

    from fresco_b200.shard import ShardedNUwU, weight_factor_sum

    x, radii, Sk, V, L = _pattern(ndim, N, K, seed=ndim + 40)
    e_ref, g_ref = O.NUwU(radii, K, Sk, V, L).get_energy_gradient(x)
    parts = _shards(x, radii, ndim, cuts)
    totals = (N, sum(weight_factor_sum(r, ndim) for _, r in parts))
    shards = [ShardedNUwU(r, K, Sk, V, L, eps=eps, precision=prec, totals=totals) for _, r in parts]
    rhos = [s.rho(torch.tensor(p, device="cuda")) for s, (p, _) in zip(shards, parts)]
    rho = torch.stack(rhos).sum(0)
    out = [s.finish(rho.clone()) for s in shards]
    es = [float(e.item()) for e, _ in out]
    g = np.concatenate([gg.cpu().numpy() for _, gg in out])
    for e in es:
        assert abs(e - e_ref) <= tol * abs(e_ref), (e, e_ref)
    assert np.linalg.norm(g - g_ref) <= tol * np.linalg.norm(g_ref)
    assert all(s.status() == 0 for s in shards)


def test_single_shard_matches_nuwu_and_rejects_partial_evaluation():
    """A shard holding every point is the pattern's NUwU; a partial shard refuses the plain call."""
    from fresco_b200 import NUwU
    from fresco_b200.shard import ShardedNUwU

    x, radii, Sk, V, L = _pattern(2, 1500, 128, seed=3)  # fine grid 512: NUwU takes the band transforms
    whole = ShardedNUwU(radii, 128, Sk, V, L, eps=1e-12)
    e, g = whole.get_energy_gradient(x)
    e_ref, g_ref = NUwU(radii, 128, Sk, V, L, eps=1e-12).get_energy_gradient(x)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-10 * np.linalg.norm(g_ref)
    assert abs(whole.get_energy(x) - e_ref) <= 1e-10 * abs(e_ref)
    with pytest.raises(ValueError):
        ShardedNUwU(radii, 128, Sk, V, L, totals=(10, 1.0))  # fewer points in total than in this shard


def test_nonfinite_coordinate_on_one_shard_reaches_every_shard():
    import torch

    from fresco_b200.shard import ShardedNUwU, weight_factor_sum

    x, radii, Sk, V, L = _pattern(2, 800, 10, seed=9)
    x = x.copy()
    x[5] = np.nan
    parts = _shards(x, radii, 2, [400])
    totals = (800, sum(weight_factor_sum(r, 2) for _, r in parts))
    shards = [ShardedNUwU(r, 10, Sk, V, L, totals=totals) for _, r in parts]
    rho = sum(s.rho(torch.tensor(p, device="cuda")) for s, (p, _) in zip(shards, parts))
    for s in shards:
        e, _ = s.finish(rho.clone())
        assert np.isnan(float(e.item()))
