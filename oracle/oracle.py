"""CPU oracle for the FReSCo loss-and-gradient path (test infrastructure only).

This module is a plain-numpy restatement of the reference's arithmetic, used
only by ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg, to check results against.  Nothing in the product package imports it.

Every transform here is an exact FP64 direct sum (a NUDFT), i.e. the quantity
FINUFFT approximates to tolerance ``eps``.  The glue around the transforms
(coordinate maps, mode ordering, weights, loss and gradient factors, and the
reference's quirks) follows the reference source line by line; each function
cites the file:line it restates.  All paths are relative to the reference
project root.

Parity pinning: the restatement is checked against golden vectors produced by
the reference's own C++ (``source/fresco/*.hpp``, ``source/lbfgs.cpp``,
``source/modified_fire.cpp``) compiled unchanged against this project's
FINUFFT/FFTW API shim (``oracle/Makefile``, ``tests/golden/make_golden.py``),
and the repulsion against the reference's own known answers
(``cpp_tests/source/test_inversepower.cpp:41-42``).
"""
from __future__ import annotations

import math

import numpy as np

TWO_PI = 2.0 * np.pi


# ---------------------------------------------------------------------------
# setup helpers
# ---------------------------------------------------------------------------

def modes_per_dim(v_size: int, ndim: int) -> int:
    """Odd mode count n = 2K+1 derived from len(V).

    Restates ``NUwU::calculate_Kvec`` (source/fresco/nuwu.hpp:54-79): K is the
    truncated ``(sqrt(len V) - 1)/2`` (cbrt in 3D); modes run -K..K.
    """
    if ndim == 1:
        k = int((v_size - 1) // 2)
    elif ndim == 2:
        k = int((math.sqrt(v_size) - 1) / 2)
    elif ndim == 3:
        k = int((np.cbrt(v_size) - 1) / 2)
    else:
        raise RuntimeError(f"Invalid dimension: {ndim}")
    return 2 * k + 1


def point_weights(radii, ndim: int) -> np.ndarray:
    """Point weights c_i, normalised so that sum(c) = N.

    Restates ``initialize_c`` (source/fresco/nuwu.hpp:125-149): the area (2D)
    or volume (3D) factor is multiplied in once per dimension (quirk kept),
    summed in index order, then every weight is scaled by N/sum.
    """
    radii = np.asarray(radii, dtype=np.float64)
    n = radii.size
    c = np.ones(n, dtype=np.float64)
    for _ in range(ndim):
        if ndim == 2:
            c = c * np.pi * radii * radii
        elif ndim == 3:
            c = c * np.pi * radii * radii * radii * 4.0 / 3.0
    s = 0.0
    for v in c:  # sequential sum, same order as the reference loop
        s += v
    return c * (n / s)


def coord_map(points, L, energy: bool) -> np.ndarray:
    """Per-dimension NUFFT coordinates of the points, shape (ndim, N).

    Restates the maps of source/fresco/nuwu.hpp:157-187 (energy:
    ``(p - round(p/L) + L) * 2pi/L``) and :216-250 (gradient:
    ``(p - round(p/L)) * 2pi/L``).  ``round(p/L)`` is not multiplied by L
    (quirk kept).  ``np.round`` rounds half to even while C's ``round`` rounds
    half away from zero, so C rounding is restated explicitly.
    """
    L = np.asarray(L, dtype=np.float64)
    ndim = L.size
    p = np.asarray(points, dtype=np.float64).reshape(-1, ndim)
    out = np.empty((ndim, p.shape[0]))
    for a in range(ndim):
        q = p[:, a] / L[a]
        r = np.sign(q) * np.floor(np.abs(q) + 0.5)  # C round(): half away from zero
        if energy:
            out[a] = (p[:, a] - r + L[a]) * TWO_PI / L[a]
        else:
            out[a] = (p[:, a] - r) * TWO_PI / L[a]
    return out


def mode_values(n: int) -> np.ndarray:
    """Integer mode values in FINUFFT's default (modeord=0) order: -floor(n/2) ..."""
    return np.arange(n) - n // 2


# ---------------------------------------------------------------------------
# exact transforms (what FINUFFT approximates)
# ---------------------------------------------------------------------------

def _phase(k, x, iflag):
    return np.exp(1j * iflag * np.outer(x, k))  # (N, n)


def nudft1(x, c, n_modes, iflag):
    """Type 1: f[k] = sum_j c_j exp(iflag i k.x_j); output flat with dim 0 fastest."""
    ndim = len(n_modes)
    c = np.asarray(c, dtype=np.complex128)
    e = [_phase(mode_values(n_modes[a]), x[a], iflag) for a in range(ndim)]
    if ndim == 1:
        f = c @ e[0]
    elif ndim == 2:
        f = np.einsum("j,jx,jy->yx", c, e[0], e[1], optimize=True)
    else:
        f = np.einsum("j,jx,jy,jz->zyx", c, e[0], e[1], e[2], optimize=True)
    return f.reshape(-1)


def nudft2(x, f, n_modes, iflag):
    """Type 2: c_j = sum_k f[k] exp(iflag i k.x_j); f flat with dim 0 fastest."""
    ndim = len(n_modes)
    e = [_phase(mode_values(n_modes[a]), x[a], iflag) for a in range(ndim)]
    f = np.asarray(f, dtype=np.complex128).reshape(tuple(reversed(n_modes)))
    if ndim == 1:
        return e[0] @ f
    if ndim == 2:
        a = e[0] @ f.T  # (N, ny)
        return np.sum(a * e[1], axis=1)
    a = np.einsum("jx,zyx->jzy", e[0], f, optimize=True)
    a = np.einsum("jzy,jy->jz", a, e[1], optimize=True)
    return np.sum(a * e[2], axis=1)


def nudft3(x, c, s, iflag):
    """Type 3: f_k = sum_j c_j exp(iflag i s_k.x_j); x (ndim,N), s (ndim,M)."""
    ph = np.zeros((x.shape[1], s.shape[1]))
    for a in range(x.shape[0]):
        ph += np.outer(x[a], s[a])
    return np.asarray(c, dtype=np.complex128) @ np.exp(1j * iflag * ph)


# ---------------------------------------------------------------------------
# loss pieces
# ---------------------------------------------------------------------------

def _loss_terms(absrho2_over_norm, sk0, v):
    """d = (S - S0)/S0' and phi, S0' = S0 where S0 != 0 else 1 (nuwu.hpp:262-271)."""
    d = absrho2_over_norm - sk0
    nz = sk0 != 0
    d = np.where(nz, d / np.where(nz, sk0, 1.0), d)
    phi = float(np.sum(v * d * d))
    return d, phi


class NUwU:
    """Points -> uniform k-grid loss (source/fresco/nuwu.hpp:17-318)."""

    def __init__(self, radii, K, Sk, V, L, eps=1e-6):
        self.L = np.asarray(L, dtype=np.float64)
        self.ndim = self.L.size
        self.Sk = np.asarray(Sk, dtype=np.float64).ravel()
        self.V = np.asarray(V, dtype=np.float64).ravel()
        assert len(self.Sk) == len(self.V)  # nuwu.pyx:17
        self.N = len(radii)
        self.n = modes_per_dim(self.V.size, self.ndim)
        self.nm = self.n ** self.ndim
        self.c = point_weights(radii, self.ndim)
        self.kvec = mode_values(self.n)

    def rho(self, points, energy=False):
        x = coord_map(points, self.L, energy)
        return nudft1(x, self.c, [self.n] * self.ndim, +1)  # iflag +1, nuwu.hpp:50

    def get_energy(self, points):
        """nuwu.hpp:152-208."""
        rho = self.rho(points, energy=True)
        _, phi = _loss_terms(np.abs(rho) ** 2 / self.N, self.Sk[: self.nm], self.V[: self.nm])
        return phi

    def get_energy_gradient(self, points):
        """nuwu.hpp:210-317: type 1, mode loop, d type-2 transforms (iflag -1)."""
        x = coord_map(points, self.L, energy=False)
        n = self.n
        rho = nudft1(x, self.c, [n] * self.ndim, +1)
        sk0 = self.Sk[: self.nm]
        v = self.V[: self.nm]
        d, phi = _loss_terms(np.abs(rho) ** 2 / self.N, sk0, v)
        factor = (4.0 / self.N) * v * d * rho
        factor = np.where(sk0 != 0, factor / np.where(sk0 != 0, sk0, 1.0), factor)
        idx = np.arange(self.nm)
        comps = [self.kvec[idx % n]]
        if self.ndim == 2:
            comps.append(self.kvec[idx // n])
        elif self.ndim == 3:
            comps.append(self.kvec[(idx % (n * n)) // n])
            comps.append(self.kvec[idx // (n * n)])
        grad = np.zeros(self.N * self.ndim)
        for a, ka in enumerate(comps):
            fa = ka * factor * (-1j)
            cx = nudft2(x, fa, [n] * self.ndim, -1)
            grad[a :: self.ndim] = np.real(cx * np.conj(self.c))
        return phi, grad

    def active_modes(self):
        """Flat indices of the modes with V != 0 and their integer k, shape (ndim, A)."""
        n = self.n
        act = np.nonzero(self.V[: self.nm])[0]
        comps = [self.kvec[act % n]]
        if self.ndim >= 2:
            comps.append(self.kvec[(act // n) % n])
        if self.ndim == 3:
            comps.append(self.kvec[act // (n * n)])
        return act, np.stack(comps).astype(np.float64)

    def get_energy_gradient_active(self, points, chunk=1 << 15):
        """``get_energy_gradient`` summed over the modes with V != 0 only (still exact).

        A mode with V = 0 adds nothing to phi (nuwu.hpp:270) and its residual
        factor (nuwu.hpp:273-276) is zero, so it drops out of the d type-2
        transforms (nuwu.hpp:291-315).  Restricting the sums to the active
        modes gives the same energy and gradient in O(N * active) work, which
        keeps full-size point sets (N ~ 10^6) checkable when V is sparse.
        The gradient map (nuwu.hpp:216-250) is used for rho, as in
        get_energy_gradient.
        """
        rho = self.rho_active(points, self.c, chunk)
        return self.finish_active(rho, points, self.c, self.N, chunk)

    def rho_active(self, points, c, chunk=1 << 15):
        """rho at the active modes of the points `points` with weights `c` (gradient map).  It is
        linear in the points: the values of disjoint point sets add up to that of their union."""
        x = coord_map(points, self.L, energy=False)  # (ndim, n)
        _, kk = self.active_modes()
        rho = np.zeros(kk.shape[1], dtype=np.complex128)
        for s in range(0, x.shape[1], chunk):
            ph = x[:, s : s + chunk].T @ kk
            rho += np.asarray(c[s : s + chunk]) @ np.exp(1j * ph)
        return rho

    def finish_active(self, rho, points, c, n_total, chunk=1 << 15):
        """phi of the active modes from rho (nuwu.hpp:260-287, S = |rho|^2 / n_total) and the
        gradient at the points `points` with weights `c` (nuwu.hpp:291-315)."""
        x = coord_map(points, self.L, energy=False)
        act, kk = self.active_modes()
        sk0 = self.Sk[: self.nm][act]
        v = self.V[: self.nm][act]
        d, phi = _loss_terms(np.abs(rho) ** 2 / n_total, sk0, v)
        factor = (4.0 / n_total) * v * d * rho
        factor = np.where(sk0 != 0, factor / np.where(sk0 != 0, sk0, 1.0), factor)
        fa = (-1j * kk * factor[None, :]).T  # (A, ndim): -i k_a F(k)
        n = x.shape[1]
        grad = np.zeros(n * self.ndim)
        g = grad.reshape(-1, self.ndim)
        for s in range(0, n, chunk):
            e = np.exp(-1j * (x[:, s : s + chunk].T @ kk))  # iflag -1
            cx = e @ fa  # (chunk, ndim)
            g[s : s + chunk] = np.real(cx * np.conj(np.asarray(c[s : s + chunk]))[:, None])
        return phi, grad


class UwU:
    """Uniform grid -> uniform k-grid loss (source/fresco/uwu.hpp:17-195).

    ``Sk`` and ``V`` are given centred (fftshift order) and ifftshifted as in
    fresco/potentials/uwu.pyx:14-15.  Grid flattening is row-major (FFTW
    convention, uwu.hpp:48-49).
    """

    def __init__(self, N, K, Sk, V, L, eps=1e-6):
        self.shape = tuple(int(v) for v in np.asarray(N).ravel())
        self.L = np.asarray(L, dtype=np.float64)
        self.Sk = np.fft.ifftshift(np.asarray(Sk, dtype=np.float64)).ravel()
        self.V = np.fft.ifftshift(np.asarray(V, dtype=np.float64)).ravel()
        assert len(self.Sk) == len(self.V)

    def _rho(self, points):
        x = np.asarray(points, dtype=np.float64).reshape(self.shape)
        # FFTW sign +1, unnormalised: n * ifftn
        rho = np.fft.ifftn(x) * x.size
        return x, rho.ravel(), float(np.sum(x))

    def get_energy(self, points):
        _, rho, rtot = self._rho(points)
        _, phi = _loss_terms(np.abs(rho) ** 2 / rtot, self.Sk, self.V)
        return phi

    def get_energy_gradient(self, points):
        """uwu.hpp:152-194 (f = 2/R V d rho / S0'; grad = Re FFT_-(f))."""
        _, rho, rtot = self._rho(points)
        d, phi = _loss_terms(np.abs(rho) ** 2 / rtot, self.Sk, self.V)
        f = 2.0 / rtot * self.V * d * rho
        f = np.where(self.Sk != 0, f / np.where(self.Sk != 0, self.Sk, 1.0), f)
        g = np.fft.fftn(f.reshape(self.shape))  # sign -1, unnormalised
        return phi, np.real(g).ravel()


class UwNU:
    """Uniform grid -> non-uniform k-points (source/fresco/uwnu.hpp:17-158)."""

    def __init__(self, N, K, Sk, V, L, eps=1e-6):
        self.L = np.asarray(L, dtype=np.float64)
        self.ndim = self.L.size
        self.N = [int(v) for v in np.asarray(N).ravel()]
        Kf = np.asarray(K, dtype=np.float64).ravel()
        self.Sk = np.asarray(Sk, dtype=np.float64).ravel()
        self.V = np.asarray(V, dtype=np.float64).ravel()
        assert len(self.Sk) == len(self.V)
        nk = self.Sk.size
        # uwnu.hpp:243-276: k~ = K * 2pi / L per dim
        self.kt = np.stack([Kf[a :: self.ndim][:nk] * TWO_PI / self.L[a] for a in range(self.ndim)])

    def get_energy(self, points):
        rho = nudft2(self.kt, points, self.N[: self.ndim], +1)  # type 2, iflag +1
        _, phi = _loss_terms(np.abs(rho) ** 2, self.Sk, self.V)  # rhotot == 1
        return phi

    def get_energy_gradient(self, points):
        """uwnu.hpp:314-355: f = 4 V d rho/S0', grad = Re(type1_-(f))/(2 pi)."""
        rho = nudft2(self.kt, points, self.N[: self.ndim], +1)
        d, phi = _loss_terms(np.abs(rho) ** 2, self.Sk, self.V)
        f = 4.0 * self.V * d * rho
        f = np.where(self.Sk != 0, f / np.where(self.Sk != 0, self.Sk, 1.0), f)
        c = nudft1(self.kt, f, self.N[: self.ndim], -1)
        return phi, np.real(c) / TWO_PI

    def get_energy_gradient_active(self, points):
        """``get_energy_gradient`` over the k-points with V != 0 only (2D, exact).

        k-points with V = 0 add nothing to phi and have a zero residual
        f = 4 V d rho / S0' (uwnu.hpp:314-349), so they drop out of the
        type-1 transform back to the grid (uwnu.hpp:350-355).  The sums over
        the grid are separable, exp(i (k0 m0 + k1 m1)) = exp(i k0 m0)
        exp(i k1 m1), so rho and the gradient are two matrix products each:
        O(G * active) work for a full-size grid.
        """
        if self.ndim != 2:
            raise ValueError("active-k-point sums are written for 2D grids")
        act = np.nonzero(self.V)[0]
        k0, k1 = self.kt[0][act], self.kt[1][act]
        m0, m1 = mode_values(self.N[0]), mode_values(self.N[1])
        grid = np.asarray(points, dtype=np.float64).reshape(self.N[1], self.N[0])  # dim 0 fastest
        b = grid @ np.exp(1j * np.outer(m0, k0))  # (N1, A), iflag +1
        rho = np.sum(b * np.exp(1j * np.outer(m1, k1)), axis=0)
        sk0, v = self.Sk[act], self.V[act]
        d, phi = _loss_terms(np.abs(rho) ** 2, sk0, v)
        f = 4.0 * v * d * rho
        f = np.where(sk0 != 0, f / np.where(sk0 != 0, sk0, 1.0), f)
        c = (np.exp(-1j * np.outer(m1, k1)) * f[None, :]) @ np.exp(-1j * np.outer(k0, m0))  # iflag -1
        return phi, np.real(c).ravel() / TWO_PI


class NUwNU:
    """Points -> non-uniform k-points (source/fresco/nuwnu.hpp:17-291)."""

    def __init__(self, radii, K, Sk, V, L, eps=1e-6):
        self.L = np.asarray(L, dtype=np.float64)
        self.ndim = self.L.size
        self.Sk = np.asarray(Sk, dtype=np.float64).ravel()
        self.V = np.asarray(V, dtype=np.float64).ravel()
        assert len(self.Sk) == len(self.V)
        self.N = len(radii)
        Kf = np.asarray(K, dtype=np.float64).ravel()
        self.nk = Kf.size // self.ndim
        # nuwnu.hpp:47-76: frequencies used as given (no 2pi/L scaling)
        self.s = np.stack([Kf[a :: self.ndim][: self.nk] for a in range(self.ndim)])
        self.c = point_weights(radii, self.ndim)

    def get_energy(self, points):
        x = coord_map(points, self.L, energy=True)
        rho = nudft3(x, self.c, self.s, +1)
        _, phi = _loss_terms(np.abs(rho) ** 2 / self.N, self.Sk[: self.nk], self.V[: self.nk])
        return phi

    def get_energy_gradient(self, points):
        """nuwnu.hpp:184-289; the energy map is used here too, and conj(c) is omitted (:269)."""
        x = coord_map(points, self.L, energy=True)
        rho = nudft3(x, self.c, self.s, +1)
        sk0 = self.Sk[: self.nk]
        v = self.V[: self.nk]
        d, phi = _loss_terms(np.abs(rho) ** 2 / self.N, sk0, v)
        factor = (-4.0j / self.N) * v * d * rho
        factor = np.where(sk0 != 0, factor / np.where(sk0 != 0, sk0, 1.0), factor)
        grad = np.zeros(self.N * self.ndim)
        for a in range(self.ndim):
            # type 3 from k-points back to the points, iflag -1
            cx = nudft3(self.s, self.s[a] * factor, x, -1)
            grad[a :: self.ndim] = np.real(cx)
        return phi, grad


# ---------------------------------------------------------------------------
# soft-sphere repulsion
# ---------------------------------------------------------------------------

def _round_half_even(v):
    return np.round(v)  # round_fast rounds half to even (distance.hpp:32-36)


class InversePower:
    """E = sum_{i<j, r<d_ij} eps/a (1 - r/d_ij)^a with d_ij = r_i + r_j.

    Restates InversePowerInteraction::energy_gradient
    (source/fresco/inversepower_potential.hpp:44-58), the pair accumulator
    (source/fresco/cell_list_potential.hpp:154-181) and the min-image rule
    (source/fresco/distance.hpp:179, round_fast :32-36) as an O(N^2) sum,
    which the cell list reproduces exactly (cpp_tests test_cell_lists.cpp:317-332).
    """

    def __init__(self, a, eps, radii, boxv, use_cell_lists=False, ncellx_scale=None,
                 balance_omp=True, method="periodic"):
        self.a = float(a)
        self.eps = float(eps)
        self.radii = np.asarray(radii, dtype=np.float64)
        self.boxv = np.asarray(boxv, dtype=np.float64)
        self.ndim = self.boxv.size
        self.periodic = str(method).lower().endswith("periodic")

    def _pairs(self, x):
        x = np.asarray(x, dtype=np.float64).reshape(-1, self.ndim)
        n = x.shape[0]
        i, j = np.triu_indices(n, k=1)
        # get_rij(r_ij, r_i, r_j) = r_i - r_j with min image (meta_periodic_distance)
        dr = x[i] - x[j]
        if self.periodic:
            dr = dr - _round_half_even(dr / self.boxv) * self.boxv
        return i, j, dr

    def get_energy_gradient(self, x):
        x = np.asarray(x, dtype=np.float64)
        if not (np.isfinite(x[0]) and np.isfinite(x[-1])):  # cell_list_potential.hpp:452-455
            return float("nan"), np.full(x.size, np.nan)
        i, j, dr = self._pairs(x)
        r2 = np.sum(dr * dr, axis=1)
        rs = self.radii[i] + self.radii[j]
        m = r2 < rs * rs
        r = np.sqrt(r2[m])
        rsm = rs[m]
        factor = np.power(1.0 - r / rsm, self.a) * self.eps
        e = float(np.sum(factor / self.a))
        gij = -factor / ((r - rsm) * r)
        g = np.zeros_like(x).reshape(-1, self.ndim)
        contrib = dr[m] * gij[:, None]
        np.add.at(g, i[m], -contrib)
        np.add.at(g, j[m], contrib)
        return e, g.ravel()

    def get_energy(self, x):
        return self.get_energy_gradient(x)[0]

    def get_energy_gradient_tree(self, x):
        """The same pair sum with the candidate pairs found by a k-d tree (scipy).

        Only pairs closer than twice the largest radius can interact, so
        searching them with scipy's ``cKDTree`` (periodic ``boxsize`` for the
        periodic box) leaves the O(N^2) restatement above unchanged in value
        (summation order aside) and makes N ~ 10^6 checkable.  The pair
        vectors and the min-image rule are those of ``_pairs``.
        """
        from scipy.spatial import cKDTree

        x = np.asarray(x, dtype=np.float64)
        if not (np.isfinite(x[0]) and np.isfinite(x[-1])):
            return float("nan"), np.full(x.size, np.nan)
        p = x.reshape(-1, self.ndim)
        if self.periodic:
            w = p - np.floor(p / self.boxv) * self.boxv
            w = np.where((w >= self.boxv) | (w < 0), 0.0, w)
            tree = cKDTree(w, boxsize=self.boxv)
        else:
            tree = cKDTree(p)
        ij = tree.query_pairs(2.0 * float(np.max(self.radii)) * (1 + 1e-9), output_type="ndarray")
        i, j = ij[:, 0], ij[:, 1]
        dr = p[i] - p[j]
        if self.periodic:
            dr = dr - _round_half_even(dr / self.boxv) * self.boxv
        r2 = np.sum(dr * dr, axis=1)
        rs = self.radii[i] + self.radii[j]
        m = r2 < rs * rs
        r = np.sqrt(r2[m])
        rsm = rs[m]
        factor = np.power(1.0 - r / rsm, self.a) * self.eps
        e = float(np.sum(factor / self.a))
        gij = -factor / ((r - rsm) * r)
        contrib = dr[m] * gij[:, None]
        n = p.shape[0]
        g = np.stack([np.bincount(i[m], -contrib[:, a], minlength=n) + np.bincount(j[m], contrib[:, a], minlength=n)
                      for a in range(self.ndim)], axis=1)
        return e, g.ravel()


class CombinedPotential:
    """Sum of potentials (source/fresco/combine_potentials.hpp:16-59)."""

    def __init__(self):
        self.pots = []

    def add_potential(self, p):
        self.pots.append(p)

    def get_energy(self, x):
        return float(sum(p.get_energy(x) for p in self.pots))

    def get_energy_gradient(self, x):
        e = 0.0
        g = np.zeros(np.asarray(x).size)
        for p in self.pots:
            ei, gi = p.get_energy_gradient(x)
            e += ei
            g += np.asarray(gi)
        return e, g


# ---------------------------------------------------------------------------
# optimisers
# ---------------------------------------------------------------------------

class LBFGS:
    """Restates source/lbfgs.cpp:9-258 and source/fresco/optimizer.hpp:55-241."""

    def __init__(self, x0, pot, tol=1e-5, M=4, maxstep=0.1, maxErise=1e-4, H0=0.1,
                 nsteps=10000, rel_energy=False):
        self.pot = pot
        self.x = np.array(x0, dtype=np.float64)
        self.n = self.x.size
        self.tol, self.M, self.maxstep, self.maxErise = tol, M, maxstep, maxErise
        self.H0 = H0
        self.maxiter = nsteps
        self.rel = rel_energy
        self.s = np.zeros((M, self.n))
        self.y = np.zeros((M, self.n))
        self.rho = np.zeros(M)
        self.k = 0
        self.iter = 0
        self.nfev = 0
        self.f = 0.0
        self.g = np.zeros(self.n)
        self.rms = 1e10
        self.init = False

    def _eval(self, x):
        self.nfev += 1
        f, g = self.pot.get_energy_gradient(x)
        return float(f), np.array(g, dtype=np.float64)

    def _initialize(self):
        self.f, self.g = self._eval(self.x)
        self.rms = math.sqrt(float(self.g @ self.g) / self.n)
        self.init = True

    def stop_criterion_satisfied(self):
        if not self.init:
            self._initialize()
        return self.rms <= self.tol

    def _step(self):
        g = self.g
        if self.k == 0:  # lbfgs.cpp:109-124
            gnorm = math.sqrt(float(g @ g))
            if gnorm > 1.0:
                gnorm = 1.0 / gnorm
            return -gnorm * self.H0 * g
        step = g.copy()
        jmin, jmax = max(0, self.k - self.M), self.k
        alpha = np.zeros(self.M)
        for j in range(jmax - 1, jmin - 1, -1):
            i = j % self.M
            alpha[i] = self.rho[i] * float(self.s[i] @ step)
            step -= alpha[i] * self.y[i]
        step *= -self.H0
        for j in range(jmin, jmax):
            i = j % self.M
            beta = -self.rho[i] * float(self.y[i] @ step)
            step -= self.s[i] * (alpha[i] - beta)
        return step

    def one_iteration(self):
        if not self.init:
            self._initialize()
        xold, gold = self.x.copy(), self.g.copy()
        step = self._step()
        if float(step @ self.g) > 0.0:  # lbfgs.cpp:177-189
            step = -step
        factor = 1.0
        stepnorm = math.sqrt(float(step @ step))
        if factor * stepnorm > self.maxstep:
            factor = self.maxstep / stepnorm
        for _ in range(10):  # lbfgs.cpp:199-229
            self.x = xold + factor * step
            fnew, self.g = self._eval(self.x)
            df = fnew - self.f
            if self.rel:
                df /= abs(self.f) if self.f != 0 else 1e-100
            if df < self.maxErise:
                break
            factor *= 0.5
        self.f = fnew
        self.rms = math.sqrt(float(self.g @ self.g)) / math.sqrt(self.n)
        # update_memory, lbfgs.cpp:66-105
        kl = self.k % self.M
        self.y[kl] = self.g - gold
        self.s[kl] = self.x - xold
        ys = float(self.y[kl] @ self.s[kl])
        yy = float(self.y[kl] @ self.y[kl])
        if ys == 0.0:
            ys = 1.0
        self.rho[kl] = 1.0 / ys
        if yy == 0.0:
            yy = 1.0
        self.H0 = ys / yy
        self.k += 1
        self.iter += 1

    def run(self, niter=None):
        if not self.init:
            self._initialize()
        if niter is None:
            niter = self.maxiter - self.iter
        for _ in range(niter):
            if self.stop_criterion_satisfied():
                break
            self.one_iteration()
        return self.x


class ModifiedFire:
    """Restates source/fresco/modified_fire.hpp:84-230 and source/modified_fire.cpp:43-118."""

    def __init__(self, x0, pot, dtstart=0.1, dtmax=1.0, maxstep=0.5, Nmin=5, finc=1.1,
                 fdec=0.5, fa=0.99, astart=0.1, tol=1e-3, stepback=True, nsteps=10000):
        self.pot = pot
        self.x = np.array(x0, dtype=np.float64)
        self.N = self.x.size
        self.dtstart = self.dt = dtstart
        self.dtmax, self.maxstep, self.Nmin = dtmax, maxstep, Nmin
        self.finc, self.fdec, self.fa = finc, fdec, fa
        self.astart = self.a = astart
        self.tol, self.stepback = tol, stepback
        self.maxiter = nsteps
        self.v = np.zeros(self.N)
        self.g = np.zeros(self.N)
        self.f = 0.0
        self.fold = 0.0
        self.xold = self.x.copy()
        self.gold = self.g.copy()
        self.fire_iter = 0
        self.iter = 0
        self.nfev = 0
        self.rms = 1e10
        self.init = False
        self.ifnorm = 0.0
        self.vnorm = 0.0

    def _initialize(self):
        self.nfev += 1
        f, g = self.pot.get_energy_gradient(self.x)
        self.f, self.g = float(f), np.array(g, dtype=np.float64)
        self.fold = self.f
        self.v = -self.g * self.dt
        gnorm = float(self.g @ self.g)
        self.ifnorm = 1.0 / math.sqrt(gnorm)
        self.vnorm = math.sqrt(float(self.v @ self.v))
        self.rms = 1.0 / (self.ifnorm * math.sqrt(self.N))
        self.init = True

    def stop_criterion_satisfied(self):
        if not self.init:
            self._initialize()
        return self.rms <= self.tol

    def one_iteration(self):
        # modified_fire.hpp:160-178 does not initialise f and g here (LBFGS
        # does, lbfgs.cpp:38-40): before run() it steps from f = 0, g = 0.
        self.nfev += 1
        self.iter += 1
        self.fire_iter += 1
        self.fold = self.f
        self.xold = self.x.copy()
        self.v = (1.0 - self.a) * self.v - self.a * self.g * self.ifnorm * self.vnorm
        # forward Euler, modified_fire.hpp:136-158
        self.v = self.v - self.dt * self.g
        dx = self.dt * self.v
        self.gold = self.g.copy()
        normdx = math.sqrt(float(dx @ dx))
        factor = 1.0
        if normdx > self.maxstep:
            factor = self.maxstep / normdx
        self.x = self.x + dx * factor
        f, g = self.pot.get_energy_gradient(self.x)
        self.f, self.g = float(f), np.array(g, dtype=np.float64)
        P = -float(self.v @ self.g)
        if P > 0:
            if self.fire_iter > self.Nmin:
                self.dt = min(self.dt * self.finc, self.dtmax)
                self.a *= self.fa
            gnorm = float(self.g @ self.g)
            self.vnorm = math.sqrt(float(self.v @ self.v))
            self.ifnorm = 1.0 / math.sqrt(gnorm)
            self.rms = 1.0 / (self.ifnorm * math.sqrt(self.N))
        else:
            self.dt *= self.fdec
            self.a = self.astart
            self.fire_iter = 0
            self.v = np.zeros(self.N)
            if self.stepback:
                self.f = self.fold
                self.x = self.xold
                self.g = self.gold

    def run(self, niter=None):
        if not self.init:
            self._initialize()
        if niter is None:
            niter = self.maxiter - self.iter
        for _ in range(niter):
            if self.stop_criterion_satisfied():
                break
            self.one_iteration()
        return self.x


# ---------------------------------------------------------------------------
# seeded workloads
# ---------------------------------------------------------------------------

def stealthy_nuwu_inputs(N, K, kmax, ndim=2, seed=1, L=None, radius=1.0):
    """Uniform points in [0, L)^d and a stealthy target S0=0, V=1 for 0<|k|<=kmax."""
    rng = np.random.default_rng(seed)
    if L is None:
        L = np.full(ndim, TWO_PI)
    L = np.asarray(L, dtype=np.float64)
    x = (rng.random((N, ndim)) * L).ravel()
    kv = np.arange(-K, K + 1)
    grids = np.meshgrid(*([kv] * ndim), indexing="ij")
    kmag = np.sqrt(sum(g.astype(np.float64) ** 2 for g in grids))
    V = ((kmag <= kmax) & (kmag > 0)).astype(np.float64)
    Sk = np.zeros_like(V)
    radii = np.full(N, radius)
    return x, radii, Sk, V, L


# ---------------------------------------------------------------------------
# structure measurement (fresco/utils/utils.py:16-52, 138-152), exact sums
# ---------------------------------------------------------------------------

def radial_profile(data, center=None):
    """utils.py:138-152: mean over integer radii int(|idx - center|), radii > R = shape[0]/2 pooled and dropped."""
    data = np.asarray(data)
    ndim = data.ndim
    R = int(data.shape[0] / 2)
    if center is None:
        center = np.array(data.shape) / 2
    center = np.asarray(center)
    for _ in range(ndim):
        center = np.expand_dims(center, axis=-1)
    idx = np.indices(data.shape)
    r = np.sqrt(np.sum((idx - center) ** 2, axis=0)).astype(int)
    r = np.where(r <= R, r, R + 1)
    tbin = np.bincount(r.ravel(), data.ravel())
    nr = np.bincount(r.ravel())
    return np.unique(r).ravel()[:-1], (tbin / nr)[:-1]


def export_structure(r, L, Nk=1001, radii=None):
    """utils.py:16-52 with the type-1 transform as an exact sum (finufft.nufft{2,3}d1, isign +1)."""
    ndim = len(L)
    LL = np.asarray(L, dtype=np.float64).reshape(1, -1)
    rr = np.array(r, dtype=np.float64).reshape(-1, ndim) / LL
    if np.amax(rr) > 1:
        rr -= 0.5
    rr *= TWO_PI
    N = rr.shape[0]
    if radii is None:
        c = np.ones(N)
    else:
        radii = np.asarray(radii, dtype=np.float64)
        c = np.pi * radii ** 2 if ndim == 2 else 4.0 / 3.0 * np.pi * radii ** 3
        c = c * (N / np.sum(c))
    f = nudft1([rr[:, a] for a in range(ndim)], c, [Nk] * ndim, +1)
    rho = f.reshape((Nk,) * ndim).transpose(tuple(range(ndim))[::-1])  # -> [k0, k1, (k2)]
    Sk = np.abs(rho) ** 2 / N
    gr = np.fft.ifftn(np.fft.ifftshift(Sk) - 1.0, (Nk,) * ndim)
    gr = np.real(np.fft.fftshift(gr)) * (Nk ** ndim) * np.prod(L) / N
    center = int(Nk / 2)
    q, S = radial_profile(Sk, center=[center] * ndim)
    rq, g = radial_profile(gr, center=[center] * ndim)
    return q, S, Sk, rq / Nk, g, gr


# ---------------------------------------------------------------------------
# point-pattern statistics and overlap checks
# ---------------------------------------------------------------------------

class MT19937_64:
    """The 64-bit Mersenne Twister of the C++ standard ([rand.eng.mers], std::mt19937_64:
    w=64, n=312, m=156, r=31; Matsumoto & Nishimura), with its integer seeding.  The reference draws
    its window centres from it (point_pattern_statistics.hpp:45, 72-77)."""

    _N, _M = 312, 156
    _A = 0xB5026F5AA96619E9
    _UPPER, _LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF
    _MASK = (1 << 64) - 1

    def __init__(self, seed=5489):
        self.seed(seed)

    def seed(self, s):
        mt = [int(s) & self._MASK]
        for i in range(1, self._N):
            prev = mt[-1]
            mt.append((6364136223846793005 * (prev ^ (prev >> 62)) + i) & self._MASK)
        self._mt = mt
        self._i = self._N

    def _twist(self):
        mt, n, m = self._mt, self._N, self._M
        for i in range(n):
            y = (mt[i] & self._UPPER) | (mt[(i + 1) % n] & self._LOWER)
            mt[i] = mt[(i + m) % n] ^ (y >> 1) ^ (self._A if y & 1 else 0)
        self._i = 0

    def __call__(self):
        if self._i >= self._N:
            self._twist()
        y = self._mt[self._i]
        self._i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & self._MASK


def uniform_real(gen, a, b):
    """std::uniform_real_distribution<double>(a, b)(gen) for a 64-bit engine as libstdc++ computes it:
    generate_canonical<double, 53> takes one draw, u = double(draw) / 2^64 (u = 1 becomes the largest
    double below 1), then u * (b - a) + a."""
    u = float(gen()) / 18446744073709551616.0
    if u >= 1.0:
        u = np.nextafter(1.0, 0.0)
    return u * (b - a) + a


def window_centres(gen, boxv, n):
    """n window centres, in the reference's draw order (point_pattern_statistics.hpp:72-77)."""
    boxv = [float(v) for v in np.asarray(boxv, dtype=np.float64).ravel()]
    out = np.empty((n, len(boxv)))
    for k in range(n):
        for a, L in enumerate(boxv):
            out[k, a] = uniform_real(gen, 0.0, L) - L / 2
    return out


def periodic_dist2(r1, r2, boxv):
    """|r1 - r2|^2 with periodic_distance::get_rij (distance.hpp:170-192; ibox = 1 / L, round half to even)
    and the dot from 0 in axis order (vecN.hpp:283-291), every operation rounded on its own."""
    boxv = np.asarray(boxv, dtype=np.float64)
    d = np.asarray(r1, dtype=np.float64) - np.asarray(r2, dtype=np.float64)
    ibox = 1.0 / boxv
    d = d - np.rint(d * ibox) * boxv
    s = np.zeros(d.shape[:-1])
    for a in range(d.shape[-1]):
        s = s + d[..., a] * d[..., a]
    return s


class Moments:
    """moments.hpp:28-52: running means of x and x^2; variance = E[x^2] - E[x]^2."""

    def __init__(self):
        self.mean = 0.0
        self.mean2 = 0.0
        self.count = 0

    def update(self, v):
        v = float(v)
        self.mean = (self.mean * float(self.count) + v) / float(self.count + 1)
        self.mean2 = (self.mean2 * float(self.count) + v * v) / float(self.count + 1)
        self.count += 1

    def variance(self):
        return self.mean2 - self.mean * self.mean


def window_counts(coords, boxv, radii, centres):
    """Number of points within each radius of each centre: counts[k, i] = #{j : dist2(c_k, x_j) <= r_i^2}
    (point_pattern_statistics.hpp:78-90; batch_pointstats.hpp:82-118 cumulated over sorted radii)."""
    boxv = np.asarray(boxv, dtype=np.float64)
    x = np.asarray(coords, dtype=np.float64).reshape(-1, boxv.size)
    r2 = np.asarray(radii, dtype=np.float64) ** 2
    out = np.empty((len(centres), r2.size), dtype=np.int64)
    for k, c in enumerate(centres):
        d2 = periodic_dist2(c[None, :], x, boxv)
        out[k] = (d2[:, None] <= r2[None, :]).sum(axis=0)
    return out


class BatchPPS:
    """PointPatternStatistics / BatchPPS restated (point_pattern_statistics.hpp:36-111,
    batch_pointstats.hpp:29-150) without the reference's data race on the shared counter
    (point_pattern_statistics.hpp:82-89) and with its uninitialised loop counters read as 0
    (batch_pointstats.hpp:50, 76, 130, 139, 148)."""

    def __init__(self, coords, boxv, radii, rseed):
        self.coords = np.asarray(coords, dtype=np.float64)
        self.boxv = np.asarray(boxv, dtype=np.float64)
        self.radii = np.atleast_1d(np.asarray(radii, dtype=np.float64))
        self.gen = MT19937_64(rseed)
        self.moments = [Moments() for _ in self.radii]

    def run(self, n):
        centres = window_centres(self.gen, self.boxv, n)
        counts = window_counts(self.coords, self.boxv, self.radii, centres)
        for k in range(n):
            for i, m in enumerate(self.moments):
                m.update(counts[k, i])
        return counts

    def mean(self):
        return np.array([m.mean for m in self.moments])

    def variance(self):
        return np.array([m.variance() for m in self.moments])


def overlapping_particles(coords, radii, boxv, periodic=True, changed=None):
    """Sorted indices i with |r_ij|^2 < (r_i + r_j)^2 for some j != i (check_overlap.hpp:53-101); with
    changed atoms only the pairs (i changed, any j != i) count, and both members are reported."""
    boxv = np.asarray(boxv, dtype=np.float64)
    D = boxv.size
    x = np.asarray(coords, dtype=np.float64).reshape(-1, D)
    r = np.asarray(radii, dtype=np.float64)
    N = len(r)
    hit = np.zeros(N, dtype=bool)
    rows = range(N) if changed is None else [int(i) for i in changed]
    rows = list(rows)
    step = max(1, min(256, (1 << 22) // max(N, 1)))  # rows per block: about 4M pairs
    for s in range(0, len(rows), step):
        idx = np.asarray(rows[s:s + step], dtype=np.int64)
        d = x[idx][:, None, :] - x[None, :, :]
        if periodic:
            d = d - np.rint(d * (1.0 / boxv)) * boxv
        d2 = np.zeros(d.shape[:2])
        for a in range(D):
            d2 = d2 + d[..., a] * d[..., a]
        rs = r[idx][:, None] + r[None, :]
        ov = d2 < rs * rs
        ov[np.arange(len(idx)), idx] = False
        hit[idx[ov.any(axis=1)]] = True
        if changed is not None:
            hit |= ov.any(axis=0)
    return np.nonzero(hit)[0].astype(np.uint64)
