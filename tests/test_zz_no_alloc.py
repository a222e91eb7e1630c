"""The allocation-free NUwNU entry point against the handle-based one, through the C ABI.

fresco_nuwnu_energy_gradient_noalloc serves callers that cannot allocate device memory where they
need the loss (a host whose memory pool owns the GPU, a loop that must not call cudaFree because it
waits for the whole device).  Its per-k-point sums live in a static device array shared by all
calls, so two calls in a row are checked: the second must not see the first one's sums.  This file
is collected last so that it also runs after every other GPU test in one process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_K = 4096  # the documented limit of the static array


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _weights(radii, ndim):
    # per-point weights as the reference derives them from the radii (nuwnu.hpp:81-105)
    c = np.ones_like(radii)
    for _ in range(ndim):
        c = c * (np.pi * radii**2 if ndim == 2 else 4.0 / 3.0 * np.pi * radii**3 if ndim == 3 else 1.0)
    return c * (len(c) / c.sum())


def _handle_eval(lib, h, x_d, n, stream, torch):
    g = torch.empty(n, dtype=torch.float64, device="cuda")
    e = torch.empty(1, dtype=torch.float64, device="cuda")
    rc = lib.fresco_potential_energy_gradient_device(h, C.c_void_p(x_d.data_ptr()), n, C.c_void_p(g.data_ptr()),
                                                     C.c_void_p(e.data_ptr()), 0, C.c_void_p(stream))
    assert rc == 0, lib.fresco_last_error()
    return g, e


def _noalloc_eval(lib, x_d, N, ndim, w_d, k_d, sk_d, v_d, nk, L, mode, stream, torch):
    g = torch.full((N * ndim,), 7.0, dtype=torch.float64, device="cuda")  # stale values must be overwritten
    e = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    Lc = np.ascontiguousarray(L, dtype=np.float64)
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    rc = lib.fresco_nuwnu_energy_gradient_noalloc(ptr(x_d), N, ndim, ptr(w_d), ptr(k_d), ptr(sk_d), ptr(v_d), nk,
                                                   Lc.ctypes.data_as(C.POINTER(C.c_double)), mode, ptr(g), ptr(e),
                                                   0, C.c_void_p(stream))
    assert rc == 0, lib.fresco_last_error()
    return g, e


@pytest.mark.parametrize("ndim,N,nk,equal_radii,mode", [(2, 3000, 40, False, 0), (3, 1500, MAX_K, True, 1),
                                                         (1, 700, 9, False, 1)])
def test_noalloc_matches_handle_on_two_calls(ndim, N, nk, equal_radii, mode):
    import torch

    from fresco_b200._lib import lib

    rng = np.random.default_rng(100 + ndim)
    radii = np.full(N, 0.8) if equal_radii else 0.5 + rng.random(N)
    K = (rng.random(nk * ndim) - 0.5) * 60
    Sk = rng.random(nk) * N * (rng.random(nk) < 0.5)
    V = rng.random(nk)
    L = 0.7 + rng.random(ndim)
    h = C.c_void_p()
    dp = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    rc = lib.fresco_nuwnu_create(dp(radii), N, dp(K), nk, dp(Sk), dp(V), dp(L), ndim, 1e-12, 0, C.byref(h))
    assert rc == 0, lib.fresco_last_error()
    try:
        assert lib.fresco_potential_set_gradient_mode(h, mode) == 0
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()  # noqa: E731
        w_d = None if equal_radii else dev(_weights(radii, ndim))
        k_d, sk_d, v_d = dev(K), dev(Sk), dev(V)
        stream = torch.cuda.current_stream().cuda_stream
        # two calls in a row on different coordinates: the second reuses the static sums of the first
        for call in range(2):
            x_d = dev(rng.random(ndim * N) * 1.4 - 0.2)
            g0, e0 = _handle_eval(lib, h, x_d, N * ndim, stream, torch)
            g1, e1 = _noalloc_eval(lib, x_d, N, ndim, w_d, k_d, sk_d, v_d, nk, L, mode, stream, torch)
            torch.cuda.synchronize()
            assert _rel(e1.cpu().numpy(), e0.cpu().numpy()) < 1e-11, call
            assert _rel(g1.cpu().numpy(), g0.cpu().numpy()) < 1e-10, call
    finally:
        lib.fresco_potential_destroy(h)


def test_noalloc_rejects_more_kpoints_than_the_static_array_holds():
    import torch

    from fresco_b200._lib import FRESCO_ERR_INVALID, lib

    nk, N, ndim = MAX_K + 1, 10, 2
    x = torch.zeros(N * ndim, dtype=torch.float64, device="cuda")
    k = torch.zeros(nk * ndim, dtype=torch.float64, device="cuda")
    sv = torch.zeros(nk, dtype=torch.float64, device="cuda")
    g = torch.zeros(N * ndim, dtype=torch.float64, device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    L = np.ones(ndim)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    rc = lib.fresco_nuwnu_energy_gradient_noalloc(p(x), N, ndim, None, p(k), p(sv), p(sv), nk,
                                                   L.ctypes.data_as(C.POINTER(C.c_double)), 0, p(g), p(e), 0, None)
    assert rc == FRESCO_ERR_INVALID
    assert b"4096" in lib.fresco_last_error()


def _setup(ndim, N, nk, seed, torch, lib):
    rng = np.random.default_rng(seed)
    radii = 0.5 + rng.random(N)
    K = (rng.random(nk * ndim) - 0.5) * 40
    Sk = rng.random(nk) * N * (rng.random(nk) < 0.5)
    V = rng.random(nk)
    L = 0.7 + rng.random(ndim)
    h = C.c_void_p()
    dp = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    rc = lib.fresco_nuwnu_create(dp(radii), N, dp(K), nk, dp(Sk), dp(V), dp(L), ndim, 1e-12, 0, C.byref(h))
    assert rc == 0, lib.fresco_last_error()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()  # noqa: E731
    arrays = dict(w_d=dev(_weights(radii, ndim)), k_d=dev(K), sk_d=dev(Sk), v_d=dev(V))
    x_d = dev(rng.random(ndim * N) * 1.4 - 0.2)
    return h, arrays, L, x_d


def _noalloc_raw(lib, x_d, N, ndim, a, nk, L, g, e, acc, stream):
    Lc = np.ascontiguousarray(L, dtype=np.float64)
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    rc = lib.fresco_nuwnu_energy_gradient_noalloc(ptr(x_d), N, ndim, ptr(a["w_d"]), ptr(a["k_d"]), ptr(a["sk_d"]),
                                                   ptr(a["v_d"]), nk, Lc.ctypes.data_as(C.POINTER(C.c_double)), 0,
                                                   ptr(g), ptr(e), acc, C.c_void_p(stream))
    assert rc == 0, lib.fresco_last_error()


def test_noalloc_accumulates_into_preset_outputs():
    """accumulate = 1 adds the loss and gradient to what the output arrays hold, on two calls in a row."""
    import torch

    from fresco_b200._lib import lib

    ndim, N, nk = 2, 2000, 64
    h, a, L, x_d = _setup(ndim, N, nk, 7, torch, lib)
    try:
        stream = torch.cuda.current_stream().cuda_stream
        g0, e0 = _handle_eval(lib, h, x_d, N * ndim, stream, torch)
        for call in range(2):
            preset_g = torch.linspace(-3.0, 5.0, N * ndim, dtype=torch.float64, device="cuda")
            preset_e = torch.full((1,), 11.5, dtype=torch.float64, device="cuda")
            g, e = preset_g.clone(), preset_e.clone()
            _noalloc_raw(lib, x_d, N, ndim, a, nk, L, g, e, 1, stream)
            torch.cuda.synchronize()
            assert _rel((e - preset_e).cpu().numpy(), e0.cpu().numpy()) < 1e-11, call
            assert _rel((g - preset_g).cpu().numpy(), g0.cpu().numpy()) < 1e-10, call
    finally:
        lib.fresco_potential_destroy(h)


def test_noalloc_energy_only():
    """A NULL gradient pointer computes the energy alone, equal to the handle form's."""
    import torch

    from fresco_b200._lib import lib

    ndim, N, nk = 3, 1200, 100
    h, a, L, x_d = _setup(ndim, N, nk, 8, torch, lib)
    try:
        stream = torch.cuda.current_stream().cuda_stream
        _, e0 = _handle_eval(lib, h, x_d, N * ndim, stream, torch)
        for call in range(2):
            e = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
            _noalloc_raw(lib, x_d, N, ndim, a, nk, L, None, e, 0, stream)
            torch.cuda.synchronize()
            assert _rel(e.cpu().numpy(), e0.cpu().numpy()) < 1e-11, call
    finally:
        lib.fresco_potential_destroy(h)


def test_noalloc_nonfinite_call_then_finite_call():
    """A NaN coordinate makes that call's energy and gradient NaN; the status it leaves in the shared
    array must not leak into the next, finite call, whose results equal the handle form's."""
    import torch

    from fresco_b200._lib import lib

    ndim, N, nk = 2, 1500, 50
    h, a, L, x_d = _setup(ndim, N, nk, 9, torch, lib)
    try:
        stream = torch.cuda.current_stream().cuda_stream
        g0, e0 = _handle_eval(lib, h, x_d, N * ndim, stream, torch)
        bad = x_d.clone()
        bad[17] = float("nan")
        g = torch.empty(N * ndim, dtype=torch.float64, device="cuda")
        e = torch.empty(1, dtype=torch.float64, device="cuda")
        _noalloc_raw(lib, bad, N, ndim, a, nk, L, g, e, 0, stream)
        torch.cuda.synchronize()
        assert torch.isnan(e).all() and torch.isnan(g).all()
        _noalloc_raw(lib, x_d, N, ndim, a, nk, L, g, e, 0, stream)
        torch.cuda.synchronize()
        assert torch.isfinite(e).all() and torch.isfinite(g).all()
        assert _rel(e.cpu().numpy(), e0.cpu().numpy()) < 1e-11
        assert _rel(g.cpu().numpy(), g0.cpu().numpy()) < 1e-10
    finally:
        lib.fresco_potential_destroy(h)
