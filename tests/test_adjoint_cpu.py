"""Differentiation workload host logic and the PyTorch reference model, no GPU."""
import numpy as np
import pytest

from spectral_analyzer_b200.adjoint import (boundary_absorption, boundary_mask,
                                            differentiation_problem, gaussian_random_field)


def small_problem(n=(20, 18, 22), steps=120, seed=3, n_pml=4):
    return differentiation_problem(n, n_steps=steps, seed=seed, n_rec=2, n_pml=n_pml, corr=3.0)


def test_absorption_field_shape_and_range():
    a = boundary_absorption((40, 36, 44), 10, 8.0, 5)
    inside = ~boundary_mask((40, 36, 44), 10)
    assert np.all(a[inside] == 0)
    assert a[~inside].min() >= 0.05 and a[~inside].max() <= 0.5
    assert np.array_equal(a, boundary_absorption((40, 36, 44), 10, 8.0, 5))
    g = gaussian_random_field((32, 32, 32), 8.0, 1)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1) < 1e-12


def test_problem_places_points_inside():
    p = differentiation_problem(n=128, n_steps=4000)
    for q in [p.src] + p.receivers:
        assert all(12 <= c < 116 for c in q)
    assert len(p.receivers) == 4 and p.a.dtype == np.float32
    moved = (p.a_target != p.a)[p.a > 0].mean()
    assert moved > 0.9
    assert np.all(p.a_target[p.a == 0] == 0)


def test_torch_reference_matches_double_oracle():
    torch = pytest.importorskip("torch")
    from oracle import OracleFDTD
    from spectral_analyzer_b200.precision import pressure_taps
    from torch_reference import traces
    p = small_problem()
    nx, ny, nz = p.shape
    idx, w = pressure_taps(nx, ny, nz, np.asarray(p.receivers, np.float32))
    o = OracleFDTD(nx, ny, nz, p.dx, p.c, p.rho, n_pml=p.n_pml, precision="f64")
    o.set_cell_absorption(p.a.astype(np.float64))
    ref = o.run(p.n_steps, p.flat(p.src), p.signal().astype(np.float64), idx, w.astype(np.float64))
    got = traces(torch.as_tensor(p.a, dtype=torch.float64), p, idx, w, torch.float64, segment=50)
    got = got.detach().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_torch_reference_gradient_matches_finite_differences():
    torch = pytest.importorskip("torch")
    from spectral_analyzer_b200.precision import pressure_taps
    from torch_reference import loss_and_grad, traces
    p = small_problem(n=(12, 11, 14), steps=60, n_pml=3)
    nx, ny, nz = p.shape
    idx, w = pressure_taps(nx, ny, nz, np.asarray(p.receivers, np.float32))
    tgt = traces(torch.as_tensor(p.a_target, dtype=torch.float64), p, idx, w, torch.float64).detach().numpy()
    L, g = loss_and_grad(p.a, p, idx, w, tgt, device="cpu")
    a = p.a.astype(np.float64)
    for cell in [(0, 0, 0), (1, 4, 6), (11, 10, 13), (2, 2, 12)]:
        h = 1e-4
        ap, am = a.copy(), a.copy()
        ap[cell] += h
        am[cell] -= h
        Lp, _ = loss_and_grad(ap, p, idx, w, tgt, device="cpu")
        Lm, _ = loss_and_grad(am, p, idx, w, tgt, device="cpu")
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - g[cell]) <= 1e-5 * abs(g[cell]) + 1e-9 * L, (cell, fd, g[cell])
