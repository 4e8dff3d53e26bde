"""Adjoint kernels on the GPU: the float forward is the float oracle bit for
bit, the double adjoint is torch.autograd's gradient of the same model, the
float adjoint agrees with central finite differences, the checkpoint interval
does not change a bit, and the autograd.Function hands the gradient to torch."""
import numpy as np
import pytest

from spectral_analyzer_b200.adjoint import differentiation_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch


def problem(n=(40, 36, 44), steps=300, seed=7, n_pml=6, corr=4.0):
    return differentiation_problem(n, n_steps=steps, seed=seed, n_rec=4, n_pml=n_pml, corr=corr)


def targets_for(prob, double=True):
    from spectral_analyzer_b200.adjoint import AdjointRoom
    r = AdjointRoom(prob, double=double)
    r.set_absorption(prob.a_target)
    t = r.forward(keep_checkpoints=False)
    r.close()
    return t


def test_float_forward_is_the_oracle(cuda):
    from oracle import OracleFDTD
    from spectral_analyzer_b200.adjoint import AdjointRoom
    prob = problem()
    r = AdjointRoom(prob)
    r.set_absorption(prob.a)
    y = r.forward()
    nx, ny, nz = prob.shape
    o = OracleFDTD(nx, ny, nz, prob.dx, prob.c, prob.rho, n_pml=prob.n_pml)
    assert r.dt == pytest.approx(o.dt, rel=0, abs=0)
    o.set_cell_absorption(prob.a)
    idx, w = r.taps
    ref = o.run(prob.n_steps, prob.flat(prob.src), prob.signal(), idx, w.astype(np.float32))
    assert np.array_equal(y.astype(np.float32).view(np.uint32), ref.view(np.uint32))


def test_double_adjoint_is_torch_autograd(cuda):
    from spectral_analyzer_b200.adjoint import AdjointRoom
    from torch_reference import loss_and_grad
    prob = problem(n=(28, 24, 30), steps=220, n_pml=5)
    tgt = targets_for(prob)
    r = AdjointRoom(prob, double=True, checkpoint_every=50)
    r.set_absorption(prob.a)
    y = r.forward()
    g = r.backward(2.0 * (y - tgt))
    L_ref, g_ref = loss_and_grad(prob.a, prob, *r.taps, tgt, device="cuda", segment=50)
    assert float(np.sum((y - tgt) ** 2)) == pytest.approx(L_ref, rel=1e-12)
    assert np.linalg.norm(g - g_ref) <= 1e-9 * np.linalg.norm(g_ref)
    # the gradient lives on the absorbing layer only through the field's support
    assert np.count_nonzero(g) > 0


def test_float_adjoint_matches_finite_differences(cuda):
    from spectral_analyzer_b200.adjoint import AdjointRoom
    prob = problem(n=(32, 32, 32), steps=400, n_pml=6, seed=8)
    tgt = targets_for(prob)
    r = AdjointRoom(prob, double=False)
    r.set_absorption(prob.a)
    y = r.forward()
    g = r.backward(2.0 * (y - tgt))
    d = AdjointRoom(prob, double=True)
    d.set_absorption(prob.a.astype(np.float64))
    yd = d.forward()
    gd = d.backward(2.0 * (yd - tgt))
    # float adjoint vs double adjoint over the whole field
    assert np.linalg.norm(g - gd) <= 2e-3 * np.linalg.norm(gd)
    rng = np.random.default_rng(3)
    layer = np.argwhere(prob.a > 0)
    big = layer[np.argsort(-np.abs(gd[tuple(layer.T)]))[:200]]
    cells = big[rng.choice(len(big), 6, replace=False)]
    a = prob.a.astype(np.float64)
    for c in map(tuple, cells):
        h = 1e-4
        ap, am = a.copy(), a.copy()
        ap[c] += h
        am[c] -= h
        fd = (d.loss(ap, tgt) - d.loss(am, tgt)) / (2 * h)
        assert abs(gd[c] - fd) <= 1e-5 * abs(fd), (c, gd[c], fd)
        assert abs(g[c] - fd) <= 1e-2 * abs(fd), (c, g[c], fd)


def test_checkpoint_interval_changes_nothing(cuda):
    from spectral_analyzer_b200.adjoint import AdjointRoom
    prob = problem(n=(24, 20, 26), steps=150, n_pml=5, seed=9)
    tgt = targets_for(prob, double=False)
    out = []
    for K in (7, 50, 150):
        r = AdjointRoom(prob, checkpoint_every=K)
        r.set_absorption(prob.a)
        y = r.forward()
        out.append(r.backward(2.0 * (y - tgt)))
        r.close()
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[1], out[2])


def test_autograd_function(cuda):
    torch = cuda
    from spectral_analyzer_b200.adjoint import AdjointRoom, trace_loss
    prob = problem(n=(24, 22, 20), steps=120, n_pml=5, seed=10)
    tgt = targets_for(prob, double=False)
    r = AdjointRoom(prob)
    a = torch.tensor(prob.a, device="cuda", requires_grad=True)
    loss = trace_loss(a, r, tgt)
    loss.backward()
    r2 = AdjointRoom(prob)
    r2.set_absorption(prob.a)
    y = r2.forward()
    g = r2.backward(2.0 * (y - tgt))
    assert float(loss.detach()) == pytest.approx(float(np.sum((y - tgt) ** 2)), rel=1e-12)
    assert a.grad.dtype == torch.float32
    assert np.array_equal(a.grad.cpu().numpy(), g.astype(np.float32))
    assert r.launch_count > 0


def test_invalid_calls(cuda):
    from spectral_analyzer_b200 import _native
    from spectral_analyzer_b200.adjoint import AdjointRoom
    lib = _native.load()
    assert not lib.fdtd_b200_adj_create(8, 8, 8, 0.01, 343.0, 1.21, 0, 0, 0)
    prob = problem(n=(20, 20, 20), steps=10, n_pml=4)
    r = AdjointRoom(prob)
    with pytest.raises(RuntimeError):            # no checkpointed forward yet
        r.backward(np.zeros((0, 4)))
    r.steps = 10
    with pytest.raises(RuntimeError):
        r.backward(np.zeros((10, 4)))
    with pytest.raises(ValueError):
        r.set_absorption(np.zeros(5, np.float32))
    with pytest.raises(RuntimeError):            # longer than the trace capacity
        r.forward(11)
