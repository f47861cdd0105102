"""Differentiation form on the GPU: gradients of a marginal loss with respect to every
beam splitter's (theta, phi) and eta, from the library's forward and its hand-written
adjoint, against the pure-torch FP64 autograd reference and central finite differences
of the library's forward."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import torch_reference as tr  # noqa: E402
from bosonsampling_b200 import adjoint, interferometer  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.set_device(0)


def _setup(n, d, chi, seed):
    _, bs, ph = interferometer.circuit(n, seed)
    rng = np.random.default_rng(seed)
    target = rng.dirichlet(np.ones(d), size=n)
    th = np.array([b[2] for b in bs])
    phi = np.array([b[3] for b in bs])
    return bs, ph, th, phi, target


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_gate_angle_gradient_matches_finite_differences():
    d, rng = 5, np.random.default_rng(1)
    th, ph = rng.uniform(0.1, 1.4, 6), rng.uniform(0, 6.2, 6)
    ubar = torch.as_tensor(rng.standard_normal((6, d, d, d)) + 1j * rng.standard_normal((6, d, d, d)), device="cuda")
    g_th, g_ph = adjoint.angle_grads(d, th, ph, ubar)
    h = 1e-6
    for i in range(6):
        def f(t, p):
            u = adjoint.gate_tensor(d, t, p, "cuda")
            return float((torch.conj(ubar[i]) * u).real.sum())
        fd_t = (f(th[i] + h, ph[i]) - f(th[i] - h, ph[i])) / (2 * h)
        fd_p = (f(th[i], ph[i] + h) - f(th[i], ph[i] - h)) / (2 * h)
        assert abs(float(g_th[i]) - fd_t) <= 1e-7 * max(1.0, abs(fd_t))
        assert abs(float(g_ph[i]) - fd_p) <= 1e-7 * max(1.0, abs(fd_p))


@pytest.mark.parametrize("n,d,chi,seed", [(6, 3, 12, 11), (7, 3, 10, 12)])
def test_circuit_gradient_matches_torch_autograd_and_finite_differences(n, d, chi, seed):
    bs, ph, th, phi, target = _setup(n, d, chi, seed)
    photons, eta = list(range(0, n, 2)), 0.6
    circ = adjoint.DiffCircuit(n, d, chi, photons, bs, ph)
    try:
        loss, g_th, g_ph, g_eta = circ.loss_and_grad(th, phi, eta, target)
        # the pure-torch FP64 autograd reference
        t_th = torch.tensor(th, dtype=torch.float64, requires_grad=True)
        t_ph = torch.tensor(phi, dtype=torch.float64, requires_grad=True)
        t_eta = torch.tensor(eta, dtype=torch.float64, requires_grad=True)
        trace, P = tr.circuit(n, d, chi, photons, t_eta, bs, t_th, t_ph, ph)
        ref_loss = ((P.real / trace.real - torch.as_tensor(target)) ** 2).sum()
        ref_loss.backward()
        ref = float(ref_loss.detach())
        assert abs(loss - ref) <= 1e-10 * max(1.0, abs(ref))
        assert _rel(g_th.cpu(), t_th.grad) < 1e-6
        assert _rel(g_ph.cpu(), t_ph.grad) < 1e-6
        assert abs(g_eta - float(t_eta.grad)) <= 1e-6 * max(1.0, abs(float(t_eta.grad)))

        # central finite differences of the library's own forward (h = 1e-6, FP64)
        def L(t, p, e):
            trc, Pm = circ.run(t, p, e)
            return float(((Pm.real / trc.real - target) ** 2).sum())
        h = 1e-6
        for i in (0, len(th) // 2, len(th) - 1):
            tp, tm = th.copy(), th.copy()
            tp[i] += h
            tm[i] -= h
            fd = (L(tp, phi, eta) - L(tm, phi, eta)) / (2 * h)
            assert abs(float(g_th[i]) - fd) <= 1e-5 * max(abs(fd), 1e-3)
            pp, pm = phi.copy(), phi.copy()
            pp[i] += h
            pm[i] -= h
            fd = (L(th, pp, eta) - L(th, pm, eta)) / (2 * h)
            assert abs(float(g_ph[i]) - fd) <= 1e-5 * max(abs(fd), 1e-3)
        fd = (L(th, phi, eta + h) - L(th, phi, eta - h)) / (2 * h)
        assert abs(g_eta - fd) <= 1e-5 * max(abs(fd), 1e-3)
    finally:
        circ.close()


def test_autograd_function_agrees_with_loss_and_grad():
    n, d, chi, seed = 6, 3, 12, 13
    bs, ph, th, phi, target = _setup(n, d, chi, seed)
    circ = adjoint.DiffCircuit(n, d, chi, list(range(0, n, 2)), bs, ph)
    try:
        _, g_th, g_ph, g_eta = circ.loss_and_grad(th, phi, 0.55, target)
        t_th = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
        t_ph = torch.tensor(phi, dtype=torch.float64, device="cuda", requires_grad=True)
        t_eta = torch.tensor(0.55, dtype=torch.float64, device="cuda", requires_grad=True)
        trace, P = adjoint.CircuitMarginals.apply(t_th, t_ph, t_eta, circ)
        ((P.real / trace.real - torch.as_tensor(target, device="cuda")) ** 2).sum().backward()
        assert _rel(t_th.grad.cpu(), g_th.cpu()) < 1e-12
        assert _rel(t_ph.grad.cpu(), g_ph.cpu()) < 1e-12
        assert abs(float(t_eta.grad) - g_eta) <= 1e-12 * max(1.0, abs(g_eta))
    finally:
        circ.close()


def test_deep_circuit_early_parameters_match_finite_differences():
    """N=24, d=4, chi=256, 8 layers (truncating, degenerate spectra at eta = 0.5): the
    gradients of the first layer's angles and of eta pass through every later update."""
    n, d, chi = 24, 4, 256
    _, bs, ph = interferometer.circuit(n, 1005)
    bs = [b for b in bs if b[0] < 8]
    target = np.random.default_rng(0).dirichlet(np.ones(d), size=n)
    th = np.array([b[2] for b in bs])
    phi = np.array([b[3] for b in bs])
    circ = adjoint.DiffCircuit(n, d, chi, list(range(0, n, 2)), bs, ph)
    try:
        _, g_th, g_ph, g_eta = circ.loss_and_grad(th, phi, 0.5, target)

        def L(t, p, e):
            trc, Pm = circ.run(t, p, e)
            return float(((Pm.real / trc.real - target) ** 2).sum())
        h = 1e-6
        for i in (0, 1, len(th) // 2):
            tp, tm = th.copy(), th.copy()
            tp[i] += h
            tm[i] -= h
            fd = (L(tp, phi, 0.5) - L(tm, phi, 0.5)) / (2 * h)
            assert abs(float(g_th[i]) - fd) <= 1e-5 * max(abs(fd), 1e-3)
        fd = (L(th, phi, 0.5 + h) - L(th, phi, 0.5 - h)) / (2 * h)
        assert abs(g_eta - fd) <= 1e-5 * max(abs(fd), 1e-3)
    finally:
        circ.close()
