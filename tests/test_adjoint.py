"""The hand-written adjoint of one update (bosonsampling_b200.adjoint.update_backward)
against torch autograd through the pure-torch reference update, on the CPU: gradients of
a gauge-invariant loss with respect to both input sites, the right Lambda and the gate
tensor.  (The circuit-level gradients are checked on the GPU in test_gpu_adjoint.py.)"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import torch_reference as tr  # noqa: E402
from bosonsampling_b200 import adjoint  # noqa: E402


def _state(n, d, chi, seed):
    rng = np.random.default_rng(seed)
    st = tr.canonicalize(tr.product_state(n, d, chi, list(range(0, n, 2)), torch.tensor(0.6, dtype=torch.float64)))
    for m in list(range(0, n - 1, 2)) + list(range(1, n - 1, 2)):
        th, ph = torch.tensor(rng.uniform(0.2, 1.3)), torch.tensor(rng.uniform(0, 6.28))
        st, _ = tr.bs_update(st, m, tr.gate(th, ph, d))
    return tr.TState(n, d, chi, st.G.detach(), st.Lam.detach(), st.charge)


def _rel(a, b):
    return float((a - b).abs().max() / max(float(b.abs().max()), 1e-300))


@pytest.mark.parametrize("n,d,chi,mode,seed", [(5, 3, 8, 1, 3), (6, 3, 12, 2, 4), (6, 4, 10, 0, 5), (5, 3, 6, 3, 6)])
def test_update_adjoint_matches_autograd(n, d, chi, mode, seed):
    st = _state(n, d, chi, seed)
    rng = np.random.default_rng(seed + 100)
    GL = st.G[mode].clone().requires_grad_(True)
    GR = st.G[mode + 1].clone().requires_grad_(True)
    inner_R = mode + 2 < n
    LR = st.Lam[mode + 1].clone().requires_grad_(True) if inner_R else None
    U3 = tr.gate(torch.tensor(0.7), torch.tensor(1.1), d).detach().requires_grad_(True)
    G = torch.cat([st.G[:mode], GL[None], GR[None], st.G[mode + 2:]])
    Lam = torch.cat([st.Lam[:mode + 1], LR[None], st.Lam[mode + 2:]]) if inner_R else st.Lam
    out, kept = tr.bs_update(tr.TState(n, d, chi, G, Lam, st.charge), mode, U3)
    # a gauge-invariant loss of the outputs: the two-site product and the new spectrum
    A = torch.as_tensor(rng.standard_normal((chi, chi)) + 1j * rng.standard_normal((chi, chi)))
    c = torch.as_tensor(rng.standard_normal(chi))
    oL = out.G[mode].detach().requires_grad_(True)
    oR = out.G[mode + 1].detach().requires_grad_(True)
    oS = out.Lam[mode].detach().requires_grad_(True)

    def loss(gl, gr, s):
        return (torch.conj(A) * (gl @ gr)).real.sum() + (c * s).sum() + ((gl @ gr).abs() ** 2).sum()

    loss(oL, oR, oS).backward()
    loss(out.G[mode], out.G[mode + 1], out.Lam[mode]).backward()
    # the adjoint from the output gradients
    before = adjoint.StateT(st.G, st.Lam, st.charge, d)
    after = adjoint.StateT(out.G.detach(), out.Lam.detach(), out.charge, d)
    Gbar = torch.zeros((n, chi, chi), dtype=torch.complex128)
    Lbar = torch.zeros((n - 1, chi), dtype=torch.float64)
    Gbar[mode], Gbar[mode + 1], Lbar[mode] = oL.grad, oR.grad, oS.grad
    ubar = adjoint.update_backward(before, after, mode, U3.detach(), Gbar, Lbar)
    assert sum(kept) > 0
    assert _rel(Gbar[mode], GL.grad) < 1e-9
    assert _rel(Gbar[mode + 1], GR.grad) < 1e-9
    if inner_R:
        assert _rel(Lbar[mode + 1], LR.grad) < 1e-9
    assert _rel(ubar, U3.grad) < 1e-9
    assert float(Lbar[mode].abs().max()) == 0.0


def test_svd_backward_truncated_matches_autograd():
    rng = np.random.default_rng(7)
    th = torch.as_tensor(rng.standard_normal((9, 6)) + 1j * rng.standard_normal((9, 6))).requires_grad_(True)
    U, S, _ = torch.linalg.svd(th, full_matrices=False)
    k = 3
    V, s = U[:, :k], S[:k]
    A = torch.as_tensor(rng.standard_normal((9, 9)) + 1j * rng.standard_normal((9, 9)))
    w = torch.as_tensor(rng.standard_normal(k))
    # gauge invariant: through the projector V V^H and the kept spectrum
    L = (torch.conj(A) * (V @ V.conj().transpose(0, 1))).real.sum() + (w * s).sum()
    Vl = V.detach().requires_grad_(True)
    sl = s.detach().requires_grad_(True)
    ((torch.conj(A) * (Vl @ Vl.conj().transpose(0, 1))).real.sum() + (w * sl).sum()).backward()
    L.backward()
    g = adjoint.svd_backward(th.detach(), V.detach(), Vl.grad, sl.grad)
    assert _rel(g, th.grad) < 1e-9


def _circuit_adjoint_cpu(n, d, chi, photons, eta, mesh, th, ph, phases, target):
    """The library's reverse sweep (update_backward in reverse order) driven by the torch
    reference's forward states, on the CPU; returns (dtheta, dphi, deta)."""
    st = tr.product_state(n, d, chi, photons, torch.tensor(eta, dtype=torch.float64))
    prod = tr.TState(n, d, chi, st.G.detach(), st.Lam.detach(), st.charge)
    recs, gates, modes = [prod], [], []
    cur = prod
    ident = tr.fock_tensor(torch.eye(2, dtype=torch.complex128), d)
    for m in range(n - 2, -1, -1):
        cur, _ = tr.bs_update(cur, m, ident)
        recs.append(cur); gates.append(ident); modes.append(m)
    for i, (_, m, _, _) in enumerate(mesh):
        u = tr.gate(torch.tensor(th[i]), torch.tensor(ph[i]), d)
        cur, _ = tr.bs_update(cur, m, u)
        recs.append(cur); gates.append(u); modes.append(m)
    G = cur.G.detach().clone().requires_grad_(True)
    trace, P = tr.marginals(tr.TState(n, d, chi, G, cur.Lam.detach(), cur.charge), phases)
    ((P.real / trace.real - torch.as_tensor(target)) ** 2).sum().backward()
    Gbar, Lbar = G.grad.clone(), torch.zeros((n - 1, chi), dtype=torch.float64)
    ubars = []
    for t in range(len(modes) - 1, -1, -1):
        b = adjoint.StateT(recs[t].G.detach(), recs[t].Lam.detach(), recs[t].charge, d)
        a = adjoint.StateT(recs[t + 1].G.detach(), recs[t + 1].Lam.detach(), recs[t + 1].charge, d)
        ubars.append(adjoint.update_backward(b, a, modes[t], gates[t].detach(), Gbar, Lbar))
    ubars = ubars[::-1][n - 1:]             # the mesh's gates, in mesh order
    # angles through torch autograd of the gate tensor alone (the device kernel is checked
    # on the GPU); eta through the product state's entries
    dth, dph = [], []
    for i in range(len(mesh)):
        t_ = torch.tensor(th[i], requires_grad=True)
        p_ = torch.tensor(ph[i], requires_grad=True)
        (torch.conj(ubars[i]) * tr.gate(t_, p_, d)).real.sum().backward()
        dth.append(float(t_.grad)); dph.append(float(p_.grad))
    e_ = torch.tensor(eta, dtype=torch.float64, requires_grad=True)
    (Gbar.conj() * tr.product_state(n, d, chi, photons, e_).G).real.sum().backward()
    return np.array(dth), np.array(dph), float(e_.grad)


def _problem(n, d, seed):
    from bosonsampling_b200 import interferometer
    _, bs, ph = interferometer.circuit(n, seed)
    rng = np.random.default_rng(seed)
    target = rng.dirichlet(np.ones(d), size=n)
    return bs, ph, np.array([b[2] for b in bs]), np.array([b[3] for b in bs]), target


# torch's own SVD backward refuses degenerate spectra (its gauge check), which the
# canonicalised product state has at d = 4; d = 3 circuits are non-degenerate, and the
# degenerate case is checked against finite differences below
@pytest.mark.parametrize("n,d,chi,seed", [(6, 3, 12, 21), (8, 3, 10, 22)])
def test_circuit_adjoint_matches_autograd_cpu(n, d, chi, seed):
    bs, ph, th, phi, target = _problem(n, d, seed)
    photons, eta = list(range(0, n, 2)), 0.6
    dth, dph, deta = _circuit_adjoint_cpu(n, d, chi, photons, eta, bs, th, phi, ph, target)
    t_th = torch.tensor(th, requires_grad=True)
    t_ph = torch.tensor(phi, requires_grad=True)
    t_eta = torch.tensor(eta, dtype=torch.float64, requires_grad=True)
    trace, P = tr.circuit(n, d, chi, photons, t_eta, bs, t_th, t_ph, ph)
    ((P.real / trace.real - torch.as_tensor(target)) ** 2).sum().backward()
    assert _rel(torch.as_tensor(dth), t_th.grad) < 1e-7
    assert _rel(torch.as_tensor(dph), t_ph.grad) < 1e-7
    assert abs(deta - float(t_eta.grad)) <= 1e-7 * max(1.0, abs(float(t_eta.grad)))


def test_circuit_adjoint_at_degenerate_spectra_matches_finite_differences_cpu():
    """eta = 0.5 makes (1 - eta) = eta: exactly degenerate singular values, where torch's
    own SVD backward refuses (its gauge check fails) and the broadened F is needed."""
    n, d, chi = 6, 4, 12
    bs, ph, th, phi, target = _problem(n, d, 23)
    photons, eta = list(range(0, n, 2)), 0.5
    dth, dph, deta = _circuit_adjoint_cpu(n, d, chi, photons, eta, bs, th, phi, ph, target)

    def L(t, p, e):
        with torch.no_grad():
            trace, P = tr.circuit(n, d, chi, photons, torch.tensor(e, dtype=torch.float64), bs,
                                  torch.as_tensor(t), torch.as_tensor(p), ph)
            return float(((P.real / trace.real - torch.as_tensor(target)) ** 2).sum())
    h = 1e-6
    fds, ads = [], []
    for i in (0, 4, len(th) - 1):
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fds.append((L(tp, phi, eta) - L(tm, phi, eta)) / (2 * h)); ads.append(dth[i])
        pp, pm = phi.copy(), phi.copy()
        pp[i] += h
        pm[i] -= h
        fds.append((L(th, pp, eta) - L(th, pm, eta)) / (2 * h)); ads.append(dph[i])
    fds.append((L(th, phi, eta + h) - L(th, phi, eta - h)) / (2 * h)); ads.append(deta)
    scale = max(abs(x) for x in fds)
    for a_, f_ in zip(ads, fds):
        assert abs(a_ - f_) <= 1e-5 * max(abs(f_), 1e-3 * scale)


@pytest.mark.parametrize("m,n", [(7, 7), (9, 6), (6, 9)])
def test_svd_backward_small_kept_value_next_to_zeros(m, n):
    """A rank-deficient block whose smallest kept singular value is tiny: its coupling to
    the zero singular values, 1 / (0 - s_i^2), must survive the Lorentzian broadening."""
    rng = np.random.default_rng(m * 10 + n)
    r = min(m, n)
    Q1 = np.linalg.qr(rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m)))[0][:, :r]
    Q2 = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))[0][:, :r]
    s = np.zeros(r)
    s[:3] = [1.0, 0.3, 2e-9]
    lam = torch.as_tensor(rng.uniform(0.2, 1.0, n))
    C = torch.as_tensor((Q1 * s) @ Q2.conj().T / lam.numpy()[None, :]).requires_grad_(True)
    A = torch.as_tensor(rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))
    th = C * lam[None, :]
    V = torch.linalg.svd(th, full_matrices=False)[0][:, :3]
    (torch.conj(A) * (V @ (V.conj().transpose(0, 1) @ C))).real.sum().backward()
    Vd, Cd = V.detach(), C.detach()
    Vl, Wl = Vd.clone().requires_grad_(True), (Vd.conj().transpose(0, 1) @ Cd).requires_grad_(True)
    (torch.conj(A) * (Vl @ Wl)).real.sum().backward()
    Vb = Vl.grad + Cd @ Wl.grad.conj().transpose(0, 1)
    tb = adjoint.svd_backward(Cd * lam[None, :], Vd, Vb, torch.zeros(3, dtype=torch.float64))
    Cb = Vd @ Wl.grad + tb * lam[None, :]
    assert _rel(Cb, C.grad) < 1e-6
