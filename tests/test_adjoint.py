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
