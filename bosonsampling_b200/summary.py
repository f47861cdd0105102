"""Drop-ins for the reference's ``src/summary.py`` observables (device, FP64)."""
import numpy as np

from .engine import MPOSimulator


def Probability(n, d, Gamma, Lambda, charge):
    """Trace of the MPO (``src/summary.py:11-26``), computed on the device.

    Accepts host (numpy) or CUDA (torch) arrays in the layout [n, chi, chi] /
    [n-1, chi] / [n+1, chi, 2]; returns a complex scalar.
    """
    chi = Gamma.shape[-1]
    with MPOSimulator(n, d, chi) as sim:
        if hasattr(Gamma, "data_ptr"):
            sim.load(Gamma, Lambda, charge)
        else:
            sim.load_host(np.asarray(Gamma, dtype=np.complex128), np.asarray(Lambda, dtype=np.float64),
                          np.asarray(charge, dtype=np.int32))
        return sim.trace()


def EntanglementEntropy(Lambda):
    """Per-bond von Neumann entropy of the normalised Lambda^2 (``src/summary.py:3-9``)."""
    import torch
    L = torch.as_tensor(Lambda, dtype=torch.float64)
    if torch.cuda.is_available():
        L = L.cuda()
    p = L * L
    p = p / p.sum(dim=1, keepdim=True).clamp_min(1e-300)
    h = torch.where(p > 0, -p * torch.log2(torch.where(p > 0, p, torch.ones_like(p))), torch.zeros_like(p))
    return h.sum(dim=1).cpu().numpy()
