"""Device-resident MPO simulator over libbsmpo (the product path).

``MPOSimulator`` owns one libbsmpo handle: the MPO lives in HBM for the whole run,
every beam-splitter update runs as CUDA kernels, and only the per-update kept counts
(and observables, when asked for) come back to the host.  PyTorch provides device
memory and the current stream; it does no arithmetic on the update path.
"""
import ctypes

import numpy as np

from . import _capi


def lossy_single_photon_rhos(n_modes, photon_modes, eta, d):
    """(1-eta)|0><0| + eta|1><1| on ``photon_modes``, vacuum elsewhere."""
    pm = set(int(m) for m in photon_modes)
    out = []
    for i in range(n_modes):
        rho = np.zeros((d, d), dtype=np.complex128)
        if i in pm:
            rho[0, 0] = 1.0 - eta
            if d > 1:
                rho[1, 1] = eta
        else:
            rho[0, 0] = 1.0
        out.append(rho)
    return out


def clements_t(theta, phi):
    """2x2 block of T(theta, phi) = [[e^{i phi} cos, -sin], [e^{i phi} sin, cos]]."""
    c, s = np.cos(theta), np.sin(theta)
    e = np.exp(1j * phi)
    return np.array([[e * c, -s], [e * s, c]], dtype=np.complex128)


def _m8(S):
    S = np.asarray(S, dtype=np.complex128)
    return np.array([S[0, 0].real, S[0, 0].imag, S[0, 1].real, S[0, 1].imag,
                     S[1, 0].real, S[1, 0].imag, S[1, 1].real, S[1, 1].imag], dtype=np.float64)


class MPOSimulator:
    """One n-mode, cutoff-d, bond-dimension-chi MPO resident on the current CUDA device."""

    def __init__(self, n, d, chi, cutoff=0.0):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("MPOSimulator needs a CUDA device (no CPU path exists)")
        self.torch = torch
        self.n, self.d, self.chi = int(n), int(d), int(chi)
        self.L = _capi.lib()
        h = ctypes.c_void_p()
        _capi.check(self.L.bsmpo_create(self.n, self.d, self.chi, 0, ctypes.byref(h)))
        self.h = h
        self.set_stream(torch.cuda.current_stream())
        self.set_cutoff(cutoff)

    # -------------------------------------------------------------- plumbing
    def _chk(self, rc):
        _capi.check(rc, self.h)

    def set_stream(self, stream):
        self._stream = stream
        self._chk(self.L.bsmpo_set_stream(self.h, ctypes.c_void_p(stream.cuda_stream)))

    def set_cutoff(self, cutoff):
        self._chk(self.L.bsmpo_set_cutoff(self.h, float(cutoff)))

    PRECISIONS = {"fp64": 0, "fp64-gram": 1, "tf32x3": 2}

    def set_precision(self, precision):
        """Sector SVD / contraction mode: 'fp64' (Jacobi, the plain path), 'fp64-gram'
        (FP64 Gram + Hermitian eigenproblem) or 'tf32x3' (the Gram route with the
        contractions on the tensor cores, 3 x TF32 split products)."""
        self._chk(self.L.bsmpo_set_precision(self.h, self.PRECISIONS[precision]))

    def set_workers(self, n_workers):
        """Beam splitters of one brick-wall layer that ``run_mesh`` runs at once."""
        self._chk(self.L.bsmpo_set_workers(self.h, int(n_workers)))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.bsmpo_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -------------------------------------------------------------- state
    def load(self, gamma, lam, charge):
        """Load device tensors (complex128 [n,chi,chi], float64 [n-1,chi], int32 [n+1,chi,2])."""
        t = self.torch
        g = gamma.to(dtype=t.complex128).contiguous()
        l = lam.to(dtype=t.float64).contiguous()
        c = charge.to(dtype=t.int32).contiguous()
        assert g.is_cuda and l.is_cuda and c.is_cuda
        assert tuple(g.shape) == (self.n, self.chi, self.chi)
        assert tuple(l.shape) == (self.n - 1, self.chi)
        assert tuple(c.shape) == (self.n + 1, self.chi, 2)
        self._chk(self.L.bsmpo_load_state(self.h, ctypes.c_void_p(g.data_ptr()),
                                          ctypes.c_void_p(l.data_ptr()),
                                          ctypes.c_void_p(c.data_ptr())))

    def load_host(self, gamma, lam, charge):
        t = self.torch
        dev = t.device("cuda", t.cuda.current_device())
        self.load(t.from_numpy(np.ascontiguousarray(gamma)).to(dev),
                  t.from_numpy(np.ascontiguousarray(lam)).to(dev),
                  t.from_numpy(np.ascontiguousarray(charge)).to(dev))

    def store(self):
        """Device tensors (Gamma, Lambda, charge) copied out of the handle."""
        t = self.torch
        dev = t.device("cuda", t.cuda.current_device())
        g = t.empty((self.n, self.chi, self.chi), dtype=t.complex128, device=dev)
        l = t.empty((self.n - 1, self.chi), dtype=t.float64, device=dev)
        c = t.empty((self.n + 1, self.chi, 2), dtype=t.int32, device=dev)
        self._chk(self.L.bsmpo_store_state(self.h, ctypes.c_void_p(g.data_ptr()),
                                           ctypes.c_void_p(l.data_ptr()),
                                           ctypes.c_void_p(c.data_ptr())))
        return g, l, c

    def get_site(self, site, out=None):
        """Gamma[site] (complex128 chi x chi device tensor, ``out`` if given)."""
        t = self.torch
        if out is None:
            out = t.empty((self.chi, self.chi), dtype=t.complex128, device=t.device("cuda", t.cuda.current_device()))
        assert out.is_cuda and out.dtype == t.complex128 and out.is_contiguous() and out.numel() == self.chi ** 2
        self._chk(self.L.bsmpo_get_site(self.h, int(site), ctypes.c_void_p(out.data_ptr())))
        return out

    def put_site(self, site, gamma):
        t = self.torch
        assert gamma.is_cuda and gamma.dtype == t.complex128 and gamma.is_contiguous() and gamma.numel() == self.chi ** 2
        self._chk(self.L.bsmpo_put_site(self.h, int(site), ctypes.c_void_p(gamma.data_ptr())))

    def get_bond(self, bond, lam=None, charge=None):
        """(Lambda float64 [chi], charges int32 [chi, 2]) of bond 1..n-1, device tensors."""
        t = self.torch
        dev = t.device("cuda", t.cuda.current_device())
        if lam is None:
            lam = t.empty(self.chi, dtype=t.float64, device=dev)
        if charge is None:
            charge = t.empty((self.chi, 2), dtype=t.int32, device=dev)
        self._check_bond_tensors(lam, charge)
        self._chk(self.L.bsmpo_get_bond(self.h, int(bond), ctypes.c_void_p(lam.data_ptr()),
                                        ctypes.c_void_p(charge.data_ptr())))
        return lam, charge

    def put_bond(self, bond, lam, charge):
        self._check_bond_tensors(lam, charge)
        self._chk(self.L.bsmpo_put_bond(self.h, int(bond), ctypes.c_void_p(lam.data_ptr()),
                                        ctypes.c_void_p(charge.data_ptr())))

    def _check_bond_tensors(self, lam, charge):
        t = self.torch
        assert lam.is_cuda and lam.dtype == t.float64 and lam.is_contiguous() and lam.numel() == self.chi
        assert charge.is_cuda and charge.dtype == t.int32 and charge.is_contiguous() and charge.numel() == 2 * self.chi

    def init_product(self, rho_sites, total_photons=None, canonicalize=True):
        """Product-state MPO of the per-mode density matrices ``rho_sites`` (n of d x d),
        built on the device (``bsmpo_init_product``), then canonicalised."""
        rho = np.ascontiguousarray(np.asarray(rho_sites, dtype=np.complex128))
        assert rho.shape == (self.n, self.d, self.d)
        tp = -1 if total_photons is None else int(total_photons)
        self._chk(self.L.bsmpo_init_product(self.h, _capi.dptr(rho.view(np.float64)), tp))
        if canonicalize:
            self.canonicalize()

    def init_single_photons(self, photon_modes, eta, total_photons=None, canonicalize=True):
        """Lossy single photons (transmissivity eta) in ``photon_modes``, canonicalised."""
        self.init_product(lossy_single_photon_rhos(self.n, photon_modes, eta, self.d), total_photons,
                          canonicalize)

    def canonicalize(self):
        """Right-to-left sweep of identity-gate updates (``src/MPO.py:137-155``)."""
        self._chk(self.L.bsmpo_canonicalize(self.h))

    # -------------------------------------------------------------- updates
    def bs_update(self, mode, S):
        """Apply the 2x2 single-particle unitary ``S`` to modes (mode, mode+1)."""
        m = _m8(S)
        self._chk(self.L.bsmpo_bs_update(self.h, int(mode), _capi.dptr(m)))

    def bs_update_tensor(self, mode, U3):
        """Apply a gate given as a device tensor U[new_a, new_b, old_a] (complex128 d^3)."""
        u = U3.to(dtype=self.torch.complex128).contiguous()
        assert u.is_cuda and u.numel() == self.d ** 3
        self._chk(self.L.bsmpo_bs_update_tensor(self.h, int(mode), ctypes.c_void_p(u.data_ptr())))

    def run_mesh(self, modes, theta, phi):
        modes = np.ascontiguousarray(modes, dtype=np.int32)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        self._chk(self.L.bsmpo_run_mesh(self.h, len(modes), _capi.iptr(modes), _capi.dptr(theta),
                                        _capi.dptr(phi)))

    def run_mesh_host(self, modes, theta, phi, state_in, state_out=None):
        """``run_mesh`` over a host-resident state (``bsmpo_run_mesh_host``): ``state_in``
        = (Gamma complex128 [n,chi,chi], Lambda float64 [n-1,chi], charge int32
        [n+1,chi,2]) CPU tensors, page-locked for the copies to overlap the updates;
        the resulting state goes to ``state_out`` (same shapes, may be ``state_in``;
        new pinned tensors if None), which is returned.  The device keeps the state."""
        t = self.torch
        shapes = [(self.n, self.chi, self.chi), (self.n - 1, self.chi), (self.n + 1, self.chi, 2)]
        dtypes = [t.complex128, t.float64, t.int32]
        if state_out is None:
            state_out = tuple(t.empty(sh, dtype=dt, pin_memory=True) for sh, dt in zip(shapes, dtypes))
        for x in list(state_in) + list(state_out):
            assert not x.is_cuda and x.is_contiguous()
        for x, y, sh, dt in zip(state_in, state_out, shapes, dtypes):
            assert tuple(x.shape) == sh and tuple(y.shape) == sh and x.dtype == dt and y.dtype == dt
        modes = np.ascontiguousarray(modes, dtype=np.int32)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        ptr = [ctypes.c_void_p(x.data_ptr()) for x in list(state_in) + list(state_out)]
        self._chk(self.L.bsmpo_run_mesh_host(self.h, len(modes), _capi.iptr(modes), _capi.dptr(theta),
                                             _capi.dptr(phi), *ptr))
        return state_out

    def mesh_truncation(self):
        """Truncation weight of every update of the last ``run_mesh`` call (mesh order)."""
        n = self.L.bsmpo_mesh_truncation(self.h, None, 0)
        if n < 0:
            _capi.check(n, self.h)
        out = np.zeros(max(n, 1))
        n2 = self.L.bsmpo_mesh_truncation(self.h, _capi.dptr(out), len(out))
        if n2 < 0:
            _capi.check(n2, self.h)
        return out[:n]

    def apply_phases(self, phases):
        ph = np.ascontiguousarray(phases, dtype=np.float64)
        assert ph.shape == (self.n,)
        self._chk(self.L.bsmpo_apply_phases(self.h, _capi.dptr(ph)))

    # -------------------------------------------------------------- results
    def observables(self, marginals=True):
        """(trace complex, P[n, d] complex or None) in FP64."""
        tr = np.zeros(2)
        P = np.zeros((self.n, self.d, 2)) if marginals else None
        self._chk(self.L.bsmpo_observables(self.h, _capi.dptr(tr),
                                           _capi.dptr(P) if marginals else None))
        Pc = (P[..., 0] + 1j * P[..., 1]) if marginals else None
        return complex(tr[0], tr[1]), Pc

    def trace(self):
        return self.observables(marginals=False)[0]

    def last_update_info(self):
        ns = ctypes.c_int()
        self._chk(self.L.bsmpo_last_update_info(self.h, ctypes.byref(ns), None, None, None, None, 0,
                                                None, None))
        n = ns.value
        cc = np.zeros((max(n, 1), 2), dtype=np.int32)
        shape = np.zeros((max(n, 1), 2), dtype=np.int32)
        slen = np.zeros(max(n, 1), dtype=np.int32)
        kept = np.zeros(max(n, 1), dtype=np.int32)
        tw = np.zeros(1)
        self._chk(self.L.bsmpo_last_update_info(self.h, ctypes.byref(ns), _capi.iptr(cc),
                                                _capi.iptr(shape), _capi.iptr(slen), None, 0,
                                                _capi.iptr(kept), _capi.dptr(tw)))
        sig = np.zeros(max(int(slen[:n].sum()), 1))
        self._chk(self.L.bsmpo_last_update_info(self.h, ctypes.byref(ns), None, None, None,
                                                _capi.dptr(sig), len(sig), None, None))
        offs = np.concatenate([[0], np.cumsum(slen[:n])])
        return {
            "sectors": [tuple(int(x) for x in cc[i]) for i in range(n)],
            "shape": [tuple(int(x) for x in shape[i]) for i in range(n)],
            "sigma": [sig[offs[i]:offs[i + 1]].copy() for i in range(n)],
            "kept": [int(k) for k in kept[:n]],
            "trunc_weight": float(tw[0]),
        }

    def last_update_work(self):
        g, s, b = np.zeros(1), np.zeros(1), np.zeros(1)
        self._chk(self.L.bsmpo_last_update_work(self.h, _capi.dptr(g), _capi.dptr(s), _capi.dptr(b)))
        return {"gemm_flops": float(g[0]), "svd_flops": float(s[0]), "min_bytes": float(b[0])}

    def bond_dims(self):
        out = np.zeros(self.n + 1, dtype=np.int32)
        self._chk(self.L.bsmpo_bond_dims(self.h, _capi.iptr(out)))
        return [int(x) for x in out]

    def svd_routes(self):
        """(updates solved by the Jacobi SVD, by the Gram route) since creation."""
        c = (ctypes.c_int64 * 2)()
        self._chk(self.L.bsmpo_svd_routes(self.h, c))
        return int(c[0]), int(c[1])

    def workspace_stats(self):
        """(device allocations, pinned allocations, device bytes held, pinned bytes held)."""
        c = (ctypes.c_int64 * 4)()
        self._chk(self.L.bsmpo_workspace_stats(self.h, c))
        return tuple(int(x) for x in c)

    def kernel_launches(self):
        return int(self.L.bsmpo_kernel_launches(self.h))

    def set_timing(self, on=True):
        self._chk(self.L.bsmpo_set_timing(self.h, 1 if on else 0))

    def jacobi_timing(self):
        """(device ms, algorithmic flops, launches) of the Jacobi phase since set_timing()."""
        ms, fl = np.zeros(1), np.zeros(1)
        n = ctypes.c_int64()
        self._chk(self.L.bsmpo_jacobi_timing(self.h, _capi.dptr(ms), _capi.dptr(fl), ctypes.byref(n)))
        return float(ms[0]), float(fl[0]), int(n.value)

    def tridiag_timing(self):
        """(device ms, streamed bytes, zhetrd flops, phases) of the Gram route's
        tridiagonalisation since set_timing()."""
        ms, by, fl = np.zeros(1), np.zeros(1), np.zeros(1)
        n = ctypes.c_int64()
        self._chk(self.L.bsmpo_tridiag_timing(self.h, _capi.dptr(ms), _capi.dptr(by), _capi.dptr(fl),
                                              ctypes.byref(n)))
        return float(ms[0]), float(by[0]), float(fl[0]), int(n.value)

    def stage_times(self):
        """Per-stage milliseconds (only with BSMPO_PROFILE=1 at creation)."""
        ms = np.zeros(10)
        self._chk(self.L.bsmpo_stage_times(self.h, _capi.dptr(ms), 10))
        names = ["plan", "theta_gemm", "mix", "jacobi", "select_sync", "v_w", "scatter", "unused"]
        out = {k: float(v) for k, v in zip(names, ms[:8])}
        out["jacobi_rounds"] = int(ms[8])
        out["updates"] = int(ms[9])
        return out


def batch_circuits(n_circuits=64, seed=1004, chis=(128, 256, 512), d=4):
    """Independent seeded circuits of uneven size: N uniform in [16, 48], single photons in
    every second mode, transmissivity uniform in [0.2, 0.8], chi drawn from ``chis``; the
    Haar unitary of circuit i is seeded by ``seed * 1000 + i``."""
    from . import interferometer
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_circuits):
        n = int(rng.integers(16, 49))
        eta = float(rng.uniform(0.2, 0.8))
        chi = int(rng.choice(np.asarray(chis)))
        U, bs, ph = interferometer.circuit(n, seed * 1000 + i)
        specs.append(dict(n=n, d=d, chi=chi, eta=eta, photon_modes=list(range(0, n, 2)), mesh=bs, phases=ph))
    return specs


def batch_cost(spec):
    """Relative work of a circuit for ordering a batch: beam splitters x chi^3 (the
    per-sector eigen/SVD work grows with the cube of the sector sizes, which chi caps)."""
    return len(spec["mesh"]) * float(spec["chi"]) ** 3


def run_batch(specs, concurrency=8, precision="fp64-gram", workers=4, timing=None, largest_first=False):
    """Runs independent circuits (``batch_circuits`` entries) side by side on the current
    device: ``concurrency`` circuits at a time, each on its own handle, host thread and
    stream (the library's calls release the GIL), each handle overlapping its own updates
    on ``workers`` streams.  Handles are created and initialised first and released last,
    outside the concurrent phase (allocating or freeing device memory synchronises the
    whole device).  ``largest_first`` starts the circuits in decreasing ``batch_cost``
    (longest-first list scheduling: the batch does not end on one large circuit running
    alone).  Returns ``[(trace, marginals)]`` in input order; every circuit computes
    exactly what it computes alone.  ``timing`` (a dict), if given, receives the
    wall-clock seconds of the concurrent phase (the meshes, phases and observables)."""
    import time
    from concurrent.futures import ThreadPoolExecutor

    import torch
    dev = torch.cuda.current_device()
    streams = [torch.cuda.Stream() for _ in specs]
    sims = []
    try:
        for sp, st in zip(specs, streams):
            with torch.cuda.stream(st):
                sim = MPOSimulator(sp["n"], sp["d"], sp["chi"])
                sims.append(sim)
                sim.set_precision(precision)
                sim.set_workers(workers)
                sim.init_single_photons(sp["photon_modes"], sp["eta"])
        torch.cuda.synchronize()
        out = [None] * len(specs)

        def one(i):
            sp, sim = specs[i], sims[i]
            torch.cuda.set_device(dev)
            with torch.cuda.stream(streams[i]):
                m = sp["mesh"]
                sim.run_mesh([b[1] for b in m], [b[2] for b in m], [b[3] for b in m])
                sim.apply_phases(sp["phases"])
                out[i] = sim.observables()

        order = list(range(len(specs)))
        if largest_first:
            order.sort(key=lambda i: -batch_cost(specs[i]))
        t0 = time.perf_counter()
        if concurrency <= 1:
            for i in order:
                one(i)
        else:
            with ThreadPoolExecutor(max_workers=concurrency) as ex:
                list(ex.map(one, order))
        torch.cuda.synchronize()
        if timing is not None:
            timing["seconds"] = time.perf_counter() - t0
        return out
    finally:
        for sim in sims:
            sim.close()
