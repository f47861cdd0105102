"""The run.py queue and result files (bosonsampling_b200.runner), on CPU with a fake
worker: the experiment-queue protocol, the file names and the chi-doubling rule of the
reference's run.py (run.py:81-215)."""
import os
import pickle

import numpy as np

from bosonsampling_b200 import runner


class FakeWorker:
    """Stands in for gpu_algorithm.Worker: traces that drift by `drift` over the layers."""

    def __init__(self, drift, success=True):
        self.drift, self.success, self.calls = drift, success, []

    def ExperimentInit(self, input_state_type, n_modes, n_input_states, ps, d, chi, parameters, seed):
        self.n = n_modes
        self.calls.append(chi)

    def Simulate(self):
        prob = np.linspace(1.0, 1.0 + self.drift, self.n + 1).astype(np.float32)
        EE = np.zeros((self.n - 1, self.n + 1), np.float32)
        return self.success, prob, EE, None


def _experiments(tmp_path, n=2):
    exps = [dict(input_state_type="Single photon", n_modes=6, n_input_states=3, post_selected_photon_number=None,
                 local_hilbert_space_dimension=3, bond_dimension=16, parameters={"loss": 0.2},
                 status="incomplete") for _ in range(n)]
    exps[1]["n_modes"] = 8
    path = str(tmp_path / "experiments.pickle")
    with open(path, "wb") as f:
        pickle.dump(exps, f)
    return path


def test_queue_runs_each_incomplete_experiment_once(tmp_path):
    path = _experiments(tmp_path)
    root = str(tmp_path / "Results")
    done = runner.run(FakeWorker(0.5), path, seed=3, root=root)
    assert [(i, chi) for (i, chi, _) in done] == [(0, 16), (1, 16)]
    with open(path, "rb") as f:
        assert [e["status"] for e in pickle.load(f)] == ["in progress", "in progress"]
    with open(path, "rb") as f:
        exp = pickle.load(f)[0]
    prefix = runner.result_prefix(exp, root)
    assert prefix.endswith("n_6_m_3_PS_None_d_3_p_{'loss': 0.2}_")
    assert np.load(prefix + "chi.npy").tolist() == [16.0]
    assert np.load(prefix + "chi_16_prob.npy").shape == (7,)
    assert np.load(prefix + "chi_16_EE.npy").shape == (5, 7)


def test_chi_doubles_while_the_traces_drift_and_stops_when_they_agree(tmp_path):
    path = _experiments(tmp_path, n=2)
    root = str(tmp_path / "Results")
    runner.run(FakeWorker(0.5), path, root=root)           # drift 50% > 10%
    with open(path, "rb") as f:
        exps = pickle.load(f)
    for e in exps:
        e["status"] = "incomplete"
    with open(path, "wb") as f:
        pickle.dump(exps, f)
    w = FakeWorker(0.01)                                    # drift 1% after doubling
    runner.run(w, path, root=root)
    assert w.calls == [32, 32]
    prefix = runner.result_prefix(exps[0], root)
    assert np.load(prefix + "chi.npy").tolist() == [16.0, 32.0]
    assert runner.choose_chi(exps[0], root) == ("skip", 32)


def test_unsuccessful_run_goes_back_to_the_queue_and_limits_skip(tmp_path):
    path = _experiments(tmp_path, n=2)
    root = str(tmp_path / "Results")
    done = runner.run(FakeWorker(0.0, success=False), path, root=root, max_runs=1)
    assert done[0][0] == 0
    with open(path, "rb") as f:
        exps = pickle.load(f)
    assert exps[0]["status"] == "incomplete"
    big = dict(exps[1], n_modes=201)
    assert runner.choose_chi(big, root)[0] == "skip"
    assert runner.choose_chi(dict(exps[1], bond_dimension=40000), root)[0] == "skip"
