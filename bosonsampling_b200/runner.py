"""Experiment queue and result files of the reference's ``run.py``, one process, one GPU.

The reference's ``run.py`` (``main``, ``run.py:81-215``) takes the next experiment whose
``status`` is ``'incomplete'`` from ``experiments.pickle`` under a file lock, marks it
``'in progress'``, decides the bond dimension from earlier results (a stored run whose
layer-wise traces vary by more than 10% doubles chi), runs ``Worker.Simulate()`` and
saves ``Results/<type>/n_<n>_m_<m>_PS_<ps>_d_<d>_p_<params>_chi_<chi>_prob.npy``,
``..._chi_<chi>_EE.npy`` and the list of bond dimensions tried, ``...chi.npy``.  Its MPI
roles and ``comm.bcast`` are not needed with one GPU; the file formats, the queue and the
chi rule are the same, so results written here read back into ``analysis.ipynb``.

    python -m bosonsampling_b200.runner --seed 0 [--experiments experiments.pickle]
"""
import argparse
import contextlib
import fcntl
import os
import pickle

import numpy as np

MAX_CHI = 20000     # run.py:163-166
MAX_MODES = 200     # run.py:169-171


@contextlib.contextmanager
def file_lock(path):
    """An exclusive lock on ``path`` (the role of ``FileLock`` in ``run.py:91``)."""
    fd = os.open(path, os.O_CREAT | os.O_RDWR, 0o644)
    try:
        fcntl.flock(fd, fcntl.LOCK_EX)
        yield
    finally:
        fcntl.flock(fd, fcntl.LOCK_UN)
        os.close(fd)


def result_prefix(exp, root="Results"):
    """``Results/<type>/n_<n>_m_<m>_PS_<ps>_d_<d>_p_<params>_`` (``run.py:137``)."""
    return os.path.join(root, str(exp["input_state_type"]),
                        "n_{}_m_{}_PS_{}_d_{}_p_{}_".format(exp["n_modes"], exp["n_input_states"],
                                                            exp["post_selected_photon_number"],
                                                            exp["local_hilbert_space_dimension"],
                                                            exp["parameters"]))


def take_next(experiments_path, start):
    """Index and dict of the first ``'incomplete'`` experiment at or after ``start``,
    marked ``'in progress'`` in the file (``run.py:91-124``); ``(None, None)`` if none."""
    with file_lock(experiments_path + ".lock"):
        with open(experiments_path, "rb") as f:
            experiments = pickle.load(f)
        for idx in range(start, len(experiments)):
            if experiments[idx]["status"] == "incomplete":
                experiments[idx]["status"] = "in progress"
                with open(experiments_path, "wb") as f:
                    pickle.dump(experiments, f)
                exp = dict(experiments[idx])
                exp["status"] = "incomplete"
                return idx, exp
    return None, None


def release(experiments_path, idx):
    """Put an experiment back in the queue after an unsuccessful run."""
    with file_lock(experiments_path + ".lock"):
        with open(experiments_path, "rb") as f:
            experiments = pickle.load(f)
        experiments[idx]["status"] = "incomplete"
        with open(experiments_path, "wb") as f:
            pickle.dump(experiments, f)


def choose_chi(exp, root="Results"):
    """(status, chi) with the reference's rule (``run.py:141-171``): a stored run whose
    positive layer traces vary by more than 10% (max / min - 1 > 0.1) doubles the largest
    chi tried; a good stored run is skipped; chi > 20000 or n > 200 is skipped."""
    prefix = result_prefix(exp, root)
    chi = int(exp["bond_dimension"])
    status = "run"
    if os.path.isfile(prefix + "chi.npy"):
        chi = int(np.max(np.load(prefix + "chi.npy")))
        prob = np.load(prefix + "chi_{}_prob.npy".format(chi))
        prob = prob[prob > 0]
        error = np.max(prob) / np.min(prob) - 1 if len(prob) else np.inf
        if error > 0.1:
            chi *= 2
        else:
            status = "skip"
    if status == "run" and (chi > MAX_CHI or int(exp["n_modes"]) > MAX_MODES):
        status = "skip"
    return status, chi


def save_results(exp, chi, prob, EE, root="Results"):
    """``..._chi_<chi>_prob.npy``, ``..._chi_<chi>_EE.npy`` and ``...chi.npy``, only if
    some trace is positive (``run.py:193-215``).  Returns whether anything was written."""
    prefix = result_prefix(exp, root)
    if not np.sum(np.asarray(prob) > 0) > 0:
        return False
    os.makedirs(os.path.dirname(prefix), exist_ok=True)
    chis = np.load(prefix + "chi.npy") if os.path.isfile(prefix + "chi.npy") else np.array([])
    np.save(prefix + "chi_{}_prob.npy".format(chi), prob)
    np.save(prefix + "chi_{}_EE.npy".format(chi), EE)
    np.save(prefix + "chi.npy", np.append(chis, chi))
    return True


def run(worker, experiments_path="experiments.pickle", seed=0, root="Results", max_runs=None):
    """The loop of ``run.py:main``: returns the list of (index, chi, saved) it ran."""
    done = []
    start = 0
    while max_runs is None or len(done) < max_runs:
        idx, exp = take_next(experiments_path, start)
        if idx is None:
            if start == 0:
                break             # nothing left to run
            start = 0             # search again from the top
            continue
        start = idx + 1
        status, chi = choose_chi(exp, root)
        if status == "skip":
            continue
        worker.ExperimentInit(exp["input_state_type"], exp["n_modes"], exp["n_input_states"],
                              exp["post_selected_photon_number"], exp["local_hilbert_space_dimension"],
                              chi, exp["parameters"], seed)
        success, prob, EE, _ = worker.Simulate()
        saved = save_results(exp, chi, prob, EE, root)
        if not success:
            release(experiments_path, idx)
        done.append((idx, chi, saved))
    return done


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--experiments", default="experiments.pickle")
    p.add_argument("--results", default="Results")
    a = p.parse_args(argv)
    from .gpu_algorithm import Worker
    for idx, chi, saved in run(Worker(), a.experiments, a.seed, a.results):
        print("experiment %d: chi %d, %s" % (idx, chi, "saved" if saved else "not saved"))


if __name__ == "__main__":
    main()
