"""BatchRun's host logic on the CPU (no solver): when a case leaves the batch -- at its step
target, or when the window means of its discharge sum (and, optionally, of its lid level)
stop changing."""
import numpy as np

from water_flow_simulation_b200.batch import BatchRun


class _Lattice:
    def __init__(self, series):
        self.series, self.k = series, 0

    def profile_sums(self, mean=False):
        q, level = self.series[self.k]
        self.k += 1
        return {"q": np.array([q]), "top_drho": np.array([level]), "top_n": np.array([1.0])}


class _Run:
    def __init__(self, series, vel=10.0):
        self.lbm = _Lattice(series)
        self.r = type("R", (), {"vel": vel})()


def _batch(series_per_case, tol=None, window=1, level_tol_cm=None, target=10 ** 9, check_every=20,
           observe_only=False):
    B = BatchRun.__new__(BatchRun)
    B.runs = [_Run(s) for s in series_per_case]
    n = len(B.runs)
    B.active = list(range(n))
    B.steps_done = [0] * n
    B.target = [target] * n
    B.samples = [[] for _ in range(n)]
    B.converged = [False] * n
    B.steps_to_converge = [None] * n
    B.level_at_stop = [None] * n
    B.observe_only = observe_only
    B.tol, B.window, B.check_every, B.level_tol_cm = tol, window, check_every, level_tol_cm
    B.rebatched = 0

    def rebatch():
        B.rebatched += 1
    B._rebatch = rebatch
    return B


def _advance(B, chunks):
    for _ in range(chunks):
        for i in B.active:
            B.steps_done[i] += 20
        B._retire()


def test_cases_leave_at_their_step_target():
    B = _batch([[(1.0, 0.0)] * 10] * 2, target=60)
    _advance(B, 2)
    assert B.active == [0, 1]
    _advance(B, 1)
    assert B.active == [] and B.rebatched == 1 and B.converged == [False, False]


def test_window_means_of_the_discharge_decide_convergence():
    steady = [(100.0, 0.0)] * 10
    noisy = [(100.0 + (5.0 if k % 2 else -5.0), 0.0) for k in range(10)]
    B = _batch([steady, noisy], tol=1e-3, window=1)
    _advance(B, 2)                                  # two samples: case 0 has converged
    assert B.converged == [True, False] and B.steps_to_converge[0] == 40 and B.active == [1]
    B = _batch([noisy], tol=1e-3, window=2)         # window means of 2 samples average the noise out
    _advance(B, 4)
    assert B.converged == [True] and B.steps_to_converge[0] == 80


def test_level_tolerance_holds_a_case_back():
    """Discharge steady, lid level still moving by 1e-4 in rho (vel 10 m/s per lattice unit:
    100/3 * 100/9.81 * 1e-4 = 0.034 cm per sample)."""
    series = [(50.0, 1e-4 * k) for k in range(10)]
    B = _batch([series], tol=1e-3, level_tol_cm=0.01)
    _advance(B, 5)
    assert B.converged == [False]
    B = _batch([series], tol=1e-3, level_tol_cm=0.05)
    _advance(B, 2)
    assert B.converged == [True]


def test_observe_only_records_the_stop_and_runs_on():
    """observe_only: the case that meets the rule stays in the batch to its target, with the
    step and the window-mean level of the stop recorded (and checked no more)."""
    B = _batch([[(1.0, 0.0)] * 6], tol=1e-3, target=120, observe_only=True)
    _advance(B, 2)
    assert B.converged == [True] and B.steps_to_converge[0] == 40 and B.active == [0]
    assert B.level_at_stop[0] is not None
    _advance(B, 4)
    assert B.active == [] and B.steps_to_converge[0] == 40 and B.steps_done[0] == 120
