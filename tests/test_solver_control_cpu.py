"""Newton control of StaticImplicitSolver on the host, driven by a scripted
residual sequence instead of the device (no GPU): the relative stop test,
the round-off floor exit of the relative mode (floor_rtol: the residual has
stopped halving below 1e-9 of the first one) and the failure return of the
absolute mode when no step is accepted."""
import torch

from fea_b200.solver import StaticImplicitSolver


class _Script:
    """An assembly whose residual at iteration k has the scripted norm."""

    def __init__(self, norms):
        self.norms = list(norms)
        self.calls = 0

    def assemble_csr(self, GC):
        k = min(self.calls, len(self.norms) - 1)
        self.calls += 1
        R = torch.zeros(4, dtype=torch.float64)
        R[0] = self.norms[k]
        return R, torch.ones(4, dtype=torch.float64)


class _Scripted(StaticImplicitSolver):
    """The solver's Newton loop with the device parts replaced: unit steps,
    a zero correction, a constant energy."""

    def __init__(self, norms, alpha=1.0, **kw):
        super().__init__(**kw)
        self.assembly = _Script(norms)
        self.alpha = alpha

    def get_total_energy(self, GC_now):
        return torch.tensor(0.0, dtype=torch.float64)

    def _scaled_rmax_dev(self, K_values, R):
        return R.abs().max()

    def _linear_request(self, K_values, R, iter_now=0, alpha0=None, dGC0=None, srmax=None):
        return torch.zeros_like(R)

    def _run_linear(self, req):
        pass

    def _linear_finish(self, req, K_values, R):
        return req

    def _line_search(self, GC0, dGC, R, energy0):
        if self.alpha == 0.0:
            return 0.0, GC0.clone(), energy0
        return self.alpha, GC0 + self.alpha * dGC, energy0


def _run(s):
    return s._solve_iteration(torch.zeros(4, dtype=torch.float64), s.tol_error)


def test_relative_stop_test():
    s = _Scripted([1.0, 1e-2, 1e-5, 1e-9, 1e-13], rtol=1e-12)
    assert not isinstance(_run(s), bool)
    assert [h["rnorm"] for h in s.history] == [1.0, 1e-2, 1e-5, 1e-9, 1e-13]


def test_round_off_floor_ends_the_relative_mode():
    # below floor_rtol (1e-9 of the first) the residual stops halving: the
    # first residual at the floor that is not half the smallest of the three
    # before it (2.5e-10 against 3e-10) ends the loop with the iterate
    norms = [1.0, 1e-3, 1e-7, 3e-10, 2.5e-10, 2.6e-10, 2.4e-10, 2.5e-10, 2.45e-10]
    s = _Scripted(norms, rtol=1e-14)
    assert not isinstance(_run(s), bool)
    assert len(s.history) == 5
    assert s.history[-1]["rnorm"] == 2.5e-10


def test_no_floor_exit_above_floor_rtol():
    # stagnation above 1e-9 of the first residual is not the floor: the loop
    # goes on until its iteration cap and reports failure
    norms = [1.0, 1e-3, 1e-6, 5e-7, 5e-7, 5e-7, 5e-7, 5e-7]
    s = _Scripted(norms, rtol=1e-14, maximum_iteration=12)
    assert _run(s) is False
    assert len(s.history) == 13


def test_absolute_mode_fails_when_no_step_is_accepted():
    s = _Scripted([1.0, 1.0], alpha=0.0, tol_error=1e-5)
    assert _run(s) is False


def test_halving_below_the_floor_goes_on_to_rtol():
    norms = [1.0, 1e-5, 5e-10, 2e-10, 9e-11, 4e-11, 1e-15]
    s = _Scripted(norms, rtol=1e-14)
    assert not isinstance(_run(s), bool)
    assert len(s.history) == 7 and s.history[-1]["rnorm"] == 1e-15
