"""Host logic of the reference-named driver routines in
oversetdevfort_b200.api (CPU only): check_convergence as
src/solveFlow.f90:192-222 writes it, the istep rules of
solmultiphasethermofluid_stag (:50-54, :109) and the setBCs entry points,
on a stand-in context that records the calls."""
import numpy as np

from oversetdevfort_b200 import api as A


def test_check_convergence_semantics():
    r0 = np.array([1.0, 2.0, 3.0, 4.0])
    tol = (1e-3, 1e-3, 1e-2, 1e-1)
    atol = (1e-12, 1e-12, 1e-13, 1e-14)
    below = np.array([1e-4, 1e-4, 1e-3, 1e-2])
    np.testing.assert_array_equal(A.check_convergence(below, r0, tol, 7, atol), [1, 1, 1, 1])
    # strict comparison: residual == tol * residual0 is not converged
    at = np.array(tol) * r0
    np.testing.assert_array_equal(A.check_convergence(at, r0, tol, 7, atol), [0, 0, 0, 0])
    # the absolute test alone: residual0 = 0 converges only below atol
    z = np.zeros(4)
    np.testing.assert_array_equal(A.check_convergence(z, z, tol, 7, atol), [1, 1, 1, 1])
    np.testing.assert_array_equal(A.check_convergence(z, z, tol, 7, (0.0,) * 4), [0, 0, 0, 0])
    # fields outside the flag stay 0
    np.testing.assert_array_equal(A.check_convergence(below, r0, tol, 3, atol), [1, 1, 1, 0])
    np.testing.assert_array_equal(A.check_convergence(below, r0, tol, 1, atol), [1, 1, 0, 0])
    np.testing.assert_array_equal(A.check_convergence(below, r0, tol, 4, atol), [0, 0, 0, 1])
    # one field above its tolerance
    mixed = below.copy()
    mixed[1] = 1.0
    np.testing.assert_array_equal(A.check_convergence(mixed, r0, tol, 7, atol), [1, 0, 1, 1])


class _Recorder:
    def __init__(self):
        self.calls = []

    def quench_newton(self, **kw):
        self.calls.append(("quench_newton", kw))
        return kw

    def apply_bcs(self, which):
        self.calls.append(("apply_bcs", which))


def test_newton_routine_istep_rules():
    ctx = _Recorder()
    kw = A.solmultiphasethermofluid_stag(ctx, 0, newton_max=4, kspace=80)
    assert kw["newton_max"] == 1 and kw["solve_tem"] is False and kw["kspace"] == 80
    kw = A.solmultiphasethermofluid_stag(ctx, 1, newton_max=4)
    assert kw["newton_max"] == 1 and kw["solve_tem"] is True
    kw = A.solmultiphasethermofluid_stag(ctx, 2, newton_max=4)
    assert kw["newton_max"] == 4 and kw["solve_tem"] is True
    kw = A.solmultiphasethermofluid_stag(ctx, 5, solve_tem=False)
    assert kw["newton_max"] == 3 and kw["solve_tem"] is False


def test_setbcs_entry_points():
    ctx = _Recorder()
    A.setBCs_NSVOF(ctx)
    A.setBCs_Tem(ctx)
    assert ctx.calls == [("apply_bcs", 1), ("apply_bcs", 2)]
