"""Host logic of the Python stepper mirrors (solver/time/ExplicitTimeStepper.cpp:36-100): which
solver calls each one makes per step (no GPU: a recording stand-in for the solver)."""

from pdekit_b200.rds import RK3TVD, ExplicitEuler


class _Recorder:
    def __init__(self):
        self.calls = []

    def assemble_lhs_and_rhs(self, cfl):
        self.calls.append(("assemble_lhs_and_rhs", cfl))

    def solve(self):
        self.calls.append(("solve",))

    def advance_rk3tvd(self, cfl, nsteps):
        self.calls.append(("advance_rk3tvd", cfl, nsteps))


def test_explicit_euler_is_assemble_then_solve():
    s = _Recorder()
    stepper = ExplicitEuler()
    stepper.setup(1, 10)
    stepper.advance_in_time(s, 0.9)
    assert s.calls == [("assemble_lhs_and_rhs", 0.9), ("solve",)]


def test_rk3tvd_is_one_device_step_per_call():
    s = _Recorder()
    stepper = RK3TVD()
    stepper.setup(4, 10)
    stepper.advance_in_time(s, 0.5)
    stepper.advance_in_time(s, 0.25)
    assert s.calls == [("advance_rk3tvd", 0.5, 1), ("advance_rk3tvd", 0.25, 1)]
