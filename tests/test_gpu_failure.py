"""Failure detection of the time step, through the C ABI.  No test here
faults, traps or hangs the GPU: the failures are planted in the inputs on the
host (a non-finite value, a zero Courant number, a momentum whose velocity
overflows) or made by the library's test hook that lets the sweep kernels'
bounded tile waits give up at once.

The reference stops its main loop on a non-positive dt (src/main.cpp:175-183)
and on a non-finite time (src/main.cpp:207-212); its CFL reduction skips a
non-finite cell through fmax (src/tstep.cpp:76-78).  This library returns
HOW_ERR_DT and HOW_ERR_NONFINITE for those and also reports a non-finite
state before stepping on it."""
import numpy as np
import pytest

from howtest import CPUOracle, active

pytestmark = pytest.mark.gpu

HOW_ERR_CUDA, HOW_ERR_NONFINITE, HOW_ERR_DT = -4, -6, -7


def _params(hm, n=(16, 16, 16), **kw):
    args = dict(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=1.0, gam=5.0 / 3.0, cour=0.4, problem="blast3d_b",
                rhomin=1e-6, pgmin=1e-6)
    args.update(kw)
    return hm.make_parameters(**args)


@pytest.mark.parametrize("value", [np.nan, np.inf], ids=["nan", "inf"])
def test_nonfinite_state_stops_the_run(value):
    import how_mhd as hm
    p = _params(hm)
    q = hm.problem_state(p)
    active(q, 16, 16, 16)[7, 5, 6, 7] = value
    with hm.Domain(p) as dom:
        dom.set_state(q)
        dom.bound(0)
        dom.initialize_bfield_from_q()
        with pytest.raises(hm.HowError) as e:
            dom.run(0.0, 3)
        assert e.value.code == HOW_ERR_NONFINITE, e.value
        with pytest.raises(hm.HowError) as e:
            dom.tstep()
        assert e.value.code == HOW_ERR_NONFINITE
        # the state was not stepped on
        np.testing.assert_array_equal(active(dom.get_state(0), 16, 16, 16), active(q, 16, 16, 16))


def test_zero_courant_number_gives_non_positive_dt():
    """cour 0: dt = 0, the reference's "non-positive dt detected" stop."""
    import how_mhd as hm
    p = _params(hm, cour=0.0)
    with hm.Domain(p) as dom:
        dom.init_problem()
        with pytest.raises(hm.HowError) as e:
            dom.run(0.0, 2)
        assert e.value.code == HOW_ERR_DT and "non-positive dt" in str(e.value)


def test_overflowing_velocity_gives_non_positive_dt():
    """A finite state whose velocity overflows to infinity: the signal speed
    is infinite, dt = cour / inf = 0 -- in the reference (checked on the
    oracle) and here."""
    import how_mhd as hm
    n = (16, 16, 16)
    p = _params(hm)
    q = hm.problem_state(p)
    a = active(q, *n)
    a[0, 4, 4, 4] = 1e-3
    a[1, 4, 4, 4] = 1e308          # vx = 1e311: overflows to inf
    o = CPUOracle(*n, rhomin=1e-6, pgmin=1e-6)
    o.set_state(q)
    assert o.tstep() == 0.0
    with hm.Domain(p) as dom:
        dom.set_state(q)
        dom.bound(0)
        dom.initialize_bfield_from_q()
        assert dom.tstep() == 0.0
        with pytest.raises(hm.HowError) as e:
            dom.run(0.0, 2)
        assert e.value.code == HOW_ERR_DT


def test_expired_tile_wait_is_reported_and_context_recovers():
    """The sweep kernels' tile waits are bounded.  The test hook makes the
    compute threads give up at once: the step returns HOW_ERR_CUDA with the
    kernel's status ("bounded TMA wait expired") instead of hanging, every
    block still waits for its copies in flight before it exits, and the same
    context then steps exactly as a fresh one."""
    import how_mhd as hm
    p = _params(hm, n=(24, 24, 24))
    with hm.Domain(p) as dom:
        dom.init_problem()
        dt = dom.tstep()
        dom.set_wait_limit(True)
        with pytest.raises(hm.HowError) as e:
            dom.ssprk(dt)
        assert e.value.code == HOW_ERR_CUDA and "bounded TMA wait expired" in str(e.value)
        dom.set_wait_limit(False)
        dom.init_problem()
        dom.run(0.0, 2)
        q = dom.get_state(0)
    with hm.Domain(p) as fresh:
        fresh.init_problem()
        fresh.run(0.0, 2)
        np.testing.assert_array_equal(fresh.get_state(0), q)
