"""Initial-guess extrapolation (initial_guess_extrapolation of the reference,
src/solvers/3d/ins_solver.cpp:342-343): the polynomial through the history
points, evaluated at the new time."""
import numpy as np
import pytest

import sipg


def _history(m, n, seed):
    rng = np.random.default_rng(seed)
    coef = rng.standard_normal((m, n))          # a polynomial of degree m-1 in t per entry
    times = np.sort(rng.uniform(0.0, 1.0, m)) + np.arange(m)
    hist = [sum(coef[k] * t ** k for k in range(m)) for t in times]
    return coef, times, hist


@pytest.mark.parametrize("m", [1, 2, 3, 4])
def test_host_extrapolation_reproduces_polynomials(m):
    coef, times, hist = _history(m, 257, seed=m)
    t_new = times[-1] + 0.7
    want = sum(coef[k] * t_new ** k for k in range(m))
    got = sipg.extrapolate_initial_guess(times, hist, t_new)
    assert np.allclose(got, want, rtol=1e-10, atol=1e-10)


def test_invalid_history_is_rejected():
    with pytest.raises(sipg.SipgError):
        sipg.extrapolate_initial_guess([1.0, 1.0], [np.zeros(3), np.ones(3)], 2.0)


@pytest.mark.gpu
@pytest.mark.parametrize("m", [1, 3])
def test_device_extrapolation_matches_host(m):
    coef, times, hist = _history(m, 10001, seed=10 + m)
    t_new = times[-1] + 0.5
    dev = [sipg.DeviceVector(h) for h in hist]
    out = sipg.DeviceVector(np.zeros(10001))
    sipg.extrapolate_initial_guess_device(times, [d.ptr for d in dev], t_new, 10001, out.ptr)
    host = sipg.extrapolate_initial_guess(times, hist, t_new)
    assert np.allclose(out.get(), host, rtol=1e-13, atol=1e-13)
