"""The parity tolerance every GPU test and smoke() apply (oracle/tolerance.py):
relative 1e-5 where the FP64 value is at least tau, absolute 1e-5 tau below."""

import numpy as np

from oracle import tolerance as TOL


def test_relative_above_tau_absolute_below():
    ref = np.zeros((2, 10))
    ref[0] = 100.0 * TOL.TAU            # well above every tau: the bound is relative
    ref[1] = 0.01 * TOL.TAU             # well below: the bound is 1e-5 tau, absolute
    just_in = ref + np.array([1e-5 * 100.0 * TOL.TAU, 1e-5 * TOL.TAU]) * 0.999
    just_out = ref + np.array([1e-5 * 100.0 * TOL.TAU, 1e-5 * TOL.TAU]) * 1.001
    assert (TOL.scaled_error(just_in, ref) <= 1.0).all()
    assert (TOL.scaled_error(just_out, ref) > 1.0).all()


def test_sign_and_shape():
    rng = np.random.default_rng(1)
    ref = rng.normal(size=(50, 10))
    x = ref + rng.normal(scale=1e-7, size=ref.shape)
    s = TOL.scaled_error(x, ref)
    assert s.shape == ref.shape
    assert np.allclose(TOL.scaled_error(-x, -ref), s)
    assert np.allclose(TOL.relative_error(x, ref), s * TOL.REL)


def test_tau_table():
    assert TOL.REL == 1e-5
    assert len(TOL.TERMS) == len(TOL.TAU) == 10
    assert set(TOL.TAU.tolist()) <= {0.05, 0.25, 0.5, 1.0}
    assert dict(zip(TOL.TERMS, TOL.TAU.tolist())) == {
        "vdw": 0.25, "ele": 0.5, "pmf": 0.25, "psp": 0.05, "hdb": 0.25,
        "hpc": 0.5, "kde": 0.05, "lhm": 0.05, "dst": 0.25, "total": 0.25}
