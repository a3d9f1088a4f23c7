"""NVT (Nose-Hoover chain) in the oracle's whole step, on the CPU.

The oracle restates NVTensemble::Solve with temp_ctrl_type NOSE_HOOVER
(nvt_ensemble.cpp:128-160, NoseHooverController): the chain scales the
velocities before the first half kick and after the second.  Checked here by
behaviour: the temperature the chain tracks is the kinetic temperature of the
velocities, the thermostat pulls a system at T = 1 to the target, a ramp
follows t_start -> t_stop, and an off thermostat is plain NVE.
"""
import numpy as np
import pytest

from rbmd_b200 import systems


def _kinetic_t(sys, vel, tdof):
    m = np.asarray(sys["mass"], float)[sys["type"]]
    return (m[:, None] * vel ** 2).sum() / tdof


@pytest.fixture(scope="module")
def sys4k():
    return systems.lj_electrolyte(4000, seed=61)


def test_thermostat_tracks_kinetic_temperature(oracle, sys4k):
    e = oracle.Engine(sys4k, seed=3)
    e.compute_forces(0)
    e.set_nose_hoover(1.2, 1.2, 0.1)
    tdof = 3 * sys4k["n"] - 3
    t0 = e.thermostat()["temperature"]
    assert abs(t0 - _kinetic_t(sys4k, sys4k["vel"], tdof)) < 1e-12 * t0
    e.step(5)
    got = e.thermostat()
    assert abs(got["temperature"] - _kinetic_t(sys4k, e.get()["vel"][np.argsort(e.get()["gid"])],
                                               tdof)) < 1e-10 * got["temperature"]
    assert (got["eta_dot"] != 0).all()


@pytest.mark.slow
def test_thermostat_reaches_target(oracle, sys4k):
    """From T = 1 toward T = 1.5 with t_damp = 20 dt: the mean over the last
    half of 400 steps is within 5 % of the target; an NVE run stays near 1."""
    out = {}
    for name, damp in (("nvt", 0.1), ("nve", 0.0)):
        e = oracle.Engine(sys4k, seed=3)
        e.compute_forces(0)
        e.set_nose_hoover(1.5, 1.5, damp)
        temps = []
        for _ in range(40):
            e.step(10)
            g = e.get()
            temps.append(_kinetic_t(sys4k, g["vel"][np.argsort(g["gid"])], 3 * sys4k["n"] - 3))
        out[name] = np.asarray(temps)
    assert abs(out["nvt"][20:].mean() - 1.5) < 0.05 * 1.5
    assert abs(out["nve"][20:].mean() - 1.5) > 0.2


def test_temperature_ramp(oracle, sys4k):
    e = oracle.Engine(sys4k, seed=3)
    e.compute_forces(0)
    e.set_nose_hoover(1.0, 2.0, 0.05, num_steps=200)
    e.step(200)
    g = e.get()
    t_end = _kinetic_t(sys4k, g["vel"][np.argsort(g["gid"])], 3 * sys4k["n"] - 3)
    assert t_end > 1.4
