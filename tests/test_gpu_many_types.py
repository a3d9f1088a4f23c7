"""More atom types than the old 16-type shared-memory tables held: the
4000-atom LJ electrolyte with its atoms spread over 40 LJ types (seeded
sigma in [0.9, 1.1], eps in [0.5, 1.5]; the ions keep their charges).  The
per-type-pair tables of the pair kernels are sized in shared memory from the
type count.  RBL engines in both forms against the oracle's RBL + RBE
evaluation (1e-9 / 1e-5 relative RMS force, exact RBL pair sets), a
Verlet-list engine's pair energies within 1e-10, and a request above the
engine's limit rejected with a clear error.
"""
import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu

NT = 40


@pytest.fixture(scope="module")
def sys_many():
    s = systems.lj_electrolyte(4000, seed=91)
    rng = np.random.default_rng(5)
    s = dict(s)
    s["type"] = rng.integers(0, NT, size=s["n"]).astype(np.int32)
    s["sigma"] = rng.uniform(0.9, 1.1, NT)
    s["eps"] = rng.uniform(0.5, 1.5, NT)
    s["mass"] = np.ones(NT)
    return s


def test_many_types_rbl_against_oracle(cuda, rbx, oracle, sys_many):
    s = sys_many
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbe_sample_philox(box, 0.16, 100, 13, 2)
    want = oracle.rbl_rbe_evaluation(s, m, epoch=2)
    for prec, tol in ((rbx.PLAIN_FP64, 1e-9), (rbx.MIXED, 1e-5)):
        e = rbx.Engine(s, precision=prec)
        e.set_k_samples(*m)
        e.compute_forces(epoch=2)
        fp, fk = e.force_parts()
        assert systems.rel_rms(fp + fk, want["force"]) < tol, prec
        gc, gs = e.rbl_pairs()
        assert np.array_equal(oracle.pair_keys(gc), want["core_keys"]), prec
        assert np.array_equal(oracle.pair_keys(gs), want["shell_keys"]), prec
        el, ec, _ = e.pair_energy()
        assert abs(el - want["e_vdwl"]) < 1e-10 * abs(want["e_vdwl"]), prec
        e.step(3)
        assert np.isfinite(e.get_state()["force"]).all()
        e.close()


def test_many_types_verlet_energy(cuda, rbx, oracle, sys_many):
    s = sys_many
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbe_sample_philox(box, 0.16, 100, 13, 2)
    want = oracle.rbl_rbe_evaluation(s, m, epoch=0)
    e = rbx.Engine(s, precision=rbx.PLAIN_FP64, neighbor="VERLET")
    e.set_k_samples(*m)
    e.compute_forces(epoch=0)
    el, ec, vp = e.pair_energy()
    assert abs(el - want["e_vdwl"]) < 1e-10 * abs(want["e_vdwl"])
    assert abs(ec - want["e_coul"]) < 1e-10 * abs(want["e_coul"])
    assert np.abs(vp - want["virial_pair"]).max() < 1e-10 * np.abs(want["virial_pair"]).max()
    e.close()


def test_type_limit_rejected(cuda, rbx, sys_many):
    s = dict(sys_many)
    big = rbx.MAX_TYPES + 1
    s["sigma"], s["eps"], s["mass"] = np.ones(big), np.ones(big), np.ones(big)
    with pytest.raises(rbx.RbxError, match="ntypes must be in"):
        rbx.Engine(s)
