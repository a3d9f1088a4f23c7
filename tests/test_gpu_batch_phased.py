"""Phase-batched replicas: one launch per phase of the MD step over the blocks
of every replica, each replica's rebuild under its own conditional node.
The replicas must end bit-identical to the same engines stepped alone, and
to the graph-branch design."""
import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu


def _engines(rbx, specs, precision, seed=9):
    syss = [systems.lj_electrolyte(n, seed=sd) for n, sd in specs]
    out = [rbx.Engine(s, precision=precision, seed=seed) for s in syss]
    for e in out:
        e.compute_forces(0)
    return out


def _assert_same(e1, e2):
    a, c = e1.get_state(), e2.get_state()
    for key in ("pos", "vel", "force"):
        assert np.array_equal(a[key], c[key]), key
    s1, s2 = e1.stats(), e2.stats()
    assert s1.steps == s2.steps and s1.rebuilds == s2.rebuilds


def test_phased_batch_matches_single_engines(cuda, rbx):
    # sizes from the two-cell box (1,000 atoms) up; they rebuild on different steps
    specs = [(1000, 5), (2600, 6), (4000, 7), (6500, 8), (9100, 9)]
    batched = _engines(rbx, specs, rbx.MIXED)
    single = _engines(rbx, specs, rbx.MIXED)
    b = rbx.Batch(batched)
    b.step(7)
    assert b.design == rbx.Batch.PHASED
    b.step(23)
    for e in single:
        e.step(7)
        e.step(23)
    for e1, e2 in zip(batched, single):
        _assert_same(e1, e2)
    assert sum(e.stats().rebuilds for e in batched) >= len(specs)
    b.close()
    for e in batched + single:
        e.close()


def test_phased_and_branch_designs_agree(cuda, rbx):
    specs = [(3000, 21), (4000, 22), (5200, 23)]
    a = _engines(rbx, specs, rbx.MIXED, seed=4)
    c = _engines(rbx, specs, rbx.MIXED, seed=4)
    ba, bc = rbx.Batch(a), rbx.Batch(c)
    bc.set_mode(rbx.Batch.BRANCHES)
    for k in (5, 15):
        ba.step(k)
        bc.step(k)
    assert ba.design == rbx.Batch.PHASED and bc.design == rbx.Batch.BRANCHES
    for e1, e2 in zip(a, c):
        _assert_same(e1, e2)
    # switching a batch's design mid-run keeps the trajectory
    ba.set_mode(rbx.Batch.BRANCHES)
    bc.set_mode(rbx.Batch.PHASED)
    ba.step(10)
    bc.step(10)
    assert ba.design == rbx.Batch.BRANCHES and bc.design == rbx.Batch.PHASED
    for e1, e2 in zip(a, c):
        _assert_same(e1, e2)
    ba.close()
    bc.close()
    for e in a + c:
        e.close()


def test_phased_mode_needs_eligible_replicas(cuda, rbx):
    mixed = _engines(rbx, [(4000, 31)], rbx.MIXED)
    plain = _engines(rbx, [(4000, 32)], rbx.PLAIN_FP64)
    b = rbx.Batch(mixed + plain)
    b.set_mode(rbx.Batch.PHASED)
    with pytest.raises(rbx.RbxError, match="mixed form"):
        b.step(1)
    b.set_mode(rbx.Batch.AUTO)  # falls back to one branch per replica
    b.step(3)
    assert b.design == rbx.Batch.BRANCHES
    b.close()
    for e in mixed + plain:
        e.close()


def test_auto_design_follows_replica_size(cuda, rbx):
    # AUTO: phased below 5,000 atoms per replica on average, branches above;
    # an explicit mode overrides it, with the same trajectories either way
    big = _engines(rbx, [(6000, 41), (7000, 42)], rbx.MIXED)
    ref = _engines(rbx, [(6000, 41), (7000, 42)], rbx.MIXED)
    b = rbx.Batch(big)
    b.step(4)
    assert b.design == rbx.Batch.BRANCHES
    b.set_mode(rbx.Batch.PHASED)
    b.step(6)
    assert b.design == rbx.Batch.PHASED
    for e in ref:
        e.step(4)
        e.step(6)
    for e1, e2 in zip(big, ref):
        _assert_same(e1, e2)
    b.close()
    for e in big + ref:
        e.close()
