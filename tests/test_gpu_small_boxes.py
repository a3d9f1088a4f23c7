"""Boxes with fewer than three cells of edge cut_off + skin along an axis:
edges between 2 and 3 times cut_off + skin (953 <= N < 3216 atoms for the
cubic LJ electrolyte at rho* = 0.8; below N = 953 the edge is shorter than
2 (cut_off + skin) and the engine rejects the box).  The candidate rows come
from an all-pairs builder with the FP64 list predicate, each pair once (the
reference's (2c + 1)^3 stencil over cells of edge (cut_off + skin) / c wraps
onto the same cell more than once along an axis with fewer than 2c + 1 cells
and lists those pairs repeatedly, tests/test_golden_rows.py; the oracle's
stencil visits each distinct cell once).

Checked: RBL + RBE forces in both forms against the oracle (1e-9 / 1e-5
relative RMS), exact RBL pair sets, the Verlet-list pair energies, steps
with rebuilds that keep the pair sets exact, a box with 2 and 3 cells on
different axes, and small replicas inside a batch bit-identical to the same
engines stepped alone.
"""
import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu


def _stretched(n, seed, scale):
    s = systems.lj_electrolyte(n, seed=seed)
    lo = np.asarray(s["lo"], float)
    sc = np.asarray(scale, float)
    hi = lo + (np.asarray(s["hi"], float) - lo) * sc
    return dict(s, lo=lo, hi=hi, pos=lo + (s["pos"] - lo) * sc)


CASES = [("cubic_n1200", 1200, (1.0, 1.0, 1.0)),        # 2 x 2 x 2 cells
         ("mixed_n2400", 2400, (0.8, 1.25, 1.0))]       # 2 x 3 x 2 cells


@pytest.mark.parametrize("name,n,scale", CASES, ids=[c[0] for c in CASES])
def test_small_box_forces_and_pairs(cuda, rbx, oracle, name, n, scale):
    s = _stretched(n, 31, scale)
    L = np.asarray(s["hi"]) - np.asarray(s["lo"])
    assert (L >= 2 * 5.3).all() and (np.floor(L / 5.3) < 3).any()
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbe_sample_philox(box, 0.16, 100, 17, 4)
    want = oracle.rbl_rbe_evaluation(s, m, epoch=4)
    for prec, tol in ((rbx.PLAIN_FP64, 1e-9), (rbx.MIXED, 1e-5)):
        e = rbx.Engine(s, precision=prec)
        e.set_k_samples(*m)
        e.compute_forces(epoch=4)
        fp, fk = e.force_parts()
        assert systems.rel_rms(fp + fk, want["force"]) < tol, prec
        gc, gs = e.rbl_pairs()
        assert np.array_equal(oracle.pair_keys(gc), want["core_keys"]), prec
        assert np.array_equal(oracle.pair_keys(gs), want["shell_keys"]), prec
        el, ec, vp = e.pair_energy()
        assert abs(el - want["e_vdwl"]) < 1e-10 * abs(want["e_vdwl"]), prec
        assert abs(ec - want["e_coul"]) < 1e-10 * abs(want["e_coul"]), prec
        e.close()


def test_small_box_steps_keep_exact_pairs(cuda, rbx, oracle):
    """Velocity-Verlet steps with list rebuilds: after each block of steps the
    engine's RBL pairs equal the oracle's lists on the engine's own positions."""
    s = systems.lj_electrolyte(1500, seed=8)
    e = rbx.Engine(s, precision=rbx.PLAIN_FP64, seed=4)
    e.compute_forces(0)
    p = s["params"]
    for k in range(4):
        e.step(15)
        st = e.get_state()
        ep = e.stats().epoch
        e.compute_forces(epoch=ep)
        gc, gs = e.rbl_pairs()
        box = oracle.Box.make(s["lo"], s["hi"])
        x, y, z = (np.ascontiguousarray(st["pos"][:, d]) for d in range(3))
        perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
        xs, ys, zs = x[perm], y[perm], z[perm]
        cnt, rows = oracle.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
        freq = oracle.rbl_params(s["n"], box, p["r_core"], p["cut_off"],
                                 p["neighbor_sample_num"])[0]
        gid = np.asarray(s["gid"])[perm]
        cc, core, sc, shell = oracle.rbl_filter(box, p["r_core"], p["cut_off"], freq, ep, gid, xs,
                                                ys, zs, cnt, rows)
        core_keys = oracle._pair_keys(gid, cc, core)
        shell_keys = oracle._pair_keys(gid, sc, shell)
        assert np.array_equal(oracle.pair_keys(gc), core_keys), k
        assert np.array_equal(oracle.pair_keys(gs), shell_keys), k
    assert e.stats().rebuilds >= 2
    e.close()


def test_small_replicas_in_batch(cuda, rbx):
    specs = [(1000, 5, rbx.MIXED), (2600, 6, rbx.PLAIN_FP64), (5000, 7, rbx.MIXED)]
    syss = [systems.lj_electrolyte(n, seed=sd) for n, sd, _ in specs]
    batched = [rbx.Engine(s, precision=p, seed=9) for s, (_, _, p) in zip(syss, specs)]
    single = [rbx.Engine(s, precision=p, seed=9) for s, (_, _, p) in zip(syss, specs)]
    for e in batched + single:
        e.compute_forces(0)
    b = rbx.Batch(batched)
    b.step(25)
    for e in single:
        e.step(25)
    for e1, e2 in zip(batched, single):
        a, c = e1.get_state(), e2.get_state()
        for key in ("pos", "vel", "force"):
            assert np.array_equal(a[key], c[key]), key
        assert e1.stats().rebuilds == e2.stats().rebuilds
    b.close()
    for e in batched + single:
        e.close()


def test_box_below_two_list_radii_rejected(cuda, rbx):
    s = systems.lj_electrolyte(900, seed=1)  # edge 10.4 < 2 (cut_off + skin) = 10.6
    with pytest.raises(rbx.RbxError, match="exceeds half the box length"):
        rbx.Engine(s)
