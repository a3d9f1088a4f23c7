"""The FP64 oracle against golden outputs of more of RBMD's kernels: linked
cells and the full candidate list, the CVFF special-bond RBL pair force, the
RBSOG far field with its virial, SHAKE / RATTLE, and the RBE + RBL path at
N = 51,200.

Fixtures come from tests/golden/make_golden.py (groups cells, special, rbsog,
shake, large), which runs the reference's .hip.cu kernels compiled in place for
sm_100a on the inputs stored in each file (the large case regenerates its
inputs from the seed and checks them against a stored digest).
"""
import hashlib
import os

import numpy as np
import pytest

from rbmd_b200 import systems

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    return dict(np.load(path))


def _pairs(gid, counts, rows):
    owner = np.repeat(np.arange(len(counts)), counts)
    flat = np.concatenate([rows[i][:counts[i]] for i in range(len(counts))])
    p = np.stack([gid[owner].astype(np.int64), gid[flat].astype(np.int64)], 1)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# --- linked cells and the full list -----------------------------------------
@pytest.mark.parametrize("name", ["ref_cells_n3328.npz", "ref_cells_n1200.npz"])
@pytest.mark.parametrize("c", [1, 3])
def test_cells_and_full_list(oracle, name, c):
    """Cell of every atom (AssignAtomsToCell with its one-cell correction),
    atoms per cell, and the list of pairs within cut_off + skin = 5.3 as a set.
    c = 3 is the RBL builder's grid (cells of edge 5.3 / 3, a 7^3 stencil).
    Where an axis holds fewer than 2c + 1 cells the reference's stencil visits
    a wrapped cell more than once and lists those pairs repeatedly; the oracle
    lists each pair once, and equals the reference's list with the repeats
    removed."""
    f = _load(name)
    box = oracle.Box.make(f["lo"], f["hi"])
    x, y, z = f["x"], f["y"], f["z"]
    dims = f[f"c{c}_dims"]
    perm, cell_sorted, cs, ce = oracle.cells_sort(box, 5.3 / c, x, y, z)
    assert np.array_equal(oracle.cell_grid(box, 5.3 / c)[1], dims)
    cell = np.empty_like(cell_sorted)
    cell[perm] = cell_sorted
    assert np.array_equal(cell, f[f"c{c}_cell"])
    assert np.array_equal(ce - cs, f[f"c{c}_cell_count"])
    # the candidate set within 5.3 from the oracle's cut_off + skin grid
    p2, c2, s2, e2 = oracle.cells_sort(box, 5.3, x, y, z)
    cnt, rows = oracle.full_list(box, 5.3, x[p2], y[p2], z[p2], c2, s2, e2)
    gid = np.asarray(f["gid"])[p2]
    pairs = _pairs(gid, cnt, rows)
    assert _sha(pairs) == str(f[f"c{c}_unique_digest"])
    dup = int(f[f"c{c}_duplicates"])
    if (dims >= 2 * c + 1).all():
        assert dup == 0
        assert str(f[f"c{c}_list_digest"]) == str(f[f"c{c}_unique_digest"])
        want = np.empty(len(x), dtype=np.int64)
        want[p2] = cnt
        assert np.array_equal(want, f[f"c{c}_list_count"].astype(np.int64))
    else:
        assert dup > 0


# --- CVFF special-bond RBL pair force ---------------------------------------
@pytest.mark.parametrize("variant", ["optimized", "reference"])
def test_special_rbl_force(oracle, variant):
    """SpecialLJCutCoulRBLForceOp, both kernels RBMD ships, on case A's atoms,
    the oracle's RBL lists and seeded special rows (weights 0, 0.5, 0.8)."""
    f = _load(f"ref_special_{variant}.npz")
    g = _load("ref_caseA.npz")
    box = oracle.Box.make(g["lo"], g["hi"])
    x, y, z = g["x"], g["y"], g["z"]
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    cnt, rows = oracle.full_list(box, 5.3, x, y, z, cell, cs, ce)
    cc, core, sc, shell = oracle.rbl_filter(box, 2.5, 5.0, int(g["freq"]), int(g["epoch"]),
                                            g["gid"], x, y, z, cnt, rows)
    assert np.array_equal(cc, f["core_count"]) and np.array_equal(sc, f["shell_count"])
    want = oracle.pair_force_rbl_special(box, 2.5, 5.0, int(g["freq"]), 0.16, 1.0, g["type"],
                                         g["sigma"], g["eps"], g["gid"], g["q"], x, y, z, cc,
                                         core, sc, shell, f["nspecial"], f["special"],
                                         tuple(f["weights"]))
    assert systems.rel_rms(f["f64_force"], want) < 1e-12
    assert systems.rel_rms(f["f32_force"], want) < 1e-4
    # the weights act: the same force without special rows differs
    plain = oracle.pair_force_rbl(box, 2.5, 5.0, int(g["freq"]), 0.16, 1.0, g["type"],
                                  g["sigma"], g["eps"], g["q"], x, y, z, cc, core, sc, shell)
    assert systems.rel_rms(plain, want) > 1e-3


# --- RBSOG far field ---------------------------------------------------------
def test_rbsog_far_field_and_virial(oracle):
    """ComputeRBSOGSampleForceOp + ComputeRBSOGDirectForceOp (force, energy,
    virial with the NPT terms over the chain's gather map) against the
    oracle's RBSOG force, energy and virial; the gather map against the
    oracle's restatement of the chain on the stored uniforms."""
    f = _load("ref_rbsog_l2.npz")
    box = oracle.Box.make(f["lo"], f["hi"])
    lvl = int(f["level"])
    m = (f["mx"], f["my"], f["mz"])
    x, y, z, q = f["x"], f["y"], f["z"], f["q"]
    prm = oracle.rbsog_params(lvl, 5.0, box)
    assert prm["S"] == pytest.approx(float(f["S"]), rel=1e-14)
    assert prm["S_npt"] == pytest.approx(float(f["S_npt"]), rel=1e-14)
    assert np.array_equal(oracle.rbsog_idx_npt(lvl, 5.0, box, m, f["u"]), f["idx"])
    force, energy = oracle.rbsog_force(lvl, 5.0, box, 1.0, q, m, x, y, z)
    self_e = -prm["self_coeff"] * float((q ** 2).sum())
    ref_f = f["f64_force_sample"] + f["f64_force_direct"]
    assert systems.rel_rms(ref_f, force) < 1e-11
    assert abs(float(f["f64_energy_parts"].sum()) + self_e - energy) < 1e-11 * abs(energy)
    vir = oracle.rbsog_virial(lvl, 5.0, box, 1.0, q, m, f["idx"], x, y, z)
    ref_v = f["f64_virial_sample"] + f["f64_virial_direct"]
    assert np.abs(ref_v - vir).max() < 1e-11 * np.abs(vir).max()
    # RBMD's FP32 build to FP32 accuracy
    ref32 = f["f32_force_sample"].astype(np.float64) + f["f32_force_direct"]
    assert systems.rel_rms(ref32, force) < 1e-4
    v32 = f["f32_virial_sample"].astype(np.float64) + f["f32_virial_direct"]
    assert np.abs(v32 - vir).max() < 1e-4 * np.abs(vir).max()


# --- RBE + RBL at N = 51,200 -------------------------------------------------
def test_large_case(oracle):
    f = _load("ref_large_n51200.npz")
    n, seed = int(f["n"]), int(f["seed"])
    s = systems.lj_electrolyte(n, seed=seed)
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    xs, ys, zs = x[perm], y[perm], z[perm]
    q, gid = s["q"][perm], s["gid"][perm].astype(np.int32)
    typ = s["type"][perm].astype(np.int32)
    h = hashlib.sha256()
    for a in (xs, ys, zs, q, gid):
        h.update(np.ascontiguousarray(a).tobytes())
    if h.hexdigest() != str(f["input_digest"]):
        pytest.skip("regenerated inputs differ from the ones the fixture was made on")
    freq = int(f["freq"])
    assert oracle.rbl_params(n, box, 2.5, 5.0, 100)[0] == freq
    m = oracle.rbe_sample_philox(box, 0.16, int(f["P"]), 1000 + seed, int(f["epoch"]))
    re, im = oracle.rbe_structure_factor(box, q, xs, ys, zs, *m)
    scale = np.sqrt((re ** 2 + im ** 2).mean())
    assert np.abs(f["rho_re"] - re).max() < 1e-10 * scale
    assert np.abs(f["rho_im"] - im).max() < 1e-10 * scale
    S = oracle.rbe_gauss_sum(box, 0.16)
    sub = f["subset"]
    fk = oracle.rbe_force(box, S, 1.0, re, im, q, *m, xs, ys, zs)
    assert systems.rel_rms(f["rbe_force"], fk[sub]) < 1e-11
    e, v = oracle.rbe_energy_virial(box, 0.16, S, 1.0, float((q ** 2).sum()), float(q.sum()), re,
                                    im, *m)
    assert abs(float(f["rbe_energy"]) - e) < 1e-11 * abs(e)
    assert np.allclose(f["rbe_virial"], v, rtol=1e-10, atol=1e-11 * np.abs(v).max())
    cnt, rows = oracle.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
    cc, core, sc, shell = oracle.rbl_filter(box, 2.5, 5.0, freq, int(f["epoch"]), gid, xs, ys,
                                            zs, cnt, rows)
    assert _sha(cc.astype(np.int32)) == str(f["core_count_digest"])
    assert _sha(sc.astype(np.int32)) == str(f["shell_count_digest"])
    assert _sha(_pairs(gid, cc, core)) == str(f["core_digest"])
    assert _sha(_pairs(gid, sc, shell)) == str(f["shell_digest"])
    fr = oracle.pair_force_rbl(box, 2.5, 5.0, freq, 0.16, 1.0, typ, s["sigma"], s["eps"], q, xs,
                               ys, zs, cc, core, sc, shell)
    assert systems.rel_rms(f["rbl_force"], fr[sub]) < 1e-12


# --- SHAKE / RATTLE ------------------------------------------------------------
def test_shake_rattle(oracle):
    """ShakeAOp (half kick, drift, constraint, periodic wrap) and ShakeBOp
    (half kick, RATTLE) on 1,000 rigid waters with seeded forces: the
    oracle's op-level restatement within 1e-9 of RBMD's FP64 kernels
    (positions by minimum image, velocities relative to their RMS), RBMD's
    FP32 build to FP32 accuracy."""
    f = _load("ref_shake_water1000.npz")
    box = oracle.Box.make(f["lo"], f["hi"])
    L = np.asarray(f["hi"]) - np.asarray(f["lo"])
    args = (box, f["gid"], f["type"], f["mass"], float(f["dt"]), float(f["fmt2v"]), f["clusters"],
            1.0, 109.47)
    pos, vel, img, fails = oracle.shake_a(*args, f["pos"], f["vel"], f["force"])
    assert fails == 0
    vb, fails_b = oracle.shake_b(*args, pos, vel, f["force"])
    assert fails_b == 0

    def close_pos(a, b, tol):
        d = a - b
        d -= L * np.rint(d / L)
        return np.abs(d).max() < tol

    vscale = np.sqrt((vel ** 2).mean())
    assert close_pos(f["f64_a_pos"], pos, 1e-9)
    assert np.abs(f["f64_a_vel"] - vel).max() < 1e-9 * vscale
    assert np.abs(f["f64_b_vel"] - vb).max() < 1e-9 * vscale
    assert close_pos(f["f32_a_pos"].astype(np.float64), pos, 1e-3)
    assert np.abs(f["f32_b_vel"] - vb).max() < 1e-3 * vscale
    # the constraints hold in the reference's output
    cl = f["clusters"]
    d = f["f64_a_pos"][cl[:, 1]] - f["f64_a_pos"][cl[:, 0]]
    d -= L * np.rint(d / L)
    assert np.abs(np.linalg.norm(d, axis=1) - 1.0).max() < 1e-4
