"""The FP64 oracle against golden outputs of RBMD's own kernels.

Fixtures tests/golden/ref_case*.npz come from tests/golden/make_golden.py,
which runs the reference's hot-path .hip.cu kernels (compiled in place for
sm_100a; FP64 with the double7 accessor repaired, and FP32 as shipped) on the
seeded inputs stored in each file.

FP64 reference: lists identical (per-atom counts and SHA-256 of the pair
sets), rho / forces / energies / virials to FP64 round-off.  FP32 reference
(RBMD's production precision): forces within FP32 accuracy; its lists may
differ from the FP64 lists only at the cutoff boundaries.
"""
import glob
import hashlib
import os

import numpy as np
import pytest

from rbmd_b200 import systems

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_case*.npz")))

pytestmark = pytest.mark.skipif(not FIXTURES, reason="golden fixtures not generated")


def _digest(gid, counts, rows):
    pairs = []
    for i in range(len(counts)):
        js = rows[i][:counts[i]]
        pairs.append(np.stack([np.full(len(js), gid[i], dtype=np.int64),
                               gid[js].astype(np.int64)], 1))
    allp = np.concatenate(pairs)
    order = np.lexsort((allp[:, 1], allp[:, 0]))
    return hashlib.sha256(np.ascontiguousarray(allp[order]).tobytes()).hexdigest()


def _oracle(oracle, f):
    box = oracle.Box.make(f["lo"], f["hi"])
    x, y, z, q = f["x"], f["y"], f["z"], f["q"]
    m = (f["mx"], f["my"], f["mz"])
    out = {}
    re, im = oracle.rbe_structure_factor(box, q, x, y, z, *m)
    S = oracle.rbe_gauss_sum(box, 0.16)
    out["rho_re"], out["rho_im"] = re, im
    out["rbe_force"] = oracle.rbe_force(box, S, 1.0, re, im, q, *m, x, y, z)
    out["rbe_energy"], out["rbe_virial"] = oracle.rbe_energy_virial(
        box, 0.16, S, 1.0, float((q ** 2).sum()), float(q.sum()), re, im, *m)
    # candidate list on the stored (cell-sorted) atoms
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    assert np.array_equal(perm, np.arange(len(x)))  # inputs are already in cell order
    cnt, rows = oracle.full_list(box, 5.3, x, y, z, cell, cs, ce)
    cc, core, sc, shell = oracle.rbl_filter(box, 2.5, 5.0, int(f["freq"]), int(f["epoch"]),
                                            f["gid"], x, y, z, cnt, rows)
    out["core_count"], out["shell_count"] = cc, sc
    out["core_digest"] = _digest(f["gid"], cc, core)
    out["shell_digest"] = _digest(f["gid"], sc, shell)
    out["rbl_force"] = oracle.pair_force_rbl(box, 2.5, 5.0, int(f["freq"]), 0.16, 1.0, f["type"],
                                             f["sigma"], f["eps"], q, x, y, z, cc, core, sc, shell)
    fv, vir, el, ec = oracle.pair_force_verlet(box, 5.0, 0.16, 1.0, f["type"], f["sigma"],
                                               f["eps"], q, x, y, z, cnt, rows)
    out["verlet_force"], out["verlet_virial"] = fv, vir
    out["verlet_evdwl"], out["verlet_ecoul"] = el, ec
    out["ewald_force"], _ = oracle.ewald_force(box, 0.16, 1.0, f["kmax"], q, x, y, z)
    return out


@pytest.fixture(scope="module", params=FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def case(request, oracle):
    f = dict(np.load(request.param))
    return f, _oracle(oracle, f)


def test_fp64_reference_lists_bit_exact(case):
    f, o = case
    assert np.array_equal(f["f64_core_count"], o["core_count"])
    assert np.array_equal(f["f64_shell_count"], o["shell_count"])
    assert str(f["f64_core_digest"]) == o["core_digest"]
    assert str(f["f64_shell_digest"]) == o["shell_digest"]


def test_fp64_reference_kspace(case):
    f, o = case
    scale = np.sqrt((o["rho_re"] ** 2 + o["rho_im"] ** 2).mean())
    assert np.abs(f["f64_rho_re"] - o["rho_re"]).max() < 1e-10 * scale
    assert np.abs(f["f64_rho_im"] - o["rho_im"]).max() < 1e-10 * scale
    assert systems.rel_rms(f["f64_rbe_force"], o["rbe_force"]) < 1e-11
    assert abs(float(f["f64_rbe_energy"]) - o["rbe_energy"]) < 1e-11 * abs(o["rbe_energy"])
    assert np.allclose(f["f64_rbe_virial"], o["rbe_virial"], rtol=1e-10,
                       atol=1e-11 * np.abs(o["rbe_virial"]).max())
    assert systems.rel_rms(f["f64_ewald_force"], o["ewald_force"]) < 1e-11


def test_fp64_reference_pair(case):
    f, o = case
    assert systems.rel_rms(f["f64_rbl_force"], o["rbl_force"]) < 1e-12
    assert systems.rel_rms(f["f64_verlet_force"], o["verlet_force"]) < 1e-12
    assert np.allclose(f["f64_verlet_virial"], o["verlet_virial"], rtol=1e-11)
    assert abs(float(f["f64_verlet_evdwl"]) - o["verlet_evdwl"]) < 1e-11 * abs(o["verlet_evdwl"])
    assert abs(float(f["f64_verlet_ecoul"]) - o["verlet_ecoul"]) < 1e-11 * abs(o["verlet_ecoul"])


def test_fp32_reference_within_fp32_accuracy(case):
    """RBMD's production FP32 build agrees with the FP64 oracle to FP32 accuracy;
    RBL lists and batches differ only for pairs at the list thresholds."""
    f, o = case
    assert systems.rel_rms(f["f32_rbe_force"], o["rbe_force"]) < 1e-4
    assert systems.rel_rms(f["f32_verlet_force"], o["verlet_force"]) < 1e-4
    assert systems.rel_rms(f["f32_ewald_force"], o["ewald_force"]) < 1e-4
    n = len(f["x"])
    dc = np.abs(f["f32_core_count"].astype(int) - o["core_count"]).sum()
    ds = np.abs(f["f32_shell_count"].astype(int) - o["shell_count"]).sum()
    assert dc <= max(2, n // 1000) and ds <= max(2, n // 1000)
