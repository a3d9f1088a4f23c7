"""The sm_100a kernels against the golden outputs of RBMD's own FP64 kernels
(tests/golden/ref_case*.npz, made by tests/golden/make_golden.py).

Lists and batches must be identical (SHA-256 of the (gid_i, gid_j) pair sets);
plain-FP64 k-space and pair forces within 1e-10 relative RMS; the mixed engine
within 1e-5 relative RMS of the reference's FP64 total force.
"""
import glob
import os

import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_case*.npz")))


def _system(f):
    n = int(f["n"])
    return {"n": n, "lo": f["lo"], "hi": f["hi"],
            "pos": np.stack([f["x"], f["y"], f["z"]], 1), "vel": np.zeros((n, 3)), "q": f["q"],
            "type": f["type"], "gid": f["gid"], "sigma": f["sigma"], "eps": f["eps"],
            "mass": np.ones(len(f["sigma"])),
            "params": {"cut_off": 5.0, "r_core": 2.5, "skin": 0.3, "neighbor_sample_num": 100,
                       "alpha": 0.16, "kspace_p": int(f["P"]), "qqr2e": 1.0, "dt": 0.005}}


def _digest(pairs):
    import hashlib

    p = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    order = np.lexsort((p[:, 1], p[:, 0]))
    return hashlib.sha256(np.ascontiguousarray(p[order]).tobytes()).hexdigest()


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_ops_against_reference(cuda, rbx, path):
    torch = cuda
    f = dict(np.load(path))
    n, P = int(f["n"]), int(f["P"])
    box = rbx.Box.make(f["lo"], f["hi"])
    T = [torch.as_tensor(np.ascontiguousarray(a)).to("cuda", torch.float64)
         for a in (f["q"], f["mx"], f["my"], f["mz"], f["x"], f["y"], f["z"])]
    re = torch.zeros(P, dtype=torch.float64, device="cuda")
    im = torch.zeros(P, dtype=torch.float64, device="cuda")
    rbx.rbe_structure_factor(box, *T, re, im)
    S = rbx.rbe_gauss_sum(box, 0.16)
    F = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3)]
    rbx.rbe_force(box, 0.16, S, 1.0, re, im, *T, *F)
    torch.cuda.synchronize()
    scale = np.sqrt((f["f64_rho_re"] ** 2 + f["f64_rho_im"] ** 2).mean())
    assert np.abs(re.cpu().numpy() - f["f64_rho_re"]).max() < 1e-10 * scale
    assert np.abs(im.cpu().numpy() - f["f64_rho_im"]).max() < 1e-10 * scale
    got = np.stack([a.cpu().numpy() for a in F], 1)
    assert systems.rel_rms(got, f["f64_rbe_force"]) < 1e-11


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
@pytest.mark.parametrize("precision", [0, 1])
def test_engine_against_reference(cuda, rbx, path, precision):
    f = dict(np.load(path))
    s = _system(f)
    e = rbx.Engine(s, precision=precision)
    e.set_k_samples(f["mx"], f["my"], f["mz"])
    e.compute_forces(epoch=int(f["epoch"]))
    assert e.stats().selection_frequency == int(f["freq"])
    core, shell = e.rbl_pairs()
    assert _digest(core) == str(f["f64_core_digest"])
    assert _digest(shell) == str(f["f64_shell_digest"])
    fp, fk = e.force_parts()  # in the order of the arrays given to the engine
    ref_k = f["f64_rbe_force"]
    rbl = f["f64_rbl_force"]
    ref_p = rbl - rbl.mean(0)  # reference mean-force removal
    tol = 1e-10 if precision == 0 else 1e-5
    assert systems.rel_rms(fk, ref_k) < (1e-11 if precision == 0 else 1e-5)
    assert systems.rel_rms(fp, ref_p) < tol
    assert systems.rel_rms(fp + fk, ref_p + ref_k) < tol
    e.close()


def test_cells_and_list_against_reference(cuda, rbx):
    """rbx_cells_sort / rbx_full_list against RBMD's LinkedCell and full-list
    kernels (tests/golden/ref_cells_n3328.npz, cells of edge cut_off + skin):
    the cell of every atom, atoms per cell and the pair set."""
    import hashlib

    torch = cuda
    path = os.path.join(HERE, "golden", "ref_cells_n3328.npz")
    if not os.path.exists(path):
        pytest.skip("cells fixture not generated")
    f = dict(np.load(path))
    n = int(f["n"])
    box = rbx.Box.make(f["lo"], f["hi"])
    dims = rbx.cell_grid(box, 5.3)
    assert list(dims) == f["c1_dims"].tolist()
    ncell = int(np.prod(dims))
    X = [torch.as_tensor(np.ascontiguousarray(f[k])).to("cuda", torch.float64) for k in "xyz"]
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    cos = torch.zeros(n, dtype=torch.int32, device="cuda")
    cst = torch.zeros(ncell + 1, dtype=torch.int32, device="cuda")
    scratch = torch.zeros(rbx.cells_scratch_bytes(n, ncell), dtype=torch.uint8, device="cuda")
    rbx.cells_sort(box, 5.3, *X, perm, cos, cst, scratch)
    hp, hc, hs = perm.cpu().numpy(), cos.cpu().numpy(), cst.cpu().numpy()
    cell = np.empty(n, dtype=np.int32)
    cell[hp] = hc
    assert np.array_equal(cell, f["c1_cell"])
    assert np.array_equal(np.diff(hs), f["c1_cell_count"])
    xs = [torch.as_tensor(np.ascontiguousarray(f[k][hp])).to("cuda", torch.float64) for k in "xyz"]
    cap = 800
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
    nb = torch.full((n, cap), -1, dtype=torch.int32, device="cuda")
    ovf = torch.zeros(1, dtype=torch.int32, device="cuda")
    rbx.full_list(box, 5.3, *xs, cst, cap, cnt, nb, ovf)
    torch.cuda.synchronize()
    assert ovf.item() == 0
    gc, gn = cnt.cpu().numpy(), nb.cpu().numpy()
    want = np.empty(n, dtype=np.int64)
    want[hp] = gc
    assert np.array_equal(want, f["c1_list_count"].astype(np.int64))
    gid = np.asarray(f["gid"], dtype=np.int64)[hp]
    owner = np.repeat(np.arange(n), gc)
    flat = np.concatenate([gn[i, :gc[i]] for i in range(n)])
    pairs = np.stack([gid[owner], gid[flat]], 1)
    pairs = pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]
    assert hashlib.sha256(np.ascontiguousarray(pairs).tobytes()).hexdigest() == \
        str(f["c1_list_digest"])
