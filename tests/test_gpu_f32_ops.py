"""The FP32 op-level entries (rbx_*_f32, for RBMD's default float build)
against the golden outputs of RBMD's own kernels compiled as shipped
(rbmd::Real = float; tests/golden/ref_case*.npz, f32_* arrays).

The inputs are the fixtures' positions, charges and samples rounded to
float, as the float build holds them.  RBL lists: the float twin of
FilterRblNeighborCandidatesOp must reproduce the float build's lists
exactly (per-atom counts and the SHA-256 of the (gid_i, gid_j) pair sets);
in case A those lists differ from the FP64 build's, so this checks the
float predicate itself.  Values: the twins compute in FP64 (real space,
energies) or in the mixed form (structure factor, RBE force) and store
float, so they are compared with the float build within its own rounding
error (relative RMS 5e-5 for pair forces, 5e-6 for the RBE force,
relative 1e-5 for energies and virials, the pair energies relative to
their total magnitude) and with the FP64 build.
"""
import glob
import hashlib
import os

import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_case*.npz")))
IDS = [os.path.basename(p) for p in FIXTURES]


def _digest(gid, counts, rows):
    pairs = [np.stack([np.full(c, gid[i], dtype=np.int64), gid[rows[i][:c]].astype(np.int64)], 1)
             for i, c in enumerate(counts)]
    allp = np.concatenate(pairs)
    order = np.lexsort((allp[:, 1], allp[:, 0]))
    return hashlib.sha256(np.ascontiguousarray(allp[order]).tobytes()).hexdigest()


def _f32(torch, a):
    return torch.as_tensor(np.ascontiguousarray(np.asarray(a, dtype=np.float32))).cuda()


def _i32(torch, a):
    return torch.as_tensor(np.ascontiguousarray(np.asarray(a, dtype=np.int32))).cuda()


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_kspace_f32_against_reference(cuda, rbx, oracle, path):
    torch = cuda
    f = dict(np.load(path))
    n, P = int(f["n"]), int(f["P"])
    box = rbx.Box.make(f["lo"], f["hi"])
    q, mx, my, mz, x, y, z = (_f32(torch, f[k]) for k in ("q", "mx", "my", "mz", "x", "y", "z"))
    re = torch.zeros(P, dtype=torch.float32, device="cuda")
    im = torch.zeros_like(re)
    rbx.rbe_structure_factor_f32(box, q, mx, my, mz, x, y, z, re, im)
    S = oracle.rbe_gauss_sum(oracle.Box.make(f["lo"], f["hi"]), 0.16)
    F = [torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    rbx.rbe_force_f32(box, 0.16, S, 1.0, re, im, q, mx, my, mz, x, y, z, *F)
    vir = torch.zeros(6, dtype=torch.float32, device="cuda")
    en = torch.zeros(1, dtype=torch.float32, device="cuda")
    qsq, qsum = float((f["q"] ** 2).sum()), float(f["q"].sum())
    rbx.rbe_energy_virial_f32(box, 0.16, S, 1.0, qsq, qsum, re, im, mx, my, mz, vir, en)
    torch.cuda.synchronize()
    scale = np.sqrt((f["f64_rho_re"] ** 2 + f["f64_rho_im"] ** 2).mean())
    for got, k in ((re, "rho_re"), (im, "rho_im")):
        g = got.cpu().numpy().astype(np.float64)
        assert np.abs(g - f["f32_" + k]).max() < 5e-6 * scale, k
        assert np.abs(g - f["f64_" + k]).max() < 5e-6 * scale, k
    fk = np.stack([a.cpu().numpy().astype(np.float64) for a in F], 1)
    assert systems.rel_rms(fk, f["f32_rbe_force"].astype(np.float64)) < 5e-6
    assert systems.rel_rms(fk, f["f64_rbe_force"]) < 5e-6
    e = float(en.cpu().numpy()[0])
    assert abs(e - float(f["f32_rbe_energy"])) < 1e-5 * abs(float(f["f64_rbe_energy"]))
    v = vir.cpu().numpy().astype(np.float64)
    vs = np.abs(f["f64_rbe_virial"]).max()
    assert np.abs(v - f["f32_rbe_virial"]).max() < 1e-5 * vs


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_real_space_f32_against_reference(cuda, rbx, oracle, path):
    torch = cuda
    f = dict(np.load(path))
    n = int(f["n"])
    box = rbx.Box.make(f["lo"], f["hi"])
    ob = oracle.Box.make(f["lo"], f["hi"])
    # the candidate rows the reference ran on: the FP64 list at cut_off + skin
    perm, cell, cs, ce = oracle.cells_sort(ob, 5.3, f["x"], f["y"], f["z"])
    assert np.array_equal(perm, np.arange(n))
    cnt, rows = oracle.full_list(ob, 5.3, f["x"], f["y"], f["z"], cell, cs, ce)
    cap = rows.shape[1]
    cstart = np.arange(n, dtype=np.int32) * cap
    x, y, z, q = (_f32(torch, f[k]) for k in ("x", "y", "z", "q"))
    gid = _i32(torch, f["gid"])
    core2 = np.float32(2.5 * 2.5) - np.float32(1e-4)  # r_core^2 - EPSILON in float
    force2 = np.float32(5.0 * 5.0) - np.float32(1e-4)
    core_end = torch.zeros(n, dtype=torch.int32, device="cuda")
    core = torch.full((n * cap,), -1, dtype=torch.int32, device="cuda")
    shell = torch.full((cap * n,), -1, dtype=torch.int32, device="cuda")
    snum, req, realloc = (torch.zeros(k, dtype=torch.int32, device="cuda") for k in (n, 1, 1))
    cs_t = _i32(torch, cstart)
    rbx.rbl_filter_f32(float(core2), float(force2), gid, x, y, z, cs_t, _i32(torch, cstart + cnt),
                       _i32(torch, rows.reshape(-1)), _i32(torch, np.full(n, cap)), cs_t,
                       core_end, core, cap, shell, snum, req, box, realloc, int(f["freq"]),
                       int(f["epoch"]))
    torch.cuda.synchronize()
    assert realloc.item() == 0
    hce = core_end.cpu().numpy() - cstart
    hcore = core.cpu().numpy().reshape(n, cap)
    hsn = snum.cpu().numpy()
    hsh = shell.cpu().numpy().reshape(cap, n).T.copy()
    assert np.array_equal(hce, f["f32_core_count"].astype(np.int64))
    assert np.array_equal(hsn, f["f32_shell_count"].astype(np.int64))
    assert _digest(f["gid"], hce, hcore) == str(f["f32_core_digest"])
    assert _digest(f["gid"], hsn, hsh) == str(f["f32_shell_digest"])
    # RBL pair force on those lists, then the mean-force removal
    typ = _i32(torch, f["type"])
    sig, eps = _f32(torch, f["sigma"]), _f32(torch, f["eps"])
    F = [torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    rbx.pair_force_rbl_f32(box, 2.5, 5.0, 100, int(f["freq"]), 0.16, 1.0, typ, sig, eps, cs_t,
                           _i32(torch, cstart + hce), core, _i32(torch, hsh.T.reshape(-1)),
                           _i32(torch, hsn), q, x, y, z, *F)
    torch.cuda.synchronize()
    fr = np.stack([a.cpu().numpy().astype(np.float64) for a in F], 1)
    ref = f["f32_rbl_force"].astype(np.float64)
    assert systems.rel_rms(fr, ref) < 5e-5
    mean = torch.zeros(3, dtype=torch.float32, device="cuda")
    rbx.fix_rbl_force_f32(*F, mean)
    torch.cuda.synchronize()
    fm = np.stack([a.cpu().numpy().astype(np.float64) for a in F], 1)
    assert systems.rel_rms(fm, ref - ref.mean(0)) < 5e-5
    assert np.abs(mean.cpu().numpy() - fr.mean(0)).max() < 1e-6 * np.abs(fr).max()
    # Verlet pair force (cut_off 5) on the candidate rows
    V = [torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    flat = torch.zeros(6 * n, dtype=torch.float32, device="cuda")
    el, ec = (torch.zeros(1, dtype=torch.float32, device="cuda") for _ in range(2))
    rbx.pair_force_verlet_f32(box, 5.0, 0.16, 1.0, typ, sig, eps, cs_t, _i32(torch, cstart + cnt),
                              _i32(torch, rows.reshape(-1)), q, x, y, z, *V, flat, el, ec)
    torch.cuda.synchronize()
    fv = np.stack([a.cpu().numpy().astype(np.float64) for a in V], 1)
    assert systems.rel_rms(fv, f["f32_verlet_force"].astype(np.float64)) < 5e-5
    vir = flat.cpu().numpy().astype(np.float64).reshape(6, n).sum(1)
    assert np.abs(vir - f["f32_verlet_virial"]).max() < 1e-5 * np.abs(f["f64_verlet_virial"]).max()
    e_scale = abs(float(f["f64_verlet_evdwl"])) + abs(float(f["f64_verlet_ecoul"]))
    assert abs(el.item() - float(f["f32_verlet_evdwl"])) < 1e-5 * e_scale
    assert abs(ec.item() - float(f["f32_verlet_ecoul"])) < 1e-5 * e_scale
