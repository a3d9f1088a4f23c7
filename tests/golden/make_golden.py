"""Generate golden fixtures by running RBMD's own hot-path kernels on a GPU.

The kernels are the reference's .hip.cu sources compiled in place for sm_100a
by oracle/ref_harness/Makefile into oracle/_ref/libref64.so (FP64, with the
double7 accessor repaired by a forced-include header) and libref32.so (FP32,
as shipped).  Inputs are seeded LJ-electrolyte systems, cell-sorted by the
oracle, with k-vectors and lists injected so both codes see the same data.
N is a multiple of 256 so ComputeRBEForce's in-branch __syncthreads never
diverges.  Usage (on a GPU machine):

    python tests/golden/make_golden.py --out tests/golden

Each case file holds the inputs and, per precision, the reference outputs:
rho(k), RBE force/energy/virial, the RBL core/shell lists (per-atom counts and a
SHA-256 of the sorted (gid_i, gid_j) pairs), the RBL pair force on those lists,
the Verlet pair force with energies and virial, and the exact-Ewald force.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

CASES = [
    # name, n, seed, P, epoch, kmax
    ("caseA", 3328, 11, 100, 5, (4, 4, 4)),
    ("caseB", 4096, 12, 400, 0, (3, 3, 3)),
]


def pair_digest(gid, rows_count, rows):
    """SHA-256 of the sorted (gid_i, gid_j) pairs of a row-major list."""
    pairs = []
    for i in range(len(rows_count)):
        js = rows[i][:rows_count[i]]
        pairs.append(np.stack([np.full(len(js), gid[i], dtype=np.int64), gid[js].astype(np.int64)],
                              1))
    allp = np.concatenate(pairs) if pairs else np.zeros((0, 2), dtype=np.int64)
    order = np.lexsort((allp[:, 1], allp[:, 0]))
    return hashlib.sha256(np.ascontiguousarray(allp[order]).tobytes()).hexdigest()


def build_inputs(name, n, seed, P, epoch, kmax):
    from oracle import oracle as O
    from rbmd_b200 import systems

    s = systems.lj_electrolyte(n, seed=seed)
    box = O.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = O.cells_sort(box, 5.3, x, y, z)
    xs, ys, zs = x[perm], y[perm], z[perm]
    cnt, rows = O.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
    freq, _, _ = O.rbl_params(n, box, 2.5, 5.0, 100)
    m = O.rbe_sample_philox(box, 0.16, P, 1000 + seed, epoch)
    return {
        "name": name, "n": n, "P": P, "epoch": epoch, "freq": freq, "kmax": np.array(kmax),
        "lo": s["lo"], "hi": s["hi"], "x": xs, "y": ys, "z": zs, "q": s["q"][perm],
        "type": s["type"][perm].astype(np.int32), "gid": s["gid"][perm].astype(np.int32),
        "mx": m[0], "my": m[1], "mz": m[2], "sigma": s["sigma"], "eps": s["eps"],
        "cand_count": cnt, "cand": rows,
    }


def run_reference(lib, real, inp):
    import torch

    dt = torch.float64 if real == 8 else torch.float32
    dev = "cuda"
    n, P = inp["n"], inp["P"]
    lo = (C.c_double * 3)(*inp["lo"])
    hi = (C.c_double * 3)(*inp["hi"])

    def R(a):
        return torch.as_tensor(np.ascontiguousarray(a)).to(device=dev, dtype=dt)

    def I(a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32)).to(device=dev)

    def p(t):
        return C.c_void_p(t.data_ptr())

    def z(*shape, dtype=None):
        return torch.zeros(*shape, dtype=dtype or dt, device=dev)

    keep = []  # every device array stays referenced until the end of the call

    def K(t):
        keep.append(t)
        return p(t)

    out = {}
    q, x, y, zz = R(inp["q"]), R(inp["x"]), R(inp["y"]), R(inp["z"])
    mx, my, mz = R(inp["mx"]), R(inp["my"]), R(inp["mz"])
    # RBE
    re, im = z(P), z(P)
    assert lib.ref_rbe_rho(lo, hi, n, P, p(q), p(mx), p(my), p(mz), p(x), p(y), p(zz), p(re),
                           p(im)) == 0
    from oracle import oracle as O

    box = O.Box.make(inp["lo"], inp["hi"])
    S = O.rbe_gauss_sum(box, 0.16)
    fk = [z(n) for _ in range(3)]
    assert lib.ref_rbe_force(lo, hi, n, P, C.c_double(0.16), C.c_double(S), C.c_double(1.0), p(re),
                             p(im), p(q), p(mx), p(my), p(mz), p(x), p(y), p(zz),
                             *[p(t) for t in fk]) == 0
    vir, en = z(6), z(1)
    qsq = float((inp["q"] ** 2).sum())
    qsum = float(inp["q"].sum())
    assert lib.ref_rbe_virial(lo, hi, P, C.c_double(0.16), C.c_double(S), C.c_double(1.0),
                              C.c_double(qsq), C.c_double(qsum), p(re), p(im), p(mx), p(my),
                              p(mz), p(vir), p(en)) == 0
    out["rho_re"], out["rho_im"] = re.cpu().numpy(), im.cpu().numpy()
    out["rbe_force"] = np.stack([t.cpu().numpy() for t in fk], 1)
    out["rbe_energy"], out["rbe_virial"] = en.cpu().numpy()[0], vir.cpu().numpy()
    # RBL filter on the oracle's candidate list (cut_off + skin = 5.3)
    cnt, rows = inp["cand_count"], inp["cand"]
    cap = rows.shape[1]
    cstart = np.arange(n, dtype=np.int32) * cap
    core_end = z(n, dtype=torch.int32)
    core = torch.full((n * cap,), -1, dtype=torch.int32, device=dev)
    shell = torch.full((cap * n,), -1, dtype=torch.int32, device=dev)
    snum, req, realloc = z(n, dtype=torch.int32), z(1, dtype=torch.int32), z(1, dtype=torch.int32)
    eps_ = 1e-4 if real == 8 else np.float32(1e-4)
    core2 = 2.5 * 2.5 - eps_
    force2 = 5.0 * 5.0 - eps_
    assert lib.ref_rbl_filter(C.c_double(core2), C.c_double(force2), n, K(I(inp["gid"])), p(x),
                              p(y), p(zz), K(I(cstart)), K(I(cstart + cnt)),
                              K(I(rows.reshape(-1))), K(I(np.full(n, cap))), K(I(cstart)),
                              p(core_end), p(core), cap, p(shell), p(snum), p(req), lo, hi,
                              p(realloc), inp["freq"], inp["epoch"]) == 0
    assert realloc.item() == 0
    hce = core_end.cpu().numpy() - cstart
    hcore = core.cpu().numpy().reshape(n, cap)
    hsn = snum.cpu().numpy()
    hsh = shell.cpu().numpy().reshape(cap, n).T.copy()
    out["core_count"], out["shell_count"] = hce.astype(np.int16), hsn.astype(np.int16)
    out["core_digest"] = pair_digest(inp["gid"], hce, hcore)
    out["shell_digest"] = pair_digest(inp["gid"], hsn, hsh)
    # RBL pair force on the reference's own lists
    fr = [z(n) for _ in range(3)]
    assert lib.ref_pair_rbl(lo, hi, C.c_double(2.5), C.c_double(5.0), n, 100, inp["freq"],
                            C.c_double(0.16), C.c_double(1.0), K(I(inp["type"])),
                            K(R(inp["sigma"])), K(R(inp["eps"])), K(I(cstart)),
                            K(I(cstart + hce)), K(I(hcore.reshape(-1))), K(I(hsh.T.reshape(-1))),
                            K(I(hsn)), p(q), p(x), p(y), p(zz), *[p(t) for t in fr]) == 0
    out["rbl_force"] = np.stack([t.cpu().numpy() for t in fr], 1)
    # Verlet pair force (cut_off 5) on the candidate list
    fv = [z(n) for _ in range(3)]
    flat, el, ec = z(6 * n), z(1), z(1)
    assert lib.ref_pair_verlet(lo, hi, C.c_double(5.0), n, C.c_double(0.16), C.c_double(1.0),
                               K(I(inp["type"])), K(R(inp["sigma"])), K(R(inp["eps"])),
                               K(I(cstart)), K(I(cstart + cnt)), K(I(rows.reshape(-1))), p(q), p(x),
                               p(y), p(zz), *[p(t) for t in fv], p(flat), p(el), p(ec)) == 0
    out["verlet_force"] = np.stack([t.cpu().numpy() for t in fv], 1)
    fl = flat.cpu().numpy().astype(np.float64).reshape(6, n)
    vsum = np.zeros(6)
    for i in range(n):  # Force::ReduceVirial order (force.h:24-41)
        vsum += fl[:, i]
    out["verlet_virial"], out["verlet_evdwl"], out["verlet_ecoul"] = (vsum, el.cpu().item(),
                                                                     ec.cpu().item())
    # exact Ewald
    kx, ky, kz = O.ewald_kvectors(box, inp["kmax"])
    nk = len(kx)
    ere, eim = z(nk), z(nk)
    assert lib.ref_ewald_rho(n, nk, p(q), p(x), p(y), p(zz), K(R(kx)), K(R(ky)), K(R(kz)), p(ere),
                             p(eim)) == 0
    fe = [z(n) for _ in range(3)]
    km = (C.c_int * 3)(*[int(v) for v in inp["kmax"]])
    assert lib.ref_ewald_force(lo, hi, n, km, C.c_double(0.16), C.c_double(1.0), p(ere), p(eim),
                               p(q), p(x), p(y), p(zz), *[p(t) for t in fe], K(z(6 * n))) == 0
    out["ewald_force"] = np.stack([t.cpu().numpy() for t in fe], 1)
    torch.cuda.synchronize()
    del keep
    return out


def load_libs():
    libs = {}
    for real, fname in ((8, "libref64.so"), (4, "libref32.so")):
        L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", fname))
        assert L.ref_real_size() == real
        libs[real] = L
    return libs


def group_cases(libs, out_dir):
    for case in CASES:
        inp = build_inputs(*case)
        save = {k: v for k, v in inp.items() if k not in ("cand", "cand_count", "name")}
        for real, L in libs.items():
            out = run_reference(L, real, inp)
            tag = "f64" if real == 8 else "f32"
            for k, v in out.items():
                if isinstance(v, np.ndarray) and v.dtype == np.float32:
                    v = v.astype(np.float32)
                save[f"{tag}_{k}"] = v
        path = os.path.join(out_dir, f"ref_{inp['name']}.npz")
        np.savez_compressed(path, **save)
        print(path, os.path.getsize(path))


def _torch_io(real):
    import torch

    dt = torch.float64 if real == 8 else torch.float32

    def R(a):
        return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dt)

    def I(a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32)).to(device="cuda")

    def z(*shape, dtype=None):
        return torch.zeros(*shape, dtype=dtype or dt, device="cuda")

    return R, I, z, (lambda t: C.c_void_p(t.data_ptr()))


# cells / full list: atoms in host order; c = 1 (a Verlet list) and
# c = ceil((cut_off + skin) / r_core) = 3 (the RBL builder's cells); the small
# box has 2 (c = 1) and 6 (c = 3) cells per axis, fewer than the 2c + 1 its
# stencil visits.
CELL_CASES = [("cells_n3328", 3328, 11), ("cells_n1200", 1200, 31)]


def group_cells(libs, out_dir):
    """LinkedCell + full list of RBMD (FP64 build) on seeded LJ electrolytes."""
    from oracle import oracle as O
    from rbmd_b200 import systems

    L = libs[8]
    R, I, z, p = _torch_io(8)
    for name, n, seed in CELL_CASES:
        s = systems.lj_electrolyte(n, seed=seed)
        box = O.Box.make(s["lo"], s["hi"])
        save = {"n": n, "seed": seed, "lo": s["lo"], "hi": s["hi"], "x": s["pos"][:, 0].copy(),
                "y": s["pos"][:, 1].copy(), "z": s["pos"][:, 2].copy(), "gid": s["gid"]}
        lo = (C.c_double * 3)(*s["lo"])
        hi = (C.c_double * 3)(*s["hi"])
        x, y, zz = R(save["x"]), R(save["y"]), R(save["z"])
        for c in (1, 3):
            dims = (C.c_int * 3)()
            L.ref_cell_dims(lo, hi, C.c_double(5.3), c, dims)
            ncell = dims[0] * dims[1] * dims[2]
            cell = np.zeros(n, dtype=np.int32)
            cs = np.zeros(ncell, dtype=np.int32)
            ce = np.zeros(ncell, dtype=np.int32)
            cnt = np.zeros(n, dtype=np.int32)
            cap = n * 1200
            nbr = np.zeros(cap, dtype=np.int32)
            realloc = C.c_int()
            hp = [C.c_void_p(a.ctypes.data) for a in (cell, cs, ce, cnt, nbr)]  # host arrays
            rc = L.ref_cells_full_list(lo, hi, C.c_double(5.3), c, C.c_double(5.3 * 5.3), n, p(x),
                                       p(y), p(zz), *hp, C.c_longlong(cap), C.byref(realloc))
            assert rc == 0 and realloc.value == 0, (rc, realloc.value)
            gid = np.asarray(s["gid"], dtype=np.int64)
            owner = np.repeat(np.arange(n), cnt)
            pairs = np.stack([gid[owner], gid[nbr[:cnt.sum()]]], 1)
            order = np.lexsort((pairs[:, 1], pairs[:, 0]))
            pairs = pairs[order]
            uniq = np.unique(pairs, axis=0)
            save[f"c{c}_dims"] = np.array(dims[:], dtype=np.int32)
            save[f"c{c}_cell"] = cell
            save[f"c{c}_cell_count"] = (ce - cs).astype(np.int32)
            save[f"c{c}_list_count"] = cnt.astype(np.int16)
            save[f"c{c}_list_digest"] = hashlib.sha256(
                np.ascontiguousarray(pairs).tobytes()).hexdigest()
            save[f"c{c}_unique_digest"] = hashlib.sha256(
                np.ascontiguousarray(uniq).tobytes()).hexdigest()
            save[f"c{c}_duplicates"] = int(len(pairs) - len(uniq))
        path = os.path.join(out_dir, f"ref_{name}.npz")
        np.savez_compressed(path, **save)
        print(path, os.path.getsize(path), {k: save[k] for k in save if k.endswith("duplicates")})


def _special_rows(n, gid, core_count, core, shell_count, shell, seed):
    """Seeded special rows: per atom up to 4 partners (global ids), mostly
    taken from its own core and shell lists, some from outside; nspecial the
    cumulative 1-2 / 1-3 / 1-4 counts."""
    rng = np.random.default_rng(seed)
    maxs = 4
    special = np.full((n, maxs), -1, dtype=np.int32)
    nspecial = np.zeros((n, 3), dtype=np.int32)
    for i in range(n):
        cand = list(core[i][:core_count[i]]) + list(shell[i][:shell_count[i]])
        k = int(rng.integers(0, maxs + 1))
        picks = []
        for _ in range(k):
            if cand and rng.random() < 0.8:
                picks.append(int(gid[cand[int(rng.integers(0, len(cand)))]]))
            else:
                picks.append(int(rng.integers(0, n)))
        picks = list(dict.fromkeys(p for p in picks if p != gid[i]))
        special[i, :len(picks)] = picks
        a = int(rng.integers(0, len(picks) + 1))
        b = int(rng.integers(a, len(picks) + 1))
        nspecial[i] = (a, b, len(picks))
    return nspecial, special


def group_special(libs, out_dir):
    """SpecialLJCutCoulRBLForceOp (both kernels RBMD ships: RBMD_PAIR_KERNEL
    optimized and reference) on case A's inputs and the FP64 oracle's RBL lists
    with seeded special rows; FP64 and FP32 builds."""
    import subprocess

    for variant in ("optimized", "reference"):
        env = dict(os.environ, RBMD_PAIR_KERNEL=variant)
        subprocess.run([sys.executable, os.path.abspath(__file__), "--out", out_dir, "--groups",
                        "special_one"], env=env, check=True)


def group_special_one(libs, out_dir):
    from oracle import oracle as O

    variant = os.environ.get("RBMD_PAIR_KERNEL", "optimized")
    inp = build_inputs(*CASES[0])
    n = inp["n"]
    box = O.Box.make(inp["lo"], inp["hi"])
    cc, core, sc, shell = O.rbl_filter(box, 2.5, 5.0, int(inp["freq"]), int(inp["epoch"]),
                                       inp["gid"], inp["x"], inp["y"], inp["z"],
                                       inp["cand_count"], inp["cand"])
    nspecial, special = _special_rows(n, inp["gid"], cc, core, sc, shell, 77)
    weights = (0.0, 0.5, 0.8)
    save = {"variant": variant, "nspecial": nspecial, "special": special,
            "weights": np.array(weights), "core_count": cc.astype(np.int32),
            "shell_count": sc.astype(np.int32)}
    nt = len(inp["sigma"])
    for real, L in libs.items():
        R, I, z, p = _torch_io(real)
        keep = []

        def K(t):
            keep.append(t)
            return p(t)

        sig = np.asarray(inp["sigma"], float)
        ep = np.asarray(inp["eps"], float)
        if real == 4:
            sig, ep = sig.astype(np.float32), ep.astype(np.float32)
        lj12 = np.zeros(nt * nt, dtype=sig.dtype)
        lj6 = np.zeros(nt * nt, dtype=sig.dtype)
        for a in range(nt):  # CVFF::Init (cvff.cpp:855-870) in the build's precision
            for b in range(nt):
                e_ab = np.sqrt(ep[a] * ep[b])
                s_ab = (sig[a] + sig[b]) * sig.dtype.type(0.5)
                s2 = s_ab * s_ab
                s6 = s2 * s2 * s2
                lj12[a * nt + b] = sig.dtype.type(48) * e_ab * s6 * s6
                lj6[a * nt + b] = sig.dtype.type(24) * e_ab * s6
        cap = core.shape[1]
        cstart = np.arange(n, dtype=np.int32) * cap
        f = [z(n) for _ in range(3)]
        lo = (C.c_double * 3)(*inp["lo"])
        hi = (C.c_double * 3)(*inp["hi"])
        assert L.ref_pair_rbl_special(
            lo, hi, C.c_double(2.5), C.c_double(5.0), n, 100, int(inp["freq"]), C.c_double(0.16),
            C.c_double(1.0), K(I(inp["type"])), K(I(inp["gid"])), nt, K(R(lj12)), K(R(lj6)),
            K(I(cstart)), K(I(cstart + cc)), K(I(core.reshape(-1))),
            K(I(shell.T.reshape(-1))), K(I(sc)), K(I(nspecial.reshape(-1))),
            K(I(special.reshape(-1))), special.shape[1], C.c_double(weights[0]),
            C.c_double(weights[1]), C.c_double(weights[2]), K(R(inp["q"])), K(R(inp["x"])),
            K(R(inp["y"])), K(R(inp["z"])), *[p(t) for t in f]) == 0
        tag = "f64" if real == 8 else "f32"
        save[f"{tag}_force"] = np.stack([t.cpu().numpy() for t in f], 1)
        del keep
    path = os.path.join(out_dir, f"ref_special_{variant}.npz")
    np.savez_compressed(path, **save)
    print(path, os.path.getsize(path))


def group_rbsog(libs, out_dir):
    """RBSOG far field of RBMD's kernels (sampled and direct: structure
    factors, forces, energies, virials with the NPT terms) at rbsog_level 2,
    P = 112, on a seeded 3,328-atom electrolyte, with the oracle's samples,
    direct vectors and weights and a gather map from the oracle's NPT chain."""
    from oracle import oracle as O
    from rbmd_b200 import systems

    n, level, P, cut = 3328, 2, 112, 5.0
    s = systems.lj_electrolyte(n, seed=23)
    box = O.Box.make(s["lo"], s["hi"])
    Ld = np.asarray(s["hi"]) - np.asarray(s["lo"])
    prm = O.rbsog_params(level, cut, box)
    m = O.rbsog_sample_philox(level, cut, box, P, 9, 4)
    u = np.random.default_rng(5).random(P)
    idx = O.rbsog_idx_npt(level, cut, box, m, u)
    save = {"n": n, "level": level, "P": P, "lo": s["lo"], "hi": s["hi"],
            "x": s["pos"][:, 0].copy(), "y": s["pos"][:, 1].copy(), "z": s["pos"][:, 2].copy(),
            "q": s["q"], "mx": m[0], "my": m[1], "mz": m[2], "u": u, "idx": idx,
            "S": prm["S"], "S_npt": prm["S_npt"], "direct_m": prm["direct_m"],
            "direct_fb": prm["direct_fb"], "direct_fb_npt": prm["direct_fb_npt"]}
    K = [m[d] * (2 * np.pi / Ld[d]) for d in range(3)]  # K_Sample * pxyz
    Kn = [k[idx] for k in K]
    dm = prm["direct_m"].astype(np.float64)
    D = [2 * np.pi * (dm[:, d] + 0.0) / Ld[d] for d in range(3)]
    lo = (C.c_double * 3)(*s["lo"])
    hi = (C.c_double * 3)(*s["hi"])
    for real, L in libs.items():
        R, I, z, p = _torch_io(real)
        keep = []

        def Kp(t):
            keep.append(t)
            return p(t)

        rho = [z(P), z(P)]
        drho = [z(6), z(6)]
        fs = [z(n) for _ in range(3)]
        fd = [z(n) for _ in range(3)]
        vs, vd, ep = z(6), z(6), z(2)
        assert L.ref_rbsog(lo, hi, n, P, C.c_double(1.0), C.c_double(prm["S"]),
                           C.c_double(prm["S_npt"]), *[Kp(R(k)) for k in K],
                           *[Kp(R(k)) for k in Kn], Kp(I(idx)), Kp(R(np.ones(P))),
                           Kp(R(np.ones(P))), 6, *[Kp(R(d)) for d in D],
                           Kp(R(prm["direct_fb"])), Kp(R(prm["direct_fb_npt"])), Kp(R(s["q"])),
                           Kp(R(save["x"])), Kp(R(save["y"])), Kp(R(save["z"])),
                           *[p(t) for t in rho], *[p(t) for t in drho], *[p(t) for t in fs],
                           *[p(t) for t in fd], p(vs), p(vd), p(ep)) == 0
        tag = "f64" if real == 8 else "f32"
        save[f"{tag}_rho_re"], save[f"{tag}_rho_im"] = (t.cpu().numpy() for t in rho)
        save[f"{tag}_drho_re"], save[f"{tag}_drho_im"] = (t.cpu().numpy() for t in drho)
        save[f"{tag}_force_sample"] = np.stack([t.cpu().numpy() for t in fs], 1)
        save[f"{tag}_force_direct"] = np.stack([t.cpu().numpy() for t in fd], 1)
        save[f"{tag}_virial_sample"] = vs.cpu().numpy()
        save[f"{tag}_virial_direct"] = vd.cpu().numpy()
        save[f"{tag}_energy_parts"] = ep.cpu().numpy()
        del keep
    path = os.path.join(out_dir, "ref_rbsog_l2.npz")
    np.savez_compressed(path, **save)
    print(path, os.path.getsize(path))


LARGE = ("large_n51200", 51200, 14, 100, 7, (2, 2, 2))
LARGE_SUBSET = 2048


def _array_digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def group_large(libs, out_dir):
    """The FP64 build at N = 51,200 (a multiple of 256).  Inputs are not
    stored: they are regenerated from the seed (systems.lj_electrolyte + the
    oracle's cell sort) and checked against the stored digest.  Stored: the
    RBL lists as per-atom count digests and pair-set digests, and rho(k), the
    RBE force and the RBL pair force on a seeded subset of 2,048 atoms."""
    inp = build_inputs(*LARGE)
    out = run_reference(libs[8], 8, inp)
    sub = np.sort(np.random.default_rng(3).choice(inp["n"], LARGE_SUBSET, replace=False))
    save = {"n": inp["n"], "seed": LARGE[2], "P": inp["P"], "epoch": inp["epoch"],
            "freq": inp["freq"], "input_digest": _array_digest(inp["x"], inp["y"], inp["z"],
                                                                inp["q"], inp["gid"]),
            "subset": sub.astype(np.int32), "rho_re": out["rho_re"], "rho_im": out["rho_im"],
            "rbe_energy": out["rbe_energy"], "rbe_virial": out["rbe_virial"],
            "rbe_force": out["rbe_force"][sub], "rbl_force": out["rbl_force"][sub],
            "core_count_digest": _array_digest(out["core_count"].astype(np.int32)),
            "shell_count_digest": _array_digest(out["shell_count"].astype(np.int32)),
            "core_digest": out["core_digest"], "shell_digest": out["shell_digest"],
            "core_total": int(out["core_count"].astype(np.int64).sum()),
            "shell_total": int(out["shell_count"].astype(np.int64).sum())}
    path = os.path.join(out_dir, f"ref_{LARGE[0]}.npz")
    np.savez_compressed(path, **save)
    print(path, os.path.getsize(path))


def group_shake(libs, out_dir):
    """ShakeAOp and ShakeBOp of RBMD on 1,000 rigid waters (3,000 atoms, REAL
    units) with seeded forces: A from the stored positions, velocities and
    forces; B on A's positions and velocities with the same forces."""
    from rbmd_b200 import systems

    s = systems.water(1000, seed=3)
    n = s["n"]
    prm = s["params"]
    force = np.random.default_rng(11).normal(size=(n, 3)) * 5.0
    save = {"n": n, "lo": s["lo"], "hi": s["hi"], "pos": s["pos"], "vel": s["vel"],
            "force": force, "type": s["type"], "gid": s["gid"], "mass": s["mass"],
            "clusters": s["clusters"], "dt": prm["dt"], "fmt2v": prm["fmt2v"]}
    lo = (C.c_double * 3)(*s["lo"])
    hi = (C.c_double * 3)(*s["hi"])
    for real, L in libs.items():
        R, I, z, p = _torch_io(real)
        keep = []

        def K(t):
            keep.append(t)
            return p(t)

        P = [R(s["pos"][:, d]) for d in range(3)]
        V = [R(s["vel"][:, d]) for d in range(3)]
        F = [R(force[:, d]) for d in range(3)]
        flags = [I(np.zeros(n)) for _ in range(3)]
        id2idx = K(I(np.arange(n)))
        mass, typ = K(R(s["mass"])), K(I(s["type"]))
        ang = K(I(np.ascontiguousarray(s["clusters"]).reshape(-1)))
        nang = len(s["clusters"])
        assert L.ref_shake_a(lo, hi, nang, C.c_double(prm["dt"]), C.c_double(prm["fmt2v"]), id2idx,
                             mass, typ, ang, *[p(t) for t in P], *[p(t) for t in V],
                             *[p(t) for t in F], *[p(t) for t in flags]) == 0
        tag = "f64" if real == 8 else "f32"
        save[f"{tag}_a_pos"] = np.stack([t.cpu().numpy() for t in P], 1)
        save[f"{tag}_a_vel"] = np.stack([t.cpu().numpy() for t in V], 1)
        save[f"{tag}_a_flags"] = np.stack([t.cpu().numpy() for t in flags], 0)
        assert L.ref_shake_b(lo, hi, nang, C.c_double(prm["dt"]), C.c_double(prm["fmt2v"]), id2idx,
                             mass, typ, ang, *[p(t) for t in P], *[p(t) for t in V],
                             *[p(t) for t in F]) == 0
        save[f"{tag}_b_vel"] = np.stack([t.cpu().numpy() for t in V], 1)
        del keep
    path = os.path.join(out_dir, "ref_shake_water1000.npz")
    np.savez_compressed(path, **save)
    print(path, os.path.getsize(path))


GROUPS = {"cases": group_cases, "cells": group_cells, "special": group_special,
          "special_one": group_special_one, "rbsog": group_rbsog, "large": group_large,
          "shake": group_shake}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--groups", default="cases",
                    help="comma-separated subset of: " + ", ".join(GROUPS))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    libs = load_libs()
    for g in args.groups.split(","):
        GROUPS[g](libs, args.out)


if __name__ == "__main__":
    main()
