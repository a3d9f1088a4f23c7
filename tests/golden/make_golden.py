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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    libs = {}
    for real, fname in ((8, "libref64.so"), (4, "libref32.so")):
        L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", fname))
        assert L.ref_real_size() == real
        libs[real] = L
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
        path = os.path.join(args.out, f"ref_{inp['name']}.npz")
        np.savez_compressed(path, **save)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
