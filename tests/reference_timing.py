"""Time RBMD's own hot-path kernels next to this library on the same GPU.

The reference kernels are the .hip.cu sources compiled in place for sm_100a by
oracle/ref_harness/Makefile (oracle/_ref/libref32.so as shipped, FP32, and
libref64.so, FP64).  One MD step of the reference's RBL + RBE force path with a
reused candidate list (skin > 0, LJCutCoulKspace::ComputeLJRBL and
KSpaceCalculator::ComputeRBE, lj_cut_coul_kspace.cpp:494-573,
kspace_calculator.cpp:532-588) launches:

    FilterRblNeighborCandidatesOp      RBL core list + hashed shell sample
    LJCutCoulRBLForceOp                pair force on those lists
    FixRBLForceOp                      mean-force removal (the three thrust
                                       reductions before it are not timed)
    ComputePnumberChargeStructureFactorOp   rho(k)
    ComputeRBEForceOp                  k-space force

The k-vector sampling (host MH chains), the list rebuild and the integrator are
not timed on the reference side.  This library's step is timed whole (engine
phases, CUDA events): real space (fused filter + pair force + mean partials)
and k-space (device sampling, rho(k), finalize, force, combine and half kick);
the skin check, rebuild and kick/drift phases are listed apart.

N = 200,192 (a multiple of 256: ComputeRBEForce has __syncthreads inside a
branch on i < N), the 200k LJ electrolyte recipe otherwise.  Usage on a GPU
machine: python tests/reference_timing.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

N = 200192
REPS = 20


def _median_ms(fn, reps=REPS):
    import torch

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        ev[0].record()
        fn()
        ev[1].record()
        torch.cuda.synchronize()
        ts.append(ev[0].elapsed_time(ev[1]))
    return float(np.median(ts))


def reference_step(lib, real, s, cnt, rows):
    import torch

    from oracle import oracle as O

    dt = torch.float64 if real == 8 else torch.float32
    dev = "cuda"
    n, p = s["n"], s["params"]["kspace_p"]
    lo = (C.c_double * 3)(*s["lo"])
    hi = (C.c_double * 3)(*s["hi"])
    keep = []

    def T(a, dtype=None):
        t = torch.as_tensor(np.ascontiguousarray(a)).to(device=dev, dtype=dtype or dt)
        keep.append(t)
        return t

    def P(t):
        return C.c_void_p(t.data_ptr())

    box = O.Box.make(s["lo"], s["hi"])
    alpha, qqr2e = s["params"]["alpha"], s["params"]["qqr2e"]
    S = O.rbe_gauss_sum(box, alpha)
    m = O.rbe_sample_philox(box, alpha, p, 5, 0)
    x, y, z = (T(s["pos"][:, d]) for d in range(3))
    q = T(s["q"])
    mx, my, mz = (T(v) for v in m)
    typ = T(s["type"], torch.int32)
    gid = T(s["gid"], torch.int32)
    sigma, eps = T(s["sigma"]), T(s["eps"])
    cap = rows.shape[1]
    cstart = T(np.arange(n) * cap, torch.int32)
    cend = T(np.arange(n) * cap + cnt, torch.int32)
    cand = T(rows.reshape(-1), torch.int32)
    capv = T(np.full(n, cap), torch.int32)
    core_end = T(np.zeros(n), torch.int32)
    core = T(np.full(n * cap, -1), torch.int32)
    shell = T(np.full(n * cap, -1), torch.int32)
    snum, req, realloc = (T(np.zeros(k), torch.int32) for k in (n, 1, 1))
    re, im = T(np.zeros(p)), T(np.zeros(p))
    fr = [T(np.zeros(n)) for _ in range(3)]
    fk = [T(np.zeros(n)) for _ in range(3)]
    freq, _, _ = O.rbl_params(n, box, s["params"]["r_core"], s["params"]["cut_off"],
                              s["params"]["neighbor_sample_num"])
    eps_ = 1e-4
    core2, force2 = 2.5 ** 2 - eps_, 5.0 ** 2 - eps_

    def filt():
        assert lib.ref_rbl_filter(C.c_double(core2), C.c_double(force2), n, P(gid), P(x), P(y),
                                  P(z), P(cstart), P(cend), P(cand), P(capv), P(cstart), P(core_end),
                                  P(core), cap, P(shell), P(snum), P(req), lo, hi, P(realloc),
                                  freq, 0) == 0

    def pair():
        assert lib.ref_pair_rbl(lo, hi, C.c_double(2.5), C.c_double(5.0), n, 100, freq,
                                C.c_double(alpha), C.c_double(qqr2e), P(typ), P(sigma), P(eps),
                                P(cstart), P(core_end), P(core), P(shell), P(snum), P(q), P(x),
                                P(y), P(z), *[P(t) for t in fr]) == 0

    def fix():
        assert lib.ref_fix_rbl(n, C.c_double(0.0), C.c_double(0.0), C.c_double(0.0),
                               *[P(t) for t in fr]) == 0

    def rho():
        assert lib.ref_rbe_rho(lo, hi, n, p, P(q), P(mx), P(my), P(mz), P(x), P(y), P(z), P(re),
                               P(im)) == 0

    def force():
        assert lib.ref_rbe_force(lo, hi, n, p, C.c_double(alpha), C.c_double(S), C.c_double(qqr2e),
                                 P(re), P(im), P(q), P(mx), P(my), P(mz), P(x), P(y), P(z),
                                 *[P(t) for t in fk]) == 0

    filt()
    assert int(realloc.item()) == 0, "core capacity too small"
    out = {name: _median_ms(fn) for name, fn in
           (("rbl_filter", filt), ("rbl_pair_force", pair), ("fix_rbl_force", fix),
            ("rbe_structure_factor", rho), ("rbe_force", force))}
    del keep
    return out


def ours(s, precision):
    from rbmd_b200 import rbx

    e = rbx.Engine(s, precision=precision, seed=5)
    e.compute_forces(0)
    e.step(5)
    e.set_profiling(True)
    e.step(50)
    ph = e.phase_ms()
    e.close()
    return {"kick_drift": ph[0], "skin_check_rebuild": ph[1], "real_space": ph[2], "kspace": ph[3]}


def main():
    from oracle import oracle as O
    from rbmd_b200 import rbx, systems

    s = systems.lj_electrolyte(N, seed=2024)
    box = O.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = O.cells_sort(box, 5.3, x, y, z)
    srt = dict(s)
    srt.update(pos=s["pos"][perm], q=s["q"][perm], type=s["type"][perm], gid=s["gid"][perm],
               vel=s["vel"][perm])
    cnt, rows = O.full_list(box, 5.3, x[perm], y[perm], z[perm], cell, cs, ce)
    res = {}
    for real, fname in ((4, "libref32.so"), (8, "libref64.so")):
        lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", fname))
        assert lib.ref_real_size() == real
        res["reference_f32" if real == 4 else "reference_f64"] = reference_step(lib, real, srt, cnt,
                                                                                rows)
    res["ours_mixed"] = ours(s, rbx.MIXED)
    res["ours_fp64"] = ours(s, rbx.PLAIN_FP64)
    print(f"N = {N}, P = {s['params']['kspace_p']}, candidates/atom = {cnt.mean():.1f}")
    for k, v in res.items():
        tot = sum(v[c] for c in v if c not in ("kick_drift", "skin_check_rebuild"))
        print(f"{k:14s} " + "  ".join(f"{c} {t:.4f} ms" for c, t in v.items()) +
              f"  | force path {tot:.4f} ms")


if __name__ == "__main__":
    main()
