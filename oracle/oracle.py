"""ctypes wrapper of the FP64 host oracle (oracle/rbx_oracle.c).

Test infrastructure only: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker, never by the product
package.  Each wrapper names the RBMD 2.0 source it restates.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class Box(C.Structure):
    """Orthogonal periodic box (src/data_manager/include/model/box.h:5-49)."""

    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3)]

    @staticmethod
    def make(lo, hi):
        b = Box()
        for d in range(3):
            b.lo[d] = float(lo[d])
            b.hi[d] = float(hi[d])
        return b

    @property
    def length(self):
        return np.array([self.hi[d] - self.lo[d] for d in range(3)])


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        B = C.POINTER(Box)
        sig = {
            "orc_rbe_gauss_sum": (C.c_double, [B, C.c_double]),
            "orc_rbe_structure_factor": (None, [C.c_int, C.c_int, B, _dp, _dp, _dp, _dp,
                                                _dp, _dp, _dp, _dp, _dp]),
            "orc_rbe_force": (None, [C.c_int, C.c_int, B, C.c_double, C.c_double, _dp, _dp,
                                     _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_rbe_energy_virial": (None, [C.c_int, B, C.c_double, C.c_double, C.c_double,
                                             C.c_double, C.c_double, _dp, _dp, _dp, _dp, _dp,
                                             _dp, _dp]),
            "orc_ewald_num_k": (C.c_int, [_ip]),
            "orc_ewald_kvectors": (None, [_ip, B, _dp, _dp, _dp]),
            "orc_ewald_structure_factor": (None, [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp,
                                                  _dp, _dp, _dp, _dp]),
            "orc_ewald_force": (None, [C.c_int, C.c_int, B, C.c_double, C.c_double, _dp, _dp,
                                       _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_ewald_energy": (C.c_double, [C.c_int, B, C.c_double, C.c_double, C.c_double,
                                              _dp, _dp, _dp, _dp, _dp]),
            "orc_philox4x32_10": (None, [np.ctypeslib.ndpointer(np.uint32),
                                         np.ctypeslib.ndpointer(np.uint32),
                                         np.ctypeslib.ndpointer(np.uint32)]),
            "orc_rbe_sample_philox": (C.c_int, [C.c_int, B, C.c_double, C.c_uint64,
                                                C.c_int64, _dp, _dp, _dp]),
            "orc_rbe_sample_mh": (None, [C.c_int, B, C.c_double, C.c_uint64, _dp, _dp, _dp]),
            "orc_rbsog_params": (C.c_int, [C.c_int, C.c_double, B, _dp, _dp, _ip, _dp, _dp,
                                           _dp]),
            "orc_rbsog_npt_uniforms": (None, [C.c_uint64, C.c_int64, C.c_int, _dp]),
            "orc_shake_a_op": (C.c_int, [C.c_int, B, _ip, _ip, _dp, C.c_int, C.c_double,
                                         C.c_double, C.c_int, _ip, C.c_double, C.c_double, _dp,
                                         _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_void_p]),
            "orc_shake_b_op": (C.c_int, [C.c_int, B, _ip, _ip, _dp, C.c_int, C.c_double,
                                         C.c_double, C.c_int, _ip, C.c_double, C.c_double, _dp,
                                         _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_rbsog_idx_npt": (C.c_int, [C.c_int, C.c_double, B, C.c_int, _dp, _dp, _dp, _dp,
                                            _ip]),
            "orc_rbsog_virial": (C.c_int, [C.c_int, C.c_double, B, C.c_double, C.c_double,
                                           C.c_double, C.c_int, C.c_int, _dp, _dp, _dp, _dp,
                                           _ip, _dp, _dp, _dp, _dp]),
            "orc_rbsog_sample_philox": (C.c_int, [C.c_int, C.c_double, B, C.c_int, C.c_uint64,
                                                  C.c_int64, _dp, _dp, _dp]),
            "orc_rbsog_sample_mh": (C.c_int, [C.c_int, C.c_double, B, C.c_int, C.c_uint64,
                                              _dp, _dp, _dp]),
            "orc_rbsog_force": (C.c_int, [C.c_int, C.c_double, B, C.c_double, C.c_double,
                                          C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                          _dp, _dp, _dp, C.POINTER(C.c_double)]),
            "orc_rbsog_far_exact": (C.c_int, [C.c_int, C.c_double, B, C.c_double, C.c_int, _dp,
                                              _dp, _dp, _dp, C.c_int, _dp, _dp, _dp,
                                              C.POINTER(C.c_double)]),
            "orc_pair_force_verlet_sog": (None, [C.c_int, C.c_double, B, C.c_double, C.c_int,
                                                 _ip, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int,
                                                 _ip, _ip, _dp, _dp, _dp, _dp, _dp]),
            "orc_dist2": (C.c_double, [B] + [C.c_double] * 6),
            "orc_cell_grid": (C.c_int, [B, C.c_double, _ip]),
            "orc_cells_sort": (C.c_int, [C.c_int, B, C.c_double, _dp, _dp, _dp, _ip, _ip,
                                         _ip, _ip]),
            "orc_full_list": (C.c_int64, [C.c_int, B, C.c_double, _dp, _dp, _dp, _ip, _ip,
                                          _ip, C.c_int, _ip, C.c_void_p]),
            "orc_rbl_params": (C.c_int, [C.c_int, B, C.c_double, C.c_double, C.c_int,
                                         C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "orc_rbl_mix": (C.c_uint64, [C.c_uint64]),
            "orc_rbl_selected": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_rbl_filter": (None, [C.c_int, B, C.c_double, C.c_double, C.c_int, C.c_int,
                                      _ip, _dp, _dp, _dp, C.c_int, _ip, _ip, _ip, _ip, _ip,
                                      _ip]),
            "orc_pair_force_rbl": (None, [C.c_int, B, C.c_double, C.c_double, C.c_int,
                                          C.c_double, C.c_double, _ip, _dp, _dp, _dp, _dp,
                                          _dp, _dp, C.c_int, _ip, _ip, _ip, _ip, _dp, _dp,
                                          _dp]),
            "orc_fix_rbl": (None, [C.c_int, _dp, _dp, _dp, _dp]),
            "orc_pair_force_rbl_special": (None, [C.c_int, B, C.c_double, C.c_double, C.c_int,
                                                  C.c_double, C.c_double, _ip, C.c_int, _dp, _dp,
                                                  _ip, _dp, _dp, _dp, _dp, C.c_int, _ip, _ip,
                                                  _ip, _ip, _ip, _ip, C.c_int, C.c_double,
                                                  C.c_double, C.c_double, _dp, _dp, _dp]),
            "orc_pair_force_verlet": (None, [C.c_int, B, C.c_double, C.c_double, C.c_double,
                                             _ip, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, _ip,
                                             _ip, _dp, _dp, _dp, _dp,
                                             C.POINTER(C.c_double), C.POINTER(C.c_double)]),
            "orc_max_disp2": (C.c_double, [C.c_int, B, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_engine_create": (C.c_void_p, [C.c_int, B, C.c_int, _dp, _dp, _dp, C.c_double,
                                               C.c_double, C.c_double, C.c_int, C.c_double,
                                               C.c_int, C.c_double, C.c_double, C.c_uint64,
                                               C.c_int]),
            "orc_engine_destroy": (None, [C.c_void_p]),
            "orc_engine_set_state": (C.c_int, [C.c_void_p, _ip, _ip, _dp, _dp, _dp, _dp, _dp,
                                               _dp, _dp]),
            "orc_engine_compute_forces": (C.c_int, [C.c_void_p, C.c_int]),
            "orc_engine_step": (C.c_int, [C.c_void_p, C.c_int]),
            "orc_engine_get": (C.c_int, [C.c_void_p, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                         _dp, _dp]),
            "orc_engine_rebuilds": (C.c_int, [C.c_void_p]),
            "orc_engine_set_nose_hoover": (C.c_int, [C.c_void_p, C.c_double, C.c_double,
                                                     C.c_double, C.c_longlong, C.c_double,
                                                     C.c_double, C.c_double]),
            "orc_engine_get_thermostat": (None, [C.c_void_p, _dp, _dp, _dp]),
            "orc_engine_set_fmt2v": (None, [C.c_void_p, C.c_double]),
            "orc_engine_set_shake": (C.c_int, [C.c_void_p, C.c_int, _ip, C.c_double,
                                               C.c_double]),
            "orc_engine_shake_failures": (C.c_int, [C.c_void_p]),
            "orc_num_threads": (C.c_int, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def num_threads():
    return lib().orc_num_threads()


# --- k-space ---------------------------------------------------------------
def rbe_gauss_sum(box, alpha):
    """ComputeRbeGaussianSum (src/force/src/kspace_calculator.cpp:68-78)."""
    return lib().orc_rbe_gauss_sum(C.byref(box), alpha)


def rbe_structure_factor(box, q, x, y, z, mx, my, mz):
    """ComputePnumberChargeStructureFactorOpt (kspace_calculator_op.hip.cu:238-289)."""
    n, p = len(q), len(mx)
    re = np.zeros(p)
    im = np.zeros(p)
    lib().orc_rbe_structure_factor(n, p, C.byref(box), _d(q), _d(x), _d(y), _d(z), _d(mx),
                                   _d(my), _d(mz), re, im)
    return re, im


def rbe_force(box, S, qqr2e, re, im, q, mx, my, mz, x, y, z):
    """ComputeRBEForce (kspace_calculator_op.hip.cu:678-738)."""
    n, p = len(q), len(mx)
    f = [np.zeros(n) for _ in range(3)]
    lib().orc_rbe_force(n, p, C.byref(box), S, qqr2e, _d(re), _d(im), _d(q), _d(mx), _d(my),
                        _d(mz), _d(x), _d(y), _d(z), *f)
    return np.stack(f, axis=1)


def rbe_energy_virial(box, alpha, S, qqr2e, qsq, qsum, re, im, mx, my, mz):
    """ComputeRBEVirial0 (kspace_calculator_op.hip.cu:573-674)."""
    vir = np.zeros(6)
    e = np.zeros(1)
    lib().orc_rbe_energy_virial(len(mx), C.byref(box), alpha, S, qqr2e, qsq, qsum, _d(re),
                                _d(im), _d(mx), _d(my), _d(mz), vir, e)
    return float(e[0]), vir


def ewald_kvectors(box, kmax):
    km = _i(kmax)
    nk = lib().orc_ewald_num_k(km)
    k = [np.zeros(nk) for _ in range(3)]
    lib().orc_ewald_kvectors(km, C.byref(box), *k)
    return k


def ewald_force(box, alpha, qqr2e, kmax, q, x, y, z):
    """Exact Ewald reciprocal force (ComputeEwaldForceFlat, kspace_calculator_op.hip.cu:334-403)
    and energy (ComputeKspaceEnergy + self, kspace_calculator.cpp:816-907)."""
    kx, ky, kz = ewald_kvectors(box, kmax)
    nk, n = len(kx), len(q)
    re = np.zeros(nk)
    im = np.zeros(nk)
    lib().orc_ewald_structure_factor(n, nk, _d(q), _d(x), _d(y), _d(z), kx, ky, kz, re, im)
    f = [np.zeros(n) for _ in range(3)]
    lib().orc_ewald_force(n, nk, C.byref(box), alpha, qqr2e, kx, ky, kz, re, im, _d(q), _d(x),
                          _d(y), _d(z), *f)
    qsq = float(np.sum(np.asarray(q) ** 2))
    e = lib().orc_ewald_energy(nk, C.byref(box), alpha, qqr2e, qsq, kx, ky, kz, re, im)
    return np.stack(f, axis=1), e


# --- samplers ----------------------------------------------------------------
def philox4x32_10(ctr, key):
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(np.ascontiguousarray(ctr, dtype=np.uint32),
                            np.ascontiguousarray(key, dtype=np.uint32), out)
    return out


def rbe_sample_philox(box, alpha, p, seed, step):
    m = [np.zeros(p) for _ in range(3)]
    rc = lib().orc_rbe_sample_philox(p, C.byref(box), alpha, seed, step, *m)
    if rc != 0:
        raise RuntimeError("philox k-sampler failed")
    return m


def rbe_sample_mh(box, alpha, p, seed):
    """Fetch_P_Sample Metropolis-Hastings chain (src/common/RBEPSample.h:150-188)."""
    m = [np.zeros(p) for _ in range(3)]
    lib().orc_rbe_sample_mh(p, C.byref(box), alpha, seed, *m)
    return m


# --- RBSOG ---------------------------------------------------------------------
def rbsog_params(level, cut_off, box):
    """RBSOGInit / RBSOGSetup / LJCoulSOGInit parameters (kspace_calculator.cpp:988-1140)."""
    sc = np.zeros(13)
    coef = np.zeros(128)
    coef_npt = np.zeros(128)
    dm = np.zeros(18, dtype=np.int32)
    dfb = np.zeros(6)
    dfb_npt = np.zeros(6)
    if lib().orc_rbsog_params(level, cut_off, C.byref(box), sc, coef, dm, dfb, coef_npt,
                              dfb_npt) != 0:
        raise ValueError("rbsog_level outside [0, 4]")
    mmax = int(sc[0])
    return {"mmax": mmax, "b": sc[1], "sigma": sc[2], "w0": sc[3], "S": sc[4], "S_npt": sc[5],
            "self_coeff": sc[6], "taylor": sc[7:13].copy(), "coef": coef[:mmax].copy(),
            "coef_npt": coef_npt[:mmax].copy(), "direct_m": dm.reshape(6, 3), "direct_fb": dfb,
            "direct_fb_npt": dfb_npt}


def rbsog_idx_npt(level, cut_off, box, m, u):
    """The NPT gather chain of RBSOGSampleKSpace (kspace_calculator.cpp:1242-1301) on the
    samples m with the uniforms u."""
    p = len(m[0])
    idx = np.zeros(p, dtype=np.int32)
    lib().orc_rbsog_idx_npt(level, cut_off, C.byref(box), p, *[_d(v) for v in m],
                            _d(np.asarray(u, dtype=np.float64)), idx)
    return idx


def rbsog_npt_uniforms(seed, step, p):
    """The uniforms the device NPT chain draws for (seed, step)."""
    u = np.zeros(p)
    lib().orc_rbsog_npt_uniforms(seed, step, p, u)
    return u


def shake_a(box, gid, typ, mass, dt, fmt2v, clusters, bond, angle_deg, pos, vel, force):
    """ShakeAOp at op level: half kick + drift of (pos, vel) with force, then the
    constraint of the (H, O, H) global-id clusters; returns (pos, vel, images, failures)."""
    n = len(gid)
    p = [np.ascontiguousarray(pos[:, d], dtype=np.float64).copy() for d in range(3)]
    v = [np.ascontiguousarray(vel[:, d], dtype=np.float64).copy() for d in range(3)]
    f = [np.ascontiguousarray(force[:, d], dtype=np.float64) for d in range(3)]
    img = np.zeros(3 * n, dtype=np.int32)
    cl = np.ascontiguousarray(clusters, dtype=np.int32)
    fails = lib().orc_shake_a_op(n, C.byref(box), _i(np.asarray(gid, dtype=np.int32)),
                                 _i(np.asarray(typ, dtype=np.int32)),
                                 _d(np.asarray(mass, dtype=np.float64)), len(mass), dt, fmt2v,
                                 len(cl), _i(cl), bond, angle_deg, *p, *v, *f,
                                 img.ctypes.data_as(C.c_void_p))
    return np.stack(p, 1), np.stack(v, 1), img.reshape(3, n), fails


def shake_b(box, gid, typ, mass, dt, fmt2v, clusters, bond, angle_deg, pos, vel, force):
    """ShakeBOp at op level: half kick of vel with force, then RATTLE; returns (vel, failures)."""
    n = len(gid)
    p = [np.ascontiguousarray(pos[:, d], dtype=np.float64) for d in range(3)]
    v = [np.ascontiguousarray(vel[:, d], dtype=np.float64).copy() for d in range(3)]
    f = [np.ascontiguousarray(force[:, d], dtype=np.float64) for d in range(3)]
    cl = np.ascontiguousarray(clusters, dtype=np.int32)
    fails = lib().orc_shake_b_op(n, C.byref(box), _i(np.asarray(gid, dtype=np.int32)),
                                 _i(np.asarray(typ, dtype=np.int32)),
                                 _d(np.asarray(mass, dtype=np.float64)), len(mass), dt, fmt2v,
                                 len(cl), _i(cl), bond, angle_deg, *p, *v, *f)
    return np.stack(v, 1), fails


def rbsog_virial(level, cut_off, box, qqr2e, q, m, idx, x, y, z, S=0.0, S_npt=0.0):
    """RBSOG k-space virial [6] (xx, yy, zz, xy, xz, yz): sampled part with the NPT terms over
    K[idx] plus the direct vectors (kspace_calculator_op.hip.cu:1133-1190, 1308-1355)."""
    v = np.zeros(6)
    lib().orc_rbsog_virial(level, cut_off, C.byref(box), qqr2e, S, S_npt, len(q), len(m[0]),
                           _d(q), *[_d(c) for c in m], _i(np.asarray(idx, dtype=np.int32)),
                           _d(x), _d(y), _d(z), v)
    return v


def rbsog_sample_philox(level, cut_off, box, p, seed, step):
    m = [np.zeros(p) for _ in range(3)]
    if lib().orc_rbsog_sample_philox(level, cut_off, C.byref(box), p, seed, step, *m) != 0:
        raise RuntimeError("RBSOG philox sampler failed")
    return m


def rbsog_sample_mh(level, cut_off, box, p, seed):
    """RBSOGSampleKSpace's Metropolis chain (kspace_calculator.cpp:1142-1240)."""
    m = [np.zeros(p) for _ in range(3)]
    lib().orc_rbsog_sample_mh(level, cut_off, C.byref(box), p, seed, *m)
    return m


def rbsog_force(level, cut_off, box, qqr2e, q, m, x, y, z, S=0.0):
    """ComputeRBSOG's k-space force and energy for the samples m (+ the 6 direct vectors)."""
    n, p = len(q), len(m[0])
    f = [np.zeros(n) for _ in range(3)]
    e = C.c_double()
    lib().orc_rbsog_force(level, cut_off, C.byref(box), qqr2e, S, n, p, _d(q), *[_d(v) for v in m],
                          _d(x), _d(y), _d(z), *f, C.byref(e))
    return np.stack(f, axis=1), e.value


def rbsog_far_exact(level, cut_off, box, qqr2e, q, x, y, z, mcut):
    """Exact far field over |m_d| <= mcut, |m|^2 > 1; returns (F, S_full)."""
    n = len(q)
    f = [np.zeros(n) for _ in range(3)]
    sf = C.c_double()
    lib().orc_rbsog_far_exact(level, cut_off, C.byref(box), qqr2e, n, _d(q), _d(x), _d(y), _d(z),
                              mcut, *f, C.byref(sf))
    return np.stack(f, axis=1), sf.value


def pair_force_verlet_sog(level, cut_off, box, qqr2e, typ, sigma, eps, q, x, y, z, count, rows,
                          virial=False):
    """LJCutCoulForceUserOp (lj_cut_coul_kspace_op.hip.cu:196-254, 357-470): forces,
    {E_LJ, E_coul}, and with virial=True the per-atom virial [6][n] (xx, yy, zz, xy, xz, yz)."""
    n, cap = rows.shape
    f = [np.zeros(n) for _ in range(3)]
    en = np.zeros(2)
    vir = np.zeros(6 * n)
    lib().orc_pair_force_verlet_sog(level, cut_off, C.byref(box), qqr2e, n, _i(typ), _d(sigma),
                                    _d(eps), _d(q), _d(x), _d(y), _d(z), cap, _i(count), _i(rows),
                                    *f, en, vir)
    if virial:
        return np.stack(f, axis=1), en, vir.reshape(6, n)
    return np.stack(f, axis=1), en


# --- lists -------------------------------------------------------------------
def dist2(box, pi, pj):
    return lib().orc_dist2(C.byref(box), *[float(v) for v in pi], *[float(v) for v in pj])


def cell_grid(box, cutoff):
    dims = np.zeros(3, dtype=np.int32)
    n = lib().orc_cell_grid(C.byref(box), cutoff, dims)
    return n, dims


def cells_sort(box, cutoff, x, y, z):
    """LinkedCell AssignAtomsToCell + SortAtomsByCellKey + ComputeCellRangesIndices."""
    n = len(x)
    ncell, _ = cell_grid(box, cutoff)
    perm = np.zeros(n, dtype=np.int32)
    cell = np.zeros(n, dtype=np.int32)
    cs = np.zeros(max(ncell, 1), dtype=np.int32)
    ce = np.zeros(max(ncell, 1), dtype=np.int32)
    rc = lib().orc_cells_sort(n, C.byref(box), cutoff, _d(x), _d(y), _d(z), perm, cell, cs, ce)
    if rc <= 0:
        raise RuntimeError("cell grid invalid")
    return perm, cell, cs, ce


def full_list(box, cutoff, x, y, z, cell, cs, ce):
    """GenerateFullNeighborListNoWarp over sorted atoms; returns (count, rows[n, cap])."""
    n = len(x)
    count = np.zeros(n, dtype=np.int32)
    maxc = lib().orc_full_list(n, C.byref(box), cutoff, _d(x), _d(y), _d(z), _i(cell), _i(cs),
                               _i(ce), 0, count, None)
    cap = max(int(maxc), 1)
    rows = np.full((n, cap), -1, dtype=np.int32)
    lib().orc_full_list(n, C.byref(box), cutoff, _d(x), _d(y), _d(z), _i(cell), _i(cs), _i(ce),
                        cap, count, rows.ctypes.data)
    return count, rows


def rbl_params(n_global, box, r_core, cut_off, sample_num):
    """GetRblParams (rbl_full_neighbor_list_builder.cpp:193-228) -> (freq, rs_num, rc_num)."""
    rs, rc = C.c_int(), C.c_int()
    f = lib().orc_rbl_params(n_global, C.byref(box), r_core, cut_off, sample_num,
                             C.byref(rs), C.byref(rc))
    return f, rs.value, rc.value


def rbl_mix(v):
    return lib().orc_rbl_mix(C.c_uint64(v & 0xFFFFFFFFFFFFFFFF))


def rbl_selected(freq, epoch, gi, gj):
    return bool(lib().orc_rbl_selected(freq, epoch, gi, gj))


def rbl_filter(box, r_core, cut_off, freq, epoch, gid, x, y, z, cand_count, cand):
    """FilterRBLNeighborCandidates (rbl_full_neighbor_list_op.hip.cu:237-304)."""
    n, cap = cand.shape
    cc = np.zeros(n, dtype=np.int32)
    sc = np.zeros(n, dtype=np.int32)
    core = np.full((n, cap), -1, dtype=np.int32)
    shell = np.full((n, cap), -1, dtype=np.int32)
    lib().orc_rbl_filter(n, C.byref(box), r_core, cut_off, freq, epoch, _i(gid), _d(x), _d(y),
                         _d(z), cap, _i(cand_count), _i(cand), cc, core, sc, shell)
    return cc, core, sc, shell


def pair_force_rbl(box, r_core, cut_off, freq, alpha, qqr2e, typ, sigma, eps, q, x, y, z,
                   core_count, core, shell_count, shell):
    """ComputeLJCutCoulRBLForce (lj_cut_coul_kspace_op.hip.cu:569-683), no mean removal."""
    n, cap = core.shape
    assert shell.shape == core.shape
    f = [np.zeros(n) for _ in range(3)]
    lib().orc_pair_force_rbl(n, C.byref(box), r_core, cut_off, freq, alpha, qqr2e, _i(typ),
                             _d(sigma), _d(eps), _d(q), _d(x), _d(y), _d(z), cap,
                             _i(core_count), _i(core), _i(shell_count), _i(shell), *f)
    return np.stack(f, axis=1)


def pair_force_rbl_special(box, r_core, cut_off, freq, alpha, qqr2e, typ, sigma, eps, gid, q,
                           x, y, z, core_count, core, shell_count, shell, nspecial, special,
                           weights):
    """ComputeSpecialLJCutCoulRBLForce (cvff_op.hip.cu:401-533), no mean removal.
    nspecial [n, 3] / special [n, maxs] are indexed like the atoms and hold
    partner gids."""
    n, cap = core.shape
    nt = len(sigma)
    sig = np.asarray(sigma, float)
    ep = np.asarray(eps, float)
    lj12 = np.zeros(nt * nt)
    lj6 = np.zeros(nt * nt)
    for a in range(nt):  # CVFF::Init (cvff.cpp:855-870)
        for b in range(nt):
            e_ab = math.sqrt(ep[a] * ep[b])
            s_ab = (sig[a] + sig[b]) * 0.5
            s6 = (s_ab * s_ab) ** 3
            lj12[a * nt + b] = 48.0 * e_ab * s6 * s6
            lj6[a * nt + b] = 24.0 * e_ab * s6
    sp = np.ascontiguousarray(special, dtype=np.int32)
    f = [np.zeros(n) for _ in range(3)]
    lib().orc_pair_force_rbl_special(n, C.byref(box), r_core, cut_off, freq, alpha, qqr2e,
                                     _i(typ), nt, _d(lj12), _d(lj6), _i(gid), _d(q), _d(x), _d(y),
                                     _d(z), cap, _i(core_count), _i(core), _i(shell_count),
                                     _i(shell), _i(nspecial), _i(sp), sp.shape[1], *weights, *f)
    return np.stack(f, axis=1)


def fix_rbl(f):
    """Mean-force removal (lj_cut_coul_kspace.cpp:537-563, force_op.hip.cu:9-45)."""
    fx, fy, fz = (np.ascontiguousarray(f[:, d]) for d in range(3))
    mean = np.zeros(3)
    lib().orc_fix_rbl(len(fx), fx, fy, fz, mean)
    return np.stack([fx, fy, fz], axis=1), mean


def pair_force_verlet(box, cut_off, alpha, qqr2e, typ, sigma, eps, q, x, y, z, count, rows):
    """ComputeLJCutCoulForce (lj_cut_coul_kspace_op.hip.cu:256-356) + ReduceVirial."""
    n, cap = rows.shape
    f = [np.zeros(n) for _ in range(3)]
    vir = np.zeros(6)
    el, ec = C.c_double(), C.c_double()
    lib().orc_pair_force_verlet(n, C.byref(box), cut_off, alpha, qqr2e, _i(typ), _d(sigma),
                                _d(eps), _d(q), _d(x), _d(y), _d(z), cap, _i(count), _i(rows),
                                *f, vir, C.byref(el), C.byref(ec))
    return np.stack(f, axis=1), vir, el.value, ec.value


def max_disp2(box, x, y, z, x0, y0, z0):
    return lib().orc_max_disp2(len(x), C.byref(box), _d(x), _d(y), _d(z), _d(x0), _d(y0),
                               _d(z0))


class Engine:
    """Whole NVE velocity-Verlet step on the host (NVEensemble::Solve,
    src/simulate_pipeline/src/nve_ensemble.cpp:59-91), OpenMP over atoms."""

    def __init__(self, sys, *, use_rbl=True, seed=12345):
        L = lib()
        self.n = sys["n"]
        self.box = Box.make(sys["lo"], sys["hi"])
        p = sys["params"]
        self._h = L.orc_engine_create(self.n, C.byref(self.box), len(sys["sigma"]),
                                      _d(sys["sigma"]), _d(sys["eps"]), _d(sys["mass"]),
                                      p["cut_off"], p["r_core"], p["skin"],
                                      p["neighbor_sample_num"], p["alpha"], p["kspace_p"],
                                      p["qqr2e"], p["dt"], seed, int(use_rbl))
        if not self._h:
            raise RuntimeError("orc_engine_create failed")
        L.orc_engine_set_fmt2v(self._h, float(p.get("fmt2v", 1.0)))
        self._gid = np.asarray(sys["gid"], dtype=np.int32)
        L.orc_engine_set_state(self._h, _i(sys["gid"]), _i(sys["type"]), _d(sys["q"]),
                               *[_d(sys["pos"][:, d]) for d in range(3)],
                               *[_d(sys["vel"][:, d]) for d in range(3)])

    def compute_forces(self, epoch=0):
        if lib().orc_engine_compute_forces(self._h, epoch) != 0:
            raise RuntimeError("oracle force evaluation failed")

    def step(self, nsteps):
        if lib().orc_engine_step(self._h, nsteps) != 0:
            raise RuntimeError("oracle step failed")

    def get(self):
        n = self.n
        gid = np.zeros(n, dtype=np.int32)
        a = [np.zeros(n) for _ in range(9)]
        lib().orc_engine_get(self._h, gid, *a)
        return {"gid": gid, "pos": np.stack(a[0:3], 1), "vel": np.stack(a[3:6], 1),
                "force": np.stack(a[6:9], 1)}

    @property
    def rebuilds(self):
        return lib().orc_engine_rebuilds(self._h)

    def set_nose_hoover(self, t_start, t_stop, t_damp, num_steps=0, kb=1.0, mvv2e=1.0, tdof=0.0):
        """NVT Nose-Hoover chain (NVTensemble::Solve with NOSE_HOOVER)."""
        lib().orc_engine_set_nose_hoover(self._h, t_start, t_stop, t_damp, num_steps, kb, mvv2e,
                                         tdof)

    def set_shake(self, clusters, bond, angle_deg):
        """SHAKE / RATTLE clusters given as host atom indices [nc, 3], centre second."""
        gids = np.ascontiguousarray(self._gid[np.asarray(clusters)], dtype=np.int32)
        lib().orc_engine_set_shake(self._h, len(gids), _i(gids.ravel()), bond, angle_deg)

    @property
    def shake_failures(self):
        return lib().orc_engine_shake_failures(self._h)

    def thermostat(self):
        t = np.zeros(1)
        eta, eta_dot = np.zeros(3), np.zeros(3)
        lib().orc_engine_get_thermostat(self._h, t, eta, eta_dot)
        return {"temperature": t[0], "eta": eta, "eta_dot": eta_dot}

    def __del__(self):
        try:
            if self._h:
                lib().orc_engine_destroy(self._h)
                self._h = None
        except Exception:
            pass


# --- one force evaluation of the RBL + RBE path --------------------------------
def pair_keys(pairs):
    """Sorted int64 keys gid_i * 2^32 + gid_j of an [m, 2] array of gid pairs."""
    a = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    return np.sort((a[:, 0] << 32) | (a[:, 1] & 0xFFFFFFFF))


def _pair_keys(gid, count, rows):
    n, cap = rows.shape
    mask = np.arange(cap)[None, :] < count[:, None]
    gi = np.broadcast_to(np.asarray(gid, dtype=np.int64)[:, None], rows.shape)[mask]
    gj = np.asarray(gid, dtype=np.int64)[rows[mask]]
    return np.sort((gi << 32) | (gj & 0xFFFFFFFF))


def rbl_rbe_evaluation(sys, m, epoch=0, pair_energy=True):
    """One LJCutCoulKspace::Execute of the RBL + RBE path on a system dict
    (rbmd_b200.systems layout) with injected k-samples m = (mx, my, mz):
    cell sort, candidate list at cut_off + skin, RBL filter with the batch
    hash of `epoch`, RBL pair force with mean removal, RBE structure factor,
    force, energy and virial (lj_cut_coul_kspace.cpp:464-573,
    kspace_calculator.cpp:532-669).  Optionally the pair energies and virial
    over every pair within cut_off (LJCutCoulEnergyOp).  Arrays are returned
    in the order of the input atoms; the core and shell pairs as sorted keys
    (pair_keys)."""
    p = sys["params"]
    box = Box.make(sys["lo"], sys["hi"])
    n = int(sys["n"])
    rcs = p["cut_off"] + p["skin"]
    x, y, z = (np.ascontiguousarray(sys["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = cells_sort(box, rcs, x, y, z)
    xs, ys, zs = x[perm], y[perm], z[perm]
    cnt, rows = full_list(box, rcs, xs, ys, zs, cell, cs, ce)
    freq, _, _ = rbl_params(n, box, p["r_core"], p["cut_off"], p["neighbor_sample_num"])
    gid = np.asarray(sys["gid"])[perm]
    typ = np.asarray(sys["type"])[perm]
    q = np.asarray(sys["q"])[perm]
    cc, core, sc, shell = rbl_filter(box, p["r_core"], p["cut_off"], freq, epoch, gid, xs, ys, zs,
                                     cnt, rows)
    fp = pair_force_rbl(box, p["r_core"], p["cut_off"], freq, p["alpha"], p["qqr2e"], typ,
                        sys["sigma"], sys["eps"], q, xs, ys, zs, cc, core, sc, shell)
    fp, _ = fix_rbl(fp)
    S = rbe_gauss_sum(box, p["alpha"])
    re, im = rbe_structure_factor(box, q, xs, ys, zs, *m)
    fk = rbe_force(box, S, p["qqr2e"], re, im, q, *m, xs, ys, zs)
    ek, vk = rbe_energy_virial(box, p["alpha"], S, p["qqr2e"], float((q ** 2).sum()),
                               float(q.sum()), re, im, *m)
    # the sampled sum before the self term is subtracted: the scale of the
    # k-space energy's rounding error (the two nearly cancel)
    V = float(np.prod(np.asarray(sys["hi"], float) - np.asarray(sys["lo"], float)))
    e_self = p["qqr2e"] * (np.sqrt(p["alpha"]) * float((q ** 2).sum()) / np.sqrt(np.pi)
                           + 0.5 * np.pi * float(q.sum()) ** 2 / (p["alpha"] * V))
    out = {"freq": freq, "f_pair": np.zeros((n, 3)), "f_kspace": np.zeros((n, 3)),
           "e_kspace": ek, "e_kspace_scale": abs(ek + e_self), "virial_kspace": np.asarray(vk),
           "core_keys": _pair_keys(gid, cc, core), "shell_keys": _pair_keys(gid, sc, shell)}
    out["f_pair"][perm] = fp
    out["f_kspace"][perm] = fk
    out["force"] = out["f_pair"] + out["f_kspace"]
    if pair_energy:
        _, vir, el, ec = pair_force_verlet(box, p["cut_off"], p["alpha"], p["qqr2e"], typ,
                                           sys["sigma"], sys["eps"], q, xs, ys, zs, cnt, rows)
        out.update(e_vdwl=el, e_coul=ec, virial_pair=np.asarray(vir))
    return out
