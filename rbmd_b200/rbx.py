"""ctypes binding of librbx.so (the C ABI in include/rbx.h).

The engine itself is torch-free C++/CUDA; this module only marshals arguments.
Op-level wrappers take torch CUDA tensors (device pointers) so tests can drive
the drop-in kernels exactly as RBMD's op functors are driven.  There is no CPU
fallback: loading fails loudly when the library is missing, and every compute
call raises when the library reports an error.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librbx.so")
_lib = None

RBX_OK = 0
PLAIN_FP64 = 0
MIXED = 1
# largest atom-type count an engine takes (RBX_MAX_TYPES of include/rbx.h)
MAX_TYPES = 64
NEIGHBOR_VERLET = 0
NEIGHBOR_RBL = 1
NEIGHBOR_VERLET_SOG = 2
COULOMB_NONE = 0
COULOMB_RBE = 1
COULOMB_EWALD = 2
COULOMB_RBSOG = 3


class RbxError(RuntimeError):
    pass


class Box(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3)]

    @staticmethod
    def make(lo, hi):
        b = Box()
        for d in range(3):
            b.lo[d] = float(lo[d])
            b.hi[d] = float(hi[d])
        return b


class Params(C.Structure):
    _fields_ = [
        ("neighbor_type", C.c_int),
        ("cut_off", C.c_double),
        ("r_core", C.c_double),
        ("skin", C.c_double),
        ("neighbor_sample_num", C.c_int),
        ("coulomb_type", C.c_int),
        ("alpha", C.c_double),
        ("coulomb_sample_num", C.c_int),
        ("kmax", C.c_int * 3),
        ("random_seed", C.c_uint64),
        ("qqr2e", C.c_double),
        ("dt", C.c_double),
        ("precision", C.c_int),
        ("ntypes", C.c_int),
        ("sigma", C.POINTER(C.c_double)),
        ("eps", C.POINTER(C.c_double)),
        ("mass", C.POINTER(C.c_double)),
        ("fmt2v", C.c_double),
        ("rbsog_level", C.c_int),
        ("rbsog_S", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("steps", C.c_int64),
        ("force_calls", C.c_int64),
        ("rebuilds", C.c_int64),
        ("epoch", C.c_int),
        ("selection_frequency", C.c_int),
        ("candidate_capacity", C.c_int),
        ("candidates", C.c_int64),
        ("e_kspace", C.c_double),
        ("virial_kspace", C.c_double * 6),
    ]


# Every symbol include/rbx.h declares.
EXPORTS = [
    "rbx_last_error", "rbx_version", "rbx_launch_count", "rbx_rbe_gauss_sum", "rbx_rbl_params",
    "rbx_rbe_sample", "rbx_rbe_structure_factor", "rbx_rbe_force", "rbx_rbe_energy_virial",
    "rbx_ewald_force", "rbx_cell_grid", "rbx_cells_scratch_bytes", "rbx_cells_sort",
    "rbx_full_list", "rbx_rbl_filter", "rbx_pair_force_rbl", "rbx_fix_rbl_force",
    "rbx_pair_force_verlet", "rbx_engine_create", "rbx_engine_create_json",
    "rbx_engine_destroy", "rbx_engine_set_state", "rbx_engine_set_k_samples",
    "rbx_engine_compute_forces", "rbx_engine_step", "rbx_engine_step_host",
    "rbx_engine_get_state", "rbx_engine_get_force_parts", "rbx_engine_get_rbl_pairs",
    "rbx_engine_pair_energy",
    "rbx_engine_get_stats", "rbx_engine_stream", "rbx_engine_phase_ms",
    "rbx_engine_set_profiling", "rbx_rbe_structure_factor_noalloc", "rbx_engine_set_step_graph",
    "rbx_nlist_should_reuse", "rbx_batch_create", "rbx_batch_destroy", "rbx_batch_step",
    "rbx_batch_stream", "rbx_engine_force_vjp", "rbx_engine_set_lj_params",
    "rbx_engine_set_charges", "rbx_engine_set_alpha", "rbx_lammps_read", "rbx_lammps_free",
    "rbx_lammps_get_info", "rbx_lammps_get_atoms", "rbx_lammps_get_types",
    "rbx_lammps_get_topology", "rbx_lammps_write_charge", "rbx_engine_set_images",
    "rbx_engine_get_images", "rbx_engine_write_trajectory", "rbx_engine_create_from_files",
    "rbx_engine_get_system", "rbx_engine_get_atoms", "rbx_engine_get_type_params",
    "rbx_lammps_gauss_velocities", "rbx_engine_set_nose_hoover", "rbx_engine_get_thermostat",
    "rbx_engine_set_shake", "rbx_engine_get_shake", "rbx_engine_set_special", "rbx_special_build",
    "rbx_rbsog_params", "rbx_rbsog_sample", "rbx_rbsog_force", "rbx_pair_force_verlet_sog",
    "rbx_engine_autotune", "rbx_batch_autotune", "rbx_batch_set_mode", "rbx_batch_design",
    "rbx_rbe_structure_factor_f32", "rbx_rbe_force_f32", "rbx_rbe_energy_virial_f32",
    "rbx_rbl_filter_f32", "rbx_pair_force_rbl_f32", "rbx_fix_rbl_force_f32",
    "rbx_pair_force_verlet_f32", "rbx_engine_kspace_energy_exact", "rbx_force_create_json",
    "rbx_force_destroy", "rbx_force_engine", "rbx_force_execute", "rbx_force_energies",
    "rbx_rbsog_npt_chain", "rbx_rbsog_virial", "rbx_engine_rbsog_npt_map",
]


class RbsogInfo(C.Structure):
    _fields_ = [("level", C.c_int), ("mmax", C.c_int), ("b", C.c_double), ("sigma", C.c_double),
                ("w0", C.c_double), ("S", C.c_double), ("S_npt", C.c_double),
                ("self_coeff", C.c_double), ("taylor", C.c_double * 6), ("n_direct", C.c_int),
                ("S_full", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("rho_kpt", C.c_int), ("rho_blocks", C.c_int), ("force_block", C.c_int),
                ("rbl_waves", C.c_int), ("cache_hit", C.c_int), ("rho_ms", C.c_float),
                ("force_ms", C.c_float), ("rbl_ms", C.c_float), ("rho_ms_default", C.c_float),
                ("force_ms_default", C.c_float), ("rbl_ms_default", C.c_float)]


class LammpsInfo(C.Structure):
    _fields_ = [("n_atoms", C.c_int64), ("n_bonds", C.c_int64), ("n_angles", C.c_int64),
                ("n_dihedrals", C.c_int64), ("n_impropers", C.c_int64),
                ("n_atom_types", C.c_int), ("n_bond_types", C.c_int), ("n_angle_types", C.c_int),
                ("n_dihedral_types", C.c_int), ("n_improper_types", C.c_int),
                ("atom_style", C.c_int), ("has_masses", C.c_int), ("has_pair_coeffs", C.c_int),
                ("has_velocities", C.c_int), ("has_images", C.c_int), ("box", Box)]


def lib():
    """Load librbx.so (built in-tree by rbmd_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RbxError(f"{LIB_PATH} is missing: run `python -m rbmd_b200.build` "
                       "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.c_int, C.c_double
    B = C.POINTER(Box)
    L.rbx_last_error.restype = C.c_char_p
    L.rbx_launch_count.restype = C.c_uint64
    L.rbx_cells_scratch_bytes.restype = C.c_size_t
    L.rbx_cells_scratch_bytes.argtypes = [ip, ip]
    L.rbx_rbe_gauss_sum.argtypes = [B, dp, C.POINTER(C.c_double)]
    L.rbx_rbl_params.argtypes = [ip, B, dp, dp, ip, C.POINTER(C.c_int)]
    L.rbx_rbe_sample.argtypes = [B, dp, ip, C.c_uint64, C.c_int64, vp, vp, vp, vp]
    L.rbx_rbe_structure_factor.argtypes = [B, ip, ip] + [vp] * 9 + [vp]
    L.rbx_rbe_structure_factor_noalloc.argtypes = [B, ip, ip] + [vp] * 9 + [vp]
    L.rbx_rbe_force.argtypes = [B, ip, ip, dp, dp, dp] + [vp] * 12 + [vp]
    L.rbx_rbe_energy_virial.argtypes = [B, ip, dp, dp, dp, dp, dp] + [vp] * 7 + [vp]
    L.rbx_ewald_force.argtypes = [B, ip, C.POINTER(C.c_int), dp, dp] + [vp] * 8 + [vp]
    L.rbx_cell_grid.argtypes = [B, dp, C.POINTER(C.c_int)]
    L.rbx_cells_sort.argtypes = [B, dp, ip] + [vp] * 7 + [vp]
    L.rbx_full_list.argtypes = [B, dp, ip, vp, vp, vp, vp, ip, vp, vp, vp, vp]
    L.rbx_rbl_filter.argtypes = ([dp, dp, ip] + [vp] * 11 + [ip] + [vp] * 3 + [B, vp, ip, ip,
                                                                                 vp])
    L.rbx_pair_force_rbl.argtypes = [B, dp, dp, ip, ip, ip, dp, dp] + [vp] * 14 + [vp]
    L.rbx_fix_rbl_force.argtypes = [ip, vp, vp, vp, vp, vp]
    L.rbx_pair_force_verlet.argtypes = [B, dp, ip, dp, dp] + [vp] * 15 + [vp]
    L.rbx_engine_create.restype = vp
    L.rbx_engine_create.argtypes = [C.POINTER(Params), B, ip, ip]
    L.rbx_engine_create_json.restype = vp
    L.rbx_engine_create_json.argtypes = [C.c_char_p, B, ip, ip, vp, vp, vp, vp, ip, ip]
    L.rbx_engine_destroy.argtypes = [vp]
    L.rbx_engine_set_state.argtypes = [vp] * 10
    L.rbx_engine_set_k_samples.argtypes = [vp, ip, vp, vp, vp]
    L.rbx_engine_compute_forces.argtypes = [vp, ip]
    L.rbx_engine_step.argtypes = [vp, ip]
    L.rbx_engine_step_host.argtypes = [vp] * 6
    L.rbx_engine_get_state.argtypes = [vp] * 10
    L.rbx_engine_get_force_parts.argtypes = [vp, vp, vp]
    L.rbx_engine_pair_energy.argtypes = [vp, vp, vp, vp]
    L.rbx_engine_get_rbl_pairs.argtypes = [vp, vp, C.POINTER(C.c_int64), vp,
                                           C.POINTER(C.c_int64)]
    L.rbx_engine_get_stats.argtypes = [vp, C.POINTER(Stats)]
    L.rbx_engine_stream.restype = vp
    L.rbx_engine_stream.argtypes = [vp]
    L.rbx_engine_phase_ms.argtypes = [vp, C.POINTER(C.c_float)]
    L.rbx_engine_set_profiling.argtypes = [vp, ip]
    L.rbx_engine_set_step_graph.argtypes = [vp, ip]
    L.rbx_engine_force_vjp.argtypes = [vp] + [vp] * 6
    L.rbx_engine_set_lj_params.argtypes = [vp, vp, vp]
    L.rbx_engine_set_charges.argtypes = [vp, vp]
    L.rbx_engine_set_alpha.argtypes = [vp, dp]
    L.rbx_engine_set_images.argtypes = [vp, vp]
    L.rbx_engine_get_images.argtypes = [vp, vp]
    L.rbx_engine_write_trajectory.argtypes = [vp, C.c_char_p, C.c_int64, ip]
    L.rbx_engine_create_from_files.restype = vp
    L.rbx_engine_create_from_files.argtypes = [C.c_char_p, ip, ip]
    L.rbx_engine_get_system.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), B]
    L.rbx_engine_get_atoms.argtypes = [vp, vp, vp, vp]
    L.rbx_engine_get_type_params.argtypes = [vp, vp, vp, vp]
    L.rbx_lammps_gauss_velocities.argtypes = [vp, dp, C.c_char_p, ip]
    L.rbx_engine_set_nose_hoover.argtypes = [vp, dp, dp, dp, C.c_int64, dp, dp, dp]
    L.rbx_engine_get_thermostat.argtypes = [vp, vp, vp, vp]
    L.rbx_engine_set_shake.argtypes = [vp, ip, vp, dp, dp]
    L.rbx_engine_get_shake.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.rbx_engine_set_special.argtypes = [vp, ip, vp, vp, dp, dp, dp]
    L.rbx_special_build.argtypes = [ip, ip, vp, ip, vp, ip, vp, C.POINTER(C.c_int), vp, vp]
    L.rbx_rbsog_params.argtypes = [ip, dp, B, C.POINTER(RbsogInfo), vp, vp, vp]
    L.rbx_engine_autotune.argtypes = [vp, ip, C.POINTER(Tuning)]
    L.rbx_batch_autotune.argtypes = [vp]
    L.rbx_rbsog_sample.argtypes = [B, ip, dp, ip, C.c_uint64, C.c_int64, vp, vp, vp, vp]
    L.rbx_rbsog_force.argtypes = [B, ip, dp, dp, dp, dp, ip, ip] + [vp] * 10 + [
        C.POINTER(C.c_double), vp]
    L.rbx_rbsog_npt_chain.argtypes = [B, ip, dp, ip, vp, vp, vp, C.c_uint64, C.c_int64, vp, vp]
    L.rbx_rbsog_virial.argtypes = [B, ip, dp, dp, dp, dp, ip, ip] + [vp] * 8 + [vp, vp]
    L.rbx_engine_rbsog_npt_map.argtypes = [vp, C.POINTER(C.c_int), vp]
    L.rbx_pair_force_verlet_sog.argtypes = [B, ip, dp, dp, ip, ip, vp, vp] + [vp] * 5 + [
        ip, vp, vp, vp, vp, vp, vp, vp, vp]
    L.rbx_lammps_read.restype = vp
    L.rbx_lammps_read.argtypes = [C.c_char_p, C.c_char_p, vp]
    L.rbx_lammps_free.argtypes = [vp]
    L.rbx_lammps_get_info.argtypes = [vp, C.POINTER(LammpsInfo)]
    L.rbx_lammps_get_atoms.argtypes = [vp] + [vp] * 11
    L.rbx_lammps_get_types.argtypes = [vp, vp, vp, vp]
    L.rbx_lammps_get_topology.argtypes = [vp, ip, vp, vp]
    L.rbx_lammps_write_charge.argtypes = [C.c_char_p, B, ip, ip] + [vp] * 12
    L.rbx_batch_create.restype = vp
    L.rbx_batch_create.argtypes = [C.POINTER(vp), ip]
    L.rbx_batch_destroy.argtypes = [vp]
    L.rbx_batch_step.argtypes = [vp, ip]
    L.rbx_batch_stream.restype = vp
    L.rbx_batch_stream.argtypes = [vp]
    L.rbx_batch_set_mode.argtypes = [vp, ip]
    L.rbx_batch_design.argtypes = [vp]
    L.rbx_nlist_should_reuse.argtypes = [B, ip] + [vp] * 6 + [dp, C.POINTER(C.c_int),
                                                             C.POINTER(C.c_double), vp]
    L.rbx_engine_kspace_energy_exact.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.rbx_force_create_json.restype = vp
    L.rbx_force_create_json.argtypes = [C.c_char_p, B, ip, ip, vp, vp, vp, vp, ip, ip]
    L.rbx_force_destroy.restype = None
    L.rbx_force_destroy.argtypes = [vp]
    L.rbx_force_engine.restype = vp
    L.rbx_force_engine.argtypes = [vp]
    L.rbx_force_execute.argtypes = [vp, ip, ip]
    L.rbx_force_energies.argtypes = [vp, C.POINTER(C.c_double)]
    fp = C.c_float  # FP32 twins: float scalars
    L.rbx_rbe_structure_factor_f32.argtypes = [B, ip, ip] + [vp] * 9 + [vp]
    L.rbx_rbe_force_f32.argtypes = [B, ip, ip, fp, fp, fp] + [vp] * 12 + [vp]
    L.rbx_rbe_energy_virial_f32.argtypes = [B, ip, fp, fp, fp, fp, fp] + [vp] * 7 + [vp]
    L.rbx_rbl_filter_f32.argtypes = ([fp, fp, ip] + [vp] * 11 + [ip] + [vp] * 3 +
                                     [B, vp, ip, ip, vp])
    L.rbx_pair_force_rbl_f32.argtypes = [B, fp, fp, ip, ip, ip, fp, fp] + [vp] * 14 + [vp]
    L.rbx_fix_rbl_force_f32.argtypes = [ip, vp, vp, vp, vp, vp]
    L.rbx_pair_force_verlet_f32.argtypes = [B, fp, ip, fp, fp] + [vp] * 15 + [vp]
    _lib = L
    return L


def last_error() -> str:
    return lib().rbx_last_error().decode(errors="replace")


def check(rc, what=""):
    if rc != RBX_OK:
        raise RbxError(f"{what} failed (status {rc}): {last_error()}")


def launch_count() -> int:
    return int(lib().rbx_launch_count())


def _ptr(t):
    """Device pointer of a torch tensor (or None)."""
    if t is None:
        return None
    return C.c_void_p(t.data_ptr())


def _np_ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _stream(stream):
    if stream is None:
        return None
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


# ---------------------------------------------------------------------------
# host helpers
# ---------------------------------------------------------------------------
def rbe_gauss_sum(box: Box, alpha: float) -> float:
    s = C.c_double()
    check(lib().rbx_rbe_gauss_sum(C.byref(box), alpha, C.byref(s)), "rbx_rbe_gauss_sum")
    return s.value


def rbl_params(n_global, box: Box, r_core, cut_off, sample_num) -> int:
    f = C.c_int()
    check(lib().rbx_rbl_params(n_global, C.byref(box), r_core, cut_off, sample_num, C.byref(f)),
          "rbx_rbl_params")
    return f.value


def cell_grid(box: Box, cutoff: float):
    dims = (C.c_int * 3)()
    check(lib().rbx_cell_grid(C.byref(box), cutoff, dims), "rbx_cell_grid")
    return list(dims)


# ---------------------------------------------------------------------------
# op-level wrappers (torch CUDA tensors in, results written in place)
# ---------------------------------------------------------------------------
def rbe_sample(box, alpha, p, seed, step, mx, my, mz, stream=None):
    check(lib().rbx_rbe_sample(C.byref(box), alpha, p, seed, step, _ptr(mx), _ptr(my), _ptr(mz),
                               _stream(stream)), "rbx_rbe_sample")


def rbe_structure_factor(box, q, mx, my, mz, x, y, z, re, im, stream=None):
    check(lib().rbx_rbe_structure_factor(C.byref(box), q.numel(), mx.numel(), _ptr(q), _ptr(mx),
                                         _ptr(my), _ptr(mz), _ptr(x), _ptr(y), _ptr(z), _ptr(re),
                                         _ptr(im), _stream(stream)), "rbx_rbe_structure_factor")


def rbe_structure_factor_noalloc(box, q, mx, my, mz, x, y, z, re, im, stream=None):
    """Structure factors without device allocation (built-in scratch; p <= 512)."""
    check(lib().rbx_rbe_structure_factor_noalloc(C.byref(box), q.numel(), mx.numel(), _ptr(q),
                                                 _ptr(mx), _ptr(my), _ptr(mz), _ptr(x), _ptr(y),
                                                 _ptr(z), _ptr(re), _ptr(im), _stream(stream)),
          "rbx_rbe_structure_factor_noalloc")


def rbe_force(box, alpha, S, qqr2e, re, im, q, mx, my, mz, x, y, z, fx, fy, fz, stream=None):
    check(lib().rbx_rbe_force(C.byref(box), q.numel(), mx.numel(), alpha, S, qqr2e, _ptr(re),
                              _ptr(im), _ptr(q), _ptr(mx), _ptr(my), _ptr(mz), _ptr(x), _ptr(y),
                              _ptr(z), _ptr(fx), _ptr(fy), _ptr(fz), _stream(stream)),
          "rbx_rbe_force")


def rbe_energy_virial(box, alpha, S, qqr2e, qsq, qsum, re, im, mx, my, mz, virial, energy,
                      stream=None):
    check(lib().rbx_rbe_energy_virial(C.byref(box), mx.numel(), alpha, S, qqr2e, qsq, qsum,
                                      _ptr(re), _ptr(im), _ptr(mx), _ptr(my), _ptr(mz),
                                      _ptr(virial), _ptr(energy), _stream(stream)),
          "rbx_rbe_energy_virial")


def ewald_force(box, kmax, alpha, qqr2e, q, x, y, z, fx, fy, fz, energy=None, stream=None):
    km = (C.c_int * 3)(*kmax)
    check(lib().rbx_ewald_force(C.byref(box), q.numel(), km, alpha, qqr2e, _ptr(q), _ptr(x),
                                _ptr(y), _ptr(z), _ptr(fx), _ptr(fy), _ptr(fz), _ptr(energy),
                                _stream(stream)), "rbx_ewald_force")


def cells_sort(box, cutoff, x, y, z, perm, cell_of_sorted, cell_start, scratch, stream=None):
    check(lib().rbx_cells_sort(C.byref(box), cutoff, x.numel(), _ptr(x), _ptr(y), _ptr(z),
                               _ptr(perm), _ptr(cell_of_sorted), _ptr(cell_start), _ptr(scratch),
                               _stream(stream)), "rbx_cells_sort")


def cells_scratch_bytes(n, ncell) -> int:
    return int(lib().rbx_cells_scratch_bytes(n, ncell))


def nlist_should_reuse(box, x, y, z, x0, y0, z0, skin, stream=None):
    """(reuse, max squared displacement) of a list cached at x0, y0, z0."""
    reuse, d2 = C.c_int(0), C.c_double(0.0)
    check(lib().rbx_nlist_should_reuse(C.byref(box), x.numel(), _ptr(x), _ptr(y), _ptr(z),
                                       _ptr(x0), _ptr(y0), _ptr(z0), skin, C.byref(reuse),
                                       C.byref(d2), _stream(stream)), "rbx_nlist_should_reuse")
    return bool(reuse.value), d2.value


def full_list(box, cutoff, x, y, z, cell_start, cap, count, nbrs, overflow, stream=None):
    check(lib().rbx_full_list(C.byref(box), cutoff, x.numel(), _ptr(x), _ptr(y), _ptr(z),
                              _ptr(cell_start), cap, _ptr(count), _ptr(nbrs), _ptr(overflow),
                              _stream(stream)), "rbx_full_list")


def rbl_filter(core2, force2, gid, x, y, z, cstart, cend, cand, core_cap, core_start, core_end,
               core, shell_cap, shell, shell_num, required, box, realloc, freq, epoch,
               stream=None):
    check(lib().rbx_rbl_filter(core2, force2, gid.numel(), _ptr(gid), _ptr(x), _ptr(y), _ptr(z),
                               _ptr(cstart), _ptr(cend), _ptr(cand), _ptr(core_cap),
                               _ptr(core_start), _ptr(core_end), _ptr(core), shell_cap,
                               _ptr(shell), _ptr(shell_num), _ptr(required), C.byref(box),
                               _ptr(realloc), freq, epoch, _stream(stream)), "rbx_rbl_filter")


def pair_force_rbl(box, rs, rc, sample_num, pice, alpha, qqr2e, typ, sigma, eps, start, end,
                   core, shell, shell_num, q, x, y, z, fx, fy, fz, stream=None):
    check(lib().rbx_pair_force_rbl(C.byref(box), rs, rc, q.numel(), sample_num, pice, alpha, qqr2e,
                                   _ptr(typ), _ptr(sigma), _ptr(eps), _ptr(start), _ptr(end),
                                   _ptr(core), _ptr(shell), _ptr(shell_num), _ptr(q), _ptr(x),
                                   _ptr(y), _ptr(z), _ptr(fx), _ptr(fy), _ptr(fz),
                                   _stream(stream)), "rbx_pair_force_rbl")


def fix_rbl_force(fx, fy, fz, mean=None, stream=None):
    check(lib().rbx_fix_rbl_force(fx.numel(), _ptr(fx), _ptr(fy), _ptr(fz), _ptr(mean),
                                  _stream(stream)), "rbx_fix_rbl_force")


def pair_force_verlet(box, cut_off, alpha, qqr2e, typ, sigma, eps, start, end, nbrs, q, x, y, z,
                      fx, fy, fz, flat_virial, evdwl, ecoul, stream=None):
    check(lib().rbx_pair_force_verlet(C.byref(box), cut_off, q.numel(), alpha, qqr2e, _ptr(typ),
                                      _ptr(sigma), _ptr(eps), _ptr(start), _ptr(end), _ptr(nbrs),
                                      _ptr(q), _ptr(x), _ptr(y), _ptr(z), _ptr(fx), _ptr(fy),
                                      _ptr(fz), _ptr(flat_virial), _ptr(evdwl), _ptr(ecoul),
                                      _stream(stream)), "rbx_pair_force_verlet")


# FP32 twins (the reference's default float build): float tensors and scalars,
# same argument order as the FP64 wrappers above.
def rbe_structure_factor_f32(box, q, mx, my, mz, x, y, z, re, im, stream=None):
    check(lib().rbx_rbe_structure_factor_f32(C.byref(box), q.numel(), mx.numel(), _ptr(q),
                                             _ptr(mx), _ptr(my), _ptr(mz), _ptr(x), _ptr(y),
                                             _ptr(z), _ptr(re), _ptr(im), _stream(stream)),
          "rbx_rbe_structure_factor_f32")


def rbe_force_f32(box, alpha, S, qqr2e, re, im, q, mx, my, mz, x, y, z, fx, fy, fz, stream=None):
    check(lib().rbx_rbe_force_f32(C.byref(box), q.numel(), mx.numel(), alpha, S, qqr2e,
                                  _ptr(re), _ptr(im), _ptr(q), _ptr(mx), _ptr(my), _ptr(mz),
                                  _ptr(x), _ptr(y), _ptr(z), _ptr(fx), _ptr(fy), _ptr(fz),
                                  _stream(stream)), "rbx_rbe_force_f32")


def rbe_energy_virial_f32(box, alpha, S, qqr2e, qsq, qsum, re, im, mx, my, mz, virial, energy,
                          stream=None):
    check(lib().rbx_rbe_energy_virial_f32(C.byref(box), mx.numel(), alpha, S, qqr2e, qsq, qsum,
                                          _ptr(re), _ptr(im), _ptr(mx), _ptr(my), _ptr(mz),
                                          _ptr(virial), _ptr(energy), _stream(stream)),
          "rbx_rbe_energy_virial_f32")


def rbl_filter_f32(core2, force2, gid, x, y, z, cstart, cend, cand, core_cap, core_start,
                   core_end, core, shell_cap, shell, shell_num, required, box, realloc, freq,
                   epoch, stream=None):
    check(lib().rbx_rbl_filter_f32(core2, force2, gid.numel(), _ptr(gid), _ptr(x), _ptr(y),
                                   _ptr(z), _ptr(cstart), _ptr(cend), _ptr(cand), _ptr(core_cap),
                                   _ptr(core_start), _ptr(core_end), _ptr(core), shell_cap,
                                   _ptr(shell), _ptr(shell_num), _ptr(required), C.byref(box),
                                   _ptr(realloc), freq, epoch, _stream(stream)),
          "rbx_rbl_filter_f32")


def pair_force_rbl_f32(box, rs, rc, sample_num, pice, alpha, qqr2e, typ, sigma, eps, start, end,
                       core, shell, shell_num, q, x, y, z, fx, fy, fz, stream=None):
    check(lib().rbx_pair_force_rbl_f32(C.byref(box), rs, rc, q.numel(), sample_num, pice, alpha,
                                       qqr2e, _ptr(typ), _ptr(sigma), _ptr(eps), _ptr(start),
                                       _ptr(end), _ptr(core), _ptr(shell), _ptr(shell_num),
                                       _ptr(q), _ptr(x), _ptr(y), _ptr(z), _ptr(fx), _ptr(fy),
                                       _ptr(fz), _stream(stream)), "rbx_pair_force_rbl_f32")


def fix_rbl_force_f32(fx, fy, fz, mean=None, stream=None):
    check(lib().rbx_fix_rbl_force_f32(fx.numel(), _ptr(fx), _ptr(fy), _ptr(fz), _ptr(mean),
                                      _stream(stream)), "rbx_fix_rbl_force_f32")


def pair_force_verlet_f32(box, cut_off, alpha, qqr2e, typ, sigma, eps, start, end, nbrs, q, x, y,
                          z, fx, fy, fz, flat_virial, evdwl, ecoul, stream=None):
    check(lib().rbx_pair_force_verlet_f32(C.byref(box), cut_off, q.numel(), alpha, qqr2e,
                                          _ptr(typ), _ptr(sigma), _ptr(eps), _ptr(start),
                                          _ptr(end), _ptr(nbrs), _ptr(q), _ptr(x), _ptr(y),
                                          _ptr(z), _ptr(fx), _ptr(fy), _ptr(fz),
                                          _ptr(flat_virial), _ptr(evdwl), _ptr(ecoul),
                                          _stream(stream)), "rbx_pair_force_verlet_f32")


# ---------------------------------------------------------------------------
# engine
# ---------------------------------------------------------------------------
class Engine:
    """LJCutCoulKspace force plugin + NVE velocity-Verlet step on one GPU."""

    def __init__(self, sys: dict, *, precision=PLAIN_FP64, neighbor="RBL", coulomb="RBE",
                 seed=12345, device=0, json_text: str | None = None):
        L = lib()
        self.n = int(sys["n"])
        self.box = Box.make(sys["lo"], sys["hi"])
        self._sigma = np.ascontiguousarray(sys["sigma"], dtype=np.float64)
        self._eps = np.ascontiguousarray(sys["eps"], dtype=np.float64)
        self._mass = np.ascontiguousarray(sys["mass"], dtype=np.float64)
        q = np.ascontiguousarray(sys["q"], dtype=np.float64)
        if json_text is not None:
            h = L.rbx_engine_create_json(json_text.encode(), C.byref(self.box), self.n,
                                         len(self._sigma), _np_ptr(self._sigma),
                                         _np_ptr(self._eps), _np_ptr(self._mass), _np_ptr(q),
                                         precision, device)
        else:
            p = sys["params"]
            prm = Params()
            prm.neighbor_type = {"RBL": NEIGHBOR_RBL, "VERLET": NEIGHBOR_VERLET,
                                 "VERLET-SOG": NEIGHBOR_VERLET_SOG}[neighbor]
            prm.cut_off = p["cut_off"]
            prm.r_core = p["r_core"]
            prm.skin = p["skin"]
            prm.neighbor_sample_num = p["neighbor_sample_num"]
            prm.coulomb_type = {"RBE": COULOMB_RBE, "NONE": COULOMB_NONE,
                                "RBSOG": COULOMB_RBSOG}[coulomb]
            prm.rbsog_level = int(p.get("rbsog_level", 2))
            prm.rbsog_S = float(p.get("rbsog_S", 0.0))
            prm.alpha = p["alpha"]
            prm.coulomb_sample_num = p["kspace_p"]
            prm.random_seed = seed
            prm.qqr2e = p["qqr2e"]
            prm.dt = p["dt"]
            prm.precision = precision
            prm.ntypes = len(self._sigma)
            prm.sigma = self._sigma.ctypes.data_as(C.POINTER(C.c_double))
            prm.eps = self._eps.ctypes.data_as(C.POINTER(C.c_double))
            prm.mass = self._mass.ctypes.data_as(C.POINTER(C.c_double))
            prm.fmt2v = float(p.get("fmt2v", 0.0))
            h = L.rbx_engine_create(C.byref(prm), C.byref(self.box), self.n, device)
        if not h:
            raise RbxError(f"rbx_engine_create failed: {last_error()}")
        self._h = C.c_void_p(h)
        pos = np.ascontiguousarray(sys["pos"], dtype=np.float64)
        vel = np.ascontiguousarray(sys["vel"], dtype=np.float64)
        cols = [np.ascontiguousarray(pos[:, d]) for d in range(3)] + \
               [np.ascontiguousarray(vel[:, d]) for d in range(3)]
        gid = np.ascontiguousarray(sys["gid"], dtype=np.int32)
        typ = np.ascontiguousarray(sys["type"], dtype=np.int32)
        self._gid, self._typ, self._q = gid, typ, q
        check(L.rbx_engine_set_state(self._h, _np_ptr(gid), _np_ptr(typ), _np_ptr(q),
                                     *[_np_ptr(c) for c in cols]), "rbx_engine_set_state")

    @classmethod
    def from_files(cls, json_path, *, precision=PLAIN_FP64, device=0):
        """rbx_engine_create_from_files: RBMD's JSON config and the LAMMPS data
        file it names (replicate, GAUSS velocities, image flags), host order =
        file order."""
        L = lib()
        h = L.rbx_engine_create_from_files(os.fsencode(json_path), precision, device)
        if not h:
            raise RbxError(f"rbx_engine_create_from_files failed: {last_error()}")
        self = cls.__new__(cls)
        self._h = C.c_void_p(h)
        n, nt = C.c_int(0), C.c_int(0)
        self.box = Box()
        check(L.rbx_engine_get_system(self._h, C.byref(n), C.byref(nt), C.byref(self.box)),
              "rbx_engine_get_system")
        self.n = n.value
        self._sigma, self._eps, self._mass = (np.zeros(nt.value) for _ in range(3))
        check(L.rbx_engine_get_type_params(self._h, _np_ptr(self._sigma), _np_ptr(self._eps),
                                           _np_ptr(self._mass)), "rbx_engine_get_type_params")
        self._gid, self._typ = np.zeros(self.n, np.int32), np.zeros(self.n, np.int32)
        self._q = np.zeros(self.n)
        check(L.rbx_engine_get_atoms(self._h, _np_ptr(self._gid), _np_ptr(self._typ),
                                     _np_ptr(self._q)), "rbx_engine_get_atoms")
        return self

    @property
    def gid(self):
        return self._gid

    @property
    def types(self):
        return self._typ

    @property
    def charges(self):
        return self._q

    def set_positions(self, pos, vel=None):
        """New positions (host order, [n, 3]); velocities kept unless given."""
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(self.n, 3)
        vel = self.get_state()["vel"] if vel is None else np.asarray(vel, dtype=np.float64)
        cols = [np.ascontiguousarray(pos[:, d]) for d in range(3)] + \
               [np.ascontiguousarray(vel[:, d]) for d in range(3)]
        check(lib().rbx_engine_set_state(self._h, _np_ptr(self._gid), _np_ptr(self._typ),
                                         _np_ptr(self._q), *[_np_ptr(c) for c in cols]),
              "rbx_engine_set_state")

    def set_k_samples(self, mx, my, mz):
        if mx is None:
            check(lib().rbx_engine_set_k_samples(self._h, 0, None, None, None), "set_k_samples")
            return
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (mx, my, mz)]
        self._kkeep = a
        check(lib().rbx_engine_set_k_samples(self._h, len(a[0]), *[_np_ptr(v) for v in a]),
              "rbx_engine_set_k_samples")

    def compute_forces(self, epoch=0):
        check(lib().rbx_engine_compute_forces(self._h, epoch), "rbx_engine_compute_forces")

    def step(self, nsteps=1):
        check(lib().rbx_engine_step(self._h, nsteps), "rbx_engine_step")

    def step_host(self, x_in, v_in, x_out, v_out, f_out):
        """One step from host buffers laid out as [3, n] (x, y, z rows)."""
        check(lib().rbx_engine_step_host(self._h, _np_ptr(x_in), _np_ptr(v_in), _np_ptr(x_out),
                                         _np_ptr(v_out), _np_ptr(f_out)), "rbx_engine_step_host")

    def get_state(self):
        a = [np.zeros(self.n) for _ in range(9)]
        check(lib().rbx_engine_get_state(self._h, *[_np_ptr(v) for v in a]), "get_state")
        return {"pos": np.stack(a[0:3], 1), "vel": np.stack(a[3:6], 1),
                "force": np.stack(a[6:9], 1)}

    def force_parts(self):
        fp = np.zeros((self.n, 3))
        fk = np.zeros((self.n, 3))
        check(lib().rbx_engine_get_force_parts(self._h, _np_ptr(fp), _np_ptr(fk)), "force_parts")
        return fp, fk

    def pair_energy(self):
        """(E_LJ, E_coul, virial[6]) over every pair within cut_off, totals."""
        ev, ec = np.zeros(1), np.zeros(1)
        vir = np.zeros(6)
        check(lib().rbx_engine_pair_energy(self._h, _np_ptr(ev), _np_ptr(ec), _np_ptr(vir)),
              "rbx_engine_pair_energy")
        return ev[0], ec[0], vir

    def kspace_energy_exact(self, kmax):
        """Exact Ewald reciprocal energy over kmax plus the self energy."""
        km = (C.c_int * 3)(*[int(k) for k in kmax])
        out = C.c_double(0.0)
        check(lib().rbx_engine_kspace_energy_exact(self._h, km, C.byref(out)),
              "rbx_engine_kspace_energy_exact")
        return out.value

    def rbl_pairs(self):
        nc, ns = C.c_int64(0), C.c_int64(0)
        check(lib().rbx_engine_get_rbl_pairs(self._h, None, C.byref(nc), None, C.byref(ns)),
              "rbl_pairs size")
        core = np.zeros((max(nc.value, 1), 2), dtype=np.int32)
        shell = np.zeros((max(ns.value, 1), 2), dtype=np.int32)
        check(lib().rbx_engine_get_rbl_pairs(self._h, _np_ptr(core), C.byref(nc),
                                             _np_ptr(shell), C.byref(ns)), "rbl_pairs")
        return core[:nc.value], shell[:ns.value]

    def stats(self) -> Stats:
        s = Stats()
        check(lib().rbx_engine_get_stats(self._h, C.byref(s)), "get_stats")
        return s

    def rbsog_npt_map(self) -> np.ndarray:
        """RBSOG engines: the NPT gather map of the last evaluation's samples."""
        p = C.c_int()
        check(lib().rbx_engine_rbsog_npt_map(self._h, C.byref(p), None), "rbsog_npt_map")
        out = np.zeros(p.value, dtype=np.int32)
        check(lib().rbx_engine_rbsog_npt_map(self._h, C.byref(p), _np_ptr(out)), "rbsog_npt_map")
        return out

    @property
    def stream(self) -> int:
        return int(lib().rbx_engine_stream(self._h) or 0)

    def set_lj_params(self, sigma, eps):
        self._sigma = np.ascontiguousarray(sigma, dtype=np.float64)
        self._eps = np.ascontiguousarray(eps, dtype=np.float64)
        check(lib().rbx_engine_set_lj_params(self._h, _np_ptr(self._sigma), _np_ptr(self._eps)),
              "rbx_engine_set_lj_params")

    def set_charges(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        check(lib().rbx_engine_set_charges(self._h, _np_ptr(q)), "rbx_engine_set_charges")
        self._q = q

    def set_alpha(self, alpha):
        check(lib().rbx_engine_set_alpha(self._h, float(alpha)), "rbx_engine_set_alpha")

    def autotune(self, force=False):
        """rbx_engine_autotune: launch shapes timed on the current state (cached per size bin)."""
        t = Tuning()
        check(lib().rbx_engine_autotune(self._h, int(bool(force)), C.byref(t)),
              "rbx_engine_autotune")
        return {f: getattr(t, f) for f, _ in Tuning._fields_}

    def set_nose_hoover(self, t_start, t_stop, t_damp, num_steps=0, kb=1.0, mvv2e=1.0,
                        tdof=0.0):
        """NVT with RBMD's Nose-Hoover chain; t_damp <= 0 goes back to NVE."""
        check(lib().rbx_engine_set_nose_hoover(self._h, t_start, t_stop, t_damp, int(num_steps),
                                               kb, mvv2e, tdof), "rbx_engine_set_nose_hoover")

    def set_shake(self, clusters, bond=1.0, angle=109.47):
        """SHAKE / RATTLE clusters [nc, 3] of host atom indices, centre second."""
        cl = np.ascontiguousarray(clusters, dtype=np.int32).reshape(-1, 3)
        self._shake = cl
        check(lib().rbx_engine_set_shake(self._h, len(cl), _np_ptr(cl), float(bond), float(angle)),
              "rbx_engine_set_shake")

    def set_special(self, nspecial, special, weights=(0.0, 0.0, 0.0)):
        """CVFF special-bond rows (rbx_special_build's output) and weights
        (hyper_parameters.extend.special_bonds)."""
        ns = np.ascontiguousarray(nspecial, dtype=np.int32).reshape(self.n, 3)
        sp = np.ascontiguousarray(special, dtype=np.int32).reshape(self.n, -1)
        self._special = (ns, sp)
        check(lib().rbx_engine_set_special(self._h, sp.shape[1], _np_ptr(ns), _np_ptr(sp),
                                           *[float(w) for w in weights]), "rbx_engine_set_special")

    def shake_status(self):
        nc, bad = C.c_int(0), C.c_int(0)
        check(lib().rbx_engine_get_shake(self._h, C.byref(nc), C.byref(bad)), "rbx_engine_get_shake")
        return nc.value, bad.value

    def thermostat(self):
        t = np.zeros(1)
        eta, eta_dot = np.zeros(3), np.zeros(3)
        check(lib().rbx_engine_get_thermostat(self._h, _np_ptr(t), _np_ptr(eta),
                                              _np_ptr(eta_dot)), "rbx_engine_get_thermostat")
        return {"temperature": t[0], "eta": eta, "eta_dot": eta_dot}

    def images(self):
        """Periodic image counters [n, 3] (int32), host atom order."""
        out = np.zeros((self.n, 3), np.int32)
        check(lib().rbx_engine_get_images(self._h, _np_ptr(out)), "rbx_engine_get_images")
        return out

    def set_images(self, image):
        image = np.ascontiguousarray(image, dtype=np.int32).reshape(self.n, 3)
        check(lib().rbx_engine_set_images(self._h, _np_ptr(image)), "rbx_engine_set_images")

    def write_trajectory(self, path, timestep, append=True):
        """One frame of RBMD's rbmd.trj format (LAMMPS custom dump with xu yu zu)."""
        check(lib().rbx_engine_write_trajectory(self._h, os.fsencode(path), int(timestep),
                                                int(bool(append))),
              "rbx_engine_write_trajectory")

    def force_vjp(self, g):
        """dL/d(eps, sigma per type; q per atom; alpha; positions) for g = dL/dF [n, 3]."""
        g = np.ascontiguousarray(g, dtype=np.float64).reshape(self.n, 3)
        nt = len(self._sigma)
        out = {"eps": np.zeros(nt), "sigma": np.zeros(nt), "charge": np.zeros(self.n),
               "alpha": np.zeros(1), "pos": np.zeros((self.n, 3))}
        check(lib().rbx_engine_force_vjp(self._h, _np_ptr(g), _np_ptr(out["eps"]),
                                         _np_ptr(out["sigma"]), _np_ptr(out["charge"]),
                                         _np_ptr(out["alpha"]), _np_ptr(out["pos"])),
              "rbx_engine_force_vjp")
        out["alpha"] = float(out["alpha"][0])
        return out

    def set_step_graph(self, on=True):
        check(lib().rbx_engine_set_step_graph(self._h, int(on)), "set_step_graph")

    def set_profiling(self, on=True):
        check(lib().rbx_engine_set_profiling(self._h, int(on)), "set_profiling")

    def phase_ms(self):
        out = (C.c_float * 4)()
        check(lib().rbx_engine_phase_ms(self._h, out), "phase_ms")
        return list(out)

    def close(self):
        if getattr(self, "_h", None):
            lib().rbx_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Force(Engine):
    """The LJCutCoulKspace plugin behind RBMD's Force interface
    (rbx_force_*): built from the JSON config, Execute + EvaluatePotentialEnergy
    per call, energies as RBMD reports them.  The engine methods act on the
    engine the plugin drives."""

    def __init__(self, sys, json_text, *, precision=PLAIN_FP64, device=0):
        L = lib()
        self.n = int(sys["n"])
        self.box = Box.make(sys["lo"], sys["hi"])
        self._sigma = np.ascontiguousarray(sys["sigma"], dtype=np.float64)
        self._eps = np.ascontiguousarray(sys["eps"], dtype=np.float64)
        self._mass = np.ascontiguousarray(sys["mass"], dtype=np.float64)
        q = np.ascontiguousarray(sys["q"], dtype=np.float64)
        f = L.rbx_force_create_json(json_text.encode(), C.byref(self.box), self.n,
                                    len(self._sigma), _np_ptr(self._sigma), _np_ptr(self._eps),
                                    _np_ptr(self._mass), _np_ptr(q), precision, device)
        if not f:
            raise RbxError(f"rbx_force_create_json failed: {last_error()}")
        self._f = C.c_void_p(f)
        self._h = C.c_void_p(L.rbx_force_engine(self._f))
        pos = np.ascontiguousarray(sys["pos"], dtype=np.float64)
        vel = np.ascontiguousarray(sys["vel"], dtype=np.float64)
        cols = [np.ascontiguousarray(pos[:, d]) for d in range(3)] + \
               [np.ascontiguousarray(vel[:, d]) for d in range(3)]
        gid = np.ascontiguousarray(sys["gid"], dtype=np.int32)
        typ = np.ascontiguousarray(sys["type"], dtype=np.int32)
        self._gid, self._typ, self._q = gid, typ, q
        check(L.rbx_engine_set_state(self._h, _np_ptr(gid), _np_ptr(typ), _np_ptr(q),
                                     *[_np_ptr(c) for c in cols]), "rbx_engine_set_state")

    def execute(self, epoch=0, thermo_step=True):
        check(lib().rbx_force_execute(self._f, epoch, int(bool(thermo_step))), "rbx_force_execute")

    def energies(self):
        """{e_vdwl, e_coul, e_kspace, e_pe} of the last execute."""
        out = (C.c_double * 4)()
        check(lib().rbx_force_energies(self._f, out), "rbx_force_energies")
        return dict(zip(("e_vdwl", "e_coul", "e_kspace", "e_pe"), list(out)))

    def close(self):
        if getattr(self, "_f", None):
            lib().rbx_force_destroy(self._f)  # owns its engine
            self._f = None
            self._h = None


class Batch:
    """Replicas advanced by one CUDA graph launch per MD step (rbx_batch_*).
    Keeps references to its engines, which must stay open."""

    def __init__(self, engines):
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e._h.value for e in self.engines])
        self._h = lib().rbx_batch_create(arr, len(self.engines))
        if not self._h:
            raise RbxError(f"rbx_batch_create failed: {last_error()}")

    def autotune(self):
        """rbx_batch_autotune: tune each replica (one timing per size bin)."""
        check(lib().rbx_batch_autotune(self._h), "rbx_batch_autotune")

    AUTO, PHASED, BRANCHES = 0, 1, 2  # RBX_BATCH_* graph designs

    def step(self, nsteps=1):
        check(lib().rbx_batch_step(self._h, nsteps), "rbx_batch_step")

    def set_mode(self, mode):
        """rbx_batch_set_mode: AUTO, PHASED (one launch per phase over all
        replicas) or BRANCHES (one graph branch per replica)."""
        check(lib().rbx_batch_set_mode(self._h, mode), "rbx_batch_set_mode")

    @property
    def design(self) -> int:
        """rbx_batch_design: PHASED or BRANCHES once captured, else -1."""
        return lib().rbx_batch_design(self._h)

    @property
    def stream(self) -> int:
        return lib().rbx_batch_stream(self._h) or 0

    def close(self):
        if getattr(self, "_h", None):
            lib().rbx_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# LAMMPS data files
# ---------------------------------------------------------------------------
def read_lammps(path, atom_style=None, replicate=None, gauss=None) -> dict:
    """rbx_lammps_read: the data file as 0-based arrays (file order).
    gauss=(temperature, unit, seed) draws velocity_type GAUSS velocities."""
    L = lib()
    rep = (C.c_int * 3)(*replicate) if replicate is not None else None
    h = L.rbx_lammps_read(str(path).encode(), atom_style.encode() if atom_style else None, rep)
    if not h:
        raise RbxError(f"rbx_lammps_read failed: {last_error()}")
    try:
        if gauss is not None:
            check(L.rbx_lammps_gauss_velocities(h, float(gauss[0]), gauss[1].encode(),
                                                int(gauss[2])), "rbx_lammps_gauss_velocities")
        info = LammpsInfo()
        check(L.rbx_lammps_get_info(h, C.byref(info)), "rbx_lammps_get_info")
        n, nt = info.n_atoms, info.n_atom_types
        out = {"n": n, "ntypes": nt, "atom_style": ["atomic", "charge", "full"][info.atom_style],
               "lo": [info.box.lo[d] for d in range(3)], "hi": [info.box.hi[d] for d in range(3)],
               "has_velocities": bool(info.has_velocities), "has_images": bool(info.has_images),
               "id": np.zeros(n, np.int64), "type": np.zeros(n, np.int32),
               "molecule": np.zeros(n, np.int32), "q": np.zeros(n), "pos": None, "vel": None,
               "image": np.zeros((n, 3), np.int32), "mass": np.zeros(nt), "eps": np.zeros(nt),
               "sigma": np.zeros(nt)}
        cols = [np.zeros(n) for _ in range(6)]
        check(L.rbx_lammps_get_atoms(h, _np_ptr(out["id"]), _np_ptr(out["type"]),
                                     _np_ptr(out["molecule"]), _np_ptr(out["q"]),
                                     *[_np_ptr(c) for c in cols], _np_ptr(out["image"])),
              "rbx_lammps_get_atoms")
        out["pos"] = np.stack(cols[:3], 1)
        out["vel"] = np.stack(cols[3:], 1)
        check(L.rbx_lammps_get_types(h, _np_ptr(out["mass"]), _np_ptr(out["eps"]),
                                     _np_ptr(out["sigma"])), "rbx_lammps_get_types")
        for kind, name, cnt, width in ((2, "bonds", info.n_bonds, 2), (3, "angles", info.n_angles, 3),
                                       (4, "dihedrals", info.n_dihedrals, 4),
                                       (5, "impropers", info.n_impropers, 4)):
            t = np.zeros(cnt, np.int32)
            a = np.zeros((cnt, width), np.int64)
            check(L.rbx_lammps_get_topology(h, kind, _np_ptr(t), _np_ptr(a)), name)
            out[name] = (t, a)
        return out
    finally:
        L.rbx_lammps_free(h)


def write_lammps_charge(path, sys: dict):
    """rbx_lammps_write_charge of a system dict (ids written as gid + 1)."""
    n = int(sys["n"])
    box = Box.make(sys["lo"], sys["hi"])
    nt = len(sys["sigma"])
    pos = np.ascontiguousarray(sys["pos"], np.float64)
    vel = np.ascontiguousarray(sys["vel"], np.float64)
    a = [np.ascontiguousarray(sys["mass"], np.float64), np.ascontiguousarray(sys["eps"], np.float64),
         np.ascontiguousarray(sys["sigma"], np.float64),
         np.ascontiguousarray(sys["gid"], np.int64), np.ascontiguousarray(sys["type"], np.int32),
         np.ascontiguousarray(sys["q"], np.float64)] + \
        [np.ascontiguousarray(pos[:, d]) for d in range(3)] + \
        [np.ascontiguousarray(vel[:, d]) for d in range(3)]
    check(lib().rbx_lammps_write_charge(str(path).encode(), C.byref(box), n, nt,
                                        *[_np_ptr(v) for v in a]), "rbx_lammps_write_charge")


def special_build(n, bonds=None, angles=None, dihedrals=None):
    """rbx_special_build: (nspecial [n, 3], special [n, maxspecial]) from
    0-based bonds [nb, 2], angles [na, 3], dihedrals [nd, 4]."""
    L = lib()
    arrs = [np.ascontiguousarray(np.zeros((0, k)) if a is None else a, dtype=np.int64).reshape(-1, k)
            for a, k in ((bonds, 2), (angles, 3), (dihedrals, 4))]
    ms = C.c_int(0)
    args = [int(n)]
    for a in arrs:
        args += [len(a), _np_ptr(a)]
    check(L.rbx_special_build(*args, C.byref(ms), None, None), "rbx_special_build")
    ns = np.zeros((n, 3), np.int32)
    sp = np.zeros((n, max(ms.value, 1)), np.int32)
    check(L.rbx_special_build(*args, C.byref(ms), _np_ptr(ns), _np_ptr(sp)), "rbx_special_build")
    return ns, sp[:, :ms.value]


def rbsog_params(level, cut_off, box):
    """rbx_rbsog_params: the RBSOG set-up of a level at this cut_off and box (host)."""
    info = RbsogInfo()
    coef = np.zeros(128)
    dm = np.zeros(18, np.int32)
    dfb = np.zeros(6)
    check(lib().rbx_rbsog_params(level, cut_off, C.byref(box), C.byref(info), _np_ptr(coef),
                                 _np_ptr(dm), _np_ptr(dfb)), "rbx_rbsog_params")
    return {"mmax": info.mmax, "b": info.b, "sigma": info.sigma, "w0": info.w0, "S": info.S,
            "S_npt": info.S_npt, "self_coeff": info.self_coeff, "S_full": info.S_full,
            "taylor": np.array(info.taylor[:]), "coef": coef[:info.mmax].copy(),
            "direct_m": dm.reshape(6, 3), "direct_fb": dfb}


def rbsog_sample(box, level, cut_off, p, seed, step, mx, my, mz, stream=None):
    check(lib().rbx_rbsog_sample(C.byref(box), level, cut_off, p, seed, step, _ptr(mx), _ptr(my),
                                 _ptr(mz), _stream(stream)), "rbx_rbsog_sample")


def rbsog_force(box, level, cut_off, qqr2e, S, qsqsum, q, mx, my, mz, x, y, z, fx, fy, fz,
                stream=None):
    """RBSOG k-space force (sampled + direct); returns the energy."""
    e = C.c_double()
    check(lib().rbx_rbsog_force(C.byref(box), level, cut_off, qqr2e, S, qsqsum, q.numel(),
                                mx.numel(), _ptr(q), _ptr(mx), _ptr(my), _ptr(mz), _ptr(x),
                                _ptr(y), _ptr(z), _ptr(fx), _ptr(fy), _ptr(fz), C.byref(e),
                                _stream(stream)), "rbx_rbsog_force")
    return e.value


def rbsog_npt_chain(box, level, cut_off, mx, my, mz, seed, step, idx, stream=None):
    """The NPT gather map of the samples (device int32 idx, filled in place)."""
    check(lib().rbx_rbsog_npt_chain(C.byref(box), level, cut_off, mx.numel(), _ptr(mx), _ptr(my),
                                    _ptr(mz), seed, step, _ptr(idx), _stream(stream)),
          "rbx_rbsog_npt_chain")


def rbsog_virial(box, level, cut_off, qqr2e, S, S_npt, q, mx, my, mz, idx, x, y, z, stream=None):
    """RBSOG k-space virial [6] (sampled with the gather map idx + direct)."""
    v = np.zeros(6)
    check(lib().rbx_rbsog_virial(C.byref(box), level, cut_off, qqr2e, S, S_npt, q.numel(),
                                 mx.numel(), _ptr(q), _ptr(mx), _ptr(my), _ptr(mz), _ptr(idx),
                                 _ptr(x), _ptr(y), _ptr(z), _np_ptr(v), _stream(stream)),
          "rbx_rbsog_virial")
    return v


def pair_force_verlet_sog(box, level, cut_off, qqr2e, sigma, eps, typ, q, x, y, z, count, rows,
                          fx, fy, fz, flat_virial=None, stream=None):
    """VERLET-SOG pair force over row-major candidate rows [n, cap]; returns (E_LJ, E_coul).
    flat_virial (device, 6 n doubles, optional) receives the per-atom virial."""
    sg = np.ascontiguousarray(sigma, np.float64)
    ep = np.ascontiguousarray(eps, np.float64)
    en = np.zeros(2)
    check(lib().rbx_pair_force_verlet_sog(C.byref(box), level, cut_off, qqr2e, q.numel(), len(sg),
                                          _np_ptr(sg), _np_ptr(ep), _ptr(typ), _ptr(q), _ptr(x),
                                          _ptr(y), _ptr(z), rows.shape[1], _ptr(count), _ptr(rows),
                                          _ptr(fx), _ptr(fy), _ptr(fz), _np_ptr(en),
                                          _ptr(flat_virial), _stream(stream)),
          "rbx_pair_force_verlet_sog")
    return en
