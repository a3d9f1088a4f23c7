"""The C-ABI library loads and exports every symbol include/rbx.h declares;
host-only entry points work without a GPU; compute entries fail loudly."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "rbx.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rbx_\w+)\s*\(", text)))


def test_exports_match_header(rbx):
    declared = _declared()
    assert len(declared) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", rbx.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (rbx_\w+)", out))
    missing = [d for d in declared if d not in exported]
    assert not missing, missing
    assert set(rbx.EXPORTS) == set(declared)
    for name in declared:
        getattr(rbx.lib(), name)


def test_host_helpers(rbx, oracle):
    L = (4000 / 0.8) ** (1 / 3)
    b = rbx.Box.make([0, 0, 0], [L] * 3)
    ob = oracle.Box.make([0, 0, 0], [L] * 3)
    assert rbx.rbl_params(4000, b, 2.5, 5.0, 100) == oracle.rbl_params(4000, ob, 2.5, 5.0, 100)[0]
    assert rbx.rbe_gauss_sum(b, 0.16) == oracle.rbe_gauss_sum(ob, 0.16)
    assert rbx.cell_grid(b, 5.3) == [3, 3, 3]
    with pytest.raises(rbx.RbxError):
        rbx.cell_grid(rbx.Box.make([0, 0, 0], [10.0] * 3), 5.3)  # fewer than 3 cells


def test_batch_create_rejects_empty(rbx):
    assert not rbx.lib().rbx_batch_create(None, 0)
    assert "no engines" in rbx.last_error()


def test_compute_without_gpu_fails(rbx):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    b = rbx.Box.make([0, 0, 0], [20.0] * 3)
    rc = rbx.lib().rbx_rbe_sample(C.byref(b), 0.16, 4, 1, 0, None, None, None, None)
    assert rc == 5  # RBX_ERR_DEVICE: no CPU fallback
    assert "no CPU fallback" in rbx.last_error() or "device" in rbx.last_error()
    reuse, d2 = C.c_int(7), C.c_double(0.0)
    rc = rbx.lib().rbx_nlist_should_reuse(C.byref(b), 10, *([None] * 6), 0.3, C.byref(reuse),
                                          C.byref(d2), None)
    assert rc == 5 and reuse.value == 7


JSON_OK = """{
  "init_configuration": {"read_data": {"unit": "LJ", "atom_style": "charge"}},
  "hyper_parameters": {
    "force_field": {"type": "LJ/CUT/COUL/LONG"},
    "neighbor": {"type": "RBL", "cut_off": 5, "r_core": 2.5, "skin": 0.3,
                 "neighbor_sample_num": 100, "energy_rbl_flag": "no"},
    "coulomb": {"type": "RBE", "coulomb_sample_num": 100, "alpha": 0.16,
                "energy_rbe_flag": "no"}},
  "execution": {"timestep": 0.005}
}"""


@pytest.mark.parametrize("mutate,needle", [
    (lambda s: s.replace('"energy_rbl_flag": "no"', '"x": 1'), "energy_rbl_flag"),
    (lambda s: s.replace('"energy_rbe_flag": "no"', '"x": 1'), "energy_rbe_flag"),
    (lambda s: s.replace('"alpha": 0.16', '"alpha": -1'), "alpha override must be > 0"),
    (lambda s: s.replace('"alpha": 0.16', '"x": 1'), "accuracy must be defined"),
    (lambda s: s.replace('"type": "RBE"', '"type": "PPPM"'), "Unsupported coulomb type"),
    (lambda s: s.replace('"neighbor_sample_num": 100', '"neighbor_sample_num": 0'),
     "neighbor_sample_num"),
    (lambda s: s[:-3], "JSON parse error"),
    (lambda s: s.replace('"type": "RBE"', '"type": "RBSOG"'), "RBSOG requires hyper_parameters"),
    (lambda s: s.replace('"type": "RBE"', '"type": "RBSOG", "rbsog_level": 2, "accuracy": 1e-4'),
     "Legacy RBSOG config key 'accuracy'"),
    (lambda s: s.replace('"type": "RBE"', '"type": "RBSOG", "rbsog_level": 7'),
     "rbsog_level must be in [0, 4]"),
    (lambda s: s.replace('"type": "RBL"', '"type": "VERLET-SOG"'), "rbsog_level"),
])
def test_json_config_errors(rbx, mutate, needle):
    """Missing or bad keys fail the way LJCutCoulKspace::Init /
    KSpaceCalculator::Init report them (errors before any device work)."""
    from rbmd_b200 import systems

    s = systems.lj_electrolyte(4000)
    box = rbx.Box.make(s["lo"], s["hi"])
    sig = np.ones(3)
    h = rbx.lib().rbx_engine_create_json(mutate(JSON_OK).encode(), C.byref(box), 4000, 3,
                                         sig.ctypes.data, sig.ctypes.data, sig.ctypes.data,
                                         s["q"].ctypes.data, 0, 0)
    assert not h
    assert needle in rbx.last_error()


def test_json_comments_and_bom(rbx):
    """Config files as RBMD ships them ('//' and block comments, a UTF-8
    byte-order mark) parse; the first error is then the missing key."""
    from rbmd_b200 import systems

    text = "﻿// comment line\n" + JSON_OK.replace(
        '"energy_rbl_flag": "no"', '/* block */ "x": 1 // line\n')
    s = systems.lj_electrolyte(4000)
    box = rbx.Box.make(s["lo"], s["hi"])
    sig = np.ones(3)
    h = rbx.lib().rbx_engine_create_json(text.encode(), C.byref(box), 4000, 3, sig.ctypes.data,
                                         sig.ctypes.data, sig.ctypes.data, s["q"].ctypes.data,
                                         0, 0)
    assert not h
    assert "energy_rbl_flag" in rbx.last_error()


FILES_JSON = """{
  "init_configuration": {"read_data": {"file": "sys.data", "unit": "LJ",
      "atom_style": "charge", "velocity_type": "GAUSS", "replicate": [1, 1, 1]}},
  "hyper_parameters": {
    "force_field": {"type": "LJ/CUT/COUL/LONG"},
    "neighbor": {"type": "RBL", "cut_off": 5, "r_core": 2.5, "skin": 0.3,
                 "neighbor_sample_num": 100, "energy_rbl_flag": "no"},
    "coulomb": {"type": "RBE", "coulomb_sample_num": 100, "alpha": 0.16,
                "energy_rbe_flag": "no"}},
  "execution": {"timestep": 0.005, "temperature": [1.0, 1.0, 1]}
}"""


@pytest.mark.parametrize("mutate, data, needle", [
    (lambda s: s.replace('"sys.data"', '"missing.data"'), None, "missing.data"),
    (lambda s: s.replace('"atom_style": "charge", ', ""), None, "atom_style"),
    (lambda s: s.replace("[1, 1, 1]", "[1, 0, 1]"), None, "must be positive"),
    (lambda s: s.replace("[1, 1, 1]", "[1, 1]"), None, "exactly 3 integers"),
    (lambda s: s.replace('"GAUSS"', '"UNIFORM"'), "novel", "Unsupported velocity_type"),
    (lambda s: s.replace("[1.0, 1.0, 1]", "[0.0, 1.0, 1]"), "novel",
     "temperature[0] > 0"),
    (lambda s: s, "nopair", "Pair Coeffs"),
])
def test_engine_from_files_errors(rbx, tmp_path, mutate, data, needle):
    """rbx_engine_create_from_files reports config and data-file errors as the
    reader does, before any device work."""
    from rbmd_b200 import systems

    s = systems.lj_electrolyte(2000, seed=1)
    rbx.write_lammps_charge(tmp_path / "sys.data", s)
    text = (tmp_path / "sys.data").read_text()
    if data in ("novel", "nopair"):  # drop the Velocities (so GAUSS runs) or Pair Coeffs
        head, _, _ = text.partition("\nVelocities")
        text = head + "\n"
        if data == "nopair":
            a, _, rest = text.partition("\nPair Coeffs")
            text = a + "\n" + rest[rest.index("\nAtoms"):]
        (tmp_path / "sys.data").write_text(text)
    cfg = tmp_path / "rbmd.json"
    cfg.write_text(mutate(FILES_JSON))
    h = rbx.lib().rbx_engine_create_from_files(str(cfg).encode(), 0, 0)
    assert not h
    assert needle in rbx.last_error(), rbx.last_error()


@pytest.mark.parametrize("execution, needle", [
    ('"ensemble": "NPT", ', "ensemble NPT"),
    ('"ensemble": "NVT", "temp_ctrl_type": "BERENDSEN", ', "BERENDSEN"),
])
def test_engine_from_files_ensemble_errors(rbx, tmp_path, execution, needle):
    from rbmd_b200 import systems

    s = systems.lj_electrolyte(2000, seed=1)
    rbx.write_lammps_charge(tmp_path / "sys.data", s)
    cfg = tmp_path / "rbmd.json"
    cfg.write_text(FILES_JSON.replace('"execution": {', '"execution": {' + execution))
    assert not rbx.lib().rbx_engine_create_from_files(str(cfg).encode(), 0, 0)
    assert needle in rbx.last_error(), rbx.last_error()
