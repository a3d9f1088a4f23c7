"""LAMMPS data files (rbx_lammps_*), on the CPU.

The reader restates RBMD's LammpsFullReader: header counts and box, Masses,
Pair Coeffs, Atoms (atomic / charge / full, optional image flags), Velocities
and the topology sections, ids / types / molecules made 0-based.  Checked by
a write -> read round trip of a synthetic system, against an independent
parser written here on RBMD's own example data files (when the RBMD sources
are present), for replicate, and for the errors it reports.
"""
import os

import numpy as np
import pytest

from rbmd_b200 import systems

# RBMD's example inputs, read when the RBMD sources are present
EXAMPLES = os.path.join(os.environ.get("RBMD_SOURCE", "/root/reference"), "examples")


def _parse(path):
    """Independent restatement: sections by keyword, fields split on whitespace."""
    heads = ("Masses", "Pair Coeffs", "PairIJ Coeffs", "Bond Coeffs", "Angle Coeffs",
             "Dihedral Coeffs", "Improper Coeffs", "Atoms", "Velocities", "Bonds", "Angles",
             "Dihedrals", "Impropers")
    sec, style, rows = None, None, {}
    counts = {}
    with open(path) as fh:
        lines = fh.read().splitlines()[1:]
    for raw in lines:
        t = raw.strip()
        if not t:
            continue
        hit = next((h for h in heads if t.startswith(h)), None)
        if hit:
            sec = hit
            if hit == "Atoms" and "#" in t:
                style = t.split("#", 1)[1].strip()
            rows.setdefault(sec, [])
            continue
        c = t.split("#", 1)[0].split()
        if sec is None:
            if t.endswith("atoms") or t.endswith("atom types"):
                counts[" ".join(c[1:])] = int(c[0])
            continue
        rows[sec].append(c)
    return style, counts, rows


@pytest.mark.parametrize("rel", ["01-peo/peo+Li.data", "02-water-methane/H2O-CH4.data",
                                 "03-metal/Cu/Cu10_v.data"])
def test_reads_rbmd_example_files(rbx, rel):
    path = os.path.join(EXAMPLES, rel)
    if not os.path.exists(path):
        pytest.skip("RBMD example inputs not present")
    got = rbx.read_lammps(path)
    style, counts, rows = _parse(path)
    assert got["atom_style"] == style
    atoms = rows["Atoms"]
    assert got["n"] == counts["atoms"] == len(atoms)
    assert got["ntypes"] == counts["atom types"]
    full = style == "full"
    ids = np.array([int(r[0]) for r in atoms]) - 1
    qcol = {"full": 3, "charge": 2}.get(style)  # charge column
    pcol = {"full": 4, "charge": 3, "atomic": 2}[style]  # first position column
    types = np.array([int(r[2 if full else 1]) for r in atoms]) - 1
    pos = np.array([[float(v) for v in r[pcol:pcol + 3]] for r in atoms])
    assert np.array_equal(got["id"], ids)
    assert np.array_equal(got["type"], types)
    assert np.array_equal(got["pos"], pos)
    if style != "atomic":
        assert np.array_equal(got["q"], np.array([float(r[qcol]) for r in atoms]))
    if full:
        assert np.array_equal(got["molecule"], np.array([int(r[1]) - 1 for r in atoms]))
    if "Velocities" in rows:
        byid = {int(r[0]) - 1: [float(v) for v in r[1:4]] for r in rows["Velocities"]}
        assert np.array_equal(got["vel"], np.array([byid[i] for i in ids]))
    for sec, key, k in (("Bonds", "bonds", 2), ("Angles", "angles", 3),
                        ("Dihedrals", "dihedrals", 4)):
        if sec in rows:
            t, a = got[key]
            assert np.array_equal(t, np.array([int(r[1]) - 1 for r in rows[sec]]))
            assert np.array_equal(a, np.array([[int(v) - 1 for v in r[2:2 + k]]
                                               for r in rows[sec]]))
    if len(atoms[0]) == pcol + 6:  # image flags
        assert np.array_equal(got["image"], np.array([[int(v) for v in r[pcol + 3:]]
                                                      for r in atoms]))
    if "Masses" in rows:
        for r in rows["Masses"]:
            assert got["mass"][int(r[0]) - 1] == float(r[1])


def test_charge_round_trip(rbx, tmp_path):
    s = systems.lj_electrolyte(2000, seed=3)
    path = tmp_path / "sys.data"
    rbx.write_lammps_charge(path, s)
    got = rbx.read_lammps(path)
    assert got["atom_style"] == "charge" and got["n"] == s["n"]
    assert np.array_equal(got["id"], s["gid"])
    assert np.array_equal(got["type"], s["type"])
    assert np.array_equal(got["q"], s["q"])
    assert np.array_equal(got["pos"], s["pos"])
    assert np.array_equal(got["vel"], s["vel"])
    assert np.array_equal(got["lo"], s["lo"]) and np.array_equal(got["hi"], s["hi"])
    for key in ("mass", "eps", "sigma"):
        assert np.array_equal(got[key], np.asarray(s[key], float))


def test_replicate(rbx, tmp_path):
    s = systems.lj_electrolyte(2000, seed=4)
    path = tmp_path / "sys.data"
    rbx.write_lammps_charge(path, s)
    base = rbx.read_lammps(path)
    rep = rbx.read_lammps(path, replicate=(2, 1, 3))
    n = base["n"]
    assert rep["n"] == 6 * n
    L = np.asarray(base["hi"]) - np.asarray(base["lo"])
    assert np.allclose(np.asarray(rep["hi"]) - np.asarray(rep["lo"]), L * [2, 1, 3])
    span = base["id"].max() + 1
    for r, (ix, iy, iz) in enumerate((ix, iy, iz) for iz in range(3) for iy in range(1)
                                     for ix in range(2)):
        blk = slice(r * n, (r + 1) * n)
        assert np.array_equal(rep["id"][blk], base["id"] + r * span)
        want = base["pos"] + L * [ix, iy, iz]
        unwrapped = rep["pos"][blk] + rep["image"][blk] * (L * [2, 1, 3])
        assert np.allclose(unwrapped, want, atol=1e-12)


@pytest.mark.parametrize("text, needle", [
    ("title\n\n2 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n\nAtoms # charge\n\n"
     "1 1 0.0 0.1 0.1 0.1\n", "2 atoms declared, 1 read"),
    ("title\n\n1 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n\nAtoms\n\n"
     "1 1 0.0 0.1 0.1 0.1\n", "atom style"),
    ("title\n\n1 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n0 0 0 xy xz yz\n",
     "triclinic"),
    ("title\n\n1 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n\nAtoms # charge\n\n"
     "1 2 0.0 0.1 0.1 0.1\n", "type out of range"),
])
def test_reader_errors(rbx, tmp_path, text, needle):
    path = tmp_path / "bad.data"
    path.write_text(text)
    with pytest.raises(rbx.RbxError, match=needle):
        rbx.read_lammps(path)
