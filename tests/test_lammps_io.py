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

# RBMD's example inputs, read when the RBMD sources are present: $RBMD_SOURCE,
# else a "reference" directory beside this repository
_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXAMPLES = os.path.join(os.environ.get("RBMD_SOURCE") or
                        os.path.join(os.path.dirname(_ROOT), "reference"), "examples")


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


class _MT19937_64:
    """std::mt19937_64 as the C++ standard defines it ([rand.predef]: w=64,
    n=312, m=156, r=31, a=0xB5026F5AA96619E9, tempering u=29 d=0x5555...,
    s=17 b=0x71D67FFFEDA60000, t=37 c=0xFFF7EEE000000000, l=43,
    f=6364136223846793005)."""
    M = (1 << 64) - 1

    def __init__(self, seed):
        mt = [seed & self.M]
        for i in range(1, 312):
            mt.append((6364136223846793005 * (mt[-1] ^ (mt[-1] >> 62)) + i) & self.M)
        self.mt, self.i = mt, 312

    def __call__(self):
        mt = self.mt
        if self.i >= 312:
            for k in range(312):
                x = (mt[k] & ~0x7FFFFFFF & self.M) | (mt[(k + 1) % 312] & 0x7FFFFFFF)
                mt[k] = mt[(k + 156) % 312] ^ (x >> 1) ^ (0xB5026F5AA96619E9 if x & 1 else 0)
            self.i = 0
        x = mt[self.i]
        self.i += 1
        x ^= (x >> 29) & 0x5555555555555555
        x ^= (x << 17) & 0x71D67FFFEDA60000
        x ^= (x << 37) & 0xFFF7EEE000000000
        x &= self.M
        return x ^ (x >> 43)


def _normal_triplet(seed):
    """Three std::normal_distribution<double>(0, 1) draws from one fresh
    distribution on std::mt19937_64(seed): libstdc++'s Marsaglia polar method
    (two values per accepted pair, the second kept for the next call) over
    generate_canonical<double, 53>, i.e. double(g()) / 2^64."""
    import math

    g = _MT19937_64(seed)

    def uniform():
        u = float(g()) / 2.0 ** 64
        return u if u < 1.0 else math.nextafter(1.0, 0.0)

    out, saved = [], None
    while len(out) < 3:
        if saved is not None:
            out.append(saved)
            saved = None
            continue
        while True:
            x = 2.0 * uniform() - 1.0
            y = 2.0 * uniform() - 1.0
            r2 = x * x + y * y
            if not (r2 > 1.0 or r2 == 0.0):
                break
        mult = math.sqrt(-2 * math.log(r2) / r2)
        saved = x * mult
        out.append(y * mult)
    return out


def _gauss_reference(ids, types, mass, temperature, kb, mvv2e, seed):
    """velocity_type GAUSS restated (LammpsFullReader::ApplyGaussianVelocitiesIfRequested,
    lammps_full_reader.cpp:710-864 with MixVelocitySeed :134-143)."""
    M = (1 << 64) - 1
    v = np.zeros((len(ids), 3))
    m = np.asarray(mass, float)[types]
    for i, a in enumerate(ids):
        aid = int(a) + 1
        z = (seed + 0x9E3779B97F4A7C15 + (aid << 6) + (aid >> 2)) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        z ^= z >> 31
        f = 1.0 / np.sqrt(m[i])
        v[i] = [r * f for r in _normal_triplet(z)]
    p = [0.0, 0.0, 0.0]
    mt = 0.0
    for i in range(len(ids)):  # sequential sums in atom order, as the reader
        for d in range(3):
            p[d] += m[i] * v[i, d]
        mt += m[i]
    ke = 0.0
    for i in range(len(ids)):
        for d in range(3):
            v[i, d] -= p[d] / mt
        ke += m[i] * (v[i, 0] * v[i, 0] + v[i, 1] * v[i, 1] + v[i, 2] * v[i, 2])
    ke *= mvv2e
    scale = np.sqrt(temperature * (3 * len(ids) - 3) * kb / ke)
    return v * scale


@pytest.mark.parametrize("unit, kb, mvv2e", [
    ("LJ", 1.0, 1.0),
    ("REAL", 1.9872067 * 10.0 ** -3.0, 1.0 / (4.186 * 10.0 ** -4.0)),
])
def test_gauss_velocities_match_restatement(rbx, tmp_path, unit, kb, mvv2e):
    """GAUSS velocities equal a from-the-standard restatement of the
    reader's generator bit for bit; total momentum ~0 and the kinetic
    temperature is the target."""
    s = systems.lj_electrolyte(2000, seed=8)
    path = tmp_path / "sys.data"
    rbx.write_lammps_charge(path, s)
    T, seed = (1.5, 4242) if unit == "LJ" else (298.0, 12345)
    got = rbx.read_lammps(path, replicate=(1, 1, 2), gauss=(T, unit, seed))
    want = _gauss_reference(got["id"], got["type"], got["mass"], T, kb, mvv2e, seed)
    assert np.array_equal(got["vel"], want)
    m = got["mass"][got["type"]]
    assert np.abs((m[:, None] * got["vel"]).sum(0)).max() < 1e-10 * m.sum()
    temp = mvv2e * (m[:, None] * got["vel"] ** 2).sum() / ((3 * got["n"] - 3) * kb)
    assert abs(temp - T) < 1e-12 * T


@pytest.mark.parametrize("args, needle", [
    ((0.0, "LJ", 1), "temperature[0] > 0"),
    ((1.0, "LJ", 0), "positive seed"),
    ((1.0, "SI", 1), "unsupported"),
])
def test_gauss_velocities_errors(rbx, tmp_path, args, needle):
    s = systems.lj_electrolyte(2000, seed=8)
    path = tmp_path / "sys.data"
    rbx.write_lammps_charge(path, s)
    with pytest.raises(rbx.RbxError, match=needle.replace("[", r"\[").replace("]", r"\]")):
        rbx.read_lammps(path, gauss=args)


def _special_reference(n, bonds, angles, dihedrals):
    """LammpsFullReader's special rows restated (lammps_full_reader.cpp:2101-2230)."""
    rows = [[] for _ in range(n)]
    seen = set()
    for band, items, a, b in ((0, bonds, 0, 1), (1, angles, 0, 2), (2, dihedrals, 0, 3)):
        for t in items:
            i, j = int(t[a]), int(t[b])
            if i < 0 or j < 0 or i == j or (min(i, j), max(i, j)) in seen:
                continue
            seen.add((min(i, j), max(i, j)))
            rows[i].append((j, band))
            rows[j].append((i, band))
    return rows


def test_special_build_matches_reader_rule(rbx):
    rng = np.random.default_rng(3)
    n = 300
    bonds = rng.integers(0, n, size=(400, 2))
    angles = rng.integers(0, n, size=(300, 3))
    dih = rng.integers(0, n, size=(200, 4))
    ns, sp = rbx.special_build(n, bonds, angles, dih)
    rows = _special_reference(n, bonds, angles, dih)
    assert sp.shape[1] == max(len(r) for r in rows)
    for i, r in enumerate(rows):
        assert list(sp[i, :len(r)]) == [j for j, _ in r]
        c = [sum(1 for _, b in r if b == k) for k in range(3)]
        assert list(ns[i]) == [c[0], c[0] + c[1], c[0] + c[1] + c[2]]


def test_special_build_water(rbx):
    s = systems.water(50, seed=2)
    ns, sp = rbx.special_build(s["n"], s["bonds"], s["angles"])
    o = np.arange(50) * 3
    assert (sp[o] == np.stack([o + 1, o + 2], 1)).all()
    assert (sp[o + 1] == np.stack([o, o + 2], 1)).all()
    assert (ns[o + 1] == [1, 2, 2]).all()
