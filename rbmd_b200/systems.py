"""Seeded synthetic systems standing in for RBMD's benchmark data files.

The reference's LJ-electrolyte data (``benchmark/data/lj_salt.data``) lives in an
external release archive, so the benchmark systems are rebuilt from their
recipe: reduced LJ units (qqr2e = 1), number density 0.8, 90 % neutral LJ
particles and 10 % monovalent ions split +1/-1, epsilon = sigma = mass = 1,
types assigned by seeded shuffle, a simple-cubic lattice with +-0.1 sigma
jitter and Maxwell-Boltzmann velocities at T* = 1 with zero net momentum.

The JSON ``alpha`` of RBMD is g_ewald squared (``SetAlphaFromManual``,
src/force/src/kspace_calculator.cpp:105-118), so "alpha = 0.4/sigma" becomes
``alpha = 0.16``.
"""
from __future__ import annotations

import math

import numpy as np

LJ_ELECTROLYTE_PARAMS = {
    "cut_off": 5.0,          # hyper_parameters.neighbor.cut_off
    "r_core": 2.5,           # hyper_parameters.neighbor.r_core
    "skin": 0.3,             # hyper_parameters.neighbor.skin
    "neighbor_sample_num": 100,
    "alpha": 0.16,           # hyper_parameters.coulomb.alpha (= g_ewald^2)
    "kspace_p": 100,         # hyper_parameters.coulomb.coulomb_sample_num
    "qqr2e": 1.0,            # init_configuration.read_data.unit = "LJ"
    "dt": 0.005,
}


def lj_electrolyte(n: int, seed: int = 2024, density: float = 0.8, ion_fraction: float = 0.1,
                   temperature: float = 1.0, jitter: float = 0.1, **overrides) -> dict:
    """Build an N-atom LJ electrolyte in a cubic periodic box [0, L)^3."""
    rng = np.random.default_rng(seed)
    L = (n / density) ** (1.0 / 3.0)
    side = int(math.ceil(n ** (1.0 / 3.0) - 1e-9))
    while side ** 3 < n:
        side += 1
    spacing = L / side
    sites = rng.choice(side ** 3, size=n, replace=False)
    ix = sites % side
    iy = (sites // side) % side
    iz = sites // (side * side)
    pos = (np.stack([ix, iy, iz], axis=1) + 0.5) * spacing
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    pos = np.mod(pos, L)
    pos[pos >= L] -= L  # np.mod can round up to L

    n_ion = int(round(ion_fraction * n))
    n_cat = n_ion // 2
    n_an = n_ion - n_cat
    typ = np.zeros(n, dtype=np.int32)
    typ[:n_cat] = 1
    typ[n_cat:n_cat + n_an] = 2
    rng.shuffle(typ)
    charge_of_type = np.array([0.0, 1.0, -1.0])
    q = charge_of_type[typ]

    vel = rng.normal(0.0, math.sqrt(temperature), size=(n, 3))
    vel -= vel.mean(axis=0)

    params = dict(LJ_ELECTROLYTE_PARAMS)
    params.update(overrides)
    return {
        "name": f"lj_electrolyte_n{n}",
        "n": n,
        "lo": np.zeros(3),
        "hi": np.full(3, L),
        "pos": np.ascontiguousarray(pos, dtype=np.float64),
        "vel": np.ascontiguousarray(vel, dtype=np.float64),
        "q": np.ascontiguousarray(q, dtype=np.float64),
        "type": typ,
        "gid": np.arange(1, n + 1, dtype=np.int32),
        "sigma": np.ones(3),
        "eps": np.ones(3),
        "mass": np.ones(3),
        "params": params,
    }


def rel_rms(f, ref):
    """Relative 3-D vector RMS (benchmark/common/analyze_force_samples.py definitions):
    sqrt(sum|F - F_ref|^2 / N) / sqrt(sum|F_ref|^2 / N)."""
    f = np.asarray(f, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    num = np.sqrt(np.sum((f - ref) ** 2) / len(ref))
    den = np.sqrt(np.sum(ref ** 2) / len(ref))
    return float(num / den) if den > 0 else float(num)


# Rigid three-site water (SPC/E-like) in REAL units: the water workload of
# RBMD's benchmark (benchmark/systems/water.json: CVFF + RBL + RBE, SHAKE,
# Nose-Hoover at 298 K; its 72,981-atom data file is external), rebuilt from
# the recipe: O-H 1.0 A, H-O-H 109.47 deg (the geometry RBMD's ShakeA holds),
# q_O = -0.8476, q_H = +0.4238, LJ on O only.
WATER_PARAMS = {
    "cut_off": 10.0,
    "r_core": 6.5,
    "skin": 2.0,
    "neighbor_sample_num": 100,
    "alpha": 0.09,           # g_ewald = 0.3 / A
    "kspace_p": 300,
    "qqr2e": 332.06371,      # REAL
    "dt": 2.0,               # fs
    # UnitFactor<REAL> (src/common/unit_factor.cpp:37-42), the same expressions
    "fmt2v": 4.186 * 10.0 ** -4.0,
    "kb": 1.9872067 * 10.0 ** -3.0,
    "mvv2e": 1.0 / (4.186 * 10.0 ** -4.0),
}
WATER_BOND, WATER_ANGLE = 1.0, 109.47


def water(n_mol: int, seed: int = 7, density: float = 0.0334, temperature: float = 298.0,
          jitter: float = 0.15, **overrides) -> dict:
    """n_mol rigid waters (3 n_mol atoms: O, H, H per molecule, types 0 = O,
    1 = H) in a cubic box at `density` molecules / A^3, centres on a jittered
    simple-cubic lattice, random orientations redrawn for any molecule with an
    atom closer than 1.7 A to another molecule's atom (hydrogens carry no LJ
    core, so such a contact would collapse), Maxwell-Boltzmann velocities of
    the rigid bodies' atoms at `temperature` K with zero net momentum.
    Returns the lj_electrolyte-style dict plus 'clusters' (H, O, H atom
    indices per molecule), 'bonds' and 'angles' (0-based atom indices)."""
    rng = np.random.default_rng(seed)
    L = (n_mol / density) ** (1.0 / 3.0)
    side = int(math.ceil(n_mol ** (1.0 / 3.0) - 1e-9))
    while side ** 3 < n_mol:
        side += 1
    spacing = L / side
    sites = rng.choice(side ** 3, size=n_mol, replace=False)
    cen = (np.stack([sites % side, (sites // side) % side, sites // (side * side)], 1) + 0.5)
    cen = cen * spacing + rng.uniform(-jitter, jitter, size=(n_mol, 3))
    half = math.radians(WATER_ANGLE) / 2
    h1 = WATER_BOND * np.array([math.sin(half), math.cos(half), 0.0])
    h2 = WATER_BOND * np.array([-math.sin(half), math.cos(half), 0.0])
    n = 3 * n_mol

    def frames(m):
        # random orthonormal frames from normalised Gaussian quaternions
        qv = rng.normal(size=(m, 4))
        qv /= np.linalg.norm(qv, axis=1, keepdims=True)
        w, a, b, c = qv.T
        return np.stack(
            [np.stack([1 - 2 * (b * b + c * c), 2 * (a * b - c * w), 2 * (a * c + b * w)], 1),
             np.stack([2 * (a * b + c * w), 1 - 2 * (a * a + c * c), 2 * (b * c - a * w)], 1),
             np.stack([2 * (a * c - b * w), 2 * (b * c + a * w), 1 - 2 * (a * a + b * b)], 1)], 1)

    R = frames(n_mol)
    pos = np.empty((n, 3))
    mol = np.repeat(np.arange(n_mol), 3)
    for _ in range(200):
        pos[0::3] = cen
        pos[1::3] = cen + np.einsum("mij,j->mi", R, h1)
        pos[2::3] = cen + np.einsum("mij,j->mi", R, h2)
        pos = np.mod(pos, L)
        pos[pos >= L] -= L
        from scipy.spatial import cKDTree

        pairs = cKDTree(pos, boxsize=L).query_pairs(1.7, output_type="ndarray")
        pairs = pairs[mol[pairs[:, 0]] != mol[pairs[:, 1]]]
        if len(pairs) == 0:
            break
        bad = np.unique(mol[pairs.ravel()])
        R[bad] = frames(len(bad))
    else:
        raise RuntimeError("water: could not place the molecules without close contacts")
    typ = np.tile(np.array([0, 1, 1], dtype=np.int32), n_mol)
    mass = np.array([15.9994, 1.008])
    p = dict(WATER_PARAMS)
    p.update(overrides)
    m = mass[typ]
    vel = rng.normal(size=(n, 3)) * np.sqrt(p["kb"] * temperature / (m * p["mvv2e"]))[:, None]
    vel -= (m[:, None] * vel).sum(0) / m.sum()
    q = np.tile(np.array([-0.8476, 0.4238, 0.4238]), n_mol)
    o = np.arange(n_mol) * 3
    return {
        "name": f"water_m{n_mol}",
        "n": n,
        "lo": np.zeros(3),
        "hi": np.full(3, L),
        "pos": np.ascontiguousarray(pos, dtype=np.float64),
        "vel": np.ascontiguousarray(vel, dtype=np.float64),
        "q": np.ascontiguousarray(q, dtype=np.float64),
        "type": typ,
        "gid": np.arange(n, dtype=np.int32),
        "sigma": np.array([3.166, 0.0]),
        "eps": np.array([0.1553, 0.0]),
        "mass": mass,
        "params": p,
        "clusters": np.ascontiguousarray(np.stack([o + 1, o, o + 2], 1), dtype=np.int32),
        "bonds": np.stack([np.r_[o, o], np.r_[o + 1, o + 2]], 1),
        "angles": np.stack([o + 1, o, o + 2], 1),
    }
