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
