"""The force plugin (rbx_force_*: LJCutCoulKspace behind RBMD's Force
interface) reports the energies RBMD reports, against the oracle on the
4000-atom LJ electrolyte with injected k-samples:

* pair energies (LJCutCoulEnergyOp over every pair within cut_off) for a
  Verlet list every step and for RBL only with energy_rbl_flag "yes";
* the RBE k-space energy: the sampled energy (ComputeRBEVirial0), or with
  energy_rbe_flag "yes" on a thermo step the exact Ewald energy over kmax
  plus the self energy (kspace_calculator.cpp:630-645, 816-907), and the
  sampled one again on a step that is not a thermo step;
* each divided by the atom count in LJ units, totals in REAL units
  (qqr2e 332.06371), e_pe their sum (lj_cut_coul_kspace.cpp:867-878).

Relative tolerance 1e-10 (FP64), 1e-6 on the sampled k-space energy of the
mixed form relative to its sum before the self term.
"""
import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu

BASE = """{
  "init_configuration": {"read_data": {"unit": "%(unit)s", "atom_style": "charge"}},
  "hyper_parameters": {
    "force_field": {"type": "LJ/CUT/COUL/LONG"},
    "neighbor": {"type": "%(nb)s", "cut_off": 5, "r_core": 2.5, "skin": 0.3,
                 "neighbor_sample_num": 100, "energy_rbl_flag": "%(rbl)s"},
    "coulomb": {"type": "RBE", "coulomb_sample_num": 100, "alpha": 0.16,
                "energy_rbe_flag": "%(rbe)s", "kmax": [5, 5, 5]}},
  "execution": {"timestep": 0.005}
}"""

QQR2E = {"LJ": 1.0, "REAL": 332.06371}


@pytest.fixture(scope="module")
def sys4k():
    return systems.lj_electrolyte(4000, seed=41)


def _oracle(oracle, s, m, qqr2e):
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    q = np.asarray(s["q"])
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    xs, ys, zs = x[perm], y[perm], z[perm]
    cnt, rows = oracle.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
    _, _, ev, ec = oracle.pair_force_verlet(box, 5.0, 0.16, qqr2e, s["type"][perm], s["sigma"],
                                            s["eps"], q[perm], xs, ys, zs, cnt, rows)
    S = oracle.rbe_gauss_sum(box, 0.16)
    re, im = oracle.rbe_structure_factor(box, q, x, y, z, *m)
    ek, _ = oracle.rbe_energy_virial(box, 0.16, S, qqr2e, float((q ** 2).sum()), float(q.sum()),
                                     re, im, *m)
    _, ewald = oracle.ewald_force(box, 0.16, qqr2e, [5, 5, 5], q, x, y, z)
    self_e = qqr2e * np.sqrt(0.16) * float((q ** 2).sum()) / np.sqrt(np.pi)
    return ev, ec, ek, ewald, abs(ek) + self_e


@pytest.mark.parametrize("unit", ["LJ", "REAL"])
@pytest.mark.parametrize("nb,rbl", [("RBL", "yes"), ("RBL", "no"), ("Verlet-List", "yes")])
@pytest.mark.parametrize("rbe", ["no", "yes"])
@pytest.mark.parametrize("precision", [0, 1])
def test_plugin_energies(cuda, rbx, oracle, sys4k, unit, nb, rbl, rbe, precision):
    s = sys4k
    qqr2e = QQR2E[unit]
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbe_sample_philox(box, 0.16, 100, 5, 3)
    ev, ec, ek, ewald, ek_scale = _oracle(oracle, s, m, qqr2e)
    f = rbx.Force(s, BASE % {"unit": unit, "nb": nb, "rbl": rbl, "rbe": rbe},
                  precision=precision)
    f.set_k_samples(*m)
    per = 1.0 / s["n"] if unit == "LJ" else 1.0
    for thermo in (True, False):
        f.execute(epoch=3, thermo_step=thermo)
        got = f.energies()
        if nb == "Verlet-List" or rbl == "yes":
            assert abs(got["e_vdwl"] - ev * per) < 1e-10 * abs(ev * per)
            assert abs(got["e_coul"] - ec * per) < 1e-10 * abs(ec * per)
        else:
            assert got["e_vdwl"] == 0.0 and got["e_coul"] == 0.0
        if rbe == "yes" and thermo:
            assert abs(got["e_kspace"] - ewald * per) < 1e-10 * abs(ewald * per)
        else:
            tol = 1e-10 if precision == 0 else 1e-6
            assert abs(got["e_kspace"] - ek * per) < tol * ek_scale * per
        assert got["e_pe"] == pytest.approx(got["e_vdwl"] + got["e_coul"] + got["e_kspace"],
                                            rel=1e-14, abs=1e-14)
    f.close()


def test_engine_exact_kspace_energy(cuda, rbx, oracle, sys4k):
    """rbx_engine_kspace_energy_exact against the oracle's Ewald energy at two kmax."""
    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    for prec in (0, 1):
        e = rbx.Engine(s, precision=prec)
        for kmax in ([3, 4, 5], [6, 6, 6]):
            _, want = oracle.ewald_force(box, 0.16, 1.0, kmax, s["q"], x, y, z)
            assert abs(e.kspace_energy_exact(kmax) - want) < 1e-10 * abs(want)
        e.close()
