"""Parity at the headline size: the 200k-atom LJ electrolyte (rho* = 0.8,
10 % ions, RBL r_core 2.5 / cut_off 5 / skin 0.3 / p = 100, RBE alpha 0.16)
with P = 100 and P = 400 injected k-samples, one force evaluation of each
precision form against the FP64 oracle (same positions, same k-samples, same
batch epoch).

Tolerances (relative RMS over atoms of the 3-vector force; relative for
energies, the k-space energy relative to its sampled sum before the self
term; relative to the largest component for virials): plain FP64 1e-9
for forces, 1e-10 for energies and virials; mixed 1e-5 for forces, 1e-6 for
the k-space energy and virial.  The RBL core and shell pairs equal the
oracle's lists exactly in both forms.
"""
import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu

N = 200000


@pytest.fixture(scope="module")
def sys200k():
    return systems.lj_electrolyte(N, seed=2024)


def _vir_err(got, want):
    got, want = np.asarray(got, float), np.asarray(want, float)
    return float(np.abs(got - want).max() / np.abs(want).max())


@pytest.mark.parametrize("P", [100, 400])
def test_headline_forces_energies_against_oracle(cuda, rbx, oracle, sys200k, P):
    s = dict(sys200k, params=dict(sys200k["params"], kspace_p=P))
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbe_sample_philox(box, 0.16, P, 31, 7)
    epoch = 7
    want = oracle.rbl_rbe_evaluation(s, m, epoch=epoch)
    assert want["freq"] == 4
    for prec, tf, te in ((rbx.PLAIN_FP64, 1e-9, 1e-10), (rbx.MIXED, 1e-5, 1e-6)):
        e = rbx.Engine(s, precision=prec)
        e.set_k_samples(*m)
        e.compute_forces(epoch=epoch)
        fp, fk = e.force_parts()
        assert systems.rel_rms(fp + fk, want["force"]) < tf, prec
        assert systems.rel_rms(fp, want["f_pair"]) < tf, prec
        assert systems.rel_rms(fk, want["f_kspace"]) < tf, prec
        st = e.stats()
        # relative to the sampled sum before the self term, which the energy
        # nearly cancels (about 23x at this size)
        assert abs(st.e_kspace - want["e_kspace"]) < te * want["e_kspace_scale"], prec
        assert _vir_err(st.virial_kspace[:], want["virial_kspace"]) < te, prec
        el, ec, vp = e.pair_energy()  # FP64 in both forms
        assert abs(el - want["e_vdwl"]) < 1e-10 * abs(want["e_vdwl"]), prec
        assert abs(ec - want["e_coul"]) < 1e-10 * abs(want["e_coul"]), prec
        assert _vir_err(vp, want["virial_pair"]) < 1e-10, prec
        gc, gs = e.rbl_pairs()
        assert np.array_equal(oracle.pair_keys(gc), want["core_keys"]), prec
        assert np.array_equal(oracle.pair_keys(gs), want["shell_keys"]), prec
        e.close()
