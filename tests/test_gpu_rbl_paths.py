"""Every batch-hash path of the fused RBL kernel on the GPU, in both forms.

The fused filter + pair-force kernel picks its shell-batch test from the
selection frequency (GetRblParams, rbl_full_neighbor_list_builder.cpp:193-228):
freq in {1, 2, 4} reads two bits of a partial SplitMix64 hash, other powers
of two a mask, any other freq a divisibility test by multiplication.  On the
4,000-atom LJ electrolyte (rho* = 0.8, r_core 2.5, cut_off 5: n_c - n_s = 367)
neighbor_sample_num 400 / 200 / 150 / 100 / 90 / 60 / 50 / 40 gives
freq 1 / 2 / 3 / 4 / 5 / 7 / 8 / 10, which reaches all three paths.

For each, the engine's core and shell pairs (by global id) equal the
oracle's FilterRBLNeighborCandidates restatement exactly, at two epochs, and
its total force matches the oracle's RBL + RBE force within 1e-9 (plain FP64)
and 1e-5 (mixed) relative RMS.
"""
import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu

CASES = [(400, 1), (200, 2), (150, 3), (100, 4), (90, 5), (60, 7), (50, 8), (40, 10)]


@pytest.fixture(scope="module")
def base_sys():
    return systems.lj_electrolyte(4000, seed=61)


@pytest.mark.parametrize("sample_num,freq", CASES)
def test_rbl_hash_paths_pairs_and_forces(cuda, rbx, oracle, base_sys, sample_num, freq):
    s = dict(base_sys, params=dict(base_sys["params"], neighbor_sample_num=sample_num))
    box = oracle.Box.make(s["lo"], s["hi"])
    assert oracle.rbl_params(s["n"], box, 2.5, 5.0, sample_num)[0] == freq
    m = oracle.rbe_sample_philox(box, 0.16, 100, 11, 0)
    for epoch in (0, 12345):
        want = oracle.rbl_rbe_evaluation(s, m, epoch=epoch, pair_energy=False)
        assert want["freq"] == freq
        for prec, tol in ((rbx.PLAIN_FP64, 1e-9), (rbx.MIXED, 1e-5)):
            e = rbx.Engine(s, precision=prec)
            e.set_k_samples(*m)
            e.compute_forces(epoch=epoch)
            assert e.stats().selection_frequency == freq
            gc, gs = e.rbl_pairs()
            assert np.array_equal(oracle.pair_keys(gc), want["core_keys"]), (prec, epoch)
            assert np.array_equal(oracle.pair_keys(gs), want["shell_keys"]), (prec, epoch)
            err = systems.rel_rms(e.get_state()["force"], want["force"])
            assert err < tol, (prec, epoch, err)
            e.close()
