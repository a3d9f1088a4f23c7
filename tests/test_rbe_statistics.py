"""RBE force error against the full FP64 Ewald k-space force, over many samplings.

RBE replaces the Ewald k-space sum by P importance-sampled k-vectors per step,
so its force is a random estimate of the Ewald k-space force.  The error
statistics follow the definitions of RBMD's force-accuracy analysis
(benchmark/common/analyze_force_samples.py:4-5, 171-197), over M samplings
of a fixed configuration:

    mse   = sum_samples sum_atoms |F - F_ref|^2 / (M N)
    bias2 = mean_atoms |mean_samples F - F_ref|^2
    var   = mean_atoms trace(covariance of F over samples)   (divides by M)

so that mse = bias2 + var.  F_ref is the exact Ewald k-space force over the
kmax box (ComputeEwaldForceFlat, kspace_calculator_op.hip.cu:334-403).

The reference draws k-vectors with per-axis Metropolis-Hastings chains
(RBEPSample.h:19-189); this library draws them with Philox4x32-10.  Both
target the same distribution, so both estimators are unbiased and their error
must agree within sampling error.  The CPU test compares the oracle's
restatement of the reference sampler with the Philox sampler; the GPU test runs
the library's own sampler, structure factor and force (plain FP64 ops and the
mixed engine) against the same statistics.
"""
import numpy as np
import pytest

from rbmd_b200 import systems

M = 100          # samplings
KMAX = (10, 10, 10)  # exp(-k^2 / 4 alpha) < 1e-9 beyond m = 10 for the 4,000-atom box (L = 17.1, alpha = 0.16)


def _stats(samples, ref):
    """mse, bias2, var and the relative RMS error of an (M, N, 3) sample stack."""
    f = np.asarray(samples)
    mse = float(((f - ref) ** 2).sum(axis=2).mean())
    mean = f.mean(axis=0)
    bias2 = float(((mean - ref) ** 2).sum(axis=1).mean())
    var = float(((f - mean) ** 2).sum(axis=2).mean())
    ref2 = float((ref ** 2).sum(axis=1).mean())
    return {"mse": mse, "bias2": bias2, "var": var, "rel_rms": np.sqrt(mse / ref2)}


@pytest.fixture(scope="module")
def electrolyte_n4000(oracle):
    s = systems.lj_electrolyte(4000, seed=2024)
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    q = np.ascontiguousarray(s["q"])
    f_ewald, _ = oracle.ewald_force(box, p["alpha"], p["qqr2e"], KMAX, q, x, y, z)
    S = oracle.rbe_gauss_sum(box, p["alpha"])
    return s, box, (x, y, z, q), f_ewald, S


def _oracle_rbe(oracle, box, S, qqr2e, xyzq, m):
    x, y, z, q = xyzq
    re, im = oracle.rbe_structure_factor(box, q, x, y, z, *m)
    return oracle.rbe_force(box, S, qqr2e, re, im, q, *m, x, y, z)


@pytest.fixture(scope="module")
def oracle_stats(oracle, electrolyte_n4000):
    s, box, xyzq, f_ewald, S = electrolyte_n4000
    p = s["params"]
    mh = [_oracle_rbe(oracle, box, S, p["qqr2e"], xyzq,
                      oracle.rbe_sample_mh(box, p["alpha"], p["kspace_p"], 1000 + k))
          for k in range(M)]
    ph = [_oracle_rbe(oracle, box, S, p["qqr2e"], xyzq,
                      oracle.rbe_sample_philox(box, p["alpha"], p["kspace_p"], 77, k))
          for k in range(M)]
    return _stats(mh, f_ewald), _stats(ph, f_ewald)


def test_mse_decomposes_into_bias_and_variance(oracle_stats):
    for st in oracle_stats:
        assert abs(st["mse"] - st["bias2"] - st["var"]) < 1e-9 * st["mse"]


def test_both_samplers_unbiased(oracle_stats):
    # the mean over M samplings has variance var / M per atom; no systematic bias on top
    for st in oracle_stats:
        assert st["bias2"] < 3.0 * st["var"] / M


def test_reference_and_philox_sampler_errors_agree(oracle_stats):
    mh, ph = oracle_stats
    assert 0.0 < mh["rel_rms"] < 1.0
    assert abs(ph["rel_rms"] - mh["rel_rms"]) < 0.1 * mh["rel_rms"]


@pytest.mark.gpu
def test_gpu_rbe_error_matches_reference_statistics(cuda, rbx, oracle, electrolyte_n4000,
                                                    oracle_stats):
    import torch

    s, box, (x, y, z, q), f_ewald, S = electrolyte_n4000
    p = s["params"]
    mh, _ = oracle_stats
    rbox = rbx.Box.make(s["lo"], s["hi"])
    dev = "cuda"
    P = p["kspace_p"]
    X, Y, Z, Q = (torch.tensor(a, device=dev) for a in (x, y, z, q))
    mx, my, mz = (torch.empty(P, dtype=torch.float64, device=dev) for _ in range(3))
    re, im = (torch.empty(P, dtype=torch.float64, device=dev) for _ in range(2))
    fx, fy, fz = (torch.empty(len(x), dtype=torch.float64, device=dev) for _ in range(3))
    S_dev = rbx.rbe_gauss_sum(rbox, p["alpha"])
    assert abs(S_dev - S) < 1e-12 * S
    plain, mixed, samples = [], [], []
    for k in range(M):
        rbx.rbe_sample(rbox, p["alpha"], P, 77, k, mx, my, mz)
        rbx.rbe_structure_factor(rbox, Q, mx, my, mz, X, Y, Z, re, im)
        rbx.rbe_force(rbox, p["alpha"], S_dev, p["qqr2e"], re, im, Q, mx, my, mz, X, Y, Z, fx, fy, fz)
        plain.append(torch.stack([fx, fy, fz], 1).cpu().numpy())
        samples.append(tuple(t.cpu().numpy().copy() for t in (mx, my, mz)))
    eng = rbx.Engine(s, precision=rbx.MIXED)
    for m in samples:  # the mixed engine's k-space force on the same samples
        eng.set_k_samples(*m)
        eng.compute_forces(0)
        _, fk = eng.force_parts()
        mixed.append(fk)
    eng.close()
    for st in (_stats(plain, f_ewald), _stats(mixed, f_ewald)):
        assert st["bias2"] < 3.0 * st["var"] / M
        assert abs(st["rel_rms"] - mh["rel_rms"]) < 0.1 * mh["rel_rms"]
