"""RBSOG on the CPU: the library's host set-up against the oracle's, the
reference's S against an independent computation, the samplers (the exact
Philox mixture sampler and the restated Metropolis chain) against the target
density, and the sampled force against the exact far-field sum."""
import math

import numpy as np
import pytest

from rbmd_b200 import systems


def _box(L):
    from oracle import oracle as O

    return O.Box.make([0, 0, 0], [L, L, L * 1.1])


@pytest.mark.parametrize("level", [0, 1, 2, 3, 4])
def test_params_match_oracle(rbx, oracle, level):
    box_o = _box(30.0)
    box_l = rbx.Box.make([0, 0, 0], [30.0, 30.0, 33.0])
    a = rbx.rbsog_params(level, 10.0, box_l)
    b = oracle.rbsog_params(level, 10.0, box_o)
    for key in ("b", "sigma", "w0", "S", "S_npt", "self_coeff"):
        assert abs(a[key] - b[key]) <= 1e-13 * abs(b[key]), key
    assert a["mmax"] == b["mmax"]
    assert np.allclose(a["coef"], b["coef"], rtol=1e-14, atol=0)
    assert np.allclose(a["taylor"], b["taylor"], rtol=1e-13, atol=0)
    assert np.array_equal(a["direct_m"], b["direct_m"])
    assert np.allclose(a["direct_fb"], b["direct_fb"], rtol=1e-14, atol=0)


def test_params_errors(rbx):
    box = rbx.Box.make([0, 0, 0], [30.0] * 3)
    with pytest.raises(rbx.RbxError, match=r"rbsog_level must be in \[0, 4\]"):
        rbx.rbsog_params(5, 10.0, box)


def test_S_is_the_reference_l0_sum(oracle):
    """RBSOGSetup's S: analytic per-axis sums for the l = 0 Gaussian only (the
    loop's stop value carries over to l >= 1), minus the |m|^2 <= 1 terms of
    every Gaussian; recomputed here with numpy.  The full normalisation of the
    sampled density differs, and the ratio is reported by the force test."""
    L = np.array([30.0, 30.0, 33.0])
    p = oracle.rbsog_params(2, 10.0, _box(30.0))
    sl = math.sqrt(2.0) * p["sigma"]
    j = np.arange(1, 400)
    H, Y = [], []
    for d in range(3):
        kd = math.pi * j / L[d]
        e = np.exp(-(kd * sl) ** 2)
        H.append(1 + 2 * e.sum())
        Y.append((2 * e * 4 * kd * kd).sum())
    high = p["coef"][0] * (Y[0] * H[1] * H[2] + H[0] * Y[1] * H[2] + H[0] * H[1] * Y[2])
    low = 0.0
    for m in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
        k2 = sum((2 * math.pi * m[d] / L[d]) ** 2 for d in range(3))
        g = sum(c * math.exp(-(p["b"] ** (2 * l)) * p["sigma"] ** 2 * k2 / 2)
                for l, c in enumerate(p["coef"]))
        low += 2 * g * k2
    assert abs(p["S"] - (high - low)) < 1e-10 * abs(p["S"])


def _density(p, L, mcut):
    ms = np.arange(-mcut, mcut + 1)
    mx, my, mz = np.meshgrid(ms, ms, ms, indexing="ij")
    k2 = sum((2 * math.pi * m / L[d]) ** 2 for d, m in enumerate((mx, my, mz)))
    g = sum(c * np.exp(-(p["b"] ** (2 * l)) * p["sigma"] ** 2 * k2 / 2)
            for l, c in enumerate(p["coef"]))
    w = g * k2
    w[(mx ** 2 + my ** 2 + mz ** 2) <= 1] = 0.0
    return ms, w / w.sum()


@pytest.mark.parametrize("sampler", ["philox", "mh"])
def test_samplers_follow_the_target_density(oracle, sampler):
    """Marginal of m_x and the distribution of |m|^2 against p(m) ~ G^(m)|k|^2
    on |m|^2 > 1 (chi-square, generous for the correlated Metropolis chain)."""
    L = np.array([20.0, 20.0, 22.0])
    box = _box(20.0)
    p = oracle.rbsog_params(2, 5.0, box)
    n = 40000
    if sampler == "philox":
        m = oracle.rbsog_sample_philox(2, 5.0, box, n, 7, 3)
    else:
        m = oracle.rbsog_sample_mh(2, 5.0, box, n, 7)
    m = np.stack(m, 1).astype(int)
    assert ((m ** 2).sum(1) > 1).all()
    ms, w = _density(p, L, 30)
    px = w.sum((1, 2))
    obs = np.array([(m[:, 0] == v).sum() for v in ms])
    keep = px * n > 20
    exp = px[keep] * n
    chi2 = (((obs[keep] - exp) ** 2) / exp).sum()
    dof = keep.sum() - 1
    limit = dof + 6 * math.sqrt(2 * dof) if sampler == "philox" else 4 * dof + 60
    assert chi2 < limit, (chi2, dof)


def test_sampled_force_estimates_the_far_field(oracle):
    """Mean of the sampled k-space force over 200 draws of P = 100 against the
    exact far-field sum: unbiased with the full normalisation S_full; with
    the reference's S the mean is S / S_full times the far field."""
    s = systems.lj_electrolyte(500, seed=3)
    L = float(s["hi"][0])
    from oracle import oracle as O

    box = O.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    q = s["q"]
    p = oracle.rbsog_params(2, 3.0, box)
    far, S_full = oracle.rbsog_far_exact(2, 3.0, box, 1.0, q, x, y, z, 14)
    direct, _ = oracle.rbsog_force(2, 3.0, box, 1.0, q, oracle.rbsog_sample_philox(2, 3.0, box, 1, 1, 0),
                                   x, y, z, S=1e-300)
    acc_full = np.zeros_like(far)
    acc_ref = np.zeros_like(far)
    M = 200
    for t in range(M):
        m = oracle.rbsog_sample_philox(2, 3.0, box, 100, 11, t)
        acc_full += oracle.rbsog_force(2, 3.0, box, 1.0, q, m, x, y, z, S=S_full)[0] - direct
        acc_ref += oracle.rbsog_force(2, 3.0, box, 1.0, q, m, x, y, z)[0] - direct
    assert systems.rel_rms(acc_full / M, far) < 0.15
    ratio = p["S"] / S_full
    assert systems.rel_rms(acc_ref / M, ratio * far) < 0.15
    assert np.allclose(acc_ref, acc_full * ratio, rtol=1e-9, atol=1e-12)


def test_S_full_matches_the_exact_sum(rbx, oracle):
    """The library's S_full (the sampler's mixture total less the |m| = 1
    terms) equals the oracle's direct sum over |m|^2 > 1."""
    s = systems.lj_electrolyte(500, seed=3)
    from oracle import oracle as O

    box = O.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    _, S_full = oracle.rbsog_far_exact(2, 3.0, box, 1.0, s["q"], x, y, z, 14)
    got = rbx.rbsog_params(2, 3.0, rbx.Box.make(s["lo"], s["hi"]))
    assert abs(got["S_full"] - S_full) < 1e-9 * S_full
