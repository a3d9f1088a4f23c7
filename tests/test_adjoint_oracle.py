"""The FP64 adjoint reference (oracle/adjoint.py) against central differences.

L = sum_i g_i . F_i for a fixed random upstream g, so dL/dtheta is the
directional derivative of the force.  F is the oracle's RBL + RBE force with
fixed lists and k-samples (pair force, mean removal, rho(k), RBE force), and
the parameters are those of force-field fitting: eps and sigma per type, the
charge of each type, alpha; positions for a few atoms.  Central differences
with h = 1e-6 (relative) carry O(h^2) error.
"""
import numpy as np
import pytest

from oracle import adjoint as A
from rbmd_b200 import systems


@pytest.fixture(scope="module")
def setup(oracle):
    s = systems.lj_electrolyte(4000, seed=17)
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    L = np.asarray(s["hi"]) - np.asarray(s["lo"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    pos = s["pos"][perm].copy()
    typ = s["type"][perm].astype(np.int32)
    gid = s["gid"][perm]
    cnt, rows = oracle.full_list(box, 5.3, *(np.ascontiguousarray(pos[:, d]) for d in range(3)),
                                 cell, cs, ce)
    freq, _, _ = oracle.rbl_params(s["n"], box, p["r_core"], p["cut_off"], p["neighbor_sample_num"])
    lists = oracle.rbl_filter(box, p["r_core"], p["cut_off"], freq, 3, gid,
                              *(np.ascontiguousarray(pos[:, d]) for d in range(3)), cnt, rows)
    m = oracle.rbe_sample_philox(box, p["alpha"], p["kspace_p"], 9, 3)
    Q = np.array([0.0, 1.0, -1.0])  # charge per type of the electrolyte
    theta = {"eps": np.asarray(s["eps"], float).copy(), "sigma": np.asarray(s["sigma"], float).copy(),
             "Q": Q, "alpha": p["alpha"]}
    g = np.random.default_rng(1).normal(size=(s["n"], 3))
    return s, box, L, pos, typ, lists, freq, m, theta, g


def _force(oracle, setup, theta, pos):
    s, box, L, _, typ, (cc, core, sc, shell), freq, m, _, _ = setup
    p = s["params"]
    q = theta["Q"][typ]
    x, y, z = (np.ascontiguousarray(pos[:, d]) for d in range(3))
    fp = oracle.pair_force_rbl(box, p["r_core"], p["cut_off"], freq, theta["alpha"], p["qqr2e"],
                               typ, theta["sigma"], theta["eps"], q, x, y, z, cc, core, sc, shell)
    fp, _ = oracle.fix_rbl(fp)
    S = oracle.rbe_gauss_sum(box, theta["alpha"])
    re, im = oracle.rbe_structure_factor(box, q, x, y, z, *m)
    fk = oracle.rbe_force(box, S, p["qqr2e"], re, im, q, *m, x, y, z)
    return fp + fk


@pytest.fixture(scope="module")
def adjoint(setup):
    s, box, L, pos, typ, (cc, core, sc, shell), freq, m, theta, g = setup
    p = s["params"]
    lists = A.rbl_pairs(cc, core, sc, shell, freq)
    return A.force_vjp(pos, L, typ, theta["sigma"], theta["eps"], theta["Q"][typ], theta["alpha"],
                       p["qqr2e"], p["r_core"], p["cut_off"], freq, lists, m, g)


def _fd(oracle, setup, theta, pos, g, bump):
    h_up = bump(+1)
    h_dn = bump(-1)
    (t1, p1, h), (t2, p2, _) = h_up, h_dn
    return float((g * (_force(oracle, setup, t1, p1) - _force(oracle, setup, t2, p2))).sum()) / (2 * h)


def _close(a, b, rel=2e-5, floor=1e-7):
    assert abs(a - b) <= rel * max(abs(a), abs(b)) + floor, (a, b)


def test_parameter_gradients(oracle, setup, adjoint):
    s, box, L, pos, typ, lists, freq, m, theta, g = setup
    d_eps, d_sig, d_q, d_alpha, _ = adjoint
    for key, grad in (("eps", d_eps), ("sigma", d_sig)):
        for t in range(len(theta[key])):
            def bump(sgn, key=key, t=t):
                th = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in theta.items()}
                h = 1e-6 * th[key][t]
                th[key][t] += sgn * h
                return th, pos, h
            _close(grad[t], _fd(oracle, setup, theta, pos, g, bump))
    for t in range(3):  # dL/dQ_t = sum of dL/dq_i over atoms of type t
        def bump(sgn, t=t):
            th = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in theta.items()}
            h = 1e-6
            th["Q"][t] += sgn * h
            return th, pos, h
        _close(d_q[typ == t].sum(), _fd(oracle, setup, theta, pos, g, bump))

    def bump_alpha(sgn):
        th = dict(theta)
        h = 1e-6 * theta["alpha"]
        th["alpha"] = theta["alpha"] + sgn * h
        return th, pos, h
    _close(d_alpha, _fd(oracle, setup, theta, pos, g, bump_alpha))


def test_position_gradient(oracle, setup, adjoint):
    s, box, L, pos, typ, lists, freq, m, theta, g = setup
    d_r = adjoint[4]
    charged = np.nonzero(typ != 0)[0][:3]
    neutral = np.nonzero(typ == 0)[0][:3]
    for a in np.concatenate([charged, neutral]):
        for d in range(3):
            def bump(sgn, a=a, d=d):
                p2 = pos.copy()
                h = 1e-6
                p2[a, d] += sgn * h
                return theta, p2, h
            _close(d_r[a, d], _fd(oracle, setup, theta, pos, g, bump), rel=1e-4, floor=1e-6)
