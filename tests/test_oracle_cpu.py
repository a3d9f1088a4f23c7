"""The FP64 oracle against independent numpy restatements (small systems)."""
import numpy as np
import pytest

from rbmd_b200 import systems


@pytest.fixture(scope="module")
def sys4k():
    return systems.lj_electrolyte(4000, seed=3)


def _min_image(d, L):
    return d - L * np.where(np.abs(d) > 0.5 * L, np.sign(d), 0.0)


def test_cells_sort_stable(oracle, sys4k):
    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    assert sorted(perm.tolist()) == list(range(s["n"]))
    assert np.all(np.diff(cell) >= 0)
    for c in range(len(cs)):
        seg = perm[cs[c]:ce[c]]
        assert np.all(np.diff(seg) > 0)  # stable: old indices ascending inside a cell


def test_full_list_brute_force(oracle, sys4k):
    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    L = s["hi"][0]
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    xs, ys, zs = x[perm], y[perm], z[perm]
    cnt, rows = oracle.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
    pos = np.stack([xs, ys, zs], 1)
    for i in range(0, s["n"], 97):
        d = _min_image(pos[i] - pos, L)
        d2 = d[:, 0] ** 2 + d[:, 1] ** 2 + d[:, 2] ** 2
        want = set(np.nonzero(d2 < 5.3 ** 2)[0].tolist()) - {i}
        assert set(rows[i, :cnt[i]].tolist()) == want


def test_rbl_filter_partition(oracle, sys4k):
    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    xs, ys, zs = x[perm], y[perm], z[perm]
    gid = s["gid"][perm]
    cnt, rows = oracle.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
    cc, core, sc, shell = oracle.rbl_filter(box, 2.5, 5.0, 4, 7, gid, xs, ys, zs, cnt, rows)
    pos = np.stack([xs, ys, zs], 1)
    for i in range(0, s["n"], 131):
        cand = rows[i, :cnt[i]]
        d = _min_image(pos[i] - pos[cand], s["hi"][0])
        d2 = (d[:, 0] ** 2 + d[:, 1] ** 2) + d[:, 2] ** 2
        want_core = set(cand[d2 < 2.5 ** 2 - 1e-4].tolist())
        sel = np.array([oracle.rbl_selected(4, 7, int(gid[i]), int(gid[j])) for j in cand])
        want_shell = set(cand[(d2 >= 2.5 ** 2 - 1e-4) & (d2 < 25 - 1e-4) & sel].tolist())
        assert set(core[i, :cc[i]].tolist()) == want_core
        assert set(shell[i, :sc[i]].tolist()) == want_shell
    # the hash keeps about 1/freq of the shell
    shell_all = 0
    for i in range(s["n"]):
        cand = rows[i, :cnt[i]]
        d = _min_image(pos[i] - pos[cand], s["hi"][0])
        d2 = (d ** 2).sum(1)
        shell_all += int(((d2 >= 6.25 - 1e-4) & (d2 < 25 - 1e-4)).sum())
    assert abs(sc.sum() / shell_all - 0.25) < 0.01


def test_rbe_numpy(oracle, sys4k):
    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    L = s["hi"][0]
    x, y, z = (s["pos"][:, d] for d in range(3))
    m = oracle.rbe_sample_philox(box, 0.16, 50, 5, 3)
    re, im = oracle.rbe_structure_factor(box, s["q"], x, y, z, *m)
    k = 2 * np.pi * np.stack(m, 1) / L
    ph = s["pos"] @ k.T
    assert np.allclose(re, (s["q"][:, None] * np.cos(ph)).sum(0), rtol=1e-10, atol=1e-9)
    assert np.allclose(im, (s["q"][:, None] * np.sin(ph)).sum(0), rtol=1e-10, atol=1e-9)
    S = oracle.rbe_gauss_sum(box, 0.16)
    f = oracle.rbe_force(box, S, 1.0, re, im, s["q"], *m, x, y, z)
    k2 = (k ** 2).sum(1)
    coef = -4 * np.pi / (L ** 3 * k2) * S / 50
    t = np.cos(ph) * im - np.sin(ph) * re
    want = s["q"][:, None] * ((t * coef) @ k)
    assert np.allclose(f, want, rtol=1e-9, atol=1e-10)
    e, vir = oracle.rbe_energy_virial(box, 0.16, S, 1.0, float((s["q"] ** 2).sum()),
                                      float(s["q"].sum()), re, im, *m)
    V = L ** 3
    rho2 = re ** 2 + im ** 2
    e_want = (2 * np.pi * S / (50 * V) * rho2 / k2).sum() - np.sqrt(0.16) * (s["q"] ** 2).sum() / np.sqrt(np.pi)
    assert abs(e - e_want) < 1e-9 * abs(e_want)
    assert np.isclose(vir[0] + vir[1] + vir[2],
                      (2 * np.pi * S / (50 * V) * rho2 / k2 * (3 - 2 * k2 * (1 / (4 * 0.16) + 1 / k2))).sum())


def test_ewald_force_is_energy_gradient(oracle):
    s = systems.lj_electrolyte(300, seed=9, density=0.3)
    box = oracle.Box.make(s["lo"], s["hi"])
    pos = s["pos"].copy()
    f, e0 = oracle.ewald_force(box, 0.16, 1.0, [5, 5, 5], s["q"], *(pos[:, d] for d in range(3)))
    h = 1e-5
    ions = np.nonzero(s["q"])[0][:4]
    for i in ions:
        for d in range(3):
            p1 = pos.copy()
            p1[i, d] += h
            p2 = pos.copy()
            p2[i, d] -= h
            e1 = oracle.ewald_force(box, 0.16, 1.0, [5, 5, 5], s["q"], *(p1[:, c] for c in range(3)))[1]
            e2 = oracle.ewald_force(box, 0.16, 1.0, [5, 5, 5], s["q"], *(p2[:, c] for c in range(3)))[1]
            assert abs(-(e1 - e2) / (2 * h) - f[i, d]) < 1e-5 * max(1.0, abs(f[i, d]))


def test_samplers_distribution(oracle):
    # Philox i.i.d. draws and the restated MH chain both follow
    # P(m) ~ exp(-pi^2 m^2 / (alpha L^2)) along each axis (m = 0 vector excluded).
    L, alpha = 17.09975947, 0.16
    box = oracle.Box.make([0, 0, 0], [L] * 3)
    c = np.pi ** 2 / (alpha * L * L)
    mm = np.arange(-30, 31)
    w = np.exp(-c * mm ** 2)
    w /= w.sum()
    ph = np.concatenate([oracle.rbe_sample_philox(box, alpha, 2000, 1, st)[0] for st in range(20)])
    mh = np.concatenate([oracle.rbe_sample_mh(box, alpha, 2000, 100 + st)[0] for st in range(20)])
    for draws in (ph, mh):
        hist = np.array([(draws == v).sum() for v in mm]) / len(draws)
        var_want = (w * mm ** 2).sum()
        assert abs((draws ** 2).mean() - var_want) < 0.06 * var_want
        assert abs(hist[30] - w[30]) < 0.02


def test_pair_force_newton_and_fix(oracle, sys4k):
    s = sys4k
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    xs, ys, zs = x[perm], y[perm], z[perm]
    cnt, rows = oracle.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
    f, vir, el, ec = oracle.pair_force_verlet(box, 5.0, 0.16, 1.0, s["type"][perm], s["sigma"],
                                              s["eps"], s["q"][perm], xs, ys, zs, cnt, rows)
    # full list evaluated from both sides: momentum is conserved
    assert np.abs(f.sum(0)).max() < 1e-8 * np.abs(f).sum()
    freq = 4
    gid = s["gid"][perm]
    cc, core, sc, shell = oracle.rbl_filter(box, 2.5, 5.0, freq, 0, gid, xs, ys, zs, cnt, rows)
    fr = oracle.pair_force_rbl(box, 2.5, 5.0, freq, 0.16, 1.0, s["type"][perm], s["sigma"],
                               s["eps"], s["q"][perm], xs, ys, zs, cc, core, sc, shell)
    fr2, mean = oracle.fix_rbl(fr)
    assert np.allclose(fr2.mean(0), 0.0, atol=1e-10)
    assert np.allclose(mean, fr.mean(0))
