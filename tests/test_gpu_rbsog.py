"""RBSOG on the GPU through the C ABI against the oracle: k-samples
bit-exact, k-space force and energy (reference S and full S) within 1e-10,
VERLET-SOG pair force and energies within 1e-10."""
import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu


def _t(torch, a, dtype=None):
    a = np.ascontiguousarray(a)
    if dtype is None:
        dtype = torch.float64 if a.dtype == np.float64 else torch.int32
    return torch.as_tensor(a).to(dtype=dtype, device="cuda").contiguous()


@pytest.fixture(scope="module")
def sys4k():
    return systems.lj_electrolyte(4000, seed=29)


@pytest.mark.parametrize("level, seed, step", [(0, 1, 0), (2, 77, 5), (4, 3, 123456789)])
def test_rbsog_sampler_bit_exact(cuda, rbx, oracle, sys4k, level, seed, step):
    s = sys4k
    p = 300
    want = oracle.rbsog_sample_philox(level, 5.0, oracle.Box.make(s["lo"], s["hi"]), p, seed, step)
    m = [cuda.zeros(p, dtype=cuda.float64, device="cuda") for _ in range(3)]
    rbx.rbsog_sample(rbx.Box.make(s["lo"], s["hi"]), level, 5.0, p, seed, step, *m)
    for a, b in zip(m, want):
        assert np.array_equal(a.cpu().numpy(), b)


@pytest.mark.parametrize("S", [0.0, -1.0])
def test_rbsog_force_matches_oracle(cuda, rbx, oracle, sys4k, S):
    s = sys4k
    box_o = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbsog_sample_philox(2, 5.0, box_o, 200, 9, 1)
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    S_use = S
    if S < 0:
        S_use = rbx.rbsog_params(2, 5.0, rbx.Box.make(s["lo"], s["hi"]))["S_full"]
    want, ew = oracle.rbsog_force(2, 5.0, box_o, 1.0, s["q"], m, x, y, z, S=S_use)
    T = lambda a: _t(cuda, a)  # noqa: E731
    F = [cuda.zeros(s["n"], dtype=cuda.float64, device="cuda") for _ in range(3)]
    e = rbx.rbsog_force(rbx.Box.make(s["lo"], s["hi"]), 2, 5.0, 1.0, S, float((s["q"] ** 2).sum()),
                        T(s["q"]), *[T(v) for v in m], T(x), T(y), T(z), *F)
    got = np.stack([a.cpu().numpy() for a in F], 1)
    assert systems.rel_rms(got, want) < 1e-10
    assert abs(e - ew) < 1e-10 * abs(ew)


def test_verlet_sog_pair_force_matches_oracle(cuda, rbx, oracle, sys4k):
    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    xs, ys, zs = x[perm], y[perm], z[perm]
    cnt, rows = oracle.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
    typ, q = s["type"][perm].astype(np.int32), s["q"][perm]
    want, ew, wv = oracle.pair_force_verlet_sog(2, 5.0, box, 1.0, typ, s["sigma"], s["eps"], q,
                                                xs, ys, zs, cnt, rows, virial=True)
    T = lambda a: _t(cuda, a)  # noqa: E731
    F = [cuda.zeros(s["n"], dtype=cuda.float64, device="cuda") for _ in range(3)]
    vir = cuda.zeros(6 * s["n"], dtype=cuda.float64, device="cuda")
    en = rbx.pair_force_verlet_sog(rbx.Box.make(s["lo"], s["hi"]), 2, 5.0, 1.0, s["sigma"],
                                   s["eps"], T(typ), T(q), T(xs), T(ys), T(zs), T(cnt), T(rows),
                                   *F, flat_virial=vir)
    got = np.stack([a.cpu().numpy() for a in F], 1)
    assert systems.rel_rms(got, want) < 1e-10
    assert np.allclose(en, ew, rtol=1e-10)
    # per-atom virial (ComputeVirial of the pair force), and its total
    gv = vir.cpu().numpy().reshape(6, s["n"])
    assert np.abs(gv - wv).max() < 1e-10 * np.abs(wv).max()
    assert np.abs(gv.sum(1) - wv.sum(1)).max() < 1e-10 * np.abs(wv.sum(1)).max()


def _sog_system(n=4000, seed=29, level=2):
    s = systems.lj_electrolyte(n, seed=seed, rbsog_level=level, kspace_p=112)
    return s


def _oracle_sog_total(oracle, s, m, level):
    """VERLET-SOG pair force + RBSOG k-space force of the oracle (host order)."""
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, p["cut_off"] + p["skin"], x, y, z)
    cnt, rows = oracle.full_list(box, p["cut_off"] + p["skin"], x[perm], y[perm], z[perm], cell,
                                 cs, ce)
    fp, _ = oracle.pair_force_verlet_sog(level, p["cut_off"], box, p["qqr2e"],
                                         s["type"][perm].astype(np.int32), s["sigma"], s["eps"],
                                         s["q"][perm], x[perm], y[perm], z[perm], cnt, rows)
    pair = np.empty_like(fp)
    pair[perm] = fp
    fk, ek = oracle.rbsog_force(level, p["cut_off"], box, p["qqr2e"], s["q"], m, x, y, z)
    return pair, fk, ek


@pytest.mark.parametrize("prec", [0, 1])
def test_engine_rbsog_verlet_sog_forces(cuda, rbx, oracle, prec):
    """The engine with neighbor VERLET-SOG and coulomb RBSOG: pair part,
    k-space part and energy against the oracle on injected samples; then with
    its own device sampler at step 3 against the oracle's Philox sampler."""
    s = _sog_system()
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbsog_sample_philox(2, p["cut_off"], box, 112, 5, 0)
    pair, fk, ek = _oracle_sog_total(oracle, s, m, 2)
    e = rbx.Engine(s, precision=prec, neighbor="VERLET-SOG", coulomb="RBSOG", seed=31)
    e.set_k_samples(*m)
    e.compute_forces(0)
    fp, fkk = e.force_parts()
    tol = 1e-10 if prec == 0 else 1e-5
    assert systems.rel_rms(fp, pair) < tol
    assert systems.rel_rms(fkk, fk) < (1e-10 if prec == 0 else 2e-5)
    assert abs(e.stats().e_kspace - ek) < (1e-10 if prec == 0 else 1e-6) * abs(ek)
    e.set_k_samples(None, None, None)
    e.compute_forces(3)
    m3 = oracle.rbsog_sample_philox(2, p["cut_off"], box, 112, 31, 3)
    _, fk3, _ = _oracle_sog_total(oracle, s, m3, 2)
    assert systems.rel_rms(e.force_parts()[1], fk3) < (1e-10 if prec == 0 else 2e-5)
    e.close()


def test_engine_rbl_with_rbsog_kspace(cuda, rbx, oracle):
    """RBL real space with RBSOG k-space (a combination the reference's
    configuration allows): the k-space part against the oracle."""
    s = _sog_system(seed=31)
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbsog_sample_philox(2, p["cut_off"], box, 112, 5, 0)
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    fk, ek = oracle.rbsog_force(2, p["cut_off"], box, p["qqr2e"], s["q"], m, x, y, z)
    e = rbx.Engine(s, precision=rbx.PLAIN_FP64, coulomb="RBSOG", seed=31)
    e.set_k_samples(*m)
    e.compute_forces(0)
    assert systems.rel_rms(e.force_parts()[1], fk) < 1e-10
    e.close()


def test_engine_rbsog_graph_matches_launches(cuda, rbx):
    s = _sog_system(seed=37)
    runs = []
    for graph in (True, False):
        e = rbx.Engine(s, precision=rbx.MIXED, neighbor="VERLET-SOG", coulomb="RBSOG", seed=9)
        e.set_step_graph(graph)
        e.compute_forces(0)
        e.step(12)
        e.step(13)
        runs.append((e.get_state(), e.stats()))
        e.close()
    (a, sa), (b, sb) = runs
    for key in ("pos", "vel", "force"):
        assert np.array_equal(a[key], b[key]), key
    assert sa.rebuilds == sb.rebuilds
    assert sa.e_kspace == sb.e_kspace


def test_rbsog_npt_chain_and_virial(cuda, rbx, oracle, sys4k):
    """The NPT gather chain on the device equals the oracle's restatement of
    RBSOGSampleKSpace's chain on the same uniforms; the k-space virial
    (sampled with the gather map + direct, kspace_calculator_op.hip.cu:
    1133-1190, 1308-1355) within 1e-10 of the oracle's."""
    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    rbox = rbx.Box.make(s["lo"], s["hi"])
    P, seed, step = 112, 31, 3
    m = oracle.rbsog_sample_philox(2, 5.0, box, P, 5, 0)
    want_idx = oracle.rbsog_idx_npt(2, 5.0, box, m, oracle.rbsog_npt_uniforms(seed, step, P))
    assert 1 < len(np.unique(want_idx)) < P  # the chain both accepts and rejects
    M = [_t(cuda, v) for v in m]
    idx = cuda.zeros(P, dtype=cuda.int32, device="cuda")
    rbx.rbsog_npt_chain(rbox, 2, 5.0, *M, seed, step, idx)
    assert np.array_equal(idx.cpu().numpy(), want_idx)
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    v = rbx.rbsog_virial(rbox, 2, 5.0, 1.0, 0.0, 0.0, _t(cuda, s["q"]), *M, idx, _t(cuda, x),
                         _t(cuda, y), _t(cuda, z))
    want = oracle.rbsog_virial(2, 5.0, box, 1.0, s["q"], m, want_idx, x, y, z)
    assert np.abs(v - want).max() < 1e-10 * np.abs(want).max()


@pytest.mark.parametrize("prec", [0, 1])
def test_engine_rbsog_virial(cuda, rbx, oracle, prec):
    """The engine's k-space virial (rbx_stats.virial_kspace) with injected
    samples: its gather map equals the oracle's chain for the engine's seed
    and epoch, and the virial the oracle's on that map (1e-10 FP64, 1e-6 mixed
    relative to the largest component)."""
    s = _sog_system(seed=43)
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbsog_sample_philox(2, p["cut_off"], box, 112, 7, 0)
    e = rbx.Engine(s, precision=prec, neighbor="VERLET-SOG", coulomb="RBSOG", seed=31)
    e.set_k_samples(*m)
    e.compute_forces(5)
    idx = e.rbsog_npt_map()
    want_idx = oracle.rbsog_idx_npt(2, p["cut_off"], box, m, oracle.rbsog_npt_uniforms(31, 5, 112))
    assert np.array_equal(idx, want_idx)
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    want = oracle.rbsog_virial(2, p["cut_off"], box, p["qqr2e"], s["q"], m, want_idx, x, y, z)
    got = np.asarray(e.stats().virial_kspace[:])
    tol = 1e-10 if prec == 0 else 1e-6
    assert np.abs(got - want).max() < tol * np.abs(want).max()
    e.close()


def test_rbsog_virial_edge_cases(cuda, rbx, oracle, sys4k):
    """One sample (the gather map is [0]) and no atoms (a zero virial)."""
    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    rbox = rbx.Box.make(s["lo"], s["hi"])
    m = oracle.rbsog_sample_philox(2, 5.0, box, 1, 3, 7)
    M = [_t(cuda, v) for v in m]
    idx = cuda.full((1,), 5, dtype=cuda.int32, device="cuda")
    rbx.rbsog_npt_chain(rbox, 2, 5.0, *M, 3, 7, idx)
    assert idx.item() == 0
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    v = rbx.rbsog_virial(rbox, 2, 5.0, 1.0, 0.0, 0.0, _t(cuda, s["q"]), *M, idx, _t(cuda, x),
                         _t(cuda, y), _t(cuda, z))
    want = oracle.rbsog_virial(2, 5.0, box, 1.0, s["q"], m, np.zeros(1, dtype=np.int32), x, y, z)
    assert np.abs(v - want).max() < 1e-10 * np.abs(want).max()
    e = cuda.zeros(0, dtype=cuda.float64, device="cuda")
    assert np.array_equal(rbx.rbsog_virial(rbox, 2, 5.0, 1.0, 0.0, 0.0, e, *M, idx, e, e, e),
                          np.zeros(6))
