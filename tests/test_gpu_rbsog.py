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
    want, ew = oracle.pair_force_verlet_sog(2, 5.0, box, 1.0, typ, s["sigma"], s["eps"], q,
                                            xs, ys, zs, cnt, rows)
    T = lambda a: _t(cuda, a)  # noqa: E731
    F = [cuda.zeros(s["n"], dtype=cuda.float64, device="cuda") for _ in range(3)]
    en = rbx.pair_force_verlet_sog(rbx.Box.make(s["lo"], s["hi"]), 2, 5.0, 1.0, s["sigma"],
                                   s["eps"], T(typ), T(q), T(xs), T(ys), T(zs), T(cnt), T(rows),
                                   *F)
    got = np.stack([a.cpu().numpy() for a in F], 1)
    assert systems.rel_rms(got, want) < 1e-10
    assert np.allclose(en, ew, rtol=1e-10)
