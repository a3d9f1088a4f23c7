"""Oracle pins that need no GPU: published known-answer vectors and the
reference's closed-form parameter rules."""
import numpy as np
import pytest


# Philox4x32-10 known-answer vectors published with Random123 (Salmon et al., SC'11).
@pytest.mark.parametrize("ctr,key,out", [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
])
def test_philox_kat(oracle, ctr, key, out):
    assert list(oracle.philox4x32_10(ctr, key)) == out


def test_rbl_params_cfg(oracle):
    # GetRblParams (rbl_full_neighbor_list_builder.cpp:193-228) at rho* = 0.8,
    # r_core 2.5, cut_off 5, p = 100: n_s = 53, n_c = 420, freq = ceil(367/100) = 4
    for n in (4000, 200000):
        L = (n / 0.8) ** (1 / 3)
        box = oracle.Box.make([0, 0, 0], [L] * 3)
        assert oracle.rbl_params(n, box, 2.5, 5.0, 100) == (4, 53, 420)
    box = oracle.Box.make([0, 0, 0], [(4000 / 0.8) ** (1 / 3)] * 3)
    assert oracle.rbl_params(4000, box, 2.5, 5.0, 400)[0] == 1  # shell 367 <= 400


def _mix(v):
    M = (1 << 64) - 1
    v = (v + 0x9e3779b97f4a7c15) & M
    v = ((v ^ (v >> 30)) * 0xbf58476d1ce4e5b9) & M
    v = ((v ^ (v >> 27)) * 0x94d049bb133111eb) & M
    return v ^ (v >> 31)


def test_rbl_hash_matches_restatement(oracle):
    # MixRblSampleKey / RblShellSampleSelected (rbl_full_neighbor_list_op.hip.cu:6-30)
    rng = np.random.default_rng(1)
    for _ in range(200):
        v = int(rng.integers(0, 2**63))
        assert oracle.rbl_mix(v) == _mix(v)
    for _ in range(500):
        e, gi, gj = (int(v) for v in rng.integers(0, 200000, 3))
        f = int(rng.integers(1, 9))
        key = (e ^ _mix(gi) ^ _mix((gj + 0xd1b54a32d192ed03) & ((1 << 64) - 1)))
        want = f <= 1 or _mix(key) % f == 0
        assert oracle.rbl_selected(f, e, gi, gj) == want


def _divtest(d):
    """Host restatement of rbx::make_divtest / divisible (Granlund-Montgomery)."""
    M = (1 << 64) - 1
    k = 0
    dd = d
    while dd % 2 == 0:
        dd //= 2
        k += 1
    inv = dd
    for _ in range(6):
        inv = (inv * (2 - dd * inv)) & M
    limit = M // d

    def divisible(x):
        y = (x * inv) & M
        if k:
            y = ((y >> k) | (y << (64 - k))) & M
        return y <= limit
    return divisible


def test_divisibility_test_exact():
    rng = np.random.default_rng(2)
    for d in [2, 3, 4, 5, 6, 7, 8, 12, 13, 100, 1024, 4097, 65535]:
        f = _divtest(d)
        xs = [int(v) for v in rng.integers(0, 2**63, 300, dtype=np.int64)]
        xs += [d * int(m) for m in rng.integers(0, 2**40, 300)] + [0, d, 2 * d, (2**64 - 1)]
        for x in xs:
            x &= (1 << 64) - 1
            assert f(x) == (x % d == 0), (d, x)


def test_gauss_sum_poisson(oracle):
    # S = prod H_d - 1 equals sum_{m != 0} exp(-k^2 / (4 alpha)) (Poisson summation)
    L, alpha = 17.09975947, 0.16
    box = oracle.Box.make([0, 0, 0], [L] * 3)
    m = np.arange(-60, 61)
    w = np.exp(-(2 * np.pi * m / L) ** 2 / (4 * alpha))
    direct = w.sum() ** 3 - 1.0
    assert abs(oracle.rbe_gauss_sum(box, alpha) - direct) < 1e-9 * direct
