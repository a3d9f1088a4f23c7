"""rbx_rbe_structure_factor_noalloc: the structure-factor pass for hosts that
cannot let the library allocate device memory (they own a fixed arena or run
under a hard memory cap).  It must give the same structure factors as
rbx_rbe_structure_factor, on consecutive calls that reuse its built-in scratch.

This file is named so that pytest collects it last.
"""
import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=torch.float64)


def _inputs(torch, oracle, n, p, seed):
    s = systems.lj_electrolyte(n, seed=seed)
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbe_sample_philox(box, 0.16, p, seed, 3)
    t = [_dev(torch, a) for a in (s["q"], *m, *(s["pos"][:, d] for d in range(3)))]
    return s, t


def test_noalloc_matches_allocating_entry(cuda, rbx, oracle):
    torch = cuda
    # two calls in a row on different inputs: the shared scratch from the
    # first call must not leak into the second
    for n, p, seed in ((20000, 400, 1), (4000, 100, 2)):
        s, t = _inputs(torch, oracle, n, p, seed)
        box = rbx.Box.make(s["lo"], s["hi"])
        ref = [torch.zeros(p, dtype=torch.float64, device="cuda") for _ in range(2)]
        got = [torch.zeros(p, dtype=torch.float64, device="cuda") for _ in range(2)]
        rbx.rbe_structure_factor(box, *t, *ref)
        rbx.rbe_structure_factor_noalloc(box, *t, *got)
        torch.cuda.synchronize()
        scale = np.sqrt((ref[0].cpu().numpy() ** 2 + ref[1].cpu().numpy() ** 2).mean())
        for a, b in zip(got, ref):
            assert np.abs(a.cpu().numpy() - b.cpu().numpy()).max() < 1e-11 * scale * np.sqrt(n)


def test_noalloc_rejects_oversize(cuda, rbx, oracle):
    torch = cuda
    s, t = _inputs(torch, oracle, 1000, 513, 4)
    box = rbx.Box.make(s["lo"], s["hi"])
    out = [torch.zeros(513, dtype=torch.float64, device="cuda") for _ in range(2)]
    with pytest.raises(rbx.RbxError, match="exceeds the built-in scratch limit"):
        rbx.rbe_structure_factor_noalloc(box, *t, *out)


def test_noalloc_largest_size_then_no_atoms(cuda, rbx, oracle):
    """p_number = 512, the largest size the built-in scratch holds, against the
    allocating entry; then a call with no atoms after it, whose structure
    factors must be exactly zero whatever the previous call left behind."""
    torch = cuda
    s, t = _inputs(torch, oracle, 20000, 512, 5)
    box = rbx.Box.make(s["lo"], s["hi"])
    ref = [torch.zeros(512, dtype=torch.float64, device="cuda") for _ in range(2)]
    got = [torch.zeros(512, dtype=torch.float64, device="cuda") for _ in range(2)]
    rbx.rbe_structure_factor(box, *t, *ref)
    rbx.rbe_structure_factor_noalloc(box, *t, *got)
    torch.cuda.synchronize()
    scale = np.sqrt((ref[0].cpu().numpy() ** 2 + ref[1].cpu().numpy() ** 2).mean())
    for a, b in zip(got, ref):
        assert np.abs(a.cpu().numpy() - b.cpu().numpy()).max() < 1e-11 * scale * np.sqrt(20000)
    empty = [a[:0] for a in t[4:]]
    out = [torch.full((512,), 7.0, dtype=torch.float64, device="cuda") for _ in range(2)]
    rbx.rbe_structure_factor_noalloc(box, t[0][:0], *t[1:4], *empty, *out)
    torch.cuda.synchronize()
    for a in out:
        assert np.array_equal(a.cpu().numpy(), np.zeros(512))
