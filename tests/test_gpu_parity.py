"""GPU parity: the sm_100a kernels through the C ABI against the FP64 oracle.

Tolerances: bit-exact for lists, batch selection and k-samples; 1e-12 relative
RMS for plain-FP64 k-space, 1e-10 for plain-FP64 pair forces (the library uses
erfc where the reference kernel writes 1 - erf); 1e-6 relative RMS for the
plain-FP64 engine force; 1e-5 for the mixed engine force.
"""
import numpy as np
import pytest

from rbmd_b200 import systems

pytestmark = pytest.mark.gpu


def _t(torch, a, dtype=None):
    a = np.ascontiguousarray(a)
    if dtype is None:
        dtype = torch.float64 if a.dtype == np.float64 else torch.int32
    return torch.as_tensor(a).to(dtype=dtype, device="cuda").contiguous()


def _subcell_key(x, y, z, lo, hi, dims):
    """In-cell order of rbx_cells_sort: 4x4x4 Morton sub-cell code, then old index."""
    code = np.zeros(len(x), dtype=np.int64)
    for d, v in enumerate((x, y, z)):
        f = (v - lo[d]) * (dims[d] / (hi[d] - lo[d]))
        c = np.clip(np.floor(f), 0, dims[d] - 1)
        sub = np.clip(np.floor((f - c) * 4.0), 0, 3).astype(np.int64)
        for bit in range(2):
            code |= ((sub >> bit) & 1) << (3 * bit + d)
    return (code << 26) | np.arange(len(x))


def _sorted(oracle, s, cutoff):
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, cutoff, x, y, z)
    return box, perm, cell, cs, ce, x[perm], y[perm], z[perm]


@pytest.fixture(scope="module")
def sys4k():
    return systems.lj_electrolyte(4000, seed=21)


@pytest.fixture(scope="module")
def sys20k():
    return systems.lj_electrolyte(20000, seed=22)


# ---------------------------------------------------------------------------
# k-space ops
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("p", [1, 100, 400])
def test_rbe_sample_bit_exact(cuda, rbx, oracle, sys4k, p):
    s = sys4k
    for step in (0, 1, 12345):
        want = oracle.rbe_sample_philox(oracle.Box.make(s["lo"], s["hi"]), 0.16, p, 99, step)
        m = [cuda.zeros(p, dtype=cuda.float64, device="cuda") for _ in range(3)]
        rbx.rbe_sample(rbx.Box.make(s["lo"], s["hi"]), 0.16, p, 99, step, *m)
        cuda.cuda.synchronize()
        for d in range(3):
            assert np.array_equal(m[d].cpu().numpy(), want[d])
        assert not np.any((want[0] == 0) & (want[1] == 0) & (want[2] == 0))


@pytest.mark.parametrize("n,p", [(4000, 100), (4000, 400), (20000, 100), (1, 7), (257, 33)])
def test_rbe_kspace_ops(cuda, rbx, oracle, n, p):
    s = systems.lj_electrolyte(max(n, 2), seed=n + p)
    if n == 1:  # a single ion in a 17-sigma box
        s = systems.lj_electrolyte(4000, seed=n + p)
        s = {k: (v[:1] if isinstance(v, np.ndarray) and len(v) == 4000 else v)
             for k, v in s.items()}
        s["q"] = np.array([1.0])
        s["n"] = 1
    box = oracle.Box.make(s["lo"], s["hi"])
    rbox = rbx.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    m = oracle.rbe_sample_philox(box, 0.16, p, 3, 1)
    re, im = oracle.rbe_structure_factor(box, s["q"], x, y, z, *m)
    S = oracle.rbe_gauss_sum(box, 0.16)
    f = oracle.rbe_force(box, S, 1.0, re, im, s["q"], *m, x, y, z)
    e, vir = oracle.rbe_energy_virial(box, 0.16, S, 1.0, float((s["q"] ** 2).sum()),
                                      float(s["q"].sum()), re, im, *m)
    T = [_t(cuda, a) for a in (s["q"], *m, x, y, z)]
    dre = cuda.zeros(p, dtype=cuda.float64, device="cuda")
    dim = cuda.zeros(p, dtype=cuda.float64, device="cuda")
    rbx.rbe_structure_factor(rbox, T[0], T[1], T[2], T[3], T[4], T[5], T[6], dre, dim)
    F = [cuda.zeros(len(x), dtype=cuda.float64, device="cuda") for _ in range(3)]
    rbx.rbe_force(rbox, 0.16, S, 1.0, dre, dim, T[0], T[1], T[2], T[3], T[4], T[5], T[6], *F)
    dv = cuda.zeros(6, dtype=cuda.float64, device="cuda")
    de = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    rbx.rbe_energy_virial(rbox, 0.16, S, 1.0, float((s["q"] ** 2).sum()), float(s["q"].sum()),
                          dre, dim, T[1], T[2], T[3], dv, de)
    cuda.cuda.synchronize()
    scale = np.sqrt((re ** 2 + im ** 2).mean()) + 1e-30
    assert np.abs(dre.cpu().numpy() - re).max() < 1e-11 * scale * np.sqrt(len(x))
    assert np.abs(dim.cpu().numpy() - im).max() < 1e-11 * scale * np.sqrt(len(x))
    got = np.stack([a.cpu().numpy() for a in F], 1)
    if np.abs(f).max() > 0:
        assert systems.rel_rms(got, f) < 1e-12
    assert abs(de.item() - e) <= 1e-12 * abs(e) + 1e-14
    assert np.allclose(dv.cpu().numpy(), vir, rtol=1e-11, atol=1e-12 * np.abs(vir).max())


def test_ewald_force(cuda, rbx, oracle):
    s = systems.lj_electrolyte(500, seed=5, density=0.5)
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    f, e = oracle.ewald_force(box, 0.16, 1.0, [6, 5, 4], s["q"], x, y, z)
    T = [_t(cuda, a) for a in (s["q"], x, y, z)]
    F = [cuda.zeros(len(x), dtype=cuda.float64, device="cuda") for _ in range(3)]
    de = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    rbx.ewald_force(rbx.Box.make(s["lo"], s["hi"]), [6, 5, 4], 0.16, 1.0, *T, *F, energy=de)
    cuda.cuda.synchronize()
    assert systems.rel_rms(np.stack([a.cpu().numpy() for a in F], 1), f) < 1e-12
    assert abs(de.item() - e) < 1e-11 * abs(e)


# ---------------------------------------------------------------------------
# neighbor ops: bit-exact sets
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", [4000, 20000])
def test_cells_and_full_list(cuda, rbx, oracle, n):
    s = systems.lj_electrolyte(n, seed=n)
    rc = 5.3
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    rbox = rbx.Box.make(s["lo"], s["hi"])
    dims = rbx.cell_grid(rbox, rc)
    ncell = int(np.prod(dims))
    X = [_t(cuda, a) for a in (x, y, z)]
    perm = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    cos = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    cst = cuda.zeros(ncell + 1, dtype=cuda.int32, device="cuda")
    scratch = cuda.zeros(rbx.cells_scratch_bytes(n, ncell), dtype=cuda.uint8, device="cuda")
    rbx.cells_sort(rbox, rc, *X, perm, cos, cst, scratch)
    hp = perm.cpu().numpy()
    assert sorted(hp.tolist()) == list(range(n))
    hc = cos.cpu().numpy()
    assert np.all(np.diff(hc) >= 0)
    hs = cst.cpu().numpy()
    key = _subcell_key(x, y, z, s["lo"], s["hi"], dims)
    for c in range(ncell):
        seg = hp[hs[c]:hs[c + 1]]
        assert np.all(np.diff(key[seg]) > 0)  # (Morton sub-cell, old index) ascending
    xs = [_t(cuda, a[hp]) for a in (x, y, z)]
    cap = 800
    cnt = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    nb = cuda.full((n, cap), -1, dtype=cuda.int32, device="cuda")
    ovf = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    rbx.full_list(rbox, rc, *xs, cst, cap, cnt, nb, ovf)
    cuda.cuda.synchronize()
    assert ovf.item() == 0
    box = oracle.Box.make(s["lo"], s["hi"])
    ocnt, orows = oracle.full_list(box, rc, x[hp], y[hp], z[hp], hc, hs[:-1].copy(),
                                   hs[1:].copy())
    gc, gn = cnt.cpu().numpy(), nb.cpu().numpy()
    assert np.array_equal(gc, ocnt)
    for i in range(n):
        assert set(gn[i, :gc[i]].tolist()) == set(orows[i, :ocnt[i]].tolist())


def test_ops_without_atoms(cuda, rbx):
    """Zero atoms: structure factors are zero, the force, cell sort and list
    ops succeed and write nothing."""
    box = rbx.Box.make([0.0, 0.0, 0.0], [20.0, 21.0, 22.0])
    e = cuda.zeros(0, dtype=cuda.float64, device="cuda")
    m = [cuda.tensor([1.0, -2.0, 0.0], dtype=cuda.float64, device="cuda") for _ in range(3)]
    re = cuda.full((3,), 7.0, dtype=cuda.float64, device="cuda")
    im = cuda.full((3,), 7.0, dtype=cuda.float64, device="cuda")
    rbx.rbe_structure_factor(box, e, *m, e, e, e, re, im)
    rbx.rbe_force(box, 0.16, 1.0, 1.0, re, im, e, *m, e, e, e, e, e, e)
    dims = rbx.cell_grid(box, 5.3)
    ncell = int(np.prod(dims))
    ei = cuda.zeros(0, dtype=cuda.int32, device="cuda")
    cst = cuda.full((ncell + 1,), -1, dtype=cuda.int32, device="cuda")
    scratch = cuda.zeros(max(rbx.cells_scratch_bytes(0, ncell), 1), dtype=cuda.uint8,
                         device="cuda")
    rbx.cells_sort(box, 5.3, e, e, e, ei, ei, cst, scratch)
    ovf = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    rbx.full_list(box, 5.3, e, e, e, cst, 64, ei, ei, ovf)
    cuda.cuda.synchronize()
    assert np.all(re.cpu().numpy() == 0.0) and np.all(im.cpu().numpy() == 0.0)
    assert np.all(cst.cpu().numpy() == 0) and ovf.item() == 0


def test_cells_sort_reports_overfull_cell(cuda, rbx):
    """More atoms in one cell than the in-cell sort holds (2048): the op
    returns the capacity error and still leaves a valid permutation."""
    n = 2100
    rng = np.random.default_rng(3)
    pos = rng.uniform(1.0, 4.0, size=(n, 3))  # all inside cell (0, 0, 0)
    box = rbx.Box.make([0.0, 0.0, 0.0], [18.0, 18.0, 18.0])
    X = [_t(cuda, pos[:, d]) for d in range(3)]
    dims = rbx.cell_grid(box, 5.3)
    ncell = int(np.prod(dims))
    perm = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    cos = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    cst = cuda.zeros(ncell + 1, dtype=cuda.int32, device="cuda")
    scratch = cuda.zeros(rbx.cells_scratch_bytes(n, ncell), dtype=cuda.uint8, device="cuda")
    with pytest.raises(rbx.RbxError, match="2048"):
        rbx.cells_sort(box, 5.3, *X, perm, cos, cst, scratch)
    cuda.cuda.synchronize()
    assert sorted(perm.cpu().numpy().tolist()) == list(range(n))
    hs = cst.cpu().numpy()
    assert hs[0] == 0 and hs[1] == n and hs[-1] == n


def test_full_list_atoms_on_faces(cuda, rbx, oracle):
    """Atoms exactly on the box's lower faces, one ulp below its upper faces
    and on interior cell faces: cell sort and candidate list equal the
    oracle's as sets."""
    s = systems.lj_electrolyte(4000, seed=17)
    lo, hi = np.asarray(s["lo"], float), np.asarray(s["hi"], float)
    rc = 5.3
    dims = np.asarray(rbx.cell_grid(rbx.Box.make(lo, hi), rc))
    edge = (hi - lo) / dims
    pos = s["pos"].copy()
    rng = np.random.default_rng(5)
    idx = rng.choice(s["n"], size=300, replace=False)
    for k, a in enumerate(idx):
        d = k % 3
        if k % 3 == 0:
            pos[a, d] = lo[d]
        elif k % 3 == 1:
            pos[a, d] = np.nextafter(hi[d], -np.inf)
        else:
            pos[a, d] = lo[d] + edge[d] * (1 + k % (dims[d] - 1))
    s2 = dict(s, pos=pos)
    x, y, z = (np.ascontiguousarray(pos[:, d]) for d in range(3))
    rbox = rbx.Box.make(lo, hi)
    n = s["n"]
    ncell = int(np.prod(dims))
    X = [_t(cuda, a) for a in (x, y, z)]
    perm = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    cos = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    cst = cuda.zeros(ncell + 1, dtype=cuda.int32, device="cuda")
    scratch = cuda.zeros(rbx.cells_scratch_bytes(n, ncell), dtype=cuda.uint8, device="cuda")
    rbx.cells_sort(rbox, rc, *X, perm, cos, cst, scratch)
    hp = perm.cpu().numpy()
    xs = [_t(cuda, a[hp]) for a in (x, y, z)]
    cap = 800
    cnt = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    nb = cuda.full((n, cap), -1, dtype=cuda.int32, device="cuda")
    ovf = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    rbx.full_list(rbox, rc, *xs, cst, cap, cnt, nb, ovf)
    cuda.cuda.synchronize()
    box, operm, ocell, ocs, oce, oxs, oys, ozs = _sorted(oracle, s2, rc)
    assert np.array_equal(np.sort(hp), np.arange(n))
    assert np.array_equal(cos.cpu().numpy(), ocell)  # same cell for every sorted slot
    ocnt, orows = oracle.full_list(box, rc, oxs, oys, ozs, ocell, ocs, oce)
    gcnt, grows = cnt.cpu().numpy(), nb.cpu().numpy()
    # compare by original atom index (the in-cell orders may differ)
    want = {int(operm[i]): set(operm[orows[i, :ocnt[i]]].tolist()) for i in range(n)}
    got = {int(hp[i]): set(hp[grows[i, :gcnt[i]]].tolist()) for i in range(n)}
    assert got == want


def test_nlist_should_reuse_matches_oracle(cuda, rbx, oracle, sys4k):
    """Skin test of a cached list (ShouldReuseNeighborList): the largest
    minimum-image displacement, and reuse iff it is at most skin / 2."""
    import torch

    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    rbox = rbx.Box.make(s["lo"], s["hi"])
    L = np.asarray(s["hi"]) - np.asarray(s["lo"])
    rng = np.random.default_rng(3)
    p0 = s["pos"]
    for scale, wrap in ((0.05, False), (0.2, True)):
        p1 = p0 + rng.uniform(-scale, scale, p0.shape)
        if wrap:  # moved across the periodic boundary: the minimum image applies
            p1 = np.asarray(s["lo"]) + np.mod(p1 - np.asarray(s["lo"]), L)
        cols = [np.ascontiguousarray(a[:, d]) for a in (p1, p0) for d in range(3)]
        want = oracle.max_disp2(box, *cols)
        dev = [torch.tensor(c, device="cuda") for c in cols]
        for skin in (0.3, 2.0 * np.sqrt(want) * 0.999):
            reuse, d2 = rbx.nlist_should_reuse(rbox, *dev, skin)
            assert abs(d2 - want) <= 1e-12 * want
            assert reuse == (want <= (0.5 * skin) ** 2)  # thresholds far from the rounding


def test_full_list_overflow_flag(cuda, rbx, sys4k):
    s = sys4k
    n = s["n"]
    rbox = rbx.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    dims = rbx.cell_grid(rbox, 5.3)
    ncell = int(np.prod(dims))
    X = [_t(cuda, a) for a in (x, y, z)]
    perm = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    cos = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    cst = cuda.zeros(ncell + 1, dtype=cuda.int32, device="cuda")
    scratch = cuda.zeros(rbx.cells_scratch_bytes(n, ncell), dtype=cuda.uint8, device="cuda")
    rbx.cells_sort(rbox, 5.3, *X, perm, cos, cst, scratch)
    hp = perm.cpu().numpy()
    xs = [_t(cuda, a[hp]) for a in (x, y, z)]
    cnt = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    nb = cuda.zeros((n, 32), dtype=cuda.int32, device="cuda")
    ovf = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    rbx.full_list(rbox, 5.3, *xs, cst, 32, cnt, nb, ovf)
    cuda.cuda.synchronize()
    assert ovf.item() & 1  # capacity overflow is reported, rows stay in bounds
    assert cnt.cpu().numpy().max() > 32


def _ref_lists(oracle, s, epoch, freq):
    box, perm, cell, cs, ce, xs, ys, zs = _sorted(oracle, s, 5.3)
    cnt, rows = oracle.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
    gid = s["gid"][perm]
    cc, core, sc, shell = oracle.rbl_filter(box, 2.5, 5.0, freq, epoch, gid, xs, ys, zs, cnt,
                                            rows)
    return box, perm, xs, ys, zs, gid, cnt, rows, cc, core, sc, shell


@pytest.mark.parametrize("epoch,freq", [(0, 4), (17, 4), (3, 1), (5, 3)])
def test_rbl_filter_op_bit_exact(cuda, rbx, oracle, sys4k, epoch, freq):
    s = sys4k
    n = s["n"]
    box, perm, xs, ys, zs, gid, cnt, rows, cc, core, sc, shell = _ref_lists(oracle, s, epoch, freq)
    cap = rows.shape[1]
    cstart = np.arange(n, dtype=np.int32) * cap
    cend = cstart + cnt
    ccap = np.full(n, cap, dtype=np.int32)
    T = lambda a: _t(cuda, a)  # noqa: E731
    core_end = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    dcore = cuda.full((n * cap,), -1, dtype=cuda.int32, device="cuda")
    shell_cap = cap
    dshell = cuda.full((shell_cap * n,), -1, dtype=cuda.int32, device="cuda")
    snum = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    req = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    realloc = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    rbx.rbl_filter(2.5 ** 2 - 1e-4, 5.0 ** 2 - 1e-4, T(gid), T(xs), T(ys), T(zs), T(cstart),
                   T(cend), T(rows.reshape(-1)), T(ccap), T(cstart), core_end, dcore, shell_cap,
                   dshell, snum, req, rbx.Box.make(s["lo"], s["hi"]), realloc, freq, epoch)
    cuda.cuda.synchronize()
    assert realloc.item() == 0
    hce = core_end.cpu().numpy() - cstart
    hcore = dcore.cpu().numpy().reshape(n, cap)
    hsn = snum.cpu().numpy()
    hsh = dshell.cpu().numpy().reshape(shell_cap, n)
    assert np.array_equal(hce, cc)
    assert np.array_equal(hsn, sc)
    assert req.item() == sc.max()
    for i in range(n):
        assert hcore[i, :hce[i]].tolist() == core[i, :cc[i]].tolist()  # same order too
        assert hsh[:hsn[i], i].tolist() == shell[i, :sc[i]].tolist()


# ---------------------------------------------------------------------------
# pair-force ops
# ---------------------------------------------------------------------------
def test_pair_force_rbl_op(cuda, rbx, oracle, sys4k):
    s = sys4k
    n = s["n"]
    box, perm, xs, ys, zs, gid, cnt, rows, cc, core, sc, shell = _ref_lists(oracle, s, 2, 4)
    typ, q = s["type"][perm], s["q"][perm]
    want = oracle.pair_force_rbl(box, 2.5, 5.0, 4, 0.16, 1.0, typ, s["sigma"], s["eps"], q, xs,
                                 ys, zs, cc, core, sc, shell)
    cap = core.shape[1]
    start = np.arange(n, dtype=np.int32) * cap
    sh_sm = np.full((cap, n), -1, dtype=np.int32)
    for i in range(n):
        sh_sm[:sc[i], i] = shell[i, :sc[i]]
    T = lambda a: _t(cuda, a)  # noqa: E731
    F = [cuda.zeros(n, dtype=cuda.float64, device="cuda") for _ in range(3)]
    rbx.pair_force_rbl(rbx.Box.make(s["lo"], s["hi"]), 2.5, 5.0, 100, 4, 0.16, 1.0, T(typ),
                       T(s["sigma"]), T(s["eps"]), T(start), T(start + cc), T(core.reshape(-1)),
                       T(sh_sm.reshape(-1)), T(sc), T(q), T(xs), T(ys), T(zs), *F)
    mean = cuda.zeros(3, dtype=cuda.float64, device="cuda")
    got_raw = np.stack([a.cpu().numpy() for a in F], 1)
    assert systems.rel_rms(got_raw, want) < 1e-10
    rbx.fix_rbl_force(*F, mean=mean)
    cuda.cuda.synchronize()
    fixed, omean = oracle.fix_rbl(want)
    assert np.allclose(mean.cpu().numpy(), omean, rtol=1e-9, atol=1e-12)
    assert systems.rel_rms(np.stack([a.cpu().numpy() for a in F], 1), fixed) < 1e-10


def test_pair_force_verlet_op(cuda, rbx, oracle, sys4k):
    s = sys4k
    n = s["n"]
    box, perm, cell, cs, ce, xs, ys, zs = _sorted(oracle, s, 5.3)
    cnt, rows = oracle.full_list(box, 5.3, xs, ys, zs, cell, cs, ce)
    typ, q = s["type"][perm], s["q"][perm]
    f, vir, el, ec = oracle.pair_force_verlet(box, 5.0, 0.16, 1.0, typ, s["sigma"], s["eps"], q,
                                              xs, ys, zs, cnt, rows)
    cap = rows.shape[1]
    start = np.arange(n, dtype=np.int32) * cap
    T = lambda a: _t(cuda, a)  # noqa: E731
    F = [cuda.zeros(n, dtype=cuda.float64, device="cuda") for _ in range(3)]
    fv = cuda.zeros(6 * n, dtype=cuda.float64, device="cuda")
    e1 = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    e2 = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    rbx.pair_force_verlet(rbx.Box.make(s["lo"], s["hi"]), 5.0, 0.16, 1.0, T(typ), T(s["sigma"]),
                          T(s["eps"]), T(start), T(start + cnt), T(rows.reshape(-1)), T(q), T(xs),
                          T(ys), T(zs), *F, fv, e1, e2)
    cuda.cuda.synchronize()
    assert systems.rel_rms(np.stack([a.cpu().numpy() for a in F], 1), f) < 1e-10
    assert abs(e1.item() - el) < 1e-10 * abs(el)
    assert abs(e2.item() - ec) < 1e-10 * abs(ec)
    assert np.allclose(fv.cpu().numpy().reshape(6, n).sum(1), vir, rtol=1e-10)


# ---------------------------------------------------------------------------
# engine (the per-step fused path)
# ---------------------------------------------------------------------------
def _oracle_total(oracle, s, m, epoch):
    import __graft_entry__ as ge

    if epoch == 0:
        return ge._oracle_forces(s, m)
    raise NotImplementedError


@pytest.mark.parametrize("n", [4000, 20000])
def test_engine_forces_fp64_and_mixed(cuda, rbx, oracle, n):
    s = systems.lj_electrolyte(n, seed=100 + n)
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbe_sample_philox(box, 0.16, 100, 7, 0)
    want = _oracle_total(oracle, s, m, 0)
    for prec, tol in ((rbx.PLAIN_FP64, 1e-9), (rbx.MIXED, 1e-5)):
        e = rbx.Engine(s, precision=prec)
        e.set_k_samples(*m)
        e.compute_forces(epoch=0)
        got = e.get_state()["force"]
        err = systems.rel_rms(got, want)
        assert err < tol, (prec, err)
        fp, fk = e.force_parts()
        assert np.abs(fp.mean(0)).max() < 1e-9 * np.abs(fp).mean()  # RBL mean removed
        e.close()


def test_engine_kspace_energy_and_virial(cuda, rbx, oracle, sys20k):
    """The RBE energy and virial the engine reports with each force
    evaluation (KSpaceCalculator's energy and ComputeRBEForceVirial) against
    the oracle on the same configuration and k-samples."""
    s = sys20k
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    m = oracle.rbe_sample_philox(box, p["alpha"], 100, 5, 0)
    S = oracle.rbe_gauss_sum(box, p["alpha"])
    re, im = oracle.rbe_structure_factor(box, s["q"], x, y, z, *m)
    ek, vir = oracle.rbe_energy_virial(box, p["alpha"], S, p["qqr2e"], float((s["q"] ** 2).sum()),
                                       float(s["q"].sum()), re, im, *m)
    for prec, tol in ((rbx.PLAIN_FP64, 1e-10), (rbx.MIXED, 1e-6)):
        e = rbx.Engine(s, precision=prec)
        e.set_k_samples(*m)
        e.compute_forces(epoch=0)
        st = e.stats()
        assert abs(st.e_kspace - ek) < tol * abs(ek), prec
        assert np.allclose(np.asarray(st.virial_kspace[:]), vir, rtol=tol,
                           atol=tol * np.abs(vir).max()), prec
        e.close()


def test_engine_pair_energy(cuda, rbx, oracle):
    """Pair energies and virial over every pair within cut_off
    (rbx_engine_pair_energy, what RBMD computes with energy_rbl_flag "yes")
    against the oracle's LJCutCoulForce energies, for RBL engines in both
    forms and a Verlet-list engine, at the start and after steps that moved
    the atoms without a rebuild in between."""
    s = systems.lj_electrolyte(8000, seed=81)
    p = s["params"]
    rcs = p["cut_off"] + p["skin"]

    def want(pos):
        s2 = dict(s, pos=pos)
        box, perm, cell, cs, ce, xs, ys, zs = _sorted(oracle, s2, rcs)
        cnt, rows = oracle.full_list(box, rcs, xs, ys, zs, cell, cs, ce)
        _, vir, el, ec = oracle.pair_force_verlet(box, p["cut_off"], p["alpha"], p["qqr2e"],
                                                  s["type"][perm], s["sigma"], s["eps"],
                                                  s["q"][perm], xs, ys, zs, cnt, rows)
        return el, ec, np.asarray(vir)

    for neighbor, prec in (("RBL", rbx.PLAIN_FP64), ("RBL", rbx.MIXED), ("VERLET", rbx.MIXED)):
        e = rbx.Engine(s, precision=prec, neighbor=neighbor, seed=3)
        e.compute_forces(0)
        for k in range(2):
            if k:
                e.step(3)
            el, ec, vir = want(e.get_state()["pos"])
            gl, gc, gv = e.pair_energy()
            assert abs(gl - el) < 1e-10 * abs(el), (neighbor, prec, k)
            assert abs(gc - ec) < 1e-10 * abs(ec), (neighbor, prec, k)
            assert np.allclose(gv, vir, rtol=1e-10, atol=1e-10 * np.abs(vir).max()), (neighbor, k)
        e.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_engine_rbl_pairs_bit_exact(cuda, rbx, oracle, sys4k, prec):
    s = sys4k
    for epoch in (0, 9):
        box, perm, xs, ys, zs, gid, cnt, rows, cc, core, sc, shell = _ref_lists(oracle, s, epoch,
                                                                                4)
        e = rbx.Engine(s, precision=prec)
        e.compute_forces(epoch=epoch)
        gc, gs = e.rbl_pairs()
        want_c = {(int(gid[i]), int(gid[j])) for i in range(s["n"]) for j in core[i, :cc[i]]}
        want_s = {(int(gid[i]), int(gid[j])) for i in range(s["n"]) for j in shell[i, :sc[i]]}
        got_c = set(map(tuple, gc.tolist()))
        got_s = set(map(tuple, gs.tolist()))
        # the list predicates are the reference's FP64 ones in both forms: the
        # fixed-point screen only decides pairs outside its guard bands
        assert got_c == want_c and got_s == want_s, (prec, epoch)
        e.close()


def _orthorhombic(n, seed, scale=(1.15, 0.92, 1.0)):
    """An LJ electrolyte whose box and positions are stretched per axis."""
    s = systems.lj_electrolyte(n, seed=seed)
    lo = np.asarray(s["lo"], float)
    sc = np.asarray(scale, float)
    hi = lo + (np.asarray(s["hi"], float) - lo) * sc
    pos = lo + (s["pos"] - lo) * sc
    return dict(s, lo=lo, hi=hi, pos=pos)


@pytest.mark.parametrize("scale", [(1.15, 0.92, 1.0), (1.6, 0.8, 1.05)])
def test_engine_orthorhombic_box(cuda, rbx, oracle, scale):
    """A box with three different edge lengths (the fixed-point distance
    screen weights each axis by L_d / L_max): forces in both forms against
    the oracle, RBL pairs as exact sets in both forms, and velocity-Verlet
    steps against the oracle's engine."""
    import __graft_entry__ as ge

    s = _orthorhombic(8000, seed=61, scale=scale)
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbe_sample_philox(box, 0.16, 100, 7, 0)
    want = ge._oracle_forces(s, m)
    for prec, tol in ((rbx.PLAIN_FP64, 1e-9), (rbx.MIXED, 1e-5)):
        e = rbx.Engine(s, precision=prec)
        e.set_k_samples(*m)
        e.compute_forces(epoch=0)
        assert systems.rel_rms(e.get_state()["force"], want) < tol, prec
        freq = e.stats().selection_frequency
        p = s["params"]
        _, perm, cell, cs, ce, xs, ys, zs = _sorted(oracle, s, p["cut_off"] + p["skin"])
        cnt, rows = oracle.full_list(box, p["cut_off"] + p["skin"], xs, ys, zs, cell, cs, ce)
        gid = s["gid"][perm]
        cc, core, sc, shell = oracle.rbl_filter(box, p["r_core"], p["cut_off"], freq, 0, gid, xs,
                                                ys, zs, cnt, rows)
        gc, gs = e.rbl_pairs()
        want_c = {(int(gid[i]), int(gid[j])) for i in range(s["n"]) for j in core[i, :cc[i]]}
        want_s = {(int(gid[i]), int(gid[j])) for i in range(s["n"]) for j in shell[i, :sc[i]]}
        got_c, got_s = set(map(tuple, gc.tolist())), set(map(tuple, gs.tolist()))
        assert got_c == want_c and got_s == want_s, prec
        e.close()
    e = rbx.Engine(s, precision=rbx.PLAIN_FP64, seed=4242)
    ref = oracle.Engine(s, seed=4242)
    ref.compute_forces(0)
    e.compute_forces(0)
    for k in range(3):
        e.step(1)
        ref.step(1)
        a, b = e.get_state(), ref.get()
        order = np.argsort(b["gid"])
        assert systems.rel_rms(a["force"], b["force"][order]) < 1e-8, k
        assert np.abs(a["pos"] - b["pos"][order]).max() < 1e-10, k
    e.close()


@pytest.mark.parametrize("scale", [(1.0, 1.0, 1.0), (1.15, 0.92, 1.0)])
def test_engine_verlet_list(cuda, rbx, oracle, scale):
    """The engine with a plain Verlet list (LJ + erfc-Coulomb to cut_off over
    the candidate rows, no random batch): its pair force against the oracle's
    ComputeLJCutCoulForce restatement on a cubic and an orthorhombic box, and
    its graph step against launch-by-launch steps bit for bit."""
    s = _orthorhombic(8000, seed=71, scale=scale)
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    rcs = p["cut_off"] + p["skin"]
    _, perm, cell, cs, ce, xs, ys, zs = _sorted(oracle, s, rcs)
    cnt, rows = oracle.full_list(box, rcs, xs, ys, zs, cell, cs, ce)
    f, _, _, _ = oracle.pair_force_verlet(box, p["cut_off"], p["alpha"], p["qqr2e"],
                                          s["type"][perm], s["sigma"], s["eps"], s["q"][perm], xs,
                                          ys, zs, cnt, rows)
    want = np.empty_like(f)
    want[perm] = f
    m = oracle.rbe_sample_philox(box, p["alpha"], 100, 7, 0)
    for prec in (rbx.PLAIN_FP64, rbx.MIXED):
        e = rbx.Engine(s, precision=prec, neighbor="VERLET")
        e.set_k_samples(*m)
        e.compute_forces(epoch=0)
        fp, _ = e.force_parts()
        assert systems.rel_rms(fp, want) < 1e-10, prec  # real space is FP64 in both forms
        e.close()
    runs = []
    for graph in (True, False):
        e = rbx.Engine(s, precision=rbx.MIXED, neighbor="VERLET", seed=13)
        e.set_step_graph(graph)
        e.compute_forces(0)
        e.step(8)
        e.step(12)
        runs.append((e.get_state(), e.stats()))
        e.close()
    (a, sa), (b, sb) = runs
    for key in ("pos", "vel", "force"):
        assert np.array_equal(a[key], b[key]), key
    assert sa.rebuilds == sb.rebuilds


@pytest.mark.parametrize("prec", [0, 1])
def test_engine_rbl_pairs_between_rebuilds(cuda, rbx, oracle, prec):
    """The engine keeps its candidate rows between skin rebuilds.  After
    dynamics that moved the atoms up to skin / 2 from the list build, the core
    and shell pairs of each epoch equal the oracle's lists built from the
    current positions."""
    s = systems.lj_electrolyte(4000, seed=31, temperature=3.0)
    e = rbx.Engine(s, precision=prec, seed=5)
    e.compute_forces(epoch=0)
    checked = 0
    for k in range(8):
        e.step(6)
        st = e.get_state()
        s2 = dict(s, pos=st["pos"])
        epoch = 1000 + k
        e.compute_forces(epoch=epoch)  # keeps the rows unless the skin test fails
        *_, gid, cnt, rows, cc, core, sc, shell = _ref_lists(oracle, s2, epoch, 4)
        gc, gs = e.rbl_pairs()
        want_c = {(int(gid[i]), int(gid[j])) for i in range(s["n"]) for j in core[i, :cc[i]]}
        want_s = {(int(gid[i]), int(gid[j])) for i in range(s["n"]) for j in shell[i, :sc[i]]}
        got_c = set(map(tuple, gc.tolist()))
        got_s = set(map(tuple, gs.tolist()))
        assert got_c == want_c and got_s == want_s, (prec, k)
        checked += 1
    stats = e.stats()
    assert checked == 8 and 1 <= stats.rebuilds < stats.force_calls
    e.close()


def test_engine_philox_matches_oracle_engine(cuda, rbx, oracle, sys4k):
    """Full velocity-Verlet steps with on-device Philox k-samples and RBL
    batches: the first steps agree with the oracle's step to FP64 round-off."""
    s = sys4k
    e = rbx.Engine(s, precision=rbx.PLAIN_FP64, seed=4242)
    ref = oracle.Engine(s, seed=4242)
    ref.compute_forces(0)
    e.compute_forces(0)
    for k in range(3):
        e.step(1)
        ref.step(1)
        a, b = e.get_state(), ref.get()
        order = np.argsort(b["gid"])
        bf = b["force"][order]
        bp = b["pos"][order]
        assert systems.rel_rms(a["force"], bf) < 1e-8, k
        assert np.abs(a["pos"] - bp).max() < 1e-10
    st = e.stats()
    assert st.steps == 3 and st.selection_frequency == 4


@pytest.mark.parametrize("prec, nvt", [(0, False), (1, False), (1, True)])
def test_step_graph_matches_individual_launches(cuda, rbx, prec, nvt):
    """The CUDA-graph step (rebuild under a conditional node, device epoch,
    the Nose-Hoover chain on the device) runs the same kernels on the same
    data as the step the host drives launch by launch: the trajectories are
    bit-identical, rebuilds and thermostat included."""
    s = systems.lj_electrolyte(4000, seed=31)
    runs = []
    for graph in (True, False):
        e = rbx.Engine(s, precision=prec, seed=9)
        e.set_step_graph(graph)
        e.compute_forces(0)
        if nvt:
            e.set_nose_hoover(1.0, 1.6, 0.1, num_steps=40)
        e.step(15)
        e.step(25)
        runs.append((e.get_state(), e.stats(), e.thermostat()))
        e.close()
    (a, sa, ta), (b, sb, tb) = runs
    for key in ("pos", "vel", "force"):
        assert np.array_equal(a[key], b[key]), key
    if nvt:
        assert ta["temperature"] == tb["temperature"]
        assert np.array_equal(ta["eta_dot"], tb["eta_dot"])
    assert sa.steps == sb.steps == 40
    assert sa.rebuilds == sb.rebuilds and sa.rebuilds >= 2


@pytest.mark.parametrize("ramp", [False, True])
def test_nose_hoover_matches_oracle(cuda, rbx, oracle, sys4k, ramp):
    """NVT steps (Nose-Hoover chain of NVTensemble::Solve) agree with the
    oracle's NVT step to FP64 round-off: positions, velocities and the chain."""
    s = sys4k
    t_stop = 1.8 if ramp else 1.3
    e = rbx.Engine(s, precision=rbx.PLAIN_FP64, seed=4242)
    ref = oracle.Engine(s, seed=4242)
    for x in (e, ref):
        x.compute_forces(0)
        x.set_nose_hoover(1.3, t_stop, 0.05, num_steps=20)
    for k in range(4):
        e.step(5)
        ref.step(5)
        a, b = e.get_state(), ref.get()
        order = np.argsort(b["gid"])
        assert np.abs(a["pos"] - b["pos"][order]).max() < 1e-9, k
        assert systems.rel_rms(a["vel"], b["vel"][order]) < 1e-9, k
        ta, tb = e.thermostat(), ref.thermostat()
        assert abs(ta["temperature"] - tb["temperature"]) < 1e-9 * tb["temperature"]
        assert np.allclose(ta["eta_dot"], tb["eta_dot"], rtol=1e-7, atol=1e-12)
        assert np.allclose(ta["eta"], tb["eta"], rtol=1e-7, atol=1e-12)
    e.close()


def test_step_graph_recovers_from_list_overflow(cuda, rbx):
    """A rebuild inside the step graph that overflows the candidate rows
    (here: the host hands in a configuration compressed to 0.7 of the box,
    three times denser) is detected after the graph has run; the saved state
    comes back and the step is replayed launch by launch, growing the rows.
    The result equals the engine that never used the graph."""
    s = systems.lj_electrolyte(4000, seed=5)
    lo, hi = np.asarray(s["lo"]), np.asarray(s["hi"])
    c = 0.5 * (lo + hi)
    x = np.ascontiguousarray(s["pos"].T)
    v = np.ascontiguousarray(s["vel"].T)
    xc = np.ascontiguousarray((c + 0.7 * (s["pos"] - c)).T)
    out = []
    for graph in (True, False):
        e = rbx.Engine(s, precision=rbx.PLAIN_FP64, seed=3)
        e.set_step_graph(graph)
        e.compute_forces(0)
        cap0 = e.stats().candidate_capacity
        xo, vo, fo = np.zeros((3, s["n"])), np.zeros((3, s["n"])), np.zeros((3, s["n"]))
        e.step_host(x, v, xo, vo, fo)
        e.step_host(xc, v, xo, vo, fo)
        st = e.stats()
        assert st.candidate_capacity > cap0  # the rows grew
        out.append((xo.copy(), vo.copy(), fo.copy()))
        e.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
    assert np.isfinite(out[0][2]).all()


def test_batch_matches_single_engines(cuda, rbx):
    """Replicas of different sizes and forms advanced by one graph launch per
    step (rbx_batch) end bit-identical to the same engines stepped alone."""
    specs = [(4000, 11, rbx.MIXED), (5200, 12, rbx.PLAIN_FP64), (6500, 13, rbx.MIXED)]
    systems_ = [systems.lj_electrolyte(n, seed=sd) for n, sd, _ in specs]
    batched = [rbx.Engine(s, precision=p, seed=21) for s, (_, _, p) in zip(systems_, specs)]
    single = [rbx.Engine(s, precision=p, seed=21) for s, (_, _, p) in zip(systems_, specs)]
    for e in batched + single:
        e.compute_forces(0)
    b = rbx.Batch(batched)
    b.step(12)
    b.step(18)
    for e in single:
        e.step(12)
        e.step(18)
    for e1, e2 in zip(batched, single):
        a, c = e1.get_state(), e2.get_state()
        for key in ("pos", "vel", "force"):
            assert np.array_equal(a[key], c[key]), key
        s1, s2 = e1.stats(), e2.stats()
        assert s1.steps == s2.steps == 30 and s1.rebuilds == s2.rebuilds
    b.close()
    for e in batched + single:
        e.close()


def test_batch_follows_thermostat_set_after_capture(cuda, rbx):
    """A batch graph captured before a replica was given a thermostat is
    captured again: the replica then steps NVT, bit-identical to the same
    engine stepped alone."""
    s = systems.lj_electrolyte(4000, seed=41)
    a = rbx.Engine(s, precision=rbx.MIXED, seed=3)
    b = rbx.Engine(s, precision=rbx.MIXED, seed=3)
    for e in (a, b):
        e.compute_forces(0)
    batch = rbx.Batch([a])
    batch.step(5)
    b.step(5)
    for e in (a, b):
        e.set_nose_hoover(1.0, 1.6, 0.05, num_steps=30)
    batch.step(12)
    b.step(12)
    sa, sb = a.get_state(), b.get_state()
    for key in ("pos", "vel", "force"):
        assert np.array_equal(sa[key], sb[key]), key
    ta, tb = a.thermostat(), b.thermostat()
    assert ta["temperature"] == tb["temperature"]
    assert np.array_equal(ta["eta"], tb["eta"]) and np.any(ta["eta"] != 0)
    batch.close()
    a.close()
    b.close()


def test_engine_step_host_roundtrip(cuda, rbx, sys4k):
    s = sys4k
    e1 = rbx.Engine(s, precision=rbx.MIXED, seed=1)
    e2 = rbx.Engine(s, precision=rbx.MIXED, seed=1)
    e1.compute_forces(0)
    e2.compute_forces(0)
    n = s["n"]
    x = np.ascontiguousarray(s["pos"].T)
    v = np.ascontiguousarray(s["vel"].T)
    xo, vo, fo = np.zeros((3, n)), np.zeros((3, n)), np.zeros((3, n))
    for _ in range(3):
        e1.step_host(x, v, xo, vo, fo)
        x, v = xo.copy(), vo.copy()
        e2.step(1)
    st = e2.get_state()
    assert np.array_equal(st["pos"], xo.T)
    assert np.array_equal(st["force"], fo.T)


def test_engine_json_drop_in(cuda, rbx, sys4k):
    from tests.test_capi_cpu import JSON_OK

    s = sys4k
    e = rbx.Engine(s, json_text=JSON_OK)
    st = e.stats()
    assert st.selection_frequency == 4
    e.compute_forces(0)
    assert np.isfinite(e.get_state()["force"]).all()
    e.close()


def test_engine_energy_conservation_short(cuda, rbx):
    """Plain-FP64 RBL+RBE dynamics stays finite and the candidate list is
    rebuilt on the skin criterion."""
    s = systems.lj_electrolyte(4000, seed=77)
    e = rbx.Engine(s, precision=rbx.MIXED)
    e.step(200)
    st = e.stats()
    assert st.rebuilds >= 2
    out = e.get_state()
    assert np.isfinite(out["pos"]).all() and np.isfinite(out["vel"]).all()
    T = (out["vel"] ** 2).sum() / (3 * s["n"])
    assert 0.5 < T < 3.0


@pytest.mark.parametrize("prec", [0, 1])
def test_force_vjp_matches_oracle_adjoint(cuda, rbx, oracle, prec):
    """The engine's adjoint (rbx_engine_force_vjp) against the FP64 adjoint
    reference, itself pinned to central differences of the oracle's force:
    parameter gradients per type, dL/dq per atom and dL/dr (Hessian-vector
    product), with the same lists, batch and k-samples.  Plain FP64 within
    1e-9; the mixed form's FP32 adjoint (FP64 sums) within 2e-5."""
    from oracle import adjoint as A

    s = systems.lj_electrolyte(4000, seed=41)
    p = s["params"]
    ep = 7
    box = oracle.Box.make(s["lo"], s["hi"])
    L = np.asarray(s["hi"]) - np.asarray(s["lo"])
    m = oracle.rbe_sample_philox(box, p["alpha"], p["kspace_p"], 3, ep)
    e = rbx.Engine(s, precision=prec)
    e.set_k_samples(*m)
    e.compute_forces(epoch=ep)
    g = np.random.default_rng(5).normal(size=(s["n"], 3))
    got = e.force_vjp(g)
    e.close()
    x, y, z = (np.ascontiguousarray(s["pos"][:, d]) for d in range(3))
    perm, cell, cs, ce = oracle.cells_sort(box, 5.3, x, y, z)
    pos = s["pos"][perm]
    cnt, rows = oracle.full_list(box, 5.3, *(np.ascontiguousarray(pos[:, d]) for d in range(3)),
                                 cell, cs, ce)
    freq, _, _ = oracle.rbl_params(s["n"], box, p["r_core"], p["cut_off"],
                                   p["neighbor_sample_num"])
    cc, core, sc, shell = oracle.rbl_filter(box, p["r_core"], p["cut_off"], freq, ep, s["gid"][perm],
                                            *(np.ascontiguousarray(pos[:, d]) for d in range(3)),
                                            cnt, rows)
    lists = A.rbl_pairs(cc, core, sc, shell, freq)
    d_eps, d_sig, d_q, d_alpha, d_r = A.force_vjp(
        pos, L, s["type"][perm], np.asarray(s["sigma"], float), np.asarray(s["eps"], float),
        s["q"][perm], p["alpha"], p["qqr2e"], p["r_core"], p["cut_off"], freq, lists, m, g[perm])
    want_q = np.zeros(s["n"])
    want_q[perm] = d_q
    want_r = np.zeros((s["n"], 3))
    want_r[perm] = d_r
    # plain FP64 engine: FP64 adjoint; mixed engine: FP32 pair and k-space
    # terms (exact fixed-point phases) with FP64 sums
    tol = 1e-9 if prec == 0 else 2e-5
    assert np.allclose(got["eps"], d_eps, rtol=tol, atol=tol * np.abs(d_eps).max())
    assert np.allclose(got["sigma"], d_sig, rtol=tol, atol=tol * np.abs(d_sig).max())
    assert abs(got["alpha"] - d_alpha) < tol * abs(d_alpha)
    assert systems.rel_rms(got["charge"][:, None], want_q[:, None]) < tol
    assert systems.rel_rms(got["pos"], want_r) < tol


def test_force_vjp_against_engine_finite_differences(cuda, rbx):
    """Central differences of the engine's own FP64 force, through the
    parameter setters, against rbx_engine_force_vjp."""
    s = systems.lj_electrolyte(4000, seed=43)
    p = s["params"]
    from oracle import oracle as O

    m = O.rbe_sample_philox(O.Box.make(s["lo"], s["hi"]), p["alpha"], p["kspace_p"], 2, 4)
    e = rbx.Engine(s, precision=rbx.PLAIN_FP64)
    e.set_k_samples(*m)
    e.compute_forces(4)
    g = np.random.default_rng(8).normal(size=(s["n"], 3))
    got = e.force_vjp(g)
    sig0, eps0 = np.asarray(s["sigma"], float), np.asarray(s["eps"], float)
    Q = np.array([0.0, 1.0, -1.0])

    def L():
        e.compute_forces(4)
        return float((g * e.get_state()["force"]).sum())

    def fd(setter, base, step):
        """Central difference along `step` (scalar, or an array with one nonzero entry)."""
        h = float(np.max(np.abs(step)))
        setter(base + step)
        up = L()
        setter(base - step)
        dn = L()
        setter(base)
        return (up - dn) / (2 * h)

    def close(a, b, rel=1e-5):
        assert abs(a - b) <= rel * max(abs(a), abs(b)) + 1e-8, (a, b)

    for t in range(3):
        unit = np.eye(3)[t]
        close(got["eps"][t], fd(lambda v: e.set_lj_params(sig0, v), eps0, 1e-6 * eps0[t] * unit))
        close(got["sigma"][t], fd(lambda v: e.set_lj_params(v, eps0), sig0, 1e-6 * sig0[t] * unit))
        close(got["charge"][s["type"] == t].sum(),
              fd(lambda v: e.set_charges(v[s["type"]]), Q, 1e-6 * unit))
    close(got["alpha"], fd(e.set_alpha, p["alpha"], 1e-6 * p["alpha"]))
    pos0 = s["pos"].copy()
    for a in (0, 1234):
        for d in range(3):
            dp = np.zeros_like(pos0)
            dp[a, d] = 1e-6
            close(got["pos"][a, d], fd(e.set_positions, pos0, dp), rel=1e-4)
    e.close()


def test_autograd_function_gradients(cuda, rbx):
    """torch.autograd through RBLRBEForce gives the adjoint's gradients."""
    import torch

    from rbmd_b200.autograd import force

    s = systems.lj_electrolyte(4000, seed=44)
    p = s["params"]
    from oracle import oracle as O

    m = O.rbe_sample_philox(O.Box.make(s["lo"], s["hi"]), p["alpha"], p["kspace_p"], 6, 1)
    e = rbx.Engine(s, precision=rbx.MIXED)
    e.set_k_samples(*m)
    t64 = torch.float64
    eps = torch.tensor(s["eps"], dtype=t64, requires_grad=True)
    sig = torch.tensor(s["sigma"], dtype=t64, requires_grad=True)
    Q = torch.tensor([0.0, 1.0, -1.0], dtype=t64, requires_grad=True)
    alpha = torch.tensor(p["alpha"], dtype=t64, requires_grad=True)
    pos = torch.tensor(s["pos"], dtype=t64, requires_grad=True)
    typ = torch.as_tensor(s["type"], dtype=torch.long)
    f_ref = force(e, eps.detach() * 1.05, sig.detach() * 0.97, Q.detach()[typ] * 1.02,
                  alpha.detach(), pos.detach(), 1).detach()
    f = force(e, eps, sig, Q[typ], alpha, pos, 1)
    loss = ((f - f_ref) ** 2).mean()
    loss.backward()
    g = (2.0 * (f - f_ref) / f.numel()).detach().numpy()
    direct = e.force_vjp(g)  # same state as the forward above
    assert np.allclose(eps.grad.numpy(), direct["eps"], rtol=1e-12)
    assert np.allclose(pos.grad.numpy(), direct["pos"], rtol=1e-12, atol=1e-15)
    assert np.isfinite(Q.grad.numpy()).all() and alpha.grad is not None
    e.close()


def _read_frames(path):
    """Parse frames of the rbmd.trj format written by rbx_engine_write_trajectory."""
    lines = open(path).read().splitlines()
    frames, i = [], 0
    while i < len(lines):
        assert lines[i] == "ITEM: TIMESTEP"
        ts = int(lines[i + 1])
        assert lines[i + 2] == "ITEM: NUMBER OF ATOMS"
        n = int(lines[i + 3])
        assert lines[i + 4] == "ITEM: BOX BOUNDS pp pp pp"
        bounds = np.array([[float(v) for v in lines[i + 5 + d].split()] for d in range(3)])
        assert lines[i + 8] == "ITEM: ATOMS id type q x y z xu yu zu vx vy vz"
        rows = [r.split() for r in lines[i + 9:i + 9 + n]]
        frames.append({"timestep": ts, "bounds": bounds,
                       "id": np.array([int(r[0]) for r in rows]),
                       "type": np.array([int(r[1]) for r in rows]),
                       "data": np.array([[float(v) for v in r[2:]] for r in rows])})
        i += 9 + n
    return frames


@pytest.mark.parametrize("graph", [True, False])
def test_trajectory_frames_and_images(cuda, rbx, tmp_path, graph):
    """Image counters follow every wrap of the drift through rebuild
    permutations (graph and launch-by-launch steps alike), and the trajectory
    writer puts out RBMD's frame layout: ids and types 1-based in id order,
    positions and velocities that read back as the engine's doubles, and
    unwrapped xu = x + image * L that moves continuously across the faces."""
    s = systems.lj_electrolyte(4000, seed=41)
    perm = np.random.default_rng(2).permutation(s["n"])  # host order != id order
    s2 = dict(s)
    for key in ("pos", "vel", "type", "q", "gid"):
        s2[key] = np.ascontiguousarray(s[key][perm])
    e = rbx.Engine(s2, precision=rbx.MIXED, seed=5)
    e.set_step_graph(graph)
    e.compute_forces(0)
    L = np.asarray(s["hi"]) - np.asarray(s["lo"])
    path = tmp_path / "rbmd.trj"
    e.write_trajectory(path, 0, append=False)
    states, images = [e.get_state()], [e.images()]
    for t in (1, 2):
        e.step(60)
        e.write_trajectory(path, 60 * t)
        states.append(e.get_state())
        images.append(e.images())
    assert e.stats().rebuilds >= 2
    assert not images[0].any() and np.abs(images[-1]).sum() > 50
    frames = _read_frames(path)
    assert [f["timestep"] for f in frames] == [0, 60, 120]
    order = np.argsort(s2["gid"])
    for f, st, im in zip(frames, states, images):
        assert np.array_equal(f["bounds"], np.stack([s["lo"], s["hi"]], 1))
        assert np.array_equal(f["id"], np.sort(s2["gid"]) + 1)  # internal ids + 1
        assert np.array_equal(f["type"], s2["type"][order] + 1)
        d = f["data"]
        assert np.array_equal(d[:, 0], s2["q"][order])
        assert np.array_equal(d[:, 1:4], st["pos"][order])
        assert np.array_equal(d[:, 7:10], st["vel"][order])
        assert np.array_equal(d[:, 4:7], st["pos"][order] + im[order] * L)
    for a, b in zip(frames[:-1], frames[1:]):
        jump = np.abs(b["data"][:, 4:7] - a["data"][:, 4:7]).max()
        assert jump < 2.0  # unwrapped paths are continuous
        assert np.abs(b["data"][:, 1:4] - a["data"][:, 1:4]).max() > 0.5 * L.min()  # wraps happened
    e.close()


FILES_JSON = """{
  "init_configuration": {"read_data": {"file": "sys.data", "unit": "LJ",
      "atom_style": "charge", "velocity_type": "GAUSS", "velocity_seed": 77, "replicate": REP}},
  // RBMD's config files carry comments
  "hyper_parameters": {
    "force_field": {"type": "LJ/CUT/COUL/LONG"},
    "neighbor": {"type": "RBL", "cut_off": 5.0, "r_core": 2.5, "skin": 0.3,
                 "neighbor_sample_num": 100, "energy_rbl_flag": "no"},
    "coulomb": {"type": "RBE", "coulomb_sample_num": 100, "alpha": 0.16,
                "energy_rbe_flag": "no", "random_seed": 9}},
  "execution": {"timestep": 0.005, "temperature": [1.2, 1.2, 1]}
}"""


@pytest.mark.parametrize("rep, velocities", [((1, 1, 1), True), ((2, 1, 1), False)])
def test_engine_from_files_matches_arrays(cuda, rbx, tmp_path, rep, velocities):
    """rbx_engine_create_from_files on a data file + JSON config equals the
    engine built from the same arrays (rbx_engine_create_json): forces and a
    40-step trajectory bit for bit.  Atoms written outside the box come in
    wrapped, with the wrap in their image flags; without a Velocities section
    the GAUSS velocities are those of the reader."""
    s = systems.lj_electrolyte(4000, seed=23)
    L = np.asarray(s["hi"]) - np.asarray(s["lo"])
    moved = np.arange(0, s["n"], 397) if rep == (1, 1, 1) else np.arange(0)
    out_of_box = dict(s, pos=s["pos"].copy())
    out_of_box["pos"][moved, 0] += L[0]  # one box length out
    data = tmp_path / "sys.data"
    rbx.write_lammps_charge(data, out_of_box)
    if not velocities:
        data.write_text(data.read_text().partition("\nVelocities")[0] + "\n")
    cfg = tmp_path / "rbmd.json"
    text = FILES_JSON.replace("REP", str(list(rep)))
    if not velocities:  # and NVT with the Nose-Hoover chain
        text = text.replace('"execution": {', '"execution": {"ensemble": "NVT", '
                            '"temp_ctrl_type": "NOSE_HOOVER", ')
    cfg.write_text(text)
    a = rbx.Engine.from_files(cfg, precision=rbx.MIXED)
    ref = rbx.read_lammps(data, replicate=rep, gauss=None if velocities else (1.2, "LJ", 77))
    assert a.n == ref["n"] == s["n"] * np.prod(rep)
    assert np.array_equal(a.gid, ref["id"]) and np.array_equal(a.types, ref["type"])
    im = a.images()
    pos = ref["pos"].copy()
    Lr = np.asarray(ref["hi"]) - np.asarray(ref["lo"])
    if rep == (1, 1, 1):
        assert np.array_equal(np.nonzero(im[:, 0])[0], moved) and (im[moved, 0] == 1).all()
        pos[moved, 0] -= L[0]
    else:
        assert np.array_equal(im, ref["image"])
    sysd = {"n": ref["n"], "lo": ref["lo"], "hi": ref["hi"], "sigma": ref["sigma"],
            "eps": ref["eps"], "mass": ref["mass"], "q": ref["q"], "pos": pos, "vel": ref["vel"],
            "gid": ref["id"].astype(np.int32), "type": ref["type"]}
    b = rbx.Engine(sysd, precision=rbx.MIXED, json_text=text.replace("// RBMD's config files "
                                                                      "carry comments", ""))
    b.set_images(im)
    if not velocities:
        b.set_nose_hoover(1.2, 1.2, 1.0)
    sa, sb = a.get_state(), b.get_state()
    assert np.array_equal(sa["pos"], sb["pos"]) and np.array_equal(sa["vel"], sb["vel"])
    for e in (a, b):
        e.compute_forces(0)
        e.step(40)
    sa, sb = a.get_state(), b.get_state()
    for key in ("pos", "vel", "force"):
        assert np.array_equal(sa[key], sb[key]), key
    assert np.abs(sa["pos"] + a.images() * Lr - (sb["pos"] + b.images() * Lr)).max() == 0
    if not velocities:
        assert a.thermostat()["temperature"] == b.thermostat()["temperature"]
        assert a.thermostat()["eta_dot"][0] != 0
    a.close()
    b.close()


def _water_geometry(s, pos, vel):
    """Largest bond / H-H distance error and largest bond-direction relative
    velocity (the RATTLE condition) over all molecules."""
    L = np.asarray(s["hi"]) - np.asarray(s["lo"])
    cl = s["clusters"]

    def vec(a, b):
        d = pos[a] - pos[b]
        return d - L * np.rint(d / L)
    r01, r12, r02 = vec(cl[:, 1], cl[:, 0]), vec(cl[:, 2], cl[:, 1]), vec(cl[:, 2], cl[:, 0])
    hh = 2 * np.sin(np.radians(systems.WATER_ANGLE) / 2)
    err = max(np.abs(np.linalg.norm(r01, axis=1) - 1).max(),
              np.abs(np.linalg.norm(r12, axis=1) - 1).max(),
              np.abs(np.linalg.norm(r02, axis=1) - hh).max())
    rv = max(np.abs(((vel[cl[:, 1]] - vel[cl[:, 0]]) * r01).sum(1)).max(),
             np.abs(((vel[cl[:, 2]] - vel[cl[:, 1]]) * r12).sum(1)).max())
    return err, rv


@pytest.fixture(scope="module")
def water3k():
    return systems.water(3000, seed=11)


def _water_nvt(e, s):
    p = s["params"]
    e.set_shake(s["clusters"], systems.WATER_BOND, systems.WATER_ANGLE)
    e.compute_forces(0)
    e.set_nose_hoover(298.0, 298.0, 100.0, kb=p["kb"], mvv2e=p["mvv2e"],
                      tdof=3 * s["n"] - 3 - s["n"])


def test_shake_water_matches_oracle(cuda, rbx, oracle, water3k):
    """Rigid water (9,000 atoms, REAL units) under SHAKE / RATTLE and the
    Nose-Hoover chain: the engine's steps agree with the oracle's, the bonds
    hold to the solver's tolerance and the bond-direction velocities vanish."""
    s = water3k
    e = rbx.Engine(s, precision=rbx.PLAIN_FP64, seed=77)
    ref = oracle.Engine(s, seed=77)
    ref.set_shake(s["clusters"], systems.WATER_BOND, systems.WATER_ANGLE)
    ref.compute_forces(0)
    p = s["params"]
    ref.set_nose_hoover(298.0, 298.0, 100.0, kb=p["kb"], mvv2e=p["mvv2e"],
                        tdof=3 * s["n"] - 3 - s["n"])
    _water_nvt(e, s)
    for k in range(3):
        e.step(4)
        ref.step(4)
        a, b = e.get_state(), ref.get()
        order = np.argsort(b["gid"])
        assert np.abs(a["pos"] - b["pos"][order]).max() < 1e-8, k
        assert systems.rel_rms(a["vel"], b["vel"][order]) < 1e-8, k
        assert systems.rel_rms(a["force"], b["force"][order]) < 1e-8, k
        err, rv = _water_geometry(s, a["pos"], a["vel"])
        assert err < 1e-4 and rv < 1e-9, (err, rv)
        ta, tb = e.thermostat(), ref.thermostat()
        assert abs(ta["temperature"] - tb["temperature"]) < 1e-8 * tb["temperature"]
    assert e.shake_status() == (3000, 0) and ref.shake_failures == 0
    e.close()


def test_shake_water_graph_and_mixed(cuda, rbx, water3k):
    """The step graph with SHAKE and the thermostat equals the launch-by-launch
    step bit for bit (mixed form, rebuilds included), and holds the geometry."""
    s = water3k
    runs = []
    for graph in (True, False):
        e = rbx.Engine(s, precision=rbx.MIXED, seed=77)
        e.set_step_graph(graph)
        _water_nvt(e, s)
        e.step(10)
        e.step(15)
        runs.append((e.get_state(), e.stats(), e.images()))
        assert e.shake_status()[1] == 0
        e.close()
    (a, sa, ia), (b, sb, ib) = runs
    for key in ("pos", "vel", "force"):
        assert np.array_equal(a[key], b[key]), key
    assert np.array_equal(ia, ib)
    assert sa.rebuilds == sb.rebuilds and sa.rebuilds >= 1
    err, rv = _water_geometry(s, a["pos"], a["vel"])
    assert err < 1e-4 and rv < 1e-9, (err, rv)


def test_step_host_water_shake_nvt(cuda, rbx, water3k):
    """Host-buffer steps (positions copied out while the forces are computed)
    with SHAKE and the thermostat equal device-resident steps bit for bit,
    over enough steps for rebuilds."""
    s = water3k
    n = s["n"]
    e1 = rbx.Engine(s, precision=rbx.MIXED, seed=77)
    e2 = rbx.Engine(s, precision=rbx.MIXED, seed=77)
    for e in (e1, e2):
        _water_nvt(e, s)
    st0 = e1.get_state()
    x = np.ascontiguousarray(st0["pos"].T)
    v = np.ascontiguousarray(st0["vel"].T)
    xo, vo, fo = np.zeros((3, n)), np.zeros((3, n)), np.zeros((3, n))
    for _ in range(25):
        e1.step_host(x, v, xo, vo, fo)
        x, v = xo.copy(), vo.copy()
        e2.step(1)
    b = e2.get_state()
    assert np.array_equal(b["pos"], xo.T)
    assert np.array_equal(b["vel"], vo.T)
    assert np.array_equal(b["force"], fo.T)
    s1, s2 = e1.stats(), e2.stats()
    assert s1.steps == s2.steps == 25 and s1.rebuilds == s2.rebuilds >= 1
    assert e1.thermostat()["temperature"] == e2.thermostat()["temperature"]
    assert e1.shake_status() == e2.shake_status()
    e1.close()
    e2.close()


def _oracle_special_pair_force(oracle, s, nspecial, special, weights, epoch):
    """The oracle's CVFF RBL pair force (mean removed) in host order."""
    p = s["params"]
    box = oracle.Box.make(s["lo"], s["hi"])
    cols = [np.ascontiguousarray(s["pos"][:, d]) for d in range(3)]
    perm, cell, cs, ce = oracle.cells_sort(box, p["cut_off"] + p["skin"], *cols)
    pos = s["pos"][perm]
    xyz = [np.ascontiguousarray(pos[:, d]) for d in range(3)]
    gid = np.ascontiguousarray(s["gid"][perm], dtype=np.int32)
    cnt, rows = oracle.full_list(box, p["cut_off"] + p["skin"], *xyz, cell, cs, ce)
    freq, _, _ = oracle.rbl_params(s["n"], box, p["r_core"], p["cut_off"], p["neighbor_sample_num"])
    cc, core, sc, shell = oracle.rbl_filter(box, p["r_core"], p["cut_off"], freq, epoch, gid, *xyz,
                                            cnt, rows)
    sp_gid = np.asarray(s["gid"])[special[perm]]  # partners as gids, rows in oracle order
    f = oracle.pair_force_rbl_special(box, p["r_core"], p["cut_off"], freq, p["alpha"], p["qqr2e"],
                                      s["type"][perm].astype(np.int32), s["sigma"], s["eps"], gid,
                                      s["q"][perm], *xyz, cc, core, sc, shell,
                                      np.ascontiguousarray(nspecial[perm]), sp_gid, weights)
    f, _ = oracle.fix_rbl(f)
    out = np.empty_like(f)
    out[perm] = f
    return out


def _random_specials(s, rng, per_atom=3):
    """Symmetric special rows of random neighbour pairs within cut_off (core
    and shell), bands 1-2 / 1-3 / 1-4 drawn at random."""
    n, L = s["n"], np.asarray(s["hi"]) - np.asarray(s["lo"])
    pos = s["pos"]
    bonds, angles, dih = [], [], []
    for i in rng.choice(n, size=n // 8, replace=False):
        d = pos - pos[i]
        d -= L * np.rint(d / L)
        r = np.linalg.norm(d, axis=1)
        near = np.nonzero((r > 0) & (r < s["params"]["cut_off"]))[0]
        for j in rng.choice(near, size=per_atom, replace=False):
            band = rng.integers(3)
            if band == 0:
                bonds.append((i, j))
            elif band == 1:
                angles.append((i, -1, j))
            else:
                dih.append((i, -1, -1, j))
    return bonds, angles, dih


@pytest.mark.parametrize("prec", [0, 1])
def test_special_bonds_lj_electrolyte(cuda, rbx, oracle, prec):
    """CVFF special-bond weights on the RBL pair force (core and sampled shell
    pairs, weights 0 / 0.5 / 0.8) against the oracle's restatement of
    ComputeSpecialLJCutCoulRBLForce + mean removal."""
    s = systems.lj_electrolyte(4000, seed=19)
    rng = np.random.default_rng(5)
    bonds, angles, dih = _random_specials(s, rng)
    ns, sp = rbx.special_build(s["n"], bonds, angles, dih)
    w = (0.0, 0.5, 0.8)
    e = rbx.Engine(s, precision=prec, seed=3)
    e.set_special(ns, sp, w)
    for epoch in (0, 3):
        e.compute_forces(epoch)
        fp, _ = e.force_parts()
        want = _oracle_special_pair_force(oracle, s, ns, sp, w, epoch)
        plain = _oracle_special_pair_force(oracle, s, ns, sp, (1.0, 1.0, 1.0), epoch)
        assert systems.rel_rms(want, plain) > 1e-3  # the weights matter
        assert systems.rel_rms(fp, want) < (1e-10 if prec == 0 else 1e-5), epoch
    e.close()


def test_special_bonds_water(cuda, rbx, oracle, water3k):
    """Water with special_bonds [0, 0, 0] (the reference's water config): the
    intramolecular O-H and H-H pairs leave real space and their k-space part
    is cancelled; pair force against the oracle."""
    s = water3k
    ns, sp = rbx.special_build(s["n"], s["bonds"], s["angles"])
    assert (ns[0::3] == [2, 2, 2]).all() and (ns[1::3] == [1, 2, 2]).all()
    e = rbx.Engine(s, precision=rbx.PLAIN_FP64, seed=3)
    e.set_special(ns, sp, (0.0, 0.0, 0.0))
    e.compute_forces(2)
    fp, _ = e.force_parts()
    want = _oracle_special_pair_force(oracle, s, ns, sp, (0.0, 0.0, 0.0), 2)
    assert systems.rel_rms(fp, want) < 1e-10
    e.close()


def _write_water_full(path, s):
    """A LAMMPS data file (atom_style full) of a systems.water dict."""
    n, nm = s["n"], s["n"] // 3
    lines = ["water", "", f"{n} atoms", f"{len(s['bonds'])} bonds", f"{len(s['angles'])} angles",
             "2 atom types", "1 bond types", "1 angle types", ""]
    for d, ax in enumerate("xyz"):
        lines.append(f"{float(s['lo'][d])!r} {float(s['hi'][d])!r} {ax}lo {ax}hi")
    lines += ["", "Masses", ""] + [f"{t + 1} {float(m)!r}" for t, m in enumerate(s["mass"])]
    lines += ["", "Pair Coeffs", ""] + [f"{t + 1} {float(e)!r} {float(g)!r}"
                                        for t, (e, g) in enumerate(zip(s["eps"], s["sigma"]))]
    lines += ["", "Bond Coeffs", "", "1 450.0 1.0", "", "Angle Coeffs", "", "1 55.0 109.47"]
    lines += ["", "Atoms # full", ""]
    for i in range(n):
        x, y, z = (repr(float(v)) for v in s["pos"][i])
        lines.append(f"{s['gid'][i] + 1} {i // 3 + 1} {s['type'][i] + 1} {float(s['q'][i])!r} "
                     f"{x} {y} {z}")
    lines += ["", "Velocities", ""]
    for i in range(n):
        lines.append(f"{s['gid'][i] + 1} " + " ".join(repr(float(v)) for v in s["vel"][i]))
    lines += ["", "Bonds", ""] + [f"{k + 1} 1 {a + 1} {b + 1}" for k, (a, b) in enumerate(s["bonds"])]
    lines += ["", "Angles", ""] + [f"{k + 1} 1 {a + 1} {b + 1} {c + 1}"
                                   for k, (a, b, c) in enumerate(s["angles"])]
    path.write_text("\n".join(lines) + "\n")


WATER_JSON = """{
  "init_configuration": {"read_data": {"file": "water.data", "unit": "REAL",
                                       "atom_style": "full", "velocity_type": "NONE"}},
  "hyper_parameters": {
    "force_field": {"type": "CVFF", "mixing_rule": "arithmetic"},
    "neighbor": {"type": "RBL", "cut_off": 10, "r_core": 6.5, "neighbor_sample_num": 100,
                 "energy_rbl_flag": "no", "skin": 2},
    "coulomb": {"type": "RBE", "alpha": 0.09, "coulomb_sample_num": 300,
                "energy_rbe_flag": "no", "random_seed": 21},
    "extend": {"fix_shake": true, "special_bonds": [0, 0, 0]}},
  "execution": {"ensemble": "NVT", "temperature": [298, 298, 100],
                "temp_ctrl_type": "NOSE_HOOVER", "timestep": 2.0, "num_steps": 1000}
}"""


def test_water_config_from_files(cuda, rbx, tmp_path, water3k):
    """RBMD's water workload from its own kind of input (CVFF, RBL + RBE,
    fix_shake, special_bonds [0 0 0], NVT Nose-Hoover, REAL units, a full-style
    data file): the engine built from the files steps exactly like the one
    assembled from arrays with set_shake / set_special / set_nose_hoover."""
    s = water3k
    _write_water_full(tmp_path / "water.data", s)
    (tmp_path / "rbmd.json").write_text(WATER_JSON)
    a = rbx.Engine.from_files(tmp_path / "rbmd.json", precision=rbx.MIXED)
    assert a.shake_status() == (3000, 0)
    b = rbx.Engine(s, precision=rbx.MIXED, seed=21)
    b.set_shake(s["clusters"][:, [0, 1, 2]], 1.0, 109.47)
    ns, sp = rbx.special_build(s["n"], s["bonds"], s["angles"])
    b.set_special(ns, sp, (0.0, 0.0, 0.0))
    b.compute_forces(0)
    p = s["params"]
    b.set_nose_hoover(298.0, 298.0, 100.0, num_steps=1000, kb=p["kb"], mvv2e=p["mvv2e"],
                      tdof=2.0 * s["n"] - 3)
    a.compute_forces(0)
    for e in (a, b):
        e.step(12)
    sa, sb = a.get_state(), b.get_state()
    for key in ("pos", "vel", "force"):
        assert np.array_equal(sa[key], sb[key]), key
    assert a.thermostat()["temperature"] == b.thermostat()["temperature"]
    err, rv = _water_geometry(s, sa["pos"], sa["vel"])
    assert err < 1e-4 and rv < 1e-9
    a.close()
    b.close()


def test_autotune_keeps_parity_and_caches(cuda, rbx, oracle, sys4k):
    """The autotuner picks valid launch shapes, the forces with them still
    match the oracle, a second engine of the same size bin takes the cached
    choice without timing, and the tuned step graph equals the tuned
    launch-by-launch step bit for bit."""
    s = sys4k
    box = oracle.Box.make(s["lo"], s["hi"])
    m = oracle.rbe_sample_philox(box, 0.16, 100, 7, 0)
    import __graft_entry__ as ge

    want = ge._oracle_forces(s, m)
    e = rbx.Engine(s, precision=rbx.MIXED, seed=4)
    e.set_k_samples(*m)
    e.compute_forces(0)
    t = e.autotune(force=True)
    assert t["cache_hit"] == 0 and t["rho_kpt"] in (1, 2, 4, 8)
    assert t["force_block"] in (128, 256, 512) and t["rbl_waves"] in (2, 4, 8, 16)
    assert t["rho_blocks"] >= 1 and t["rho_ms"] <= t["rho_ms_default"] + 1e-6
    assert t["rbl_ms"] <= t["rbl_ms_default"] + 1e-6
    assert systems.rel_rms(e.get_state()["force"], want) < 1e-5
    e2 = rbx.Engine(s, precision=rbx.MIXED, seed=4)
    e2.compute_forces(0)
    t2 = e2.autotune()
    assert t2["cache_hit"] == 1
    for k in ("rho_kpt", "rho_blocks", "force_block", "rbl_waves"):
        assert t2[k] == t[k], k
    runs = []
    for graph in (True, False):
        x = rbx.Engine(s, precision=rbx.MIXED, seed=9)
        x.set_step_graph(graph)
        x.compute_forces(0)
        x.autotune()
        x.step(10)
        runs.append(x.get_state())
        x.close()
    for key in ("pos", "vel", "force"):
        assert np.array_equal(runs[0][key], runs[1][key]), key
    e.close()
    e2.close()
