"""Pin the C restatement (oracle/alp_oracle.c) to the reference.

* against the golden fixtures written by the unmodified reference
  (tests/golden/make_golden.py) -- needs nothing but the fixtures;
* against the live compiled reference (oracle/_ref) on further seeded cases,
  when it is built;
* against the known answers the reference's own tests state.
"""
import numpy as np
import pytest

import golden_cases as G

MASK_BOOL = 1


def _replay_oracle(R, mats, name, c):
    ring = int(c["ring"])
    descr = int(c["descr"])
    vxm_form = int(c["vxm_form"])
    mat = mats[f"mat{ring}"]
    n = int(mat["n"])
    rp, col, vals, form, _ = G.gather_storage(R, mat, ring, vxm_form, descr)
    u, ua, v, va, um, uma, umc, vm, vma, vmc, vc = G.vector_args(c, n)
    rc, _ = R.mxv(ring, descr & ~G.TRANSPOSE, form, n, n, rp, col, vals, G.RING_TYPE[ring], u,
                  ua, um, uma, MASK_BOOL, umc, v, va, vc, vm, vma, MASK_BOOL, vmc)
    return rc, u, ua


@pytest.mark.parametrize("name", sorted(G.mxv_cases()[1].keys()))
def test_restatement_matches_reference_mxv_golden(oracle, name):
    mats, cases = G.mxv_cases()
    c = cases[name]
    rc, u, ua = _replay_oracle(oracle, mats, name, c)
    assert rc == 0
    ua_ref = c["ua_out"].astype(bool)
    if ua is not None:
        np.testing.assert_array_equal(ua.astype(bool), ua_ref)
    else:
        assert ua_ref.all()
    if G.RING_TYPE[int(c["ring"])] == G.FP64:
        # same storage order; the reference build contracts a*x+s into FMAs
        np.testing.assert_allclose(u[ua_ref], c["u_out"][ua_ref], rtol=1e-12, atol=0)
    else:
        np.testing.assert_array_equal(u[ua_ref], c["u_out"][ua_ref])


def test_restatement_matches_reference_cg_golden(oracle):
    g = G.load("cg_27pt_16.npz")["cg"]
    m = 16 ** 3
    rp, col, vals = oracle.coo_to_crs(m, g["I"], g["J"], g["V"], G.FP64)
    rc, x, it, res = oracle.cg(rp, col, vals, g["b"], np.zeros(m), 500, 1e-10)
    assert rc == 0
    assert it == int(g["iterations"])
    assert abs(res - float(g["residual"])) <= 1e-6 * float(g["residual"])
    np.testing.assert_allclose(x, g["x"], rtol=0, atol=1e-12)


def test_restatement_matches_reference_pagerank_golden(oracle):
    g = G.load("pagerank_rmat_s10.npz")["pr"]
    n = int(g["n"])
    rp, col, vals = oracle.coo_to_crs(n, g["I"], g["J"], g["V"], G.FP64)
    cp, row, tv = oracle.coo_to_crs(n, g["J"], g["I"], g["V"], G.FP64)
    rc, pr, it, res = oracle.pagerank(rp, col, vals, cp, row, tv, 0.85, 1e-9, 1000)
    assert rc == 0
    assert it == int(g["iterations"])
    np.testing.assert_allclose(pr, g["pr"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("ring", [0, 1, 2])
@pytest.mark.parametrize("scale", [6, 10])
def test_restatement_matches_live_reference(oracle, reference, ring, scale):
    from oracle.oracle import crs_to_coo
    t = G.RING_TYPE[ring]
    rp, col, vals = oracle.rmat(scale, edge_factor=8, seed=100 + scale, vtype=t)
    n = len(rp) - 1
    I, J = crs_to_coo(rp, col)
    v = oracle.values(n, t, 3, lo=0, hi=1000)
    u0 = oracle.values(n, t, 4, lo=0, hi=1000)
    rp2, col2, vals2 = oracle.coo_to_crs(n, I, J, vals, t)
    u = u0.copy()
    rc, _ = oracle.mxv(ring, 0, 2, n, n, rp2, col2, vals2, t, u, v=v)
    uref = u0.copy()
    rc2, _ = reference.mxv(ring, 0, 0, n, n, I, J, vals, uref, None, v)
    assert rc == rc2 == 0
    if t == G.FP64:
        np.testing.assert_allclose(u, uref, rtol=1e-12, atol=0)
    else:
        np.testing.assert_array_equal(u, uref)


@pytest.mark.parametrize("ring", [5, 6, 7])
@pytest.mark.parametrize("scale", [6, 10])
@pytest.mark.parametrize("vxm_form", [0, 1], ids=["mxv", "vxm"])
def test_new_rings_restatement_matches_live_reference(oracle, reference, ring, scale, vxm_form):
    """The Pregel degree and message rings and the switched (times, plus)
    ring: the C restatement against grb::mxv / grb::vxm of the compiled
    reference on the same triples."""
    t = G.RING_TYPE[ring]
    n, I, J, V, v, u0 = G.new_ring_case(oracle, ring, scale, 300 + scale)
    rp, col, vals = oracle.coo_to_crs(n, I, J, V, t)
    if vxm_form:
        rp, col, vals = oracle.transpose(n, n, rp, col, vals, t)
    u = u0.copy()
    rc, _ = oracle.mxv(ring, 0, 1 if vxm_form else 2, n, n, rp, col, vals, t, u, v=v)
    uref = u0.copy()
    rc2, _ = reference.mxv(ring, 0, vxm_form, n, n, I, J, V, uref, None, v)
    assert rc == rc2 == 0
    if t == G.FP64:
        np.testing.assert_allclose(u, uref, rtol=1e-12, atol=0)
    else:
        np.testing.assert_array_equal(u, uref)
    assert not np.array_equal(u, u0)


def test_generators_are_deterministic(oracle):
    a = oracle.rmat(8, seed=9)
    b = oracle.rmat(8, seed=9)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    rp, col, _ = a
    assert rp[0] == 0 and np.all(np.diff(rp) >= 0)
    # rows sorted and deduplicated
    for i in range(len(rp) - 1):
        seg = col[rp[i]:rp[i + 1]]
        assert np.all(np.diff(seg.astype(np.int64)) > 0)


def test_stencil_nnz_matches_reference_probe(oracle):
    # 27-point 32^3: nnz = 94^3 = 830,584 (measured on the reference build)
    I, _, _ = oracle.stencil_coo((32, 32, 32))
    assert len(I) == 94 ** 3
    I, _, _ = oracle.stencil_coo((64, 64, 64))
    assert len(I) == 6_859_000
