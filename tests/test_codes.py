"""Hypergraph-product codes and the check-list file format (CPU)."""
import numpy as np

from joint_bp_plus_pp_b200.codes import (hgp_code, hypergraph_product, random_regular_ldpc, read_checks,
                                         to_check_lists, write_checks)


def test_random_regular_ldpc_degrees_and_seed():
    H = random_regular_ldpc(48, 3, 4, seed=5)
    assert H.shape == (36, 48)
    assert (H.sum(0) == 3).all() and (H.sum(1) == 4).all()
    assert (random_regular_ldpc(48, 3, 4, seed=5) == H).all()
    assert not (random_regular_ldpc(48, 3, 4, seed=6) == H).all()


def test_hypergraph_product_is_a_css_code():
    H1 = random_regular_ldpc(32, 3, 4, seed=1)
    HX, HZ = hypergraph_product(H1)
    assert HX.shape == (24 * 32, 32 * 32 + 24 * 24) == HZ.shape
    assert not ((HX.astype(np.int64) @ HZ.T.astype(np.int64)) % 2).any()
    assert (HX.sum(1) == 7).all() and (HZ.sum(1) == 7).all()
    assert set(np.unique(HX.sum(0))) == {3, 4} and set(np.unique(HZ.sum(0))) == {3, 4}


def test_quantum_sizes_of_the_mixed_workload():
    for nc, nq in ((32, 1600), (48, 3600), (64, 6400), (96, 14400)):
        assert hgp_code(nc, 0)[0] == nq


def test_check_file_round_trip(tmp_path):
    n, xo, xv, zo, zv = hgp_code(32, 3)
    f = tmp_path / "code.checks"
    write_checks(f, n, xo, xv, zo, zv)
    n2, xo2, xv2, zo2, zv2 = read_checks(f)
    assert n2 == n and all((a == b).all() for a, b in ((xo, xo2), (xv, xv2), (zo, zo2), (zv, zv2)))


def test_oracle_decodes_a_hypergraph_product_code(oracle):
    """The oracle's generic check-list path on an irregular code: k = n - rank_x - rank_z, and a
    low-weight error is decoded."""
    from oracle_bind import Oracle
    n, xo, xv, zo, zv = hgp_code(32, 1)
    o = Oracle.from_checks(n, xo, xv, zo, zv)
    k = n - o.bx.rank - o.bz.rank
    assert k > 0
    err = np.zeros(n, np.uint8)
    err[[5, 300, 1200]] = [1, 2, 3]
    sx, sz = o.syndrome(err)
    r = o.decode(sx, sz, 0.02, 50, enable_pp=False)
    assert r["syndrome_ok"] == 1
