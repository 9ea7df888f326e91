"""Start-up graph checks (orthogonality of Hx and Hz, Tanner-graph girth) on the host, against
the reference's known answers for the shipped code (its README start-up block and the golden
fixtures: Hx Hz^T = 0, girth 8 on both sides) and a plain breadth-first search on small
hypergraph-product codes."""
from collections import deque

import numpy as np
import pytest

from joint_bp_plus_pp_b200 import graph_checks
from joint_bp_plus_pp_b200.codes import hgp_code


def test_shipped_code_known_answers(oracle):
    xo, xv = oracle.checks(0)
    zo, zv = oracle.checks(1)
    r = graph_checks(9216, xo, xv, zo, zv)
    assert r == {"odd_pairs": 0, "girth_x": 8, "girth_z": 8}


def girth_bfs(n, off, var):
    """Shortest cycle of the Tanner graph by BFS from every node (small graphs only)."""
    m = len(off) - 1
    adj = [[] for _ in range(n + m)]
    for c in range(m):
        for e in range(off[c], off[c + 1]):
            adj[var[e]].append(n + c)
            adj[n + c].append(int(var[e]))
    best = None
    for s in range(n + m):
        dist, par = {s: 0}, {s: -1}
        q = deque([s])
        while q:
            u = q.popleft()
            for w in adj[u]:
                if w not in dist:
                    dist[w], par[w] = dist[u] + 1, u
                    q.append(w)
                elif w != par[u]:
                    cyc = dist[u] + dist[w] + 1
                    best = cyc if best is None else min(best, cyc)
    return best or 0


@pytest.mark.parametrize("nc,seed,dv,dc", [(8, 1, 3, 4), (12, 2, 3, 4), (8, 3, 3, 3)])
def test_hypergraph_products_against_bfs(nc, seed, dv, dc):
    n, xo, xv, zo, zv = hgp_code(nc, seed, dv=dv, dc=dc)
    r = graph_checks(n, xo, xv, zo, zv)
    assert r["odd_pairs"] == 0                      # a hypergraph product is a valid CSS code
    assert r["girth_x"] == girth_bfs(n, xo, xv) and r["girth_z"] == girth_bfs(n, zo, zv)


def test_non_orthogonal_pair_is_counted():
    # X check {0, 1} and Z check {1, 2} share one variable
    r = graph_checks(3, np.array([0, 2]), np.array([0, 1]), np.array([0, 2]), np.array([1, 2]))
    assert r["odd_pairs"] == 1 and r["girth_x"] == 0 and r["girth_z"] == 0
