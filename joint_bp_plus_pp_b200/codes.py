"""Codes beyond the params-file APM construction: seeded random regular classical LDPC codes,
their hypergraph product (the mixed-size workload of quantum CSS codes with n from 1.6k to 14.4k),
and a plain sparse check-list file format.

Check-list file format (text):
    n mx mz
    mx lines: the variables of one X check (space separated, 0-based)
    mz lines: the variables of one Z check
"""
import numpy as np


def random_regular_ldpc(n, dv=3, dc=4, seed=0, max_tries=10000):
    """Parity-check matrix (m x n, m = n*dv/dc) with every column of weight dv and every row
    of weight dc, drawn by the configuration model from a seeded generator; draws with a
    repeated (row, column) pair are rejected and redrawn."""
    if (n * dv) % dc:
        raise ValueError("n * dv must be a multiple of dc")
    m = n * dv // dc
    rng = np.random.default_rng(seed)
    sockets = np.repeat(np.arange(n), dv)
    for _ in range(max_tries):
        perm = rng.permutation(sockets)
        rows = perm.reshape(m, dc)
        if all(len(set(r)) == dc for r in rows):
            H = np.zeros((m, n), np.uint8)
            for i, r in enumerate(rows):
                H[i, r] = 1
            return H
    raise RuntimeError("no simple regular graph found")


def hypergraph_product(H1):
    """CSS code HX = [H1 (x) I_n | I_m (x) H1^T], HZ = [I_n (x) H1 | H1^T (x) I_m] of a classical
    m x n matrix H1: n_q = n^2 + m^2 qubits, m*n checks per side; with H1 (dv, dc)-regular
    every check has dv + dc variables and the variables have degree dv or dc."""
    H1 = np.asarray(H1, np.uint8)
    m, n = H1.shape
    In, Im = np.eye(n, dtype=np.uint8), np.eye(m, dtype=np.uint8)
    HX = np.concatenate([np.kron(H1, In), np.kron(Im, H1.T)], axis=1)
    HZ = np.concatenate([np.kron(In, H1), np.kron(H1.T, Im)], axis=1)
    return HX, HZ


def to_check_lists(H):
    """(offsets, variables) of a dense 0/1 check matrix, variables ascending per check."""
    off = [0]
    var = []
    for row in np.asarray(H):
        nz = np.nonzero(row)[0]
        var.extend(int(v) for v in nz)
        off.append(len(var))
    return np.asarray(off, np.int32), np.asarray(var, np.int32)


def hgp_code(n_classical, seed, dv=3, dc=4):
    """Check lists of the hypergraph product of a seeded random (dv, dc)-regular code:
    (n_q, x_off, x_var, z_off, z_var)."""
    HX, HZ = hypergraph_product(random_regular_ldpc(n_classical, dv, dc, seed))
    xo, xv = to_check_lists(HX)
    zo, zv = to_check_lists(HZ)
    return HX.shape[1], xo, xv, zo, zv


def write_checks(path, n, x_off, x_var, z_off, z_var):
    with open(path, "w") as f:
        f.write(f"{n} {len(x_off) - 1} {len(z_off) - 1}\n")
        for off, var in ((x_off, x_var), (z_off, z_var)):
            for c in range(len(off) - 1):
                f.write(" ".join(str(int(v)) for v in var[off[c]:off[c + 1]]) + "\n")


def read_checks(path):
    with open(path) as f:
        n, mx, mz = (int(t) for t in f.readline().split())
        lists = []
        for m in (mx, mz):
            off, var = [0], []
            for _ in range(m):
                var.extend(int(t) for t in f.readline().split())
                off.append(len(var))
            lists.append((np.asarray(off, np.int32), np.asarray(var, np.int32)))
    return n, lists[0][0], lists[0][1], lists[1][0], lists[1][1]
