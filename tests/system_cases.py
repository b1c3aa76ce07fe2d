"""Raw systems of the reference's solver tests (crates/solidfem-solve/tests/solver/pcg.rs and
multigrid.rs), as scalar CSR arrays: the 1-D Laplacian, a 2x2 indefinite matrix and the block
chain of 3x3 couplings."""
import numpy as np


def csr(n, entries):
    """Scalar CSR from {(row, col): value}, each row's columns ascending."""
    rows = [[] for _ in range(n)]
    for (r, c), v in sorted(entries.items()):
        rows[r].append((c, v))
    starts = np.zeros(n + 1, dtype=np.uint64)
    cols, vals = [], []
    for r in range(n):
        for c, v in rows[r]:
            cols.append(c)
            vals.append(v)
        starts[r + 1] = len(cols)
    return starts, np.array(cols, dtype=np.uint32), np.array(vals, dtype=np.float64)


def laplacian(n):
    """The tridiagonal [-1, 2, -1] matrix (pcg.rs:8-20)."""
    e = {}
    for i in range(n):
        e[(i, i)] = 2.0
        if i + 1 < n:
            e[(i, i + 1)] = -1.0
            e[(i + 1, i)] = -1.0
    return csr(n, e)


def unit_end_load(n):
    b = np.zeros(n)
    b[n - 1] = 1.0
    return b


def indefinite():
    """Positive diagonal, eigenvalues 1 +/- 3 (pcg.rs:90-101)."""
    return csr(2, {(0, 0): 1.0, (1, 1): 1.0, (0, 1): 3.0, (1, 0): 3.0})


def block_chain(nodes, first_block=None):
    """Nodes in a chain with 4 I diagonal blocks and -I couplings, stored as whole 3x3 blocks
    (multigrid.rs:12-29); `first_block` replaces node 0's diagonal block."""
    e = {}
    for node in range(nodes):
        for other in (node - 1, node, node + 1):
            if 0 <= other < nodes:
                for p in range(3):
                    for q in range(3):
                        v = 0.0
                        if p == q:
                            v = 4.0 if other == node else -1.0
                        e[(3 * node + p, 3 * other + q)] = v
    if first_block is not None:
        for p in range(3):
            for q in range(3):
                e[(p, q)] = first_block[p][q]
    return csr(3 * nodes, e)


def positions_for(nodes):
    return np.array([[float(i), 0.0, 0.0] for i in range(nodes)])


def modes_for(size):
    """multigrid.rs:35-39: (i mod 7) + 1 for every (row, mode)."""
    return np.array([i % 7 + 1.0 for i in range(size * 6)])
