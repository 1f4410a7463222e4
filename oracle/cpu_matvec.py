"""Multi-threaded CPU port of the reference's structured matvec (oracle; test infrastructure).

Restates mat_vec_node_basis_parallel_wcon (core/_ops.py:330-368): one parallel task per
node, summing over the node's elements the K0 rows of its local corner against the
element's unconstrained DOFs, constrained rows -> identity.  Node/element adjacency is
computed from the structured numbering (core/_geom.py:29-59) instead of the reference's
sorter/node_ids arrays.  Used only as the timed CPU baseline of bench.py (Numba parallel,
all host threads), never on the product path.
"""
import numpy as np
from numba import njit, prange

_C3 = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
               dtype=np.int64)


@njit(parallel=True, cache=True)
def matvec3d(nelx, nely, nelz, K0, E, u, cons, out, C3):
    nx, ny, nz = nelx + 1, nely + 1, nelz + 1
    for j in prange(ny):
        for i in range(nx):
            for k in range(nz):
                node = (j * nx + i) * nz + k
                for c in range(3):
                    out[node * 3 + c] = u[node * 3 + c] if cons[node * 3 + c] else 0.0
                for a in range(8):
                    ei, ej, ek = i - C3[a, 0], j - C3[a, 1], k - C3[a, 2]
                    if ei < 0 or ej < 0 or ek < 0 or ei >= nelx or ej >= nely or ek >= nelz:
                        continue
                    w = E[(ei * nely + ej) * nelz + ek]
                    for c in range(3):
                        if cons[node * 3 + c]:
                            continue
                        val = 0.0
                        for b in range(8):
                            nb = ((ej + C3[b, 1]) * nx + (ei + C3[b, 0])) * nz + ek + C3[b, 2]
                            for d in range(3):
                                kk = nb * 3 + d
                                if cons[kk]:
                                    continue
                                val += K0[a * 3 + c, b * 3 + d] * u[kk]
                        out[node * 3 + c] += val * w


def time_matvec(nel, K0, reps=2, seed=0):
    """Seconds per matvec at grid nel (3-D), random E in [0.2, 1], x=0 face constrained."""
    import time
    nelx, nely, nelz = nel
    n_nodes = (nelx + 1) * (nely + 1) * (nelz + 1)
    rng = np.random.default_rng(seed)
    E = rng.uniform(0.2, 1.0, nelx * nely * nelz)
    u = rng.standard_normal(n_nodes * 3)
    cons = np.zeros(n_nodes * 3, dtype=np.bool_)
    out = np.zeros(n_nodes * 3)
    matvec3d(2, 2, 2, K0, np.ones(8), np.zeros(81), np.zeros(81, np.bool_), np.zeros(81), _C3)  # JIT warm-up
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        matvec3d(nelx, nely, nelz, K0, E, u, cons, out, _C3)
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts)), out
