"""FE-DVR radial grid with an optional exterior-complex-scaled Laguerre-Radau tail.

Host-side setup (runs once per grid).  Same construction and same outputs as the
reference's ``make_grid`` (python/fedvr.py:36-77), written independently:

* each finite element carries Gauss-Lobatto nodes of its own order; element
  kinetic blocks D^T W D / h are assembled into a global matrix with shared
  bridge nodes (python/fedvr.py:47-51);
* an infinite element starts at ``edges[-1]``: tail+1 Radau points of the
  generalised Laguerre weight (bridge node included), scaled by
  h = exp(i*theta)/alpha (python/fedvr.py:54-69), with the exact diagonal of the
  barycentric derivative (python/fedvr.py:63-66);
* the origin is Dirichlet; a finite outer end is Dirichlet too
  (python/fedvr.py:70-72);
* the kinetic matrix is normalised by the complex square root of the assembled
  weights, bridge node included (python/fedvr.py:73-74), and tiny entries are
  cleared at 1e-13.

The returned :class:`Grid` has the reference's field names, so code written
against the reference (``grid.r``, ``grid.weights``, ``grid.kinetic``,
``grid.interior_weights`` ...) keeps working.
"""
from dataclasses import dataclass
from functools import lru_cache

import numpy as np
from scipy.sparse import csr_matrix
from scipy.special import eval_laguerre, eval_legendre, roots_genlaguerre, roots_jacobi


def derivative(nodes):
    """Lagrange differentiation matrix on ``nodes`` (barycentric form).

    D[i, j] = (b_j / b_i) / (x_i - x_j) for i != j with barycentric weights
    b_i = 1 / prod_{k != i}(x_i - x_k); the diagonal is minus the row sum
    (python/fedvr.py:12-18)."""
    x = np.asarray(nodes, dtype=float)
    diff = x[:, None] - x[None, :]
    np.fill_diagonal(diff, 1.0)
    bary = 1.0 / np.prod(diff, axis=1)
    D = (bary[None, :] / bary[:, None]) / diff
    np.fill_diagonal(D, 0.0)
    np.fill_diagonal(D, -D.sum(axis=1))
    return D


@dataclass
class Grid:
    """Radial grid: nodes, assembled quadrature weights, normalised kinetic matrix
    (fields as in python/fedvr.py:20-28)."""
    r: np.ndarray
    weights: np.ndarray
    kinetic: csr_matrix
    real_radius: float
    order: int | tuple
    ecs_angle: float
    interior_weights: np.ndarray | None = None


@lru_cache(None)
def lobatto(order):
    """Gauss-Lobatto nodes/weights/derivative for ``order`` intervals
    (order+1 nodes; python/fedvr.py:30-34)."""
    inner = roots_jacobi(order - 1, 1, 1)[0]
    x = np.concatenate(([-1.0], inner, [1.0]))
    w = 2.0 / (order * (order + 1) * eval_legendre(order, x) ** 2)
    return x, w, derivative(x)


def _tail_element(tail, edge, ecs_angle, alpha):
    """Nodes, weights and kinetic block of the infinite Laguerre-Radau element."""
    y = np.concatenate(([0.0], roots_genlaguerre(tail, 1)[0]))
    wy = 1.0 / ((tail + 1) * eval_laguerre(tail, y) ** 2)
    h = np.exp(1j * ecs_angle) / alpha
    nodes = edge + h * y
    wp = wy * np.exp(y)
    dy = derivative(y)
    # Exact diagonal for the zeros of x*L^1_tail(x): 1/2 off the origin,
    # -tail/2 at the bridge node (avoids the cancellation of row sums).
    np.fill_diagonal(dy, 0.5)
    dy[0, 0] = -tail / 2.0
    d = dy * np.exp((y[None, :] - y[:, None]) / 2.0) - np.eye(tail + 1) / 2.0
    block = d.T @ (wp[:, None] * d) / (2.0 * h)
    return nodes, h * wp, block


def make_grid(edges, order=8, ecs_angle=0.0, tail=0, alpha=1.0):
    """Build the normalised FE-DVR grid (python/fedvr.py:36-77 semantics,
    including its argument validation and error messages)."""
    edges = np.asarray(edges, dtype=float)
    bad = (edges.ndim != 1 or len(edges) < 2 or not np.all(np.isfinite(edges)) or edges[0] != 0
           or np.any(np.diff(edges) <= 0) or tail < 0 or alpha <= 0)
    if bad:
        raise ValueError('increasing edges starting at 0; order>=2; tail>=0; alpha>0')
    nelem = len(edges) - 1
    orders = np.full(nelem, order) if np.ndim(order) == 0 else np.asarray(order)
    if orders.shape != (nelem,) or np.any(orders < 2) or np.any(orders != np.round(orders)):
        raise ValueError('one integer order >=2 is required per finite element')
    orders = orders.astype(int)
    if not 0 <= ecs_angle < np.pi / 2:
        raise ValueError('absorbing ECS angle must be in [0,pi/2)')
    if ecs_angle and not tail:
        raise ValueError('ECS requires a tail element')
    total = int(orders.sum()) + 1 + tail
    r = np.zeros(total, complex)
    weights = np.zeros(total, complex)
    K = np.zeros((total, total), complex)
    start = 0
    for e in range(nelem):
        p = int(orders[e])
        x, w, D = lobatto(p)
        a, b = edges[e], edges[e + 1]
        width = b - a
        sl = slice(start, start + p + 1)
        r[sl] = a + width * (x + 1.0) / 2.0
        weights[sl] += w * width / 2.0
        K[sl, sl] += D.T @ (w[:, None] * D) / width
        start += p
    interior = weights.real.copy()
    if tail:
        nodes, wt, block = _tail_element(tail, edges[-1], ecs_angle, alpha)
        sl = slice(total - tail - 1, total)
        r[sl] = nodes
        weights[sl] += wt
        K[sl, sl] += block
    keep = np.arange(1, total if tail else total - 1)
    r = r[keep]
    weights = weights[keep]
    K = K[np.ix_(keep, keep)]
    K /= np.sqrt(weights[:, None] * weights[None, :])
    K[np.abs(K) < 1e-13] = 0
    label = int(orders[0]) if np.ndim(order) == 0 else tuple(int(o) for o in orders)
    return Grid(r, weights, csr_matrix(K), float(edges[-1]), label, ecs_angle, interior[keep])
