"""He+ (ionic) channel operators for channel-resolved tSURFF (host setup).

Drop-in for the reference's ``Ionic`` (python/surface3d.py:8-48): the inner-electron
states are the sorted distinct (l, m) of electron 1 over the product channels (optionally
only the given m), and the object carries

* ``h0``: the ionic radial Hamiltonian, one block T + V_l per state, V_l = -2 cut / r +
  l (l + 1) / (2 r^2);
* ``P[axis]``: velocity-gauge dipole couplings i (p_axis) between states, built here as
  Kronecker products over (state, radial node): P = C (x) i[T, r] + (C o dL) (x) i / (2r),
  with C[a, b] the Cartesian component of <a| r_hat |b> (kept above 1e-14) and
  dL[a, b] = l_a (l_a + 1) - l_b (l_b + 1);
* ``matrix(A)`` = h0 + |A|^2 / 2 + sum_axis A_axis P[axis];
* ``final_states(labels)``: hydrogenic (Z = 2) bound states r R_nl(r) sqrt(w) on the complex
  grid in the state's block, one column per (n, l, m) label, and ``dual_final_states``
  their element-wise conjugates: on the exterior-scaled contour the bound functions are
  paired with the ket without conjugating the radial argument (python/surface3d.py:37-42),
  so the backward propagation starts from conj(phi).
"""
import numpy as np
from scipy.sparse import csr_matrix, diags, eye, kron

from .angular import cartesian, radial_hydrogen

PRUNE = 1e-14


def _selector(na, a):
    """na x na matrix with a single 1 at (a, a)."""
    return csr_matrix(([1.], ([a], [a])), shape=(na, na))


class Ionic:
    def __init__(self, h, magnetic_numbers=None):
        self.h = h
        inner = {a for a, _ in h.ch if magnetic_numbers is None or a[1] in magnetic_numbers}
        self.states = sorted(inner)
        self.index = {s: k for k, s in enumerate(self.states)}
        self.n, self.na = h.n, len(self.states)
        r = h.r
        self.T = h.grid.kinetic.tocsr()
        self.h0 = sum(kron(_selector(self.na, a), self.T + diags(-2 * h.cut / r + l * (l + 1) / (2 * r * r)))
                      for a, (l, _) in enumerate(self.states)).tocsr()
        # angular factors between states, per Cartesian axis
        C = np.array([[cartesian(a, b) for b in self.states] for a in self.states]).transpose(2, 0, 1)
        C = np.where(np.abs(C) > PRUNE, C, 0)
        ll1 = np.array([l * (l + 1) for l, _ in self.states], float)
        dL = ll1[:, None] - ll1[None, :]
        commutator = 1j * (self.T @ diags(r) - diags(r) @ self.T)
        centrifugal = diags(1j / (2 * r))
        self.P = [(kron(csr_matrix(C[axis]), commutator) + kron(csr_matrix(C[axis] * dL), centrifugal)).tocsr()
                  for axis in range(3)]
        self.identity = eye(self.n * self.na, format='csr')

    def final_states(self, labels):
        """Columns (na * n, len(labels)): label (n, l, m) in the (l, m) state's block."""
        r, w = self.h.r, self.h.grid.weights
        out = np.zeros((self.na, self.n, len(labels)), complex)
        for column, (n, l, m) in enumerate(labels):
            out[self.index[(l, m)], :, column] = r * radial_hydrogen(n, l, r) * np.sqrt(w)
        return out.reshape(self.na * self.n, len(labels))

    def dual_final_states(self, labels):
        return np.conj(self.final_states(labels))

    def matrix(self, A):
        """Ionic Hamiltonian at vector potential A (3 components), CSR."""
        H = self.h0 + (0.5 * float(np.dot(A, A))) * self.identity
        for component, P in zip(A, self.P):
            if component != 0:
                H = H + component * P
        return H.tocsr()
