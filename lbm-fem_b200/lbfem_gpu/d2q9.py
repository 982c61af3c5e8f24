"""D2Q9 lattice in numpy: velocities, weights, moments and the second-order
equilibrium, in the numbering of include/lbfem/d2q9.h:15-55 (Lee & Lin 2001,
Fig. 1 / Eq. (3)). Lattice units: |e_x| = 1, c_s^2 = 1/3."""
import numpy as np

Q = 9
CS2 = 1.0 / 3.0
# d2q9.h:18-19
E = np.array([[0, 0], [1, 0], [1, 1], [0, 1], [-1, 1], [-1, 0], [-1, -1], [0, -1], [1, -1]], dtype=np.float64)
# d2q9.h:21-22
W = np.array([4 / 9, 1 / 9, 1 / 36, 1 / 9, 1 / 36, 1 / 9, 1 / 36, 1 / 9, 1 / 36], dtype=np.float64)


def moments(f):
    """rho, ux, uy of populations f with shape (9, ...) (d2q9.h:30-41)."""
    rho = f.sum(axis=0)
    mx = np.tensordot(E[:, 0], f, axes=(0, 0))
    my = np.tensordot(E[:, 1], f, axes=(0, 0))
    return rho, mx / rho, my / rho


def equilibrium(rho, ux, uy):
    """feq with shape (9, ...) (d2q9.h:44-55)."""
    rho, ux, uy = np.broadcast_arrays(np.asarray(rho, float), np.asarray(ux, float), np.asarray(uy, float))
    uu = ux * ux + uy * uy
    out = np.empty((Q,) + rho.shape)
    for a in range(Q):
        eu = E[a, 0] * ux + E[a, 1] * uy
        out[a] = W[a] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu)
    return out


def lattice_tensor(*index):
    """sum_a w_a e_a[i1] ... e_a[ik] (d2q9.h:69-77)."""
    s = 0.0
    for a in range(Q):
        t = W[a]
        for i in index:
            t *= E[a, i]
        s += t
    return s
