"""CPU oracle (test infrastructure only) for the pixel-space products, radial
sums and harmonic weightings: a numpy restatement of the reference's Cython
kernels, one function per kernel, each citing the lines it follows.

Pinned against the reference's own kernels compiled from its sources by
oracle/build_ref.sh into oracle/_ref (tests/test_pixel_oracle.py); the GPU
tests compare libpscuda with this module and, where oracle/_ref is present,
with the compiled reference as well.
"""
import numpy as np


# ----------------------------------------------------------- tauNL_utils.pyx
def apply_fl_weights(ls, flX, h_lm, weight):
    """tauNL_utils.pyx:80-98: out[r, lm] = w Sum_X flX[l, X, r] h[X, lm] over X = T only
    (npol 1) or X = T, E (npol 2 or 3: the reference ignores a third column)."""
    npol = flX.shape[1]
    nlm = h_lm.shape[1]
    f = flX[np.asarray(ls)[:nlm]]  # [nlm, npol, nr]
    if npol > 1:
        out = np.einsum("lxr,xl->rl", f[:, :2], h_lm[:2])
    else:
        out = f[:, 0, :].T * h_lm[0][None, :]
    return out * weight


def multiply(m1, m2, m3):  # tauNL_utils.pyx:103-113
    return m1 * m2 * m3


def multiply_asym(m1A, m1B, m3A, m3B):  # :116-126
    return m1A * (2 * m1B * m3A + m1A * m3B)


def multiplyC(m1, m2, m3c):  # :129-139
    return m1 * m2 * m3c


def multiplyC_asym(m1A, m1B, m3cA, m3cB):  # :142-152
    return m1A * (2 * m1B * m3cA + m1A * m3cB)


def multiplyCC(m1, m2, m3c):  # :155-165
    return m1 * (m2 ** 2 + np.real(m3c * np.conj(m3c)))


def multiplyCC_asym(m1A, m1B, m2A, m2B, m3cA, m3cB):  # :168-178
    return 2 * m1A * (m2A * m2B + np.real(np.conj(m3cA) * m3cB)) + m1B * (m2A * m2A + np.real(m3cA * np.conj(m3cA)))


def multiply2(B1, B2, C1, C2):  # :181-191
    return B1 * B2 + np.real(C1 * np.conj(C2))


def multiply2R(A, B):  # :194-204
    return A * B


def multiply2C(Ac, B):  # :207-217
    return Ac * B


def radial_sum(ls, lm_map, r_weights, flXs):
    """tauNL_utils.pyx:220-237: out[X, lm] = Sum_r lm_map[r, lm] flXs[l, X, r] w_r."""
    nr, nlm = lm_map.shape
    f = flXs[np.asarray(ls)[:nlm]][:, :, :nr]  # [nlm, npol, nr]
    return np.einsum("rl,lxr,r->xl", lm_map, f, np.asarray(r_weights)[:nr])


def radial_sum_spin1(ls, lm_map, r_weights, flXs):
    """tauNL_utils.pyx:240-255."""
    return 0.5 * radial_sum(ls, lm_map[0] - lm_map[1], r_weights, flXs)


def _rsum(w, per_r):
    return float(np.sum(np.asarray(w)[:len(per_r)] * per_r))


def gnl_loc_sum(w, P, Q):  # :260-272
    return _rsum(w, np.sum(P ** 3 * Q, axis=1))


def gnl_loc_disc_sum(w, P1, P2, Q1, Q2):  # :275-287
    return _rsum(w, np.sum(P1 ** 2 * P2 * Q2 + P2 ** 2 * P1 * Q1, axis=1))


def gnl_con_sum(w, R):  # :290-302
    return _rsum(w, np.sum(R ** 4, axis=1))


def gnl_con_disc_sum(w, R1, R2):  # :305-317
    return _rsum(w, np.sum(R1 ** 2 * R2 ** 2, axis=1))


def gnl_dotdot_sum(w, tau, A):  # :320-332
    return _rsum(np.asarray(tau) ** 4 * np.asarray(w), np.sum(A ** 4, axis=1))


def gnl_dotdot_disc_sum(w, tau, A1, A2):  # :335-347
    return _rsum(np.asarray(tau) ** 4 * np.asarray(w), np.sum(A1 ** 2 * A2 ** 2, axis=1))


def gnl_dotdel_sum(w, tau, A, B, C):  # :350-362
    return _rsum(np.asarray(tau) ** 2 * np.asarray(w), np.sum(A ** 2 * (B ** 2 + np.real(C * np.conj(C))), axis=1))


def gnl_dotdel_disc_sum(w, tau, A1, A2, B1, B2, C1, C2):  # :365-377
    return _rsum(np.asarray(tau) ** 2 * np.asarray(w),
                 np.sum(A1 * A2 * (B1 * B2 + np.real(C1 * np.conj(C2))), axis=1))


def gnl_deldel_sum(w, B, C):  # :380-392
    return _rsum(w, np.sum((B ** 2 + np.real(C * np.conj(C))) ** 2, axis=1))


def gnl_deldel_disc_sum(w, B1, B2, B3, B4, C1, C2, C3, C4):  # :395-405
    return _rsum(w, np.sum((B1 * B2 + np.real(C1 * np.conj(C2))) * (B3 * B4 + np.real(C3 * np.conj(C4))), axis=1))


# ----------------------------------------------------------- ideal_fisher.pyx
def r2c(re, im):  # ideal_fisher.pyx:18-26
    return re + 1j * im


def r2cstar(re, im):  # :30-38
    return re - 1j * im


def multiplyRC(R, C):  # :52-60
    return R * C


def multiplyRCstar(R, C, fac):  # :64-72
    return fac * R * np.conj(C)


def multiplyRC_sym(R, C, R2, C2):  # :76-84
    return R * C + R2 * C2


def multiplyRCstar_sym(R, C, R2, C2, fac):  # :88-96
    return fac * (R * np.conj(C) + R2 * np.conj(C2))


def multiplyRR(a, b):  # :100-108
    return a * b


def multiplyRR_sym(a, b, ab, bb):  # :112-120
    return a * b + ab * bb


def _phi_one(U, V):
    out = 2 * U[0] * np.conj(V[0])
    if U.shape[0] == 3:
        out = out + (U[1] * np.conj(V[1]) - np.conj(U[1]) * V[2]) + 1j * (U[2] * np.conj(V[1]) + np.conj(U[2]) * V[2])
    return out


def lens_phi_sum(U, V):  # :124-139
    return _phi_one(U, V)


def lens_phi_sum_sym(U1, U2, V1, V2):  # :142-157
    return _phi_one(U1, V2) + _phi_one(U2, V1)


def outer_product(Qa, Qb, sym=False):
    """ideal_fisher.pyx:423-460."""
    c = np.array([[1, 0, 0, -3], [0, 1, -3, 0], [0, -3, 9, 0], [-3, 0, 0, 9]], dtype=np.float64)
    f = np.real(np.einsum("paj,pq,qbj->ab", np.conj(Qa), c, Qb)) / 24. / 48.
    if sym:
        f = np.triu(f) + np.triu(f, 1).T
    return f
