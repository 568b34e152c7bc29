"""Seeded inputs for the pixel-product / radial-sum parity tests (shared by the
CPU oracle pin and the GPU tests)."""
import numpy as np

# op -> input kinds ('r' float64 map, 'c' complex128 map), extra scalar (fac) or None
PRODUCTS = {
    "multiply": ("rrr", None), "multiply_asym": ("rrrr", None), "multiplyC": ("rrc", None),
    "multiplyC_asym": ("rrcc", None), "multiplyCC": ("rrc", None), "multiplyCC_asym": ("rrrrcc", None),
    "multiply2": ("rrcc", None), "multiply2R": ("rr", None), "multiply2C": ("cr", None),
    "multiplyRC": ("rc", None), "multiplyRCstar": ("rc", 0.75), "multiplyRC_sym": ("rcrc", None),
    "multiplyRCstar_sym": ("rcrc", -1.25), "multiplyRR": ("rr", None), "multiplyRR_sym": ("rrrr", None),
    "r2c": ("rr", None), "r2cstar": ("rr", None),
}
# tauNL_utils methods among the products (the rest are ideal_fisher module functions)
TAUNL_PRODUCTS = {"multiply", "multiply_asym", "multiplyC", "multiplyC_asym", "multiplyCC", "multiplyCC_asym",
                  "multiply2", "multiply2R", "multiply2C"}
# radial sums: kinds of the maps, whether tau is an argument
SUMS = {
    "gnl_loc_sum": ("rr", False), "gnl_loc_disc_sum": ("rrrr", False), "gnl_con_sum": ("r", False),
    "gnl_con_disc_sum": ("rr", False), "gnl_dotdot_sum": ("r", True), "gnl_dotdot_disc_sum": ("rr", True),
    "gnl_dotdel_sum": ("rrc", True), "gnl_dotdel_disc_sum": ("rrrrcc", True), "gnl_deldel_sum": ("rc", False),
    "gnl_deldel_disc_sum": ("rrrrcccc", False),
}


def maps(kinds, shape, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k in kinds:
        x = rng.normal(size=shape)
        if k == "c":
            x = x + 1j * rng.normal(size=shape)
        out.append(np.ascontiguousarray(x))
    return out


def lm_setup(lmax):
    """l_arr, m_arr of the m-major order and the int32 constructor arguments of tauNL_utils."""
    m = np.concatenate([np.full(lmax + 1 - mm, mm) for mm in range(lmax + 1)]).astype(np.int32)
    l = np.concatenate([np.arange(mm, lmax + 1) for mm in range(lmax + 1)]).astype(np.int32)
    return l, m


def taunl_args(nr, lmax):
    l, m = lm_setup(lmax)
    return (1, nr, l, m, 0, lmax, l, m, l, m, 1)
