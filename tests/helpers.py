import numpy as np


def rel_l2(a: np.ndarray, ref: np.ndarray) -> float:
    """||a - ref||_2 / ||ref||_2 (0 when both are zero)."""
    den = float(np.sqrt(np.sum(np.abs(ref) ** 2)))
    num = float(np.sqrt(np.sum(np.abs(a - ref) ** 2)))
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return num / den


def mode_fields(mode: int):
    """(E names, H names, D names, B names) carried by a mode."""
    from fdtd_b200.problem import TE, TM
    if mode == TM:
        return ["Ez"], ["Hx", "Hy"], ["Dz"], ["Bx", "By"]
    if mode == TE:
        return ["Ex", "Ey"], ["Hz"], ["Dx", "Dy"], ["Bz"]
    return ["Ex", "Ey", "Ez"], ["Hx", "Hy", "Hz"], ["Dx", "Dy", "Dz"], ["Bx", "By", "Bz"]
