"""Helpers shared by the tests: golden fixtures and error metrics."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("x", "y", "z", "m", "vx", "vy", "vz")
GOLDEN_SIZES = (1, 2, 33, 127, 1024)


def golden(n: int) -> dict:
    with np.load(os.path.join(GOLDEN, f"ref_ic_n{n}.npz")) as z:
        return {k: z[k] for k in z.files}


def state_of(g: dict) -> dict:
    return {k: np.array(g[k]) for k in FIELDS}


def vec_rel(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-body |a - b| / |b| over (3, n) vector blocks (vector norms)."""
    num = np.sqrt(((a - b) ** 2).sum(axis=0))
    den = np.sqrt((b ** 2).sum(axis=0))
    return num / np.where(den > 0, den, 1.0)


def derivs_rel(d: np.ndarray, ref: np.ndarray) -> tuple:
    """(max acc error, max jerk error), per-body vector-relative."""
    return vec_rel(d[:3], ref[:3]).max(), vec_rel(d[3:], ref[3:]).max()


def pos_of(s: dict) -> np.ndarray:
    return np.stack([s["x"], s["y"], s["z"]])


def vel_of(s: dict) -> np.ndarray:
    return np.stack([s["vx"], s["vy"], s["vz"]])
