"""Shared helpers of the parity tests (oracle = CPU restatement in oracle/)."""
import numpy as np

from coldplate_b200 import cases

FIELD_NAMES = ("u", "v", "p", "uStar", "vStar", "pStar", "dE", "dN")


def small_cases():
    """Small versions of the three single-field workloads."""
    return {
        "straight": cases.straight_channel(16, 48),
        "network": cases.random_network(48, 96, seed=3),
        "density": cases.density_field(40, 80, seed=1),
    }


def oracle_for(case, prec="f64", **over):
    from oracle import Oracle
    prm = case.params(**over)
    return Oracle(prec, prm, cellType=case.cellType, hy=case.hy, hx=case.hx, U=case.U, Ht=case.Ht)


def gpu_for(case, **over):
    from coldplate_b200 import Simple
    prm = case.params(**over)
    return Simple(cellType=case.cellType, **prm)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    if nb == 0.0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / nb)
