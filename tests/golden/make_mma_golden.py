"""Generate tests/golden/mma.npz: the reference optimiser's own density
filter and MMA update (mma_optimizer.py density_filter_fast :370-388,
mma_update :589-718, imported from the reference checkout) on seeded inputs,
so that coldplate_b200.mma is pinned without the reference at test time.

    REF_DIR=<reference checkout> python tests/golden/make_mma_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ref = os.environ["REF_DIR"]
    sys.dont_write_bytecode = True
    sys.path.insert(0, ref)
    import mma_optimizer as mo
    rng = np.random.default_rng(11)
    M, N = 24, 40
    x0 = rng.uniform(0.0, 1.0, (M, N))
    filt = {f"filter_r{r}": mo.density_filter_fast(x0, r) for r in (1.5, 3.0)}
    xmin, xmax = np.zeros((M, N)), np.ones((M, N))
    xmax[:2] = 0.0
    xmax[-2:] = 0.0
    x = np.clip(x0, xmin, xmax)
    st = mo.MMAState(M * N)
    out = {"x0": x0, "xmin": xmin, "xmax": xmax, **filt}
    for k in range(4):
        df0 = rng.standard_normal(M * N) * (1.0 + k)
        dg = np.ones(M * N) / (M * N)
        g = float(x.mean() - 0.4)
        xn = mo.mma_update(x.ravel(), 0.0, df0, g, dg, xmin.ravel(), xmax.ravel(), st, move_limit=0.2)
        out[f"df0_{k}"], out[f"g_{k}"], out[f"x_{k + 1}"] = df0, g, xn
        x = xn.reshape(M, N)
    np.savez_compressed(os.path.join(HERE, "mma.npz"), **out)
    print("wrote", os.path.join(HERE, "mma.npz"))


if __name__ == "__main__":
    main()
