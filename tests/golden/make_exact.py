"""Writes tests/golden/exact_riemann.npz with the reference's own exact Riemann solver (python/fenice/exact.py of the
reference, imported from its source tree):

    python tests/golden/make_exact.py /path/to/fenice

Inputs: Sod's problem and 24 seeded pairs drawn as the batched shock tubes draw them (rho ~ U[0.1, 1], p ~ U[0.05, 1],
u ~ U[-1, 1]), sampled at 257 points of [0, 1] at t = 0.15. The fixture pins oracle/exact_riemann.py."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "python"))
    from fenice import exact  # the reference's module

    rng = np.random.default_rng(77)
    pairs = [((1.0, 0.0, 1.0), (0.125, 0.0, 0.1))]
    for _ in range(24):
        pairs.append(((rng.uniform(0.1, 1), rng.uniform(-1, 1), rng.uniform(0.05, 1)), (rng.uniform(0.1, 1), rng.uniform(-1, 1), rng.uniform(0.05, 1))))
    x = (np.arange(257) + 0.5) / 257
    out = {"x": x, "t": np.array(0.15), "left": np.array([p[0] for p in pairs]), "right": np.array([p[1] for p in pairs])}
    sol = np.empty((len(pairs), 3, x.size))
    for k, (lft, rgt) in enumerate(pairs):
        sol[k] = exact.riemann(x, 0.15, left=lft, right=rgt, gamma=1.4, x0=0.5)
    out["solution"] = sol
    np.savez_compressed(os.path.join(HERE, "exact_riemann.npz"), **out)
    print(f"{len(pairs)} problems written")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FENICE_REF", ""))
