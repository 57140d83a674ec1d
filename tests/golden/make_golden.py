"""Generate tests/golden/ref1d_pointwise.npz: outputs of the reference's own
shipped Model.H / Numerics.H (1-D SME level 0), compiled from the reference
tree into oracle/_ref/liboracle_ref.so, on seeded random inputs (wet, dry
and near-dry states).  Run in a container where the reference is mounted:

    make -C oracle ref REF=<reference source tree> && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle_py as O  # noqa: E402


def inputs(n=400, seed=7):
    rng = np.random.default_rng(seed)
    rows = []
    for t in range(n):
        wet = t % 4 != 0

        def st():
            b = rng.uniform(-0.5, 0.5)
            h = rng.uniform(0, 2) if wet else rng.choice([0.0, 1e-15, 1e-9, 1e-5, 0.005, 0.02, -1e-3])
            hu = rng.uniform(-2, 2) * (h if wet else 1.0)
            return [b, h, hu]

        qL, qR = st(), st()
        p = [9.81, rng.uniform(0.5, 2), rng.uniform(0, 1), rng.uniform(0, 1), rng.uniform(-0.1, 0.1)]
        aL = [0.0, 0.0, 0.0, rng.uniform(0, 2)]
        aR = [0.0, 0.0, 0.0, rng.uniform(0, 2)]
        nx = rng.choice([-1.0, 1.0])
        rows.append(qL + qR + aL + aR + p + [nx, rng.uniform(1e-4, 0.1)])
    return np.array(rows)


def evaluate(model, X, ref):
    out = {}
    for fn in O.FN:
        res = []
        for r in X:
            qL, qR, aL, aR, p, nx, s = r[0:3], r[3:6], r[6:10], r[10:14], r[14:19], r[19], r[20]
            res.append(O.pointwise(model, fn, qL, aL, p, np.array([nx, 0, 0]), qR, aR, s=s, ref=ref))
        out[fn] = np.array(res)
    return out


if __name__ == "__main__":
    X = inputs()
    out = evaluate("ref1d", X, ref=True)
    np.savez_compressed(os.path.join(HERE, "ref1d_pointwise.npz"), inputs=X, **out)
    print("wrote", os.path.join(HERE, "ref1d_pointwise.npz"), {k: v.shape for k, v in out.items()})
