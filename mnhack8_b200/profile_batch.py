"""A short run of the batched mixed-precision solver for profiling: one N=128
instance (the bench problem: lognormal k sigma 1, correlation 8 elements,
Gaussian IC sigma 0.15, dt 1e-4) for a few steps to rtol 1e-8.

    python -m mnhack8_b200.profile_batch [--N 128] [--steps 2]
"""
import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=128)
    ap.add_argument("--steps", type=int, default=2)
    a = ap.parse_args(argv)
    from mnhack8_b200 import _lib
    from mnhack8_b200.fields import FieldSpec, make_field
    N = a.N
    k, r, _ = make_field(FieldSpec(n=N, model="lognormal", mu=0.0, sigma=1.0, L=8.0 / N, seed=1))
    b = _lib.Batch(rtol=1e-8)
    s = b.add(N, 1e-4, k.ravel(), r.ravel(), T0=_lib.gaussian_ic(N, 0.15), steps=a.steps)
    ms = 0.0
    while True:
        n, t = b.step()
        if not n:
            break
        ms += t
    inf = b.info(s)
    b.close()
    print(json.dumps({"N": N, "steps": a.steps, "ms": ms, "inner_iters": inf["inner_iters"],
                      "outer_iters": inf["outer_iters"], "rel_residual": inf["rel_residual"]}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
