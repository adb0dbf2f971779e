"""Generates the golden fixtures of tests/golden (run: python tests/golden/make_golden.py).

hobson.json       closed forms of the Hobson solid harmonics Υ_n^m, Θ_n^m for n ≤ 2 at a few
                  points (the values test/test_harmonics.jl:21-23 of the reference checks)
direct_small.npz  1000 seeded uniform points, N(0,1) charges, and their FP64 direct-sum
                  potential and gradient (self excluded) computed here with numpy
                  (src/kernels.jl:479-487 restated: K = 1/(4π r), ∇ = −(t − s)/(4π r³))
"""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def hobson_closed_forms(x):
    x1, x2, z = x
    r2 = x1 * x1 + x2 * x2 + z * z
    r = np.sqrt(r2)
    w = complex(x1, x2)
    Y = {(0, 0): 1, (1, 0): z, (1, 1): -w / 2, (2, 0): (3 * z * z - r2) / 4, (2, 1): -z * w / 2, (2, 2): w * w / 8}
    T = {(0, 0): 1 / r, (1, 0): z / r ** 3, (1, 1): -w / r ** 3, (2, 0): (3 * z * z - r2) / r ** 5,
         (2, 1): -3 * z * w / r ** 5, (2, 2): 3 * w * w / r ** 5}
    for D in (Y, T):
        for (n, m) in list(D):
            if m > 0:
                D[(n, -m)] = (-1) ** m * np.conj(complex(D[(n, m)]))
    enc = lambda D: {f"{n},{m}": [complex(v).real, complex(v).imag] for (n, m), v in D.items()}
    return {"x": list(map(float, x)), "regular": enc(Y), "irregular": enc(T)}


def main():
    cases = [hobson_closed_forms(x) for x in ([0.3, -0.5, 0.4], [0.7, 0.2, -0.1], [-0.25, 0.6, 0.9])]
    with open(os.path.join(HERE, "hobson.json"), "w") as f:
        json.dump({"cases": cases}, f, indent=1)
    rng = np.random.default_rng(20240101)
    pts = rng.random((1000, 3))
    tau = rng.standard_normal(1000)
    d = pts[:, None, :] - pts[None, :, :]          # target − source
    r = np.sqrt((d * d).sum(-1))
    np.fill_diagonal(r, np.inf)
    ir = 1.0 / r
    pot = (ir * tau[None, :]).sum(1) / (4 * np.pi)
    grad = -((ir ** 3 * tau[None, :])[:, :, None] * d).sum(1) / (4 * np.pi)
    np.savez(os.path.join(HERE, "direct_small.npz"), points=pts, tau=tau, pot=pot, grad=grad)


if __name__ == "__main__":
    main()
