"""Generate tests/golden/binning_ref.json from the reference's own Binning
(util/inc/WireCellUtil/Binning.h compiled from the reference source tree into
oracle/_ref/libref_binning.so by oracle/Makefile).

Run from the repository root:  python tests/golden/make_golden.py
The vectors pin the bin-index arithmetic (bin, edge, sample_bin_range) and
the Gaussian helpers the oracle and the GPU path restate."""

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402
import ctypes as C  # noqa: E402


def main():
    O.build()
    R = O.ref()
    if R is None:
        raise SystemExit("reference Binning harness not built (reference tree absent)")
    rng = np.random.default_rng(12345)
    cases = []
    # binnings of the kinds used on the path: readout ticks and impact bins
    binnings = [
        (6000, 0.0, 3.0e6),
        (10000, 0.0, 5.0e6),
        (9600, -2299.2, 2299.2),
        (8000, -1868.0 - 2.335, 1868.0 + 2.335),
        (20010, -3001.5, 3001.5),
        (20, -10.0, 10.0),
    ]
    for (n, lo, hi) in binnings:
        bs = R.ref_binsize(n, lo, hi)
        vals = list(lo + (hi - lo) * rng.uniform(-0.05, 1.05, 200))
        # values on and near bin edges
        for k in rng.integers(0, n + 1, 50):
            e = R.ref_edge(n, lo, hi, int(k))
            vals += [e, np.nextafter(e, -np.inf), np.nextafter(e, np.inf)]
        for v in vals:
            v = float(v)
            r = (C.c_int * 2)()
            w = float(v + abs(rng.normal(0, 3 * bs)))
            R.ref_sample_bin_range(n, lo, hi, v, w, r)
            cases.append(dict(n=n, lo=lo, hi=hi, v=v, w=w, bin=R.ref_bin(n, lo, hi, v), sbr=[r[0], r[1]]))
    edges = []
    for (n, lo, hi) in binnings:
        for k in [0, 1, n // 2, n - 1, n]:
            edges.append(dict(n=n, lo=lo, hi=hi, k=k, edge=R.ref_edge(n, lo, hi, k), center=R.ref_center(n, lo, hi, k)))
    gauss = []
    for (L, m, s) in [(0, 0, 1), (10, 0, 1), (5, 5, 30), (300, 5, 30), (-1.3, 0.2, 0.7)]:
        gauss.append(dict(kind="gcumulative", args=[L, m, s], value=R.ref_gcumulative(L, m, s)))
    for (a, b, m, s) in [(-1, 1, 0, 1), (1, -1, 0, 1), (0, 10, 0, 1), (-10, 0, 0, 1), (2.0, 2.5, 0.3, 0.4)]:
        gauss.append(dict(kind="gbounds", args=[a, b, m, s], value=R.ref_gbounds(a, b, m, s)))
    out = np.zeros(20)
    tot = R.ref_gaussian_sum(20, -10.0, 10.0, 0.0, 1.0, out.ctypes.data)
    gauss.append(dict(kind="gaussian", args=[20, -10.0, 10.0, 0.0, 1.0], value=tot, bins=out.tolist()))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "binning_ref.json")
    with open(path, "w") as f:
        json.dump(dict(source="util/inc/WireCellUtil/Binning.h (compiled from the reference tree)",
                       cases=cases, edges=edges, gauss=gauss), f)
    print("wrote", path, len(cases), "cases")


if __name__ == "__main__":
    main()
