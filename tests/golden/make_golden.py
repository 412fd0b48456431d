"""Generates the golden fixtures in tests/golden/ by running the reference
KORAL sources (compiled with oracle/ref/build_ref.sh from the read-only
reference tree).  Needs the reference tree; run from the repository root:

    python tests/golden/make_golden.py

Fixtures written:
  ot16_ref.npz   relativistic Orszag-Tang, 16x16, full u/p arrays after
                 steps 0, 1, 2, 10, 50 and the dt of every step
  ot128_ref.npz  the 128x128 benchmark problem: per-variable sums, sums of
                 absolute values and extrema of the domain u/p after steps
                 0, 1, 10, 100, the dt sequence, and the full state after
                 step 1 for the first 8 rows (bit-level spot check)
"""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.koral_oracle import REF_DIR, RefKoral  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def build(name, *flags):
    lib = os.path.join(REF_DIR, name)
    subprocess.check_call([os.path.join(ROOT, "oracle", "ref", "build_ref.sh"), "ORSZAGREL", lib, *flags])
    return name


def domain(R, a):
    ng = R.ng
    return a[0, ng:ng + R.ny, ng:ng + R.nx, :].copy()


def main():
    n16 = build("libkref_orszagrel_16.so", "-DTNX=16", "-DTNY=16")
    R = RefKoral(n16)
    R.init()
    snaps = {}
    dts = []
    for step in range(51):
        if step in (0, 1, 2, 10, 50):
            snaps[f"u_{step}"] = R.array("u").copy()
            snaps[f"p_{step}"] = R.array("p").copy()
        if step == 50:
            break
        R.step(1)
        dts.append(R.scalar("dt"))
    np.savez_compressed(os.path.join(OUT, "ot16_ref.npz"), dts=np.array(dts), **snaps)

    n128 = build("libkref_orszagrel_128.so")
    R = RefKoral(n128)
    R.init()
    out = {}
    dts = []
    for step in range(101):
        if step in (0, 1, 10, 100):
            for nm in ("u", "p"):
                d = domain(R, R.array(nm))
                out[f"{nm}_sum_{step}"] = d.sum(axis=(0, 1))
                out[f"{nm}_abs_{step}"] = np.abs(d).sum(axis=(0, 1))
                out[f"{nm}_min_{step}"] = d.min(axis=(0, 1))
                out[f"{nm}_max_{step}"] = d.max(axis=(0, 1))
            if step == 1:
                out["u_rows_1"] = domain(R, R.array("u"))[:8]
                out["p_rows_1"] = domain(R, R.array("p"))[:8]
        if step == 100:
            break
        R.step(1)
        dts.append(R.scalar("dt"))
    np.savez_compressed(os.path.join(OUT, "ot128_ref.npz"), dts=np.array(dts), **out)
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
