"""Generates the golden fixtures in this folder from the reference itself.

Each scenario of tests/scenarios.py.REFERENCE_SCENARIOS is run through
oracle/_ref/ref_runner -- the reference's own update functors compiled from
its headers (oracle/Makefile) -- and the final fields are stored as
<name>.npz. Run from the repository root, where the reference tree exists:

    make -C oracle _ref/ref_runner && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import pyoracle  # noqa: E402
import scenarios  # noqa: E402

KEEP = ["Dx", "Dy", "Dz", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "Hx", "Hy", "Hz", "Px", "Py", "Pz", "Jx", "Jy", "Jz"]


def main():
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for make in scenarios.REFERENCE_SCENARIOS:
        p = make()
        ref = pyoracle.run_reference(p)
        arrays = {k: ref[k] for k in KEEP + pyoracle.PSI_NAMES + pyoracle.SURFACE_NAMES if np.any(ref[k] != 0)}
        np.savez_compressed(os.path.join(out_dir, p.name + ".npz"), steps=p.steps, **arrays)
        print(p.name, sorted(arrays))


if __name__ == "__main__":
    main()
