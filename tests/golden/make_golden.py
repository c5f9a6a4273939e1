"""Generates the golden fixtures in this folder from the reference itself.

Each scenario of tests/scenarios.py.REFERENCE_SCENARIOS is run through
oracle/_ref/ref_runner -- the reference's own update functors compiled from
its headers (oracle/Makefile) -- and the final fields are stored as
<name>.npz. Run from the repository root, where the reference tree exists:

    make -C oracle REF=$FDTD_REFERENCE_DIR ref && python tests/golden/make_golden.py [scenario ...]

(with scenario names, only those scenarios' fixtures are rewritten)

Each scenario of FORWARD_SCENARIOS, with its Lorentz materials replaced
(scenarios.forward_materials), is run the same way and then the reference's
forward material updates (XUpdate<Mode, ft, true>) of E and of H are applied
to every interior cell: <name>_fwd.npz.

It also writes config_*.xml: the reference's own XML writers (print_summary
of MaterialMap, PMLOptions, BoundaryOptions) run on config_spec.txt by
oracle/_ref/ref_xml, the fixtures of the config loaders.
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


def write_config_fixtures(out_dir):
    """config_{materials,pml,boundaries}.xml: the reference's own
    print_summary writers (oracle/_ref/ref_xml) on config_spec.txt."""
    import subprocess
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_xml")
    text = subprocess.run([exe, os.path.join(out_dir, "config_spec.txt")], check=True, capture_output=True,
                          text=True).stdout
    sections, cur = {}, None
    for line in text.splitlines():
        if line.startswith("=== "):
            cur = line[4:]
            sections[cur] = []
        else:
            sections[cur].append(line)
    for name, lines in sections.items():
        with open(os.path.join(out_dir, f"config_{name}.xml"), "w") as f:
            f.write("\n".join(lines) + "\n")
        print("config", name)


def main(names=None):
    """All fixtures, or (names given) only those scenarios' .npz files."""
    out_dir = os.path.dirname(os.path.abspath(__file__))
    if not names:
        write_config_fixtures(out_dir)
    for make in scenarios.REFERENCE_SCENARIOS:
        if names and make.__name__ not in names:
            continue
        p = make()
        ref = pyoracle.run_reference(p)
        arrays = {k: ref[k] for k in KEEP + pyoracle.PSI_NAMES + pyoracle.SURFACE_NAMES if np.any(ref[k] != 0)}
        np.savez_compressed(os.path.join(out_dir, p.name + ".npz"), steps=p.steps, **arrays)
        print(p.name, sorted(arrays))
    for make in scenarios.FORWARD_SCENARIOS:
        p = scenarios.forward_materials(make)
        if names and p.name not in names:
            continue
        ref = pyoracle.run_reference(p, explicit=True)
        arrays = {k: ref[k] for k in KEEP + pyoracle.PSI_NAMES if np.any(ref[k] != 0)}
        np.savez_compressed(os.path.join(out_dir, p.name + ".npz"), steps=p.steps, **arrays)
        print(p.name, sorted(arrays))


if __name__ == "__main__":
    main(sys.argv[1:])
