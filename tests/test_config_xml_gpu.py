"""A grid configured from the reference's XML documents (materials with a
magnetic ConstantUpdate beside vacuum, Drude and Lorentz cells, CPML faces
and boundary faces) runs on the GPU as on the oracle: FP64 bit-identical, FP32
within 1e-4."""
import math
import os

import numpy as np
import pytest

from fdtd_b200 import config_xml as C
from fdtd_b200 import problem as P
from helpers import rel_l2

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _problem(mode):
    mmap = C.read_material_map(os.path.join(GOLDEN, "config_materials.xml"))
    names = ["air", "ferrite", "silver", "magdye"]
    three = mode == P.THREED
    n = (22, 20, 18) if three else (40, 44, 1)
    # 5 nm cells: the silver Drude (1.37e16 rad/s) needs wp*dt well below 1
    dt = P.courant_dt(5e-9, 0.99 / math.sqrt(3.0 if three else 2.0))
    p = P.Problem(mode, n, 5e-9, dt, name="from_xml")
    p.materials = C.materials_for(mmap, names)
    ids = np.zeros((n[2], n[1], n[0]), np.uint8)
    if three:
        ids[4:8, 5:9, 4:10] = 1
        ids[9:13, 10:15, 6:12] = 2
        ids[4:14, 3:6, 13:18] = 3
    else:
        ids[0, 10:18, 8:16] = 1
        ids[0, 22:30, 12:26] = 2
        ids[0, 32:36, 6:30] = 3
    p.ids = ids
    C.read_pml_options(os.path.join(GOLDEN, "config_pml.xml")).apply(p)
    p.pml = {k: 4 if three else v for k, v in p.pml.items()}
    C.read_boundary_options(os.path.join(GOLDEN, "config_boundaries.xml")).apply(p)
    c = tuple(x // 2 for x in n[:2]) + ((n[2] // 2,) if three else (0,))
    p.sources.append(P.Source(2 if mode != P.TE else 0, c, P.gaussian_pulse(50, 18, 6), "E"))
    p.steps = 50
    return p


@pytest.mark.parametrize("mode", [P.TE, P.TM, P.THREED])
def test_xml_configured_grid_matches_oracle(fdtd, oracle, mode):
    p = _problem(mode)
    o = oracle.run_oracle(p)
    names = {P.TE: ["Ex", "Ey", "Hz"], P.TM: ["Ez", "Hx", "Hy"], P.THREED: ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"]}[mode]
    g = fdtd.Grid.from_problem(p, "f64")
    g.step(p.steps)
    for n in names:
        assert np.array_equal(g.get(n), o.get(n)), n
    g = fdtd.Grid.from_problem(p, "f32")
    g.step(p.steps)
    for n in names:
        assert rel_l2(g.get(n), o.get(n)) <= 1e-4, n


@pytest.mark.parametrize("sweep", ["regs", "tma", "flat", "staged"])
def test_xml_configured_3d_every_sweep(fdtd, oracle, sweep):
    """mu_r != 1 through every 3D FP32 sweep implementation."""
    p = _problem(P.THREED)
    o = oracle.run_oracle(p)
    g = fdtd.Grid.from_problem(p, "f32")
    g.set_sweep_kernel(sweep)
    g.step(p.steps)
    assert g.error_flags() == 0
    for n in ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"]:
        assert rel_l2(g.get(n), o.get(n)) <= 1e-4, n
