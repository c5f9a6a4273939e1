"""XML configuration loaders (fdtd_b200/config_xml.py) against the
reference's own writers.

The reference reads its material map, CPML options and boundary options with
tinyxml2, which is not available here; its print_summary writers produce the
same documents. tests/golden/config_*.xml are that writer's output for
tests/golden/config_spec.txt (made by tests/golden/make_golden.py through
oracle/_ref/ref_xml), and the loaders must read back the spec's values.
Where the reference tree is present the writer also runs live on random
values (printed with 6 significant digits)."""
import math
import os
import subprocess

import numpy as np
import pytest

import pyoracle

import scenarios
from fdtd_b200 import config_xml as C
from fdtd_b200 import problem as P

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
ROOT = os.path.dirname(HERE)


def _spec(path):
    """Materials, PML and boundary rows of a ref_xml spec file."""
    tok = open(path).read().split()
    mats, pml, bc = [], None, None
    q = 0
    while q < len(tok):
        if tok[q] == "nmat":
            n = int(tok[q + 1])
            q += 2
            for _ in range(n):
                name = tok[q]
                ek, K, de, f, g, mk, mK = int(tok[q + 1]), *map(float, tok[q + 2:q + 6]), int(tok[q + 6]), float(
                    tok[q + 7])
                mats.append((name, ek, K, de, f, g, mk, mK))
                q += 8
        elif tok[q] == "pml":
            pml = (int(tok[q + 1]), [int(x) for x in tok[q + 2:q + 8]])
            q += 8
        elif tok[q] == "bc":
            bc = [int(x) for x in tok[q + 1:q + 7]]
            q += 7
        else:
            raise AssertionError(tok[q])
    return mats, pml, bc


def _expected(row):
    name, ek, K, de, f, g, mk, mK = row
    mu = 1.0 if mk == 0 else mK
    if ek == 0:
        return P.Material(P.VACUUM, 1.0, mu, [])
    if ek == 1:
        return P.Material(P.CONSTANT, K, mu, [])
    if ek == 2:
        return P.Material(P.DRUDE, K, mu, [(1.0, f, g)])
    return P.Material(P.LORENTZ, K, mu, [(1.0, f, g)])


def _check(spec_path, mat_xml, pml_xml, bc_xml):
    mats, pml, bc = _spec(spec_path)
    got = C.read_material_map(mat_xml)
    assert list(got) == sorted(r[0] for r in mats)
    for row in mats:
        assert got[row[0]] == _expected(row), row[0]
    po = C.read_pml_options(pml_xml)
    assert po.N == pml[0]
    assert [po.faces[(a, s)] for a in range(3) for s in range(2)] == [bool(x) for x in pml[1]]
    bo = C.read_boundary_options(bc_xml)
    assert [bo.faces[(a, s)] for a in range(3) for s in range(2)] == [C.BOUNDARIES[k] for k in bc]


def test_golden_reference_writer_output_reads_back():
    _check(os.path.join(GOLDEN, "config_spec.txt"), os.path.join(GOLDEN, "config_materials.xml"),
           os.path.join(GOLDEN, "config_pml.xml"), os.path.join(GOLDEN, "config_boundaries.xml"))


@pytest.mark.skipif(not pyoracle.reference_tree_present(), reason="reference tree not present")
def test_reference_writer_live_random_values(tmp_path):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={pyoracle.REFERENCE_DIR}", "_ref/ref_xml"],
                   check=True)
    rng = np.random.default_rng(7)
    six = lambda v: float(f"{v:.6g}")  # the writer's default stream precision
    lines = ["nmat 8"]
    for q in range(8):
        ek = q % 4
        K, de = six(rng.uniform(1, 12)), six(rng.uniform(0.1, 2))
        f, g = six(10 ** rng.uniform(12, 16)), six(10 ** rng.uniform(10, 14))
        mk = q % 2
        mK = six(rng.uniform(1, 4))
        lines.append(f"m{q} {ek} {K!r} {de!r} {f!r} {g!r} {mk} {mK!r}")
    flags = rng.integers(0, 2, 6)
    lines.append("pml 9 " + " ".join(str(x) for x in flags))
    kinds = rng.choice([0, 2, 3, 4, 5, 6, 7], 6)
    lines.append("bc " + " ".join(str(x) for x in kinds))
    spec = tmp_path / "spec.txt"
    spec.write_text("\n".join(lines) + "\n")
    out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_xml"), str(spec)], check=True,
                         capture_output=True, text=True).stdout
    sec, cur = {}, None
    for line in out.splitlines():
        if line.startswith("=== "):
            cur = line[4:]
            sec[cur] = []
        else:
            sec[cur].append(line)
    _check(str(spec), *("\n".join(sec[k]) for k in ("materials", "pml", "boundaries")))


def test_defaults_follow_the_reference_constructors():
    po = C.read_pml_options("<PML><X><MIN>1</MIN></X></PML>")
    assert po.N == 10 and po.faces[(0, 0)] and not any(v for k, v in po.faces.items() if k != (0, 0))
    bo = C.read_boundary_options("<BoundaryConditions><Y><MAX>PMC</MAX></Y></BoundaryConditions>")
    assert bo.faces[(1, 1)] == "PMC"
    assert all(v == "PEC" for k, v in bo.faces.items() if k != (1, 1))


def test_errors():
    with pytest.raises(ValueError):
        C.read_boundary_options("<B><X><MIN>Mirror</MIN></X></B>")  # MapNameTo throws
    with pytest.raises(ValueError):
        C.read_material_map("<M><Item><Identifier>a</Identifier><MaterialPair><Electric><Glass/></Electric>"
                            "<Magnetic><Vacuum/></Magnetic></MaterialPair></Item></M>")
    with pytest.raises(C.UnsupportedConfig):
        C.read_material_map("<M><Item><Identifier>c</Identifier><MaterialPair><Electric><Conductive>"
                            "<Constant>1</Constant><Freq>5e12</Freq></Conductive></Electric>"
                            "<Magnetic><Vacuum/></Magnetic></MaterialPair></Item></M>")
    with pytest.raises(ValueError):
        C.read_pml_options("<PML><X><MIN>yes</MIN></X></PML>")
    p = scenarios.tm_cpml_sources()
    bo = C.read_boundary_options("<B><X><MIN>BlochPeriodic</MIN></X></B>")
    with pytest.raises(C.UnsupportedConfig):
        bo.apply(p)


def test_first_of_repeated_identifiers_wins():
    doc = ("<M>" + "".join(f"<Item><Identifier>a</Identifier><MaterialPair><Electric><Constant><Constant>{k}"
                           "</Constant></Constant></Electric><Magnetic><Vacuum/></Magnetic></MaterialPair></Item>"
                           for k in (2, 3)) + "</M>")
    assert C.read_material_map(doc)["a"].eps_inf == 2.0


def test_loaded_config_runs_like_the_hand_built_problem(oracle):
    """A TE problem set up from the golden XML (materials by name, CPML and
    faces) steps bit-identically to the same problem built by hand."""
    mmap = C.read_material_map(os.path.join(GOLDEN, "config_materials.xml"))
    po = C.read_pml_options(os.path.join(GOLDEN, "config_pml.xml"))
    bo = C.read_boundary_options(os.path.join(GOLDEN, "config_boundaries.xml"))
    names = ["air", "glass", "silver", "dye"]
    # 5 nm cells: the silver Drude (1.37e16 rad/s) needs wp*dt well below 1
    dt = P.courant_dt(5e-9, 0.99 / math.sqrt(2.0))

    def base():
        p = P.Problem(P.TE, (40, 44, 1), 5e-9, dt, name="te_from_xml")
        ids = np.zeros((1, 44, 40), np.uint8)
        ids[0, 10:18, 8:16] = 1
        ids[0, 22:30, 12:26] = 2
        ids[0, 32:36, 6:30] = 3
        p.ids = ids
        p.sources.append(P.Source(0, (20, 20, 0), P.gaussian_pulse(60, 20, 6), "E"))
        p.steps = 60
        return p

    a = base()
    a.materials = C.materials_for(mmap, names)
    po.apply(a)
    bo.apply(a)
    b = base()
    b.materials = [P.Material.vacuum(), P.Material.constant(2.25), P.Material.drude(1.5, 1.37e16, 1.1e14),
                   P.Material.lorentz(2.0, [(1.0, 3.1e15, 2.2e13)])]
    b.pml = {(0, 0): 12, (0, 1): 12, (1, 1): 12}
    b.boundaries = {(0, 0): "periodic", (0, 1): "periodic", (1, 0): "pec", (1, 1): "pmc"}
    assert a.pml == b.pml and a.boundaries == b.boundaries
    ga, gb = oracle.run_oracle(a), oracle.run_oracle(b)
    for n in ("Ex", "Ey", "Hz"):
        assert np.array_equal(ga.get(n), gb.get(n)), n


def test_cpp_readers_match_the_spec(tmp_path):
    """The C++ layer's readers (fdtd::xml in include/fdtd_b200.hpp) on the
    same golden documents give the same values; tests/cpp/config_xml.cpp also
    checks their errors. Compiled and run on the host, no GPU needed."""
    exe = str(tmp_path / "config_xml")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "cpp", "config_xml.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe] + [os.path.join(GOLDEN, f"config_{n}.xml") for n in ("materials", "pml", "boundaries")],
                         check=True, capture_output=True, text=True).stdout.splitlines()
    mats, pml, bc = _spec(os.path.join(GOLDEN, "config_spec.txt"))
    got = {}
    for line in out:
        f = line.split()
        if f[0] == "mat":
            got[f[1]] = P.Material(int(f[2]), float(f[3]), float(f[4]),
                                   [(1.0, float(f[6]), float(f[7]))] if int(f[5]) else [])
    assert sorted(got) == sorted(r[0] for r in mats)
    for row in mats:
        assert got[row[0]] == _expected(row), row[0]
    pml_line = [l for l in out if l.startswith("pml ")][0].split()
    assert int(pml_line[1]) == pml[0] and [int(x) for x in pml_line[2:]] == pml[1]
    bc_line = [l for l in out if l.startswith("bc ")][0].split()
    assert bc_line[1:] == [C.BOUNDARIES[k] for k in bc]
    assert [l for l in out if l.startswith("errors ")] == ["errors 31"]
