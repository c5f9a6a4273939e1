"""Readers of the reference's XML configuration files, host side.

The reference reads three documents with tinyxml2:

* a material map (``MaterialMap::readXML``, include/MaterialMap.hpp:236-282):
  ``<MaterialMap>`` of ``<Item>`` each holding an ``<Identifier>`` and a
  ``<MaterialPair>`` (``MaterialPair::readXML``, :134-181) whose
  ``<Electric>`` and ``<Magnetic>`` children name one dispersion each, read
  by that dispersion's storage (``ConstantStorage::readXML``
  include/DispersiveMaterials.hpp:411-427, ``VacuumStorage`` :466-471,
  ``LorentzStorage`` :822-865, ``DrudeStorage`` :1117-1147);
* the CPML options (``PMLOptions::readXML``, include/PML.hpp:215-281): the
  layer depth ``<N>`` and a 0/1 flag per face under ``<X>``, ``<Y>``,
  ``<Z>`` / ``<MIN>``, ``<MAX>``;
* the boundary options (``BoundaryOptions::readXML``,
  include/BoundaryUpdates.hpp:163-223): a boundary name per face.

The same documents are what the reference's ``print_summary`` writers emit.
These readers accept them and map them onto :class:`fdtd_b200.problem`
objects. Defaults follow the reference's constructors: every face PEC in
``BoundaryOptions`` (:59-65), N = 10 and no CPML face in ``PMLOptions``
(:152-156; the reference leaves the MAX flags unset, here they are off).
Unknown names raise :class:`ValueError`, as ``MapNameTo`` throws
(include/FDTDConstants.hpp:107-124); dispersions and boundaries that the GPU
path does not implement raise :class:`UnsupportedConfig`.
"""
from __future__ import annotations

import os
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from typing import Dict, Optional, Tuple, Union

from . import problem as P

# NameArray<Detail::Dispersion> (include/DispersiveMaterials.hpp:2059-2071)
DISPERSIONS = ("Vacuum", "Constant", "Conductive", "Drude", "FluidDrude", "Lorentz", "MagnetizedDrude",
               "SelfMagnetizedDrude", "MagnetizedFluidDrude", "SelfMagnetizedFluidDrude", "MultiCoefficient",
               "Anisotropic")
# NameArray<Boundary> (include/BoundaryUpdates.hpp:28-36)
BOUNDARIES = ("Periodic", "BlochPeriodic", "PEC", "PMC", "Symmetric", "Antisymmetric", "Parallel", "NONE")
_BOUNDARY_KIND = {"Periodic": "periodic", "PEC": "pec", "PMC": "pmc", "Symmetric": "symmetric",
                  "Antisymmetric": "antisymmetric"}
_AXES = ("X", "Y", "Z")
_SIDES = ("MIN", "MAX")


class UnsupportedConfig(ValueError):
    """A valid reference configuration the GPU path does not implement."""


Source = Union[str, bytes, os.PathLike]


def _root(source: Source) -> ET.Element:
    """The document element of an XML file path or an XML text."""
    if isinstance(source, bytes):
        return ET.fromstring(source)
    s = os.fspath(source)
    if s.lstrip().startswith("<"):
        return ET.fromstring(s)
    return ET.parse(s).getroot()


def _number(e: ET.Element) -> float:
    # the reference streams the first child's text into a double
    return float((e.text or "").split()[0])


def _flag(e: ET.Element) -> bool:
    # `ss >> bool` reads 0 or 1 (no boolalpha)
    tok = (e.text or "").split()
    if not tok or tok[0] not in ("0", "1"):
        raise ValueError(f"<{e.tag}> holds {e.text!r}: a 0/1 flag is expected")
    return tok[0] == "1"


@dataclass
class Dispersion:
    """One side of a MaterialPair: the dispersion's name and its numbers."""

    name: str
    K: float = 1.0
    Delta: float = 1.0
    Freq: float = 0.0
    Gamma: float = 0.0


def _dispersion(side: ET.Element) -> Dispersion:
    kids = list(side)
    if not kids:
        raise ValueError(f"<{side.tag}> names no dispersion")
    node = kids[0]
    if node.tag not in DISPERSIONS:
        raise ValueError(f"unknown dispersion {node.tag!r}")
    d = Dispersion(node.tag)
    for c in node:
        if c.tag == "Constant":
            d.K = _number(c)
        elif c.tag in ("Delta", "Freq", "Gamma"):
            setattr(d, c.tag, _number(c))
    return d


def material_from_pair(electric: Dispersion, magnetic: Dispersion) -> P.Material:
    """The Material of an (Electric, Magnetic) dispersion pair. Electric:
    Vacuum, Constant, Drude or Lorentz; magnetic: Vacuum or Constant. The
    reference reads a Lorentz <Delta> but its update does not use it
    (lorentz::LorentzUpdate::implicit_update, DispersiveMaterials.hpp:711-735,
    takes delta and never reads it), so the pole strength stays 1 here too."""
    if magnetic.name == "Vacuum":
        mu = 1.0
    elif magnetic.name == "Constant":
        mu = magnetic.K
    else:
        raise UnsupportedConfig(f"magnetic dispersion {magnetic.name!r} is not implemented on the GPU path")
    e = electric
    if e.name == "Vacuum":
        return P.Material(P.VACUUM, 1.0, mu, [])
    if e.name == "Constant":
        return P.Material(P.CONSTANT, e.K, mu, [])
    if e.name == "Drude":
        return P.Material(P.DRUDE, e.K, mu, [(1.0, e.Freq, e.Gamma)])
    if e.name == "Lorentz":
        return P.Material(P.LORENTZ, e.K, mu, [(1.0, e.Freq, e.Gamma)])
    raise UnsupportedConfig(f"electric dispersion {e.name!r} is not implemented on the GPU path")


def read_material_pair(node: ET.Element) -> P.Material:
    """A <MaterialPair> element (MaterialPair::readXML)."""
    el = mg = None
    for c in node:
        if c.tag == "Electric":
            el = _dispersion(c)
        elif c.tag == "Magnetic":
            mg = _dispersion(c)
    if el is None or mg is None:
        raise ValueError("a MaterialPair needs <Electric> and <Magnetic>")
    return material_from_pair(el, mg)


def read_material_map(source: Source) -> Dict[str, P.Material]:
    """{identifier: Material} of a <MaterialMap> document, ordered by
    identifier as the reference's std::map; the first of repeated
    identifiers is kept, as std::map::insert does."""
    root = _root(source)
    out: Dict[str, P.Material] = {}
    for item in root:
        if item.tag != "Item":
            continue
        ident, pair = None, None
        for c in item:
            if c.tag == "Identifier":
                ident = (c.text or "").strip()
            elif c.tag == "MaterialPair":
                pair = c
        if ident is None or pair is None:
            raise ValueError("an <Item> needs <Identifier> and <MaterialPair>")
        if ident not in out:
            out[ident] = read_material_pair(pair)
    return dict(sorted(out.items()))


@dataclass
class PMLOptions:
    """PMLOptions: the CPML depth and the faces that carry it."""

    N: int = 10
    faces: Dict[Tuple[int, int], bool] = field(default_factory=lambda: {(a, s): False for a in range(3)
                                                                        for s in range(2)})

    def apply(self, p: P.Problem) -> P.Problem:
        """Set N-cell CPML on the flagged faces of p's axes."""
        for (a, s), on in self.faces.items():
            if on and a < p.dim:
                p.pml[(a, s)] = int(self.N)
        return p


def read_pml_options(source: Source) -> PMLOptions:
    root = _root(source)
    po = PMLOptions()
    for c in root:
        if c.tag == "N":
            n = _number(c)
            if n != int(n) or n < 0:
                raise ValueError(f"<N> must be a cell count, got {c.text!r}")
            po.N = int(n)
        elif c.tag in _AXES:
            a = _AXES.index(c.tag)
            for m in c:
                if m.tag in _SIDES:
                    po.faces[(a, _SIDES.index(m.tag))] = _flag(m)
    return po


@dataclass
class BoundaryOptions:
    """BoundaryOptions: a boundary name per face (reference names)."""

    faces: Dict[Tuple[int, int], str] = field(default_factory=lambda: {(a, s): "PEC" for a in range(3)
                                                                       for s in range(2)})

    def apply(self, p: P.Problem) -> P.Problem:
        """Set the boundary conditions of p's axes. NONE and Parallel faces
        (a rank boundary, which the z-slab decomposition exchanges) get no
        condition; BlochPeriodic is not implemented."""
        for (a, s), name in self.faces.items():
            if a >= p.dim:
                continue
            if name == "BlochPeriodic":
                raise UnsupportedConfig("BlochPeriodic boundaries are not implemented on the GPU path")
            kind = _BOUNDARY_KIND.get(name)
            if kind is None:
                p.boundaries.pop((a, s), None)
            else:
                p.boundaries[(a, s)] = kind
        return p


def read_boundary_options(source: Source) -> BoundaryOptions:
    root = _root(source)
    bo = BoundaryOptions()
    for c in root:
        if c.tag not in _AXES:
            continue
        a = _AXES.index(c.tag)
        for m in c:
            if m.tag not in _SIDES:
                continue
            kids = list(m)
            name = kids[0].tag if kids else (m.text or "").strip()
            if name not in BOUNDARIES:
                raise ValueError(f"unknown boundary {name!r}")
            bo.faces[(a, _SIDES.index(m.tag))] = name
    return bo


def materials_for(mmap: Dict[str, P.Material], names) -> list:
    """The material table of a Problem whose cell ids index `names`."""
    return [mmap[n] for n in names]
