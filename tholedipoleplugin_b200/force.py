"""Python mirror of the plugin's TholeDipoleForce API and its XML form.

:class:`TholeDipoleForce` has the method names, argument order, enumerator
values and defaults of aehogan/tholedipoleplugin
openmmapi/include/TholeDipoleForce.h:54-428 and openmmapi/src/TholeDipoleForce.cpp
(NoCutoff, Mutual, B-spline order 5, cutoff 1 nm, Ewald tolerance 1e-4,
60 iterations, target 1e-5, OPT4 extrapolation coefficients).  The plugin's
SWIG module still describes the bond-force template it was copied from, so
this is the Python layer the force actually needs.

:func:`serialize` / :func:`deserialize` write and read the element and
attribute structure of the plugin's XML proxy
(serialization/src/TholeDipoleForceProxy.cpp:44-183, version 1): force-level
properties, ExtrapolationCoefficients/Coefficient(c), Particles/Particle with a
Dipole(x, y, z) child and CovalentMaps/CovalentMap(type)/Atom(index).
Attributes are written in name order; floats use the shortest repr that
round-trips.

:class:`Context` is the evaluation side: positions and box in, energy, forces
and the dipole/potential/moment queries out, through the CUDA kernel.
"""
from __future__ import annotations

import copy
import xml.etree.ElementTree as ET
from typing import List, Optional, Sequence

import numpy as np

from .systems import TholeSystem

OPT4 = [-0.154, 0.017, 0.658, 0.474]


class _Particle:
    __slots__ = ("charge", "dipole", "polarizability", "thole", "axisType", "z", "x", "y", "covalent")

    def __init__(self, charge, dipole, polarizability, thole, axisType, z, x, y):
        self.charge = float(charge)
        self.dipole = [float(dipole[0]), float(dipole[1]), float(dipole[2])]
        self.polarizability = float(polarizability)
        self.thole = float(thole)
        self.axisType, self.z, self.x, self.y = int(axisType), int(z), int(x), int(y)
        self.covalent: List[List[int]] = [[], [], [], []]


class TholeDipoleForce:
    NoCutoff, PME = 0, 1
    Direct, Mutual, Extrapolated = 0, 1, 2
    ZThenX, Bisector, ZBisect, ThreeFold, ZOnly, NoAxisType, LastAxisTypeIndex = 0, 1, 2, 3, 4, 5, 6
    Covalent12, Covalent13, Covalent14, Covalent15, CovalentEnd = 0, 1, 2, 3, 4

    def __init__(self):
        self._method = self.NoCutoff
        self._polarization = self.Mutual
        self._cutoff = 1.0
        self._alpha, self._nx, self._ny, self._nz = 0.0, 0, 0, 0
        self._bspline = 5
        self._max_iter = 60
        self._target = 1e-5
        self._ewald_tol = 1e-4
        self._extrap = list(OPT4)
        self._group = 0
        self._particles: List[_Particle] = []

    # -- force-level settings -------------------------------------------------------
    def getForceGroup(self) -> int:
        return self._group

    def setForceGroup(self, g: int) -> None:
        self._group = int(g)

    def getNumParticles(self) -> int:
        return len(self._particles)

    def getNonbondedMethod(self) -> int:
        return self._method

    def setNonbondedMethod(self, method: int) -> None:
        if method < 0 or method > 1:
            raise ValueError("TholeDipoleForce: Illegal value for nonbonded method")
        self._method = int(method)

    def getPolarizationType(self) -> int:
        return self._polarization

    def setPolarizationType(self, t: int) -> None:
        self._polarization = int(t)

    def getCutoffDistance(self) -> float:
        return self._cutoff

    def setCutoffDistance(self, d: float) -> None:
        self._cutoff = float(d)

    def getPMEParameters(self):
        return self._alpha, self._nx, self._ny, self._nz

    def setPMEParameters(self, alpha, nx, ny, nz) -> None:
        self._alpha, self._nx, self._ny, self._nz = float(alpha), int(nx), int(ny), int(nz)

    def getPmeBSplineOrder(self) -> int:
        return self._bspline

    def getMutualInducedMaxIterations(self) -> int:
        return self._max_iter

    def setMutualInducedMaxIterations(self, n: int) -> None:
        self._max_iter = int(n)

    def getMutualInducedTargetEpsilon(self) -> float:
        return self._target

    def setMutualInducedTargetEpsilon(self, eps: float) -> None:
        self._target = float(eps)

    def getExtrapolationCoefficients(self) -> List[float]:
        return list(self._extrap)

    def setExtrapolationCoefficients(self, c: Sequence[float]) -> None:
        self._extrap = [float(x) for x in c]

    def getEwaldErrorTolerance(self) -> float:
        return self._ewald_tol

    def setEwaldErrorTolerance(self, tol: float) -> None:
        self._ewald_tol = float(tol)

    def usesPeriodicBoundaryConditions(self) -> bool:
        return self._method == self.PME

    # -- particles --------------------------------------------------------------------
    def addParticle(self, charge, molecularDipole, polarizability, tholeDamping, axisType=5, multipoleAtomZ=-1,
                    multipoleAtomX=-1, multipoleAtomY=-1) -> int:
        self._particles.append(_Particle(charge, molecularDipole, polarizability, tholeDamping, axisType,
                                         multipoleAtomZ, multipoleAtomX, multipoleAtomY))
        return len(self._particles) - 1

    def getParticleParameters(self, index: int):
        p = self._particles[index]
        return p.charge, list(p.dipole), p.polarizability, p.thole, p.axisType, p.z, p.x, p.y

    def setParticleParameters(self, index, charge, molecularDipole, polarizability, tholeDamping, axisType,
                              multipoleAtomZ, multipoleAtomX, multipoleAtomY) -> None:
        cov = self._particles[index].covalent
        self._particles[index] = _Particle(charge, molecularDipole, polarizability, tholeDamping, axisType,
                                           multipoleAtomZ, multipoleAtomX, multipoleAtomY)
        self._particles[index].covalent = cov

    def setCovalentMap(self, index: int, typeId: int, covalentAtoms: Sequence[int]) -> None:
        self._particles[index].covalent[typeId] = [int(a) for a in covalentAtoms]

    def getCovalentMap(self, index: int, typeId: int) -> List[int]:
        return list(self._particles[index].covalent[typeId])

    def getCovalentMaps(self, index: int) -> List[List[int]]:
        return [list(c) for c in self._particles[index].covalent]

    # -- bridge to the kernels -----------------------------------------------------------
    def toSystem(self, positions, box=None, masses=None) -> TholeSystem:
        n = len(self._particles)
        P = self._particles
        b = np.zeros(3) if box is None else np.asarray(box, dtype=np.float64).reshape(-1)
        if b.size == 9:
            b = b.reshape(3, 3).diagonal().copy()
        return TholeSystem(
            positions=np.asarray(positions, dtype=np.float64).reshape(n, 3),
            charges=np.array([p.charge for p in P]), dipoles=np.array([p.dipole for p in P]).reshape(n, 3),
            polarizabilities=np.array([p.polarizability for p in P]), tholes=np.array([p.thole for p in P]),
            axis=np.array([[p.axisType, p.z, p.x, p.y] for p in P], dtype=np.int32).reshape(n, 4),
            cov12=[list(p.covalent[0]) for p in P], cov13=[list(p.covalent[1]) for p in P],
            method=self._method, box=b, cutoff=self._cutoff, ewald_tolerance=self._ewald_tol,
            polarization=self._polarization, target_eps=self._target, max_iter=self._max_iter,
            extrap=list(self._extrap), masses=None if masses is None else np.asarray(masses, dtype=np.float64))


# ---------------------------------------------------------------------------
# XML (TholeDipoleForceProxy structure, version 1).
# ---------------------------------------------------------------------------
def _fmt(v) -> str:
    return repr(float(v)) if isinstance(v, float) else str(v)


def _el(tag, parent=None, **attrs):
    e = ET.Element(tag) if parent is None else ET.SubElement(parent, tag)
    for k in sorted(attrs):
        e.set(k, _fmt(attrs[k]))
    return e


def serialize(force: TholeDipoleForce) -> str:
    a, nx, ny, nz = force.getPMEParameters()
    root = _el("Force", type="TholeDipoleForce", version=1, forceGroup=force.getForceGroup(),
               nonbondedMethod=force.getNonbondedMethod(), polarizationType=force.getPolarizationType(),
               cutoffDistance=force.getCutoffDistance(), ewaldErrorTolerance=force.getEwaldErrorTolerance(),
               mutualInducedMaxIterations=force.getMutualInducedMaxIterations(),
               mutualInducedTargetEpsilon=force.getMutualInducedTargetEpsilon(),
               pmeBSplineOrder=force.getPmeBSplineOrder(), alpha=float(a), nx=nx, ny=ny, nz=nz)
    ex = _el("ExtrapolationCoefficients", root)
    for c in force.getExtrapolationCoefficients():
        _el("Coefficient", ex, c=float(c))
    parts = _el("Particles", root)
    for i in range(force.getNumParticles()):
        q, d, pol, th, t, z, x, y = force.getParticleParameters(i)
        p = _el("Particle", parts, charge=float(q), polarizability=float(pol), tholeDamping=float(th), axisType=t,
                multipoleAtomZ=z, multipoleAtomX=x, multipoleAtomY=y)
        _el("Dipole", p, x=float(d[0]), y=float(d[1]), z=float(d[2]))
        maps = _el("CovalentMaps", p)
        for j, atoms in enumerate(force.getCovalentMaps(i)):
            if atoms:  # empty lists are not written (TholeDipoleForceProxy.cpp:99-109)
                m = _el("CovalentMap", maps, type=j)
                for k in atoms:
                    _el("Atom", m, index=k)
    ET.indent(root, space="\t")
    return '<?xml version="1.0" ?>\n' + ET.tostring(root, encoding="unicode") + "\n"


def deserialize(text: str) -> TholeDipoleForce:
    root = ET.fromstring(text)
    if root.get("version") != "1":
        raise ValueError("Unsupported version number")
    f = TholeDipoleForce()
    f.setForceGroup(int(root.get("forceGroup")))
    f.setNonbondedMethod(int(root.get("nonbondedMethod")))
    f.setPolarizationType(int(root.get("polarizationType")))
    f.setCutoffDistance(float(root.get("cutoffDistance")))
    f.setEwaldErrorTolerance(float(root.get("ewaldErrorTolerance")))
    f.setMutualInducedMaxIterations(int(root.get("mutualInducedMaxIterations")))
    f.setMutualInducedTargetEpsilon(float(root.get("mutualInducedTargetEpsilon")))
    f.setPMEParameters(float(root.get("alpha")), int(root.get("nx")), int(root.get("ny")), int(root.get("nz")))
    f.setExtrapolationCoefficients([float(c.get("c")) for c in root.find("ExtrapolationCoefficients")])
    for p in root.find("Particles"):
        d = p.find("Dipole")
        i = f.addParticle(float(p.get("charge")), [float(d.get("x")), float(d.get("y")), float(d.get("z"))],
                          float(p.get("polarizability")), float(p.get("tholeDamping")), int(p.get("axisType")),
                          int(p.get("multipoleAtomZ")), int(p.get("multipoleAtomX")), int(p.get("multipoleAtomY")))
        for m in p.find("CovalentMaps"):
            f.setCovalentMap(i, int(m.get("type")), [int(a.get("index")) for a in m])
    return f


# ---------------------------------------------------------------------------
# Evaluation.
# ---------------------------------------------------------------------------
class Context:
    """Positions/box plus a CUDA kernel for one TholeDipoleForce, with the
    queries of the plugin's Force/ForceImpl (getInducedDipoles, ...)."""

    def __init__(self, force: TholeDipoleForce, positions, box=None, masses=None, precision="mixed",
                 solver="cg"):
        from .kernel import CudaCalcTholeDipoleForceKernel
        self.force = force
        self.masses = None if masses is None else np.asarray(masses, dtype=np.float64)
        self._system = force.toSystem(positions, box, masses)
        self.kernel = CudaCalcTholeDipoleForceKernel(self._system, precision=precision, solver=solver)

    def setPositions(self, positions) -> None:
        self._system.positions = np.asarray(positions, dtype=np.float64).reshape(-1, 3)

    def setPeriodicBoxVectors(self, a, b, c) -> None:
        self.kernel.setBox(np.array([a, b, c], dtype=np.float64))

    def getState(self, getEnergy=True, getForces=True):
        e, f = self.kernel.execute(self._system.positions, include_forces=getForces)
        return e, f

    def updateParametersInContext(self) -> None:
        self.kernel.copyParametersToContext(self.force.toSystem(self._system.positions))

    def getInducedDipoles(self):
        return self.kernel.getInducedDipoles(self._system.positions)

    def getLabFramePermanentDipoles(self):
        return self.kernel.getLabFramePermanentDipoles(self._system.positions)

    def getTotalDipoles(self):
        return self.kernel.getTotalDipoles(self._system.positions)

    def getElectrostaticPotential(self, grid):
        return self.kernel.getElectrostaticPotential(grid, self._system.positions)

    def getSystemMultipoleMoments(self):
        m = self.masses if self.masses is not None else np.ones(self._system.n)
        return self.kernel.getSystemMultipoleMoments(m, self._system.positions)

    def getPMEParametersInContext(self):
        return self.kernel.getPMEParameters()

    def close(self):
        self.kernel.close()
