"""The reference's MEX routines under their own names, on the GPU.

Each function takes the same arguments, in the same order, as the MATLAB call
of the reference (solvers/scripts/dynamic/dynamicsolverdisplacementcontrolled.m
:79-105) and updates the output arrays in place, like the MEX files do. Arrays
are float64 numpy arrays in MATLAB layout (column-major nNodes x 3 node arrays,
nBonds x 2 BONDLIST with 1-based ids). Errors raise BBPDError, where MATLAB
would raise mexErrMsgTxt's error.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

_P = N.ptr


def _arr(a, name, writable=False):
    if not isinstance(a, np.ndarray) or a.dtype != np.float64:
        raise TypeError(f"{name} must be a float64 numpy array")
    if not (a.flags["F_CONTIGUOUS"] or a.ndim == 1 and a.flags["C_CONTIGUOUS"]):
        raise TypeError(f"{name} must be column-major contiguous (MATLAB layout)")
    if writable and not a.flags["WRITEABLE"]:
        raise TypeError(f"{name} is updated in place and must be writable")
    return _P(a)


def _rows(a):
    return a.shape[0]


def _sig():
    L = N.lib()
    d, i64, i = C.c_double, C.c_int64, C.c_int
    p = C.POINTER(C.c_double)
    L.bbpd_calculatedeformedlength.argtypes = [p, p, p, i64, i64, p, p, p, p, p]
    L.bbpd_calculatebsfexponential.argtypes = [p, p, p, d, d, p, p, p, p, i64]
    L.bbpd_calculatebsftrilinear.argtypes = [p, d, d, d, p, p, p, i64]
    L.bbpd_calculatebondsofteningfactor.argtypes = [p, d, d, p, p, p, i64]
    L.bbpd_calculatebondfailure.argtypes = [p, d, p, p, d, d, i64]
    L.bbpd_calculatebondforces.argtypes = [p, p, p, p, p, p, p, p, p, p, p, d, p, p, i64]
    L.bbpd_calculatenodalforces.argtypes = [p, i64, i64, p, p, p, p, i]
    L.bbpd_timeintegrationeulercromer.argtypes = [p, p, d, p, p, p, d, p, p, p, i64, i]
    L.bbpd_calculatedampingcoefficient.argtypes = [p, p, p, d, p, p, i64, p]
    L.bbpd_timeintegrationADR.argtypes = [i64, d, p, p, p, d, p, p, p, i64]
    L.bbpd_calculatedamage.argtypes = [p, p, p, i64, i64, p]
    L.bbpd_calculatedamageenergy.argtypes = [p, p, p, p, p, d, d, d, p, i64]
    return L


_L = None


def _lib():
    global _L
    if _L is None:
        _L = _sig()
    return _L


def calculatedeformedlengthMex(deformedCoordinates, BONDLIST, undeformedLength, deformedLength,
                               deformedX, deformedY, deformedZ, stretch):
    """calculatedeformedlengthMex.c:27-47 (outputs in place)."""
    N.check(_lib().bbpd_calculatedeformedlength(
        _arr(deformedCoordinates, "deformedCoordinates"), _arr(BONDLIST, "BONDLIST"),
        _arr(undeformedLength, "undeformedLength"), _rows(BONDLIST), _rows(deformedCoordinates),
        _arr(deformedLength, "deformedLength", True), _arr(deformedX, "deformedX", True),
        _arr(deformedY, "deformedY", True), _arr(deformedZ, "deformedZ", True),
        _arr(stretch, "stretch", True)))


def calculatebsfexponentialMex(stretch, s0, sc, k, alpha, bsf, bondSofteningFactor, BONDTYPE,
                               flagBondSoftening):
    """calculatebsfexponentialMex.c:26-66 (bsf, bondSofteningFactor, flag in place)."""
    N.check(_lib().bbpd_calculatebsfexponential(
        _arr(stretch, "stretch"), _arr(s0, "s0"), _arr(sc, "sc"), float(k), float(alpha),
        _arr(bsf, "bsf", True), _arr(bondSofteningFactor, "bondSofteningFactor", True),
        _arr(BONDTYPE, "BONDTYPE"), _arr(flagBondSoftening, "flagBondSoftening", True),
        _rows(stretch)))


def calculatebsftrilinear(stretch, s0, s1, sc, bondSofteningFactor, BONDTYPE, flagBondSoftening):
    """calculatebsftrilinear.m:1 on the GPU; returns (bondSofteningFactor, flagBondSoftening),
    both also updated in place."""
    N.check(_lib().bbpd_calculatebsftrilinear(
        _arr(stretch, "stretch"), float(s0), float(s1), float(sc),
        _arr(bondSofteningFactor, "bondSofteningFactor", True), _arr(BONDTYPE, "BONDTYPE"),
        _arr(flagBondSoftening, "flagBondSoftening", True), _rows(stretch)))
    return bondSofteningFactor, flagBondSoftening


def calculatebondsofteningfactor(stretch, linearElasticLimit, criticalStretchConcrete,
                                 flagBondSoftening, bondSofteningFactor, BONDTYPE):
    """calculatebondsofteningfactor.m:1 (bilinear) on the GPU; returns
    (bondSofteningFactor, flagBondSoftening), both also updated in place."""
    N.check(_lib().bbpd_calculatebondsofteningfactor(
        _arr(stretch, "stretch"), float(linearElasticLimit), float(criticalStretchConcrete),
        _arr(flagBondSoftening, "flagBondSoftening", True),
        _arr(bondSofteningFactor, "bondSofteningFactor", True), _arr(BONDTYPE, "BONDTYPE"),
        _rows(stretch)))
    return bondSofteningFactor, flagBondSoftening


def calculatebondfailureMex(fail, failureFunctionality, BONDTYPE, stretch,
                            criticalStretchConcrete, criticalStretchSteel):
    """calculatebondfailureMex.c:26-44 (fail in place)."""
    N.check(_lib().bbpd_calculatebondfailure(
        _arr(fail, "fail", True), float(failureFunctionality), _arr(BONDTYPE, "BONDTYPE"),
        _arr(stretch, "stretch"), float(criticalStretchConcrete), float(criticalStretchSteel),
        _rows(fail)))
    return fail


def calculatedamage(bondlist, fail, nFAMILYMEMBERS) -> np.ndarray:
    """calculatedamage.m:1 on the GPU: the fraction of broken bonds of every node."""
    nN = _rows(nFAMILYMEMBERS)
    damage = np.zeros(nN, dtype=np.float64)
    N.check(_lib().bbpd_calculatedamage(_arr(bondlist, "bondlist"), _arr(fail, "fail"),
                                        _arr(nFAMILYMEMBERS, "nFAMILYMEMBERS"), _rows(bondlist), nN,
                                        _arr(damage, "damage", True)))
    return damage


def calculatebondforcesMex(bForceX, bForceY, bForceZ, fail, deformedX, deformedY, deformedZ,
                           deformedLength, stretch, stretchPlastic, BONDSTIFFNESS, cellVolume,
                           VOLUMECORRECTIONFACTORS, bondSofteningFactor):
    """calculatebondforcesMex.c:26-45 (bForceX/Y/Z in place)."""
    N.check(_lib().bbpd_calculatebondforces(
        _arr(bForceX, "bForceX", True), _arr(bForceY, "bForceY", True),
        _arr(bForceZ, "bForceZ", True), _arr(fail, "fail"), _arr(deformedX, "deformedX"),
        _arr(deformedY, "deformedY"), _arr(deformedZ, "deformedZ"),
        _arr(deformedLength, "deformedLength"), _arr(stretch, "stretch"),
        _arr(stretchPlastic, "stretchPlastic"), _arr(BONDSTIFFNESS, "BONDSTIFFNESS"),
        float(cellVolume), _arr(VOLUMECORRECTIONFACTORS, "VOLUMECORRECTIONFACTORS"),
        _arr(bondSofteningFactor, "bondSofteningFactor"), _rows(bForceX)))


def calculatenodalforcesopenmpMex(BONDLIST, nodalForce, bForceX, bForceY, bForceZ,
                                  nodalForceX=None, nodalForceY=None, nodalForceZ=None):
    """calculatenodalforcesopenmpMex.c:29-85 (nodalForce accumulated in place, in the
    order of the reference's 8 OpenMP threads). The per-thread scratch arrays are
    accepted for signature compatibility and not used."""
    N.check(_lib().bbpd_calculatenodalforces(
        _arr(BONDLIST, "BONDLIST"), _rows(BONDLIST), _rows(nodalForce),
        _arr(nodalForce, "nodalForce", True), _arr(bForceX, "bForceX"), _arr(bForceY, "bForceY"),
        _arr(bForceZ, "bForceZ"), 8))


def calculatenodalforcesMex(BONDLIST, nodalForce, bForceX, bForceY, bForceZ):
    """calculatenodalforcesMex.c:19-46 (serial bond order)."""
    N.check(_lib().bbpd_calculatenodalforces(
        _arr(BONDLIST, "BONDLIST"), _rows(BONDLIST), _rows(nodalForce),
        _arr(nodalForce, "nodalForce", True), _arr(bForceX, "bForceX"), _arr(bForceY, "bForceY"),
        _arr(bForceZ, "bForceZ"), 1))


def timeintegrationeulercromerMex(nodalAcceleration, nodalForce, DAMPING, nodalVelocity, DENSITY,
                                  constraintFLAG, DT, nodalDisplacement, deformedCoordinates,
                                  undeformedCoordinates):
    """timeintegrationeulercromerMex.c:26-53 (a, v, u, x in place)."""
    nN = _rows(nodalAcceleration)
    NOD = nodalAcceleration.shape[1] if nodalAcceleration.ndim == 2 else 1
    N.check(_lib().bbpd_timeintegrationeulercromer(
        _arr(nodalAcceleration, "nodalAcceleration", True), _arr(nodalForce, "nodalForce"),
        float(DAMPING), _arr(nodalVelocity, "nodalVelocity", True), _arr(DENSITY, "DENSITY"),
        _arr(constraintFLAG, "constraintFLAG"), float(DT),
        _arr(nodalDisplacement, "nodalDisplacement", True),
        _arr(deformedCoordinates, "deformedCoordinates", True),
        _arr(undeformedCoordinates, "undeformedCoordinates"), nN, NOD))


def calculatedampingcoefficient(nodalForce, massVector, nodalForcePrevious, DT,
                                nodalVelocityPreviousHalf, nodalDisplacement) -> float:
    """calculatedampingcoefficient.m:1 (NOD = 3) on the GPU, sums in the fixed tree order."""
    cn = C.c_double()
    N.check(_lib().bbpd_calculatedampingcoefficient(
        _arr(nodalForce, "nodalForce"), _arr(massVector, "massVector"),
        _arr(nodalForcePrevious, "nodalForcePrevious"), float(DT),
        _arr(nodalVelocityPreviousHalf, "nodalVelocityPreviousHalf"),
        _arr(nodalDisplacement, "nodalDisplacement"), _rows(nodalForce),
        C.cast(C.pointer(cn), C.POINTER(C.c_double))))
    return float(cn.value)


def timeintegrationADR(iTimeStep, DT, nodalVelocityForwardHalf, nodalForce, massVector, cn,
                       nodalVelocityPreviousHalf, nodalDisplacement, CONSTRAINTFLAG):
    """timeintegrationADR.m:1 (NOD = 3); returns (nodalDisplacement,
    nodalVelocityForwardHalf), both updated in place."""
    N.check(_lib().bbpd_timeintegrationADR(
        int(iTimeStep), float(DT), _arr(nodalVelocityForwardHalf, "nodalVelocityForwardHalf", True),
        _arr(nodalForce, "nodalForce"), _arr(massVector, "massVector"), float(cn),
        _arr(nodalVelocityPreviousHalf, "nodalVelocityPreviousHalf"),
        _arr(nodalDisplacement, "nodalDisplacement", True), _arr(CONSTRAINTFLAG, "CONSTRAINTFLAG"),
        _rows(nodalForce)))
    return nodalDisplacement, nodalVelocityForwardHalf


def calculatedamageenergy(BONDSTIFFNESS, s0, sc, UNDEFORMEDLENGTH, stretch, k, alpha, cellVolume,
                          damageEnergy) -> np.ndarray:
    """calculatedamageenergy.m:1 on the GPU: the energy dissipated by every bond,
    never decreasing (damageEnergy updated in place and returned)."""
    N.check(_lib().bbpd_calculatedamageenergy(
        _arr(BONDSTIFFNESS, "BONDSTIFFNESS"), _arr(s0, "s0"), _arr(sc, "sc"),
        _arr(UNDEFORMEDLENGTH, "UNDEFORMEDLENGTH"), _arr(stretch, "stretch"), float(k), float(alpha),
        float(cellVolume), _arr(damageEnergy, "damageEnergy", True), _rows(damageEnergy)))
    return damageEnergy
