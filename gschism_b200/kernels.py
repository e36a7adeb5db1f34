"""The reference's kernel entry points (`cufunc.<name>(...)`, src/python/cuda_functions.py:140-257)
mapped onto the phases of a Model.

    k = Kernels(model, options=dict(itur=0, ibc=1, ...))   # the run's namelist switches
    k.computeTimeRamps(time, ...); k.backtrackAllNodes(); ...; k.setVelocityOpenBndNodes()

The B200 build fuses several reference kernels into one launch, so the reference's call sequence
(src/python/schism_step.py:95-334) runs unchanged and issues one launch per phase:

  computeTimeRamps                                          -> BEGIN (step clock, ramp, forcing)
  backtrackAllNodes                                         -> BTRACK
  computeElevationBoundaryConditions, computeVerticallyIntegratedVelocity,
  computeVegetationAndDragParameters, computeElemAverageGhat -> PREPARE (issued by the first)
  setupCoefficientMatrixAndRHS (+ rollUpElevation, setEssentialBC) -> ASSEMBLE
  solveWaveEquation(solver, ...)                            -> SOLVE (JCG on the device)
  updateElevation                                           -> UPDATE_ELEV
  computeHorGradientAtSide (+ solveMomentumEquations, applyMomentumBC) -> MOMENTUM
  computeVerticalVelocity                                   -> VVEL
  computeTransport(dt) / computeHorizAdvecFluxes .. nodalTracerUpdate -> TRANSPORT
  ul0UpdateZCoords (+ the other ul0*, computeNodeDensity, computeElemDensity) -> LEVELS
  zeroNodalVelocities (.. setVelocityOpenBndNodes)          -> NODAL_VEL

Names whose reference kernel does nothing under the supported physics (no tidal potential, no
bed deformation, no flow boundaries, constant viscosity, no horizontal viscosity, no baroclinic
force, drag coefficients per node) are accepted as no-ops; the switches that would give them work
are checked when the shim is made, and a run that needs one (itur != 0, ibc = 0, ntip > 0,
ihorcon != 0, ishapiro = 1, nchi != 0, iloadtide != 0, nws != 0, ifltype != 0, imm != 0, iveg != 0,
ics != 1) is refused with GS_ERR_ARG instead of running with that physics missing.  Kernels that
only such runs call (shapiroFilter1/2, setWinds) are refused too.
"""
from __future__ import annotations

from . import _lib as L

# namelist switch -> the only value this build supports
SUPPORTED = {"itur": 0, "ibc": 1, "ntip": 0, "ihorcon": 0, "ishapiro": 0, "nchi": 0, "iloadtide": 0, "nws": 0,
             "ifltype": 0, "imm": 0, "iveg": 0, "ics": 1}


class Kernels:
    def __init__(self, model, it: int = 0, options=None):
        bad = {k: v for k, v in (options or {}).items() if k in SUPPORTED and v != SUPPORTED[k]}
        if bad:
            raise L.GsError(L.GS_ERR_ARG, f"physics not supported by this build: {bad}")
        self.m = model
        self.it = it
        self._prep = False
        self._levels = False
        self._nodal = False
        self._trans = False

    def _ph(self, name, arg=None):
        self.m.phase(name, self.it if arg is None else arg)

    @staticmethod
    def _refuse(name):
        raise L.GsError(L.GS_ERR_ARG, f"{name}: not supported by this build")

    # ------------------------------------------------------------------ start of a step
    def computeTimeRamps(self, time, *a):
        self.it = int(round(time / self.m.cases[0].params.dt))
        self._prep = self._levels = self._nodal = self._trans = False
        self._ph("BEGIN", self.it)

    # reference kernels without work under the supported physics (checked in __init__)
    def scaleGravity(self, *a):          # iloadtide = 0: grav2 = grav (meshdata.cu:3945-3972)
        pass

    def computeTidalPotential(self, *a):  # ntip = 0: ETP = 0 (meshdata.cu:3994-4015)
        pass

    def computeBedDeformation(self, *a):  # imm = 0
        pass

    def getBoundaryConditions(self, *a):  # no time-history boundaries (meshdata.cu:4019-4030)
        pass

    def resetBoundaryAreas(self, *a):     # ifltype = 0: no flow boundaries
        pass

    def computeBoundaryAreas(self, *a):
        pass

    def computeFlowBcVelocities(self, *a):
        pass

    def computeBottomDragVegetation(self, *a):   # nchi = 0: Cd = drag (set in BEGIN), iveg = 0
        pass

    def computeTurbulence(self, *a):     # itur = 0: dfv = dfv0
        pass

    def computeHorizontalViscosity(self, *a):    # ihorcon = 0
        pass

    def computeDensityGradient(self):    # ibc = 1: no baroclinic force (meshdata.cu:4881-4885)
        pass

    def computeBaroclinicTerm(self):     # ibc = 1 (meshdata.cu:4963-4965)
        pass

    def shapiroFilter1(self):
        self._refuse("shapiroFilter1 (ishapiro = 1)")

    def shapiroFilter2(self):
        self._refuse("shapiroFilter2 (ishapiro = 1)")

    def setWinds(self, *a):
        self._refuse("setWinds (nws != 0; use Model.set_tau or Model.set_vortex)")

    # ------------------------------------------------------------------ phases
    def backtrackAllNodes(self):
        self._ph("BTRACK")

    def _prepare(self):
        if not self._prep:
            self._ph("PREPARE")
            self._prep = True

    def computeElevationBoundaryConditions(self, time=None):
        self._prepare()

    def computeVerticallyIntegratedVelocity(self):
        self._prepare()

    def computeVegetationAndDragParameters(self):
        self._prepare()

    def computeElemAverageGhat(self):
        self._prepare()

    def setupCoefficientMatrixAndRHS(self, time=None):
        self._prepare()
        self._ph("ASSEMBLE")

    def rollUpElevation(self):
        pass                                  # in ASSEMBLE

    def setEssentialBC(self):
        pass                                  # in ASSEMBLE

    def solveWaveEquation(self, solver=None, maxIter=None, tol=None):
        self._ph("SOLVE")
        return self.m.stats(0)["jcg_iters"]

    def updateElevation(self):
        self._ph("UPDATE_ELEV")

    def computeHorGradientAtSide(self):
        self._ph("MOMENTUM")

    def solveMomentumEquations(self, time=None):
        pass                                  # in MOMENTUM

    def applyMomentumBC(self):
        pass                                  # in MOMENTUM

    def computeVerticalVelocity(self):
        self._ph("VVEL")

    def computeTransport(self, dt=None):
        """schism_step.computeTransport (schism_step.py:78-93) in one call."""
        self._transport()

    def _transport(self):
        if not self._trans:
            self._ph("TRANSPORT")
            self._trans = True

    def computeHorizAdvecFluxes(self):
        pass                                  # in MOMENTUM (fluxes of the new velocities)

    # the kernels of schism_step.computeTransport: the whole sub-cycled transport runs in the
    # first of them; the sub-step is chosen on the device, so the minimum reported to the host
    # loop is "no limit" and the loop ends after one pass
    def horizontalAdvectionPrepare(self):
        self._transport()

    def minTransportDtKernel(self, out):
        out[0] = 1e34

    def horizontalAdvectionUpdate(self, dtb=None):
        pass

    def verticalAdvectionUpdate(self, dt=None):
        pass

    def nodalTracerUpdate(self):
        pass

    def _level(self):
        if not self._levels:
            self._ph("LEVELS")
            self._levels = True

    def ul0UpdateZCoords(self):
        self._level()

    def ul0ComputeDryElements(self):
        self._level()

    def ul0ComputeDryNodes(self):
        self._level()

    def ul0UpdateRewettedNodes(self, *a):
        self._level()

    def ul0UpdateSides(self, *a):
        self._level()

    def ul0UpdateSides2(self):
        self._level()

    def computeNodeDensity(self):
        self._level()                         # densities are computed at the end of LEVELS

    def computeElemDensity(self):
        self._level()

    def _nodal_vel(self):
        if not self._nodal:
            self._ph("NODAL_VEL")
            self._nodal = True

    def zeroNodalVelocities(self):
        self._nodal_vel()

    def computeNodalVerticalVelocities1(self):
        self._nodal_vel()

    def computeNodalVerticalVelocities2(self):
        self._nodal_vel()

    def computeNodalHorizontalVelocities1(self):
        self._nodal_vel()

    def computeNodalHorizontalVelocities2(self):
        self._nodal_vel()

    def resetVelocityOpenBndNodes(self):
        self._nodal_vel()

    def setVelocityOpenBndNodes(self):
        self._nodal_vel()
