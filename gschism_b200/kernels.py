"""The reference's kernel entry points (`cufunc.<name>(...)`, src/python/cuda_functions.py:140-257)
mapped onto the phases of a Model.

    k = Kernels(model, it)        # `it`: current step index (time = it * dt)
    k.backtrackAllNodes(); k.computeElemAverageGhat(); k.setupCoefficientMatrixAndRHS(time); ...

The B200 build fuses several reference kernels into one launch; the names that the fused launch
already covers are accepted and do nothing, so the reference's call sequence
(src/python/schism_step.py:95-334) runs unchanged:

  computeElevationBoundaryConditions, computeVerticallyIntegratedVelocity,
  computeVegetationAndDragParameters, computeElemAverageGhat  -> PREPARE (issued by the first)
  setupCoefficientMatrixAndRHS, rollUpElevation, setEssentialBC -> ASSEMBLE
  solveWaveEquation(solver, ...)                           -> SOLVE (JCG on the device)
  updateElevation                                         -> UPDATE_ELEV
  computeHorGradientAtSide, solveMomentumEquations, applyMomentumBC -> MOMENTUM
  computeVerticalVelocity                                 -> VVEL
  computeTransport(dt) / computeHorizAdvecFluxes .. nodalTracerUpdate -> TRANSPORT
  ul0UpdateZCoords .. ul0UpdateSides2                     -> LEVELS
  zeroNodalVelocities .. computeNodalHorizontalVelocities2 -> NODAL_VEL
"""
from __future__ import annotations


class Kernels:
    def __init__(self, model, it: int = 0):
        self.m = model
        self.it = it
        self._prep = False

    def _ph(self, name, arg=None):
        self.m.phase(name, self.it if arg is None else arg)

    # forcing (computeTimeRamps etc.) and the start of a step
    def computeTimeRamps(self, time, *a):
        self.it = int(round(time / self.m.cases[0].params.dt))
        self._prep = False
        self._ph("BEGIN", self.it)

    def scaleGravity(self, *a):
        pass

    def computeTidalPotential(self, *a):
        pass

    def computeBedDeformation(self, *a):
        pass

    def getBoundaryConditions(self, *a):
        pass

    def resetBoundaryAreas(self, *a):
        pass

    def computeBoundaryAreas(self, *a):
        pass

    def computeFlowBcVelocities(self, *a):
        pass

    def computeBottomDragVegetation(self, *a):
        pass

    def computeTurbulence(self, *a):
        pass

    def computeHorizontalViscosity(self, *a):
        pass

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

    def computeDensityGradient(self):
        pass

    def computeBaroclinicTerm(self):
        pass

    def computeElemAverageGhat(self):
        self._prepare()

    def setupCoefficientMatrixAndRHS(self, time=None):
        self._prepare()
        self._ph("ASSEMBLE")

    def rollUpElevation(self):
        pass                                  # fused into setupCoefficientMatrixAndRHS

    def setEssentialBC(self):
        pass                                  # fused into setupCoefficientMatrixAndRHS

    def solveWaveEquation(self, solver=None, maxIter=None, tol=None):
        self._ph("SOLVE")
        return self.m.stats(0)["jcg_iters"]

    def updateElevation(self):
        self._ph("UPDATE_ELEV")

    def computeHorGradientAtSide(self):
        pass                                  # fused into solveMomentumEquations

    def solveMomentumEquations(self, time=None):
        self._ph("MOMENTUM")

    def applyMomentumBC(self):
        pass                                  # fused into solveMomentumEquations

    def computeVerticalVelocity(self):
        self._ph("VVEL")

    def computeTransport(self, dt=None):
        self._ph("TRANSPORT")

    def computeHorizAdvecFluxes(self):
        pass                                  # fused into solveMomentumEquations

    def ul0UpdateZCoords(self):
        self._ph("LEVELS")

    def ul0ComputeDryElements(self):
        pass

    def ul0ComputeDryNodes(self):
        pass

    def ul0UpdateRewettedNodes(self, *a):
        pass

    def ul0UpdateSides(self, *a):
        pass

    def ul0UpdateSides2(self):
        pass

    def computeNodeDensity(self):
        pass

    def computeElemDensity(self):
        pass

    def zeroNodalVelocities(self):
        self._ph("NODAL_VEL")

    def computeNodalVerticalVelocities1(self):
        pass

    def computeNodalVerticalVelocities2(self):
        pass

    def computeNodalHorizontalVelocities1(self):
        pass

    def computeNodalHorizontalVelocities2(self):
        pass

    def resetVelocityOpenBndNodes(self):
        pass

    def setVelocityOpenBndNodes(self):
        pass
