"""The `cufunc` shim (gschism_b200/kernels.py) driven in the reference's call order of one step
(src/python/schism_step.py:95-334, computeTransport :78-93, minTransportDt :66-75): it issues
exactly one launch per phase in the product's phase order, and refuses physics the build lacks."""
import pytest

from gschism_b200 import _lib as L
from gschism_b200.kernels import Kernels

PHASES = ["BEGIN", "BTRACK", "PREPARE", "ASSEMBLE", "SOLVE", "UPDATE_ELEV", "MOMENTUM", "VVEL", "TRANSPORT",
          "LEVELS", "NODAL_VEL"]


class _Case:
    class params:
        dt = 100.0


class FakeModel:
    cases = [_Case()]

    def __init__(self):
        self.calls = []

    def phase(self, name, it):
        self.calls.append((name, it))

    def stats(self, member=0):
        return {"jcg_iters": 7}


def reference_step(cufunc, it, dt):
    """The cufunc calls of schism_step (schism_step.py:95-334) with nws = 0, ishapiro = 0."""
    time = it * dt
    cufunc.scaleGravity(0.0)
    cufunc.computeTimeRamps(time, 0, False, 0.0, 0.0, 0.0, 0.0, 0.5)
    cufunc.computeBedDeformation()
    cufunc.computeTidalPotential(time, None, None, None, None, None)
    cufunc.getBoundaryConditions(time)
    cufunc.resetBoundaryAreas()
    cufunc.computeBoundaryAreas()
    cufunc.computeFlowBcVelocities(time)
    cufunc.computeBottomDragVegetation()
    cufunc.computeTurbulence()
    cufunc.computeHorizontalViscosity()
    cufunc.backtrackAllNodes()
    cufunc.computeElevationBoundaryConditions(time)
    cufunc.computeVerticallyIntegratedVelocity()
    cufunc.computeVegetationAndDragParameters()
    cufunc.computeDensityGradient()
    cufunc.computeBaroclinicTerm()
    cufunc.computeElemAverageGhat()
    cufunc.setupCoefficientMatrixAndRHS(time)
    cufunc.rollUpElevation()
    cufunc.setEssentialBC()
    its = cufunc.solveWaveEquation(None, 1000, 1e-12)
    cufunc.updateElevation()
    cufunc.computeHorGradientAtSide()
    cufunc.solveMomentumEquations(time)
    cufunc.applyMomentumBC()
    cufunc.computeVerticalVelocity()
    # computeTransport(dt), schism_step.py:78-93
    cufunc.computeHorizAdvecFluxes()
    remaining, passes = dt, 0
    while remaining > 0.0:
        cufunc.horizontalAdvectionPrepare()
        out = [1e34]
        cufunc.minTransportDtKernel(out)
        dtb = min(remaining, out[0])
        cufunc.horizontalAdvectionUpdate(dtb)
        remaining -= dtb
        passes += 1
    cufunc.verticalAdvectionUpdate(dt)
    cufunc.nodalTracerUpdate()
    for name in ("ul0UpdateZCoords", "ul0ComputeDryElements", "ul0ComputeDryNodes"):
        getattr(cufunc, name)()
    cufunc.ul0UpdateRewettedNodes(it, 0)
    cufunc.ul0UpdateSides(it, 0)
    cufunc.ul0UpdateSides2()
    cufunc.computeNodeDensity()
    cufunc.computeElemDensity()
    for name in ("zeroNodalVelocities", "computeNodalVerticalVelocities1", "computeNodalVerticalVelocities2",
                 "computeNodalHorizontalVelocities1", "computeNodalHorizontalVelocities2",
                 "resetVelocityOpenBndNodes", "setVelocityOpenBndNodes"):
        getattr(cufunc, name)()
    return its, passes


def test_reference_call_order_issues_each_phase_once():
    m = FakeModel()
    k = Kernels(m)
    for it in (1, 2):
        m.calls.clear()
        its, passes = reference_step(k, it, 100.0)
        assert [c[0] for c in m.calls] == PHASES
        assert all(c[1] == it for c in m.calls)
        assert its == 7 and passes == 1


@pytest.mark.parametrize("opt", [{"itur": 3}, {"ibc": 0}, {"ntip": 2}, {"ishapiro": 1}, {"nws": 2}, {"ics": 2}])
def test_unsupported_physics_is_refused(opt):
    with pytest.raises(L.GsError) as ei:
        Kernels(FakeModel(), options=opt)
    assert ei.value.status == L.GS_ERR_ARG


def test_kernels_of_unsupported_physics_are_refused():
    k = Kernels(FakeModel())
    for name in ("shapiroFilter1", "shapiroFilter2"):
        with pytest.raises(L.GsError):
            getattr(k, name)()
    with pytest.raises(L.GsError):
        k.setWinds(None, None, None)
