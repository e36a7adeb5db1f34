"""Autotuner on the GPU (gpu): every chosen shape is accepted by the library, stream-kernel
shapes leave the results bit-identical, and a different solver tiling stays within the solver's
tolerance."""
import numpy as np
import pytest

from gschism_b200 import autotune, cases

pytestmark = pytest.mark.gpu


def test_tuned_shapes_valid_and_results_unchanged(native, tmp_path):
    from gschism_b200.model import Model
    c = cases.basin(n=120, nvrt=12, nz=4, nsteps=20)
    shapes = autotune.tuned_shapes([c], precision="fp64", warmup=2, rounds=1, path=str(tmp_path / "t.json"))
    assert set(shapes) == set(autotune.TUNE_ORDER)
    # the cache answers the second call
    assert autotune.tuned_shapes([c], precision="fp64", path=str(tmp_path / "t.json")) == shapes

    ref = Model([c], precision="fp64")
    ref.step(6)
    streams = Model([c], precision="fp64")
    autotune.apply(streams, {k: v for k, v in shapes.items() if k != "JCG_TILES"})
    assert all(streams.get_launch(k) == v for k, v in shapes.items() if k != "JCG_TILES")
    streams.step(6)
    for f in ("ETA2", "SIDE_U2", "ELEM_TR", "SIDE_BTU"):
        assert np.array_equal(streams.get(0, f), ref.get(0, f)), f

    tiled = Model([c], precision="fp64")
    tiled.set_launch("JCG_TILES", 37, 64)           # a tiling far from the default
    assert tiled.get_launch("JCG_TILES") == (37, 64)
    tiled.step(6)
    eta, eta_ref = tiled.get(0, "ETA2"), ref.get(0, "ETA2")
    assert np.abs(eta - eta_ref).max() <= 1e-10 * np.abs(eta_ref).max()


def test_invalid_shapes_rejected(native):
    from gschism_b200._lib import GsError
    from gschism_b200.model import Model
    m = Model([cases.channel()])
    for k, a, b in (("BTRACK", 256, 16), ("GHAT", 48, 16), ("GHAT", 128, 0), ("JCG_TILES", 100, 100)):
        with pytest.raises(GsError):
            m.set_launch(k, a, b)
    assert m.get_launch("BTRACK") == (128, 32)
