"""Autotuner logic on the CPU with a stand-in model: candidates the library rejects are skipped,
the shape with the smallest median phase time wins, the solver is compared per inner iteration,
and the cache round-trips."""
import pytest

from gschism_b200 import autotune
from gschism_b200._lib import GsError


class FakeModel:
    """Launch table with per-kernel limits; phase times are a function of the current shapes."""

    def __init__(self):
        self.shapes = {k: (128, 16) for k in autotune.KERNEL_PHASE}
        self.shapes["JCG_TILES"] = (592, 1024)
        self.cases = [None]

    def get_launch(self, k):
        return self.shapes[k]

    def set_launch(self, k, a, b):
        if k in ("BTRACK", "MOMENTUM", "VVEL") and a > 128:
            raise GsError(1, "block above the kernel's limit")
        self.shapes[k] = (a, b)

    def measure(self):
        t = {ph: 1.0 for ph in autotune.STEP_PHASES}
        b, g = self.shapes["BTRACK"]
        t["BTRACK"] = 5.0 + abs(b - 64) / 64 + (0.5 if g == 16 else 0.0)
        b, g = self.shapes["NODAL_VEL"]
        t["NODAL_VEL"] = 1.0 + abs(b - 256) / 256
        tiles, rows = self.shapes["JCG_TILES"]
        iters = 700 if tiles >= 888 else 600          # more tiles: more iterations, cheaper each
        t["SOLVE"] = iters * (0.03 if tiles >= 888 else 0.04)
        t["jcg_iters"] = iters
        return t


def test_tuner_picks_fastest_valid_shapes():
    m = FakeModel()
    got = autotune.tune_model(m, rounds=2, measure=m.measure)
    assert got["BTRACK"] == (64, 32)                 # 256/512 rejected by the kernel's limit
    assert got["NODAL_VEL"][0] == 256
    assert got["JCG_TILES"][0] >= 888                # per-iteration cost, not phase time
    assert all(m.get_launch(k) == v for k, v in got.items())


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    autotune.store_cache("k1", {"BTRACK": (64, 32)}, path)
    autotune.store_cache("k2", {"GHAT": (256, 16)}, path)
    data = autotune.load_cache(path)
    assert data["k1"] == {"BTRACK": [64, 32]} and data["k2"] == {"GHAT": [256, 16]}
    assert autotune.load_cache(str(tmp_path / "missing.json")) == {}


def test_cache_key_size_class():
    from gschism_b200 import cases
    c = cases.channel()
    k = autotune.cache_key([c], "fp64", "B200")
    assert k.startswith("B200|fp64|nvrt=10|ntr=1|itr_met=1|nodes~2^11")
