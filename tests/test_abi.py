"""The C ABI library loads and exports every entry point include/gschism_b200.h declares; field
and phase codes agree between the header, the Python front end and the oracle."""
import os
import re

from gschism_b200 import _lib as L
from gschism_b200.model import FIELDS

HDR = os.path.join(os.path.dirname(__file__), "..", "include", "gschism_b200.h")


def _declared():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"^\s*(?:gs_status|const char\*|size_t|void\*)\s+(gs_\w+)\s*\(", txt, re.M)))


def test_exports_every_declared_symbol(native):
    names = _declared()
    assert len(names) >= 18
    for n in names:
        assert hasattr(native, n), n
    assert set(names) == set(L.EXPORTS)


def test_field_codes_agree():
    txt = open(HDR).read()
    hdr = {m.group(1): int(m.group(2)) for m in re.finditer(r"GS_F_(\w+)\s*=\s*(\d+)", txt)}
    assert hdr == FIELDS
    from oracle.step_api import F as OF
    assert OF == FIELDS


def test_phase_codes_agree():
    txt = open(HDR).read()
    hdr = {m.group(1): int(m.group(2)) for m in re.finditer(r"GS_PHASE_(\w+)\s*=\s*(\d+)", txt)}
    assert hdr == L.PHASE


def test_config_struct_matches_header():
    txt = open(HDR).read()
    body = txt[txt.index("typedef struct {", txt.index("-- model ----")):txt.index("} gs_config;")]
    fields = re.findall(r"\b(\w+)\s*[;,]", re.sub(r"/\*.*?\*/", "", body, flags=re.S))
    assert [f for f, _ in L.GsConfig._fields_] == fields
