"""The C ABI library loads without a GPU, exports every declared entry point,
and rejects bad decks the way the reference rejects bad parameters."""
import ctypes
import re
from pathlib import Path

import pytest

import kamayan_b200
from kamayan_b200 import configs

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(kmy_[a-z0-9_]+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "kmy_create" in names and "kmy_rk_stage" in names
    assert names == set(kamayan_b200.EXPORTS) | (names - set(kamayan_b200.EXPORTS))


def test_library_exports_every_declared_symbol(kmy_lib):
    missing = [n for n in sorted(declared_symbols()) if not hasattr(kmy_lib, n)]
    assert not missing, missing


def _create(text):
    h = ctypes.c_void_p()
    rc = kamayan_b200.lib().kmy_create(text.encode(), 0, ctypes.byref(h))
    if rc == 0:
        kamayan_b200.lib().kmy_destroy(h)
    return rc


@pytest.mark.parametrize("block,key,value", [
    ("hydro", "reconstruction", "weno5"),
    ("hydro", "riemann", "hlld"),
    ("hydro", "slope_limiter", "superbee"),
    ("hydro", "ReconstructionVars", "characteristic"),
    ("physics", "MHD", "glm"),
    ("parthenon/time", "integrator", "vl2"),
    ("kamayan_b200", "precision", "fp16"),
    ("geometry", "geometry", "cylindrical"),
    ("physics", "fluid", "threeT"),
    ("parthenon/mesh", "nghost", "1"),
    ("parthenon/meshblock", "nx1", "48"),
    ("parthenon/mesh", "ix1_bc", "user"),
])
def test_bad_parameters_rejected(kmy_lib, block, key, value):
    d = configs.vortex_2d(n=64, nb=32)
    d.set(block, key, value)
    assert _create(d.text()) == 1  # KMY_ERR_BAD_PARAM, no device touched


def test_null_arguments(kmy_lib):
    L = kamayan_b200.lib()
    assert L.kmy_create(b"", 0, None) == 1
    assert L.kmy_destroy(None) == 0
    assert L.kmy_step(None, None) == 1


@pytest.mark.parametrize("block,key,value", [
    ("kamayan/refinement0", "method", "derivative_order_1"),
    ("kamayan/refinement0", "field", "velocity"),
    ("parthenon/mesh", "numlevel", "9"),
    ("parthenon/mesh", "refinement", "static"),
])
def test_bad_adaptive_parameters_rejected(kmy_lib, block, key, value):
    d = configs.blast_2d_amr(n=64, nb=8)
    d.set(block, key, value)
    assert _create(d.text()) == 1

