"""The stage-kernel autotuner's host logic (no GPU): configuration keys and
the process-wide cache with its file format (kamayan_b200/csrc/kmy_tune.cu).

The reference selects its flux loop strategy by a runtime parameter
(src/physics/hydro/hydro.cpp:75-79); the tuner selects the stage kernel by
measurement and caches the choice per device and configuration.
"""
import pytest

import kamayan_b200 as K
from kamayan_b200 import configs


@pytest.fixture(autouse=True)
def _clean_cache(kmy_lib):
    K.tune_cache_clear()
    yield
    K.tune_cache_clear()


def test_key_names_the_configuration():
    k = K.tune_key(configs.kh_3d(n=256, nb=32, precision="fp32"))
    assert k == "fp32 d3 wenoz-hllc-mc n32x32x32 g3 b512"
    k64 = K.tune_key(configs.kh_3d(n=256, nb=32, precision="fp64"))
    assert k64.startswith("fp64 ") and k64 != k
    assert "ct" in K.tune_key(configs.ot_3d(n=64, nb=32)).split()


@pytest.mark.parametrize("change", [
    ("hydro", "reconstruction", "ppm"), ("hydro", "riemann", "hll"), ("hydro", "slope_limiter", "minmod"),
    ("parthenon/meshblock", "nx2", 16)])
def test_key_changes_with_what_the_speed_depends_on(change):
    base = configs.kh_3d(n=64, nb=32, precision="fp32")
    other = configs.kh_3d(n=64, nb=32, precision="fp32")
    other.set(*change)
    assert K.tune_key(base) != K.tune_key(other)


def test_key_ignores_run_length():
    a = configs.kh_3d(n=64, nb=32, precision="fp32", nlim=5)
    b = configs.kh_3d(n=64, nb=32, precision="fp32", nlim=500)
    assert K.tune_key(a) == K.tune_key(b)


def test_key_rejects_a_bad_deck():
    d = configs.kh_3d(n=64, nb=32)
    d.set("hydro", "reconstruction", "weno9")
    with pytest.raises(K.KmyError):
        K.tune_key(d)


@pytest.mark.parametrize("block,key,value", [("kamayan_b200", "ct_update", "sideways"),
                                              ("kamayan_b200", "stage_kernel", "fastest"),
                                              ("kamayan_b200", "slab_rows", "12")])
def test_key_rejects_unknown_kernel_options(block, key, value):
    d = configs.ot_3d(n=64, nb=32)
    d.set(block, key, value)
    with pytest.raises(K.KmyError):
        K.tune_key(d)


@pytest.mark.parametrize("value", ["auto", "streamed", "per_face"])
def test_key_accepts_ct_update(value):
    d = configs.ot_3d(n=64, nb=32)
    d.set("kamayan_b200", "ct_update", value)
    assert "ct" in K.tune_key(d)


def test_cache_put_get_and_unknown_choice():
    assert K.tune_cache_get("NVIDIA B200 | x") is None
    K.tune_cache_put("NVIDIA B200 | x", "slab16", 1.25)
    assert K.tune_cache_get("NVIDIA B200 | x") == ("slab16", 1.25)
    K.tune_cache_put("NVIDIA B200 | x", "brick", 2.0)  # a later measurement replaces it
    assert K.tune_cache_get("NVIDIA B200 | x") == ("brick", 2.0)
    with pytest.raises(K.KmyError):
        K.tune_cache_put("NVIDIA B200 | y", "slab32", 1.0)
    with pytest.raises(K.KmyError):
        K.tune_cache_put("bad\tkey", "brick", 1.0)


def test_cache_file_round_trip(tmp_path):
    K.tune_cache_put("dev | a", "slab8", 0.5)
    K.tune_cache_put("dev | b", "brick", 3.0)
    f = tmp_path / "tune.txt"
    K.tune_cache_save(f)
    K.tune_cache_clear()
    assert K.tune_cache_get("dev | a") is None
    K.tune_cache_load(f)
    assert K.tune_cache_get("dev | a") == ("slab8", 0.5)
    assert K.tune_cache_get("dev | b") == ("brick", 3.0)


def test_cache_load_skips_malformed_lines(tmp_path):
    f = tmp_path / "tune.txt"
    f.write_text("dev | ok\tslab16\t1.5\n"
                 "no tabs here\n"
                 "dev | bad choice\tslab99\t1.0\n"
                 "dev | bad ms\tbrick\tfast\n"
                 "\tbrick\t1.0\n")
    K.tune_cache_load(f)
    assert K.tune_cache_get("dev | ok") == ("slab16", 1.5)
    for k in ("dev | bad choice", "dev | bad ms", ""):
        assert K.tune_cache_get(k) is None
    with pytest.raises(K.KmyError):
        K.tune_cache_load(tmp_path / "missing.txt")
