"""Deck text handling mirrors Parthenon input files and overrides."""
from kamayan_b200 import configs
from kamayan_b200.deck import Deck

SAMPLE = """
<parthenon/mesh>
refinement = none
nx1 = 64   # cells
x1min = -5.0
<hydro>
cfl = 0.8
reconstruction = wenoz
"""


def test_parse_blocks_and_comments():
    d = Deck.parse(SAMPLE)
    assert d.get("parthenon/mesh", "nx1") == "64"
    assert d.get("hydro", "reconstruction") == "wenoz"


def test_override_form():
    d = Deck.parse(SAMPLE).override("parthenon/mesh/nx1=128", "hydro/riemann=hllc")
    assert d.get("parthenon/mesh", "nx1") == "128"
    assert d.get("hydro", "riemann") == "hllc"
    again = Deck.parse(d.text())
    assert again.blocks == d.blocks


def test_override_lines_in_text_are_honoured():
    d = Deck.parse(SAMPLE + "\nhydro/cfl = 0.4\n")
    assert d.get("hydro", "cfl") == "0.4"


def test_workload_decks():
    kh = configs.kh_3d()
    assert kh.get("parthenon/mesh", "nx3") == "256"
    assert kh.get("parthenon/meshblock", "nx1") == "32"
    assert kh.get("hydro", "reconstruction") == "wenoz"
    assert kh.get("parthenon/time", "integrator") == "rk3"
    v = configs.vortex_2d()
    assert v.get("parthenon/meshblock", "nx1") == "64" and v.get("parthenon/mesh", "nghost") == "2"
    ot = configs.ot_3d()
    assert ot.get("physics", "MHD") == "ct" and ot.get("parthenon/mesh", "nghost") == "4"


def test_block_assignment_and_input_file(tmp_path):
    # the reference's params["block"] = {...} form and its write_input layout
    d = Deck()
    d["hydro"] = {"reconstruction": "wenoz", "cfl": 0.4}
    d["parthenon/mesh"] = {"nx1": 64}
    assert d["hydro"] == {"reconstruction": "wenoz", "cfl": "0.4"}
    f = tmp_path / "run.in"
    d.write(f, problem_id="vortex")
    text = f.read_text()
    assert text.splitlines()[0] == "<parthenon/job>"
    assert "problem_id = vortex" in text
    back = Deck.parse(text)
    assert back.get("hydro", "reconstruction") == "wenoz"
    assert back.get("parthenon/mesh", "nx1") == "64"
