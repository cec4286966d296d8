"""State files: the writer reproduces the reference's own files byte for
byte (tests/golden/state*_beads_*.dat, written by output_methods.save_state),
the reader reads them in 2D and 3D, and a state round-trips into a
SystemSpec that resumes the run."""
import json
import os

import numpy as np

from gliding_collective_rotation_b200 import state_io as S
from gliding_collective_rotation_b200 import workloads as W
from tests.golden_io import load

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_2d_writer_matches_the_reference_file(tmp_path):
    d, s = load("config1")
    fn = S.write_state(str(tmp_path / "state2d"), 7, 1234, 1.2345678, d["pos0"], d["tangent0"],
                       np.asarray(d["chain_id"]))
    assert os.path.basename(fn) == "state2d_beads_00000007.dat"
    assert open(fn, "rb").read() == open(os.path.join(GOLDEN, "state2d_beads_00000007.dat"), "rb").read()


def test_3d_writer_matches_the_reference_file(tmp_path):
    ref = S.read_state(os.path.join(GOLDEN, "state3d_beads_00000012.dat"))
    # rewrite what was read: the same text (values survive %.8e exactly)
    fn = S.write_state(str(tmp_path / "state3d"), 12, 99, 0.5, ref["pos"], ref["tangent"], ref["chain_id"],
                       ref["inherited_label"], ref["where_active"])
    assert open(fn).read() == open(os.path.join(GOLDEN, "state3d_beads_00000012.dat")).read()


def test_reader_2d():
    d, s = load("config1")
    st = S.read_state(os.path.join(GOLDEN, "state2d_beads_00000007.dat"))
    assert (st["stepnum"], st["filenumber"]) == (1234, 7) and abs(st["t"] - 1.23457) < 1e-12
    assert st["class_name"] == "populations.Equal_Size_Chain_Collection"
    assert np.array_equal(st["chain_id"], np.asarray(d["chain_id"]))
    assert np.allclose(st["pos"], d["pos0"], rtol=1e-8, atol=0)
    t = d["tangent0"] / np.linalg.norm(d["tangent0"], axis=1, keepdims=True)
    assert np.allclose(st["tangent"], t, atol=1e-8)
    assert np.all(st["where_active"] == 0)


def test_reader_3d_finds_columns_by_name():
    st = S.read_state(os.path.join(GOLDEN, "state3d_beads_00000012.dat"))
    assert st["pos"].shape == (72, 3) and st["orientations"].shape == (72, 2)
    assert np.allclose(np.linalg.norm(st["tangent"], axis=1), 1.0)
    L = json.load(open(os.path.join(GOLDEN, "state_index.json")))["state3d_L"]
    assert np.all((st["pos"] >= 0) & (st["pos"] < L))
    assert np.all(st["where_active"] == 0)  # not the phi column


def test_resume_spec_continues_the_step_counter(tmp_path):
    spec = W.config1(seed=0)
    fn = S.write_state(str(tmp_path / "run"), 3, 500, 0.5, spec.pos, spec.tangent, spec.chain_id)
    st = S.read_state(fn)
    resumed = S.spec_from_state(st, spec)
    assert resumed.params.step == 500 and resumed.n == spec.n
    assert np.allclose(resumed.pos, spec.pos, rtol=1e-8)
    assert S.latest_state(str(tmp_path / "run")) == fn
