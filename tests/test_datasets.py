"""The native dataset tool (gslam-data) against the reference's own scripts.

tests/golden/datasets.json holds SHA-256 digests of the files that
data/generate_citytrees.py and data/convert_slampp.py wrote for these arguments
(tests/golden/make_datasets.py); the tool must write the same bytes.
"""
import hashlib
import json
import os
import subprocess

import pytest

from conftest import load_pkg

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLDEN, "datasets.json")) as _f:
    DIGESTS = json.load(_f)


def _sha(path):
    with open(path, "rb") as f:
        data = f.read()
    return hashlib.sha256(data).hexdigest(), len(data)


@pytest.fixture(scope="module")
def G(pkg):
    return pkg


@pytest.mark.parametrize("case", DIGESTS["citytrees"], ids=lambda c: f"n{c['n_poses']}_s{c['seed']}")
def test_citytrees_bytes_match_reference_script(G, tmp_path, case):
    path = str(tmp_path / "ct.txt")
    out = G.synth.generate_citytrees(case["n_poses"], path, case["seed"])
    assert out.startswith(f"Generated {path}\n  Poses: {case['n_poses']}, Landmarks: ")
    assert _sha(path) == (case["sha256"], case["bytes"])


@pytest.mark.parametrize("case", DIGESTS["slampp"], ids=lambda c: f"{c['input'][:-4]}_delta{c['delta']}")
def test_slampp_bytes_match_reference_script(G, tmp_path, case):
    path = str(tmp_path / "conv.txt")
    out = G.synth.convert_slampp(os.path.join(GOLDEN, case["input"]), path, float(case["delta"]))
    assert out.splitlines()[1] == case["summary"]
    assert _sha(path) == (case["sha256"], case["bytes"])


def test_generated_log_reads_back(G, tmp_path):
    """The generated log is a valid reference log: one u and x record per step, steps in
    order, observations from steps that exist, landmark ids from 6 upwards."""
    path = str(tmp_path / "ct.txt")
    G.synth.generate_citytrees(1500, path, 11)
    log = G.graph.read_log(path)
    n = log.n_poses
    assert n == 1500 and log.u.shape[0] == n
    assert (log.x_step == range(n)).all()
    assert log.z_step.max() < n and log.z_lm.min() >= 6
    assert (log.z[:, 0] <= 8.5).all()


def test_tool_errors(G, tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("LANDMARK 0 1 2.0 0.1\n")
    with pytest.raises(RuntimeError, match="no ODOMETRY"):
        G.synth.convert_slampp(str(bad), str(tmp_path / "o.txt"))
    bad.write_text("ODOMETRY x 1 1.0 0.0 0.0\n")
    with pytest.raises(RuntimeError, match="malformed ODOMETRY"):
        G.synth.convert_slampp(str(bad), str(tmp_path / "o.txt"))
    with pytest.raises(RuntimeError, match="cannot read"):
        G.synth.convert_slampp(str(tmp_path / "absent.txt"), str(tmp_path / "o.txt"))
    r = subprocess.run([G.abi.DATA_TOOL_PATH, "citytrees", "0", str(tmp_path / "o.txt")], capture_output=True)
    assert r.returncode == 1
