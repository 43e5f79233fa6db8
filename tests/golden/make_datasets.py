"""Regenerates tests/golden/datasets.json: SHA-256 digests of the reference's own dataset
scripts' outputs, which the native gslam-data tool must reproduce byte for byte.

    python tests/golden/make_datasets.py

Runs data/generate_citytrees.py (several sizes and seeds) and data/convert_slampp.py
from the reference tree: on tests/golden/slampp_sample.txt (written here from a seeded
generator, with gaps, a repeated odometry record, a blank line and a foreign record) and
on tests/golden/slampp_edge_values.txt (hand-written: subnormal, largest, negative-zero,
1e-05 / 1e16 boundary and 17-digit values, so every branch of Python's float repr is
exercised).
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DATA = os.path.join(os.environ.get("GSLAM_REFERENCE", "/root/reference"), "data")
CITYTREES = [(1, 5), (80, 0), (300, 42), (1000, 7), (2500, 3), (10000, 42), (30000, 42)]
SLAMPP = [("slampp_sample.txt", "1.0"), ("slampp_sample.txt", "0.5"), ("slampp_edge_values.txt", "1.0")]


def slampp_sample(path):
    rng = np.random.default_rng(5)
    lines = []
    for i in range(200):
        if i in (37, 38, 120):
            continue
        dx, dy, dt = rng.normal(1.0, 0.1), rng.normal(0, 0.05), rng.normal(0, 0.02) if i % 7 else 0.0
        lines.append(f"ODOMETRY {i} {i + 1} {dx!r} {dy!r} {dt!r} 1 0 0 1 0 1")
        if i % 3 == 0:
            lines.append(f"LANDMARK {i} {int(rng.integers(0, 40))} {rng.uniform(1, 8)!r} "
                         f"{rng.uniform(-1.5, 1.5)!r} 1 0 1")
        if i == 50:
            lines += ["", "VERTEX2 51 0 0 0", "ODOMETRY 40 41 0.5 0.0 0.1 1 0 0 1 0 1"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def digest(path):
    with open(path, "rb") as f:
        data = f.read()
    return {"sha256": hashlib.sha256(data).hexdigest(), "bytes": len(data)}


def main():
    sample = os.path.join(HERE, "slampp_sample.txt")
    slampp_sample(sample)
    out = {"citytrees": [], "slampp": []}
    with tempfile.TemporaryDirectory() as tmp:
        for n, seed in CITYTREES:
            p = os.path.join(tmp, f"ct_{n}_{seed}.txt")
            subprocess.run([sys.executable, os.path.join(REF_DATA, "generate_citytrees.py"), str(n), p, str(seed)],
                           check=True, capture_output=True)
            out["citytrees"].append({"n_poses": n, "seed": seed, **digest(p)})
        for name, delta in SLAMPP:
            p = os.path.join(tmp, f"conv_{name}_{delta}.txt")
            r = subprocess.run([sys.executable, os.path.join(REF_DATA, "convert_slampp.py"),
                                os.path.join(HERE, name), p, delta], check=True, capture_output=True, text=True)
            out["slampp"].append({"input": name, "delta": delta, "summary": r.stdout.splitlines()[1], **digest(p)})
    with open(os.path.join(HERE, "datasets.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote datasets.json")


if __name__ == "__main__":
    main()
