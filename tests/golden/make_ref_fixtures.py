"""Regenerates the reference-data fixtures that GPU tests replay on machines without the
reference tree:

  ref_citytrees800.npz   data/cityTrees800.txt, parsed (delta, u, x, z records)
  ref_victoria_park.npz  data/victoria-park.log.txt, parsed
  ref_vp_pcg_fp64.npz    scripts/_pose_dumps_vp/cpu_pcg_fp64.txt: the reference CPU program's
                         pose dump of `GSLAM 1 1.0 200 1 victoria-park.log.txt` (116 rounds),
                         which the oracle reproduces bit for bit (tests/test_oracle_pin.py)
  ref_vp100_gj_fp64.npz  data/victoria-park-100.log.txt, parsed, with
                         scripts/_pose_dumps_vp/cpu_gj_fp64.txt: the reference's dense
                         Gauss-Jordan program's pose dump on it at lambda 0.06
                         (scripts/regen_gj_plot.py), which the oracle's dense run matches to
                         ~1e-7 (the program inverts with a parallel twin of the serial GJ)

Logs are stored as the arrays the reference's read_data yields (parsed here by
libgslam's gslam_read_log, itself checked against the oracle's parser); the tests
write them back with synth.write_log, whose shortest round-trip formatting gives the
same doubles, so a program reading the rewritten file sees exactly the reference's
inputs. This script checks that round trip before saving.

    GSLAM_REFERENCE=<reference tree> python tests/golden/make_ref_fixtures.py
"""
import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.environ.get("GSLAM_REFERENCE", "/root/reference")


def log_arrays(log):
    return dict(delta=np.float64(log.delta), u_step=log.u_step, u=log.u, x_step=log.x_step, x=log.x,
                z_step=log.z_step, z_lm=log.z_lm, z=log.z)


def main():
    G = importlib.import_module("g-slam_on_gpu_and_fpga_b200")
    G.build.build()
    for name, out in (("cityTrees800.txt", "ref_citytrees800.npz"),
                      ("victoria-park.log.txt", "ref_victoria_park.npz")):
        log = G.read_log(os.path.join(REF, "data", name))
        arrs = log_arrays(log)
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, name)
            G.synth.write_log(p, log)
            back = log_arrays(G.read_log(p))
        for k in arrs:
            a, b = np.asarray(arrs[k]), np.asarray(back[k])
            assert a.dtype == b.dtype and a.shape == b.shape and a.tobytes() == b.tobytes(), f"{name}: {k}"
        np.savez_compressed(os.path.join(HERE, out), **arrs)
        print("wrote", out, {k: np.shape(v) for k, v in arrs.items()})
    dump = np.loadtxt(os.path.join(REF, "scripts", "_pose_dumps_vp", "cpu_pcg_fp64.txt"), ndmin=2)
    np.savez_compressed(os.path.join(HERE, "ref_vp_pcg_fp64.npz"), steps=dump[:, 0].astype(np.uint32),
                        poses=dump[:, 1:].copy(), rounds=np.int32(116), lam=np.float64(1.0))
    print("wrote ref_vp_pcg_fp64.npz", dump.shape)
    log = G.read_log(os.path.join(REF, "data", "victoria-park-100.log.txt"))
    arrs = log_arrays(log)
    gj = np.loadtxt(os.path.join(REF, "scripts", "_pose_dumps_vp", "cpu_gj_fp64.txt"), ndmin=2)
    np.savez_compressed(os.path.join(HERE, "ref_vp100_gj_fp64.npz"), **arrs,
                        dump_steps=gj[:, 0].astype(np.uint32), dump_poses=gj[:, 1:].copy(), lam=np.float64(0.06))
    print("wrote ref_vp100_gj_fp64.npz", gj.shape)


if __name__ == "__main__":
    main()
