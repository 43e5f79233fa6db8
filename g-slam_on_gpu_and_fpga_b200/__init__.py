"""gslam-b200: a B200 (sm_100a) Graph-SLAM back-end.

The product is libgslam.so (C ABI: include/gslam.h, include/gslam_dropin.h) and
the GSLAM program; this package is the Python host side over that ABI:
  abi     ctypes binding of every exported entry point
  graph   PoseGraph (one resident graph) and the reference log reader
  synth   seeded city-grid pose graphs (SE(2) graphs and reference-format logs)
  build   compiles the library and program for sm_100a
The directory name is not a Python identifier; import it with
importlib.import_module("g-slam_on_gpu_and_fpga_b200").
"""
from . import abi, build, dense, graph, shard, synth, tune  # noqa: F401
from .graph import PoseGraph, PoseGraphBatch, ReferenceLog, RoundStats, read_log  # noqa: F401
