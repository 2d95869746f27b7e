"""lipika_b200 — B200-native IQ-generation backend for the lipika scene simulator.

The product is liblipika_cuda.so (lipika_b200/csrc): hand-written sm_100a
kernels for the per-chunk transmitter fan-out behind a C ABI
(include/lipika_cuda.h). This Python package is the host-side mirror of the
reference's pipeline API (src/pipeline.rs: run_scene, run_scene_to_dir,
render_window, export_truth) driving that library through ctypes.
"""
from . import config  # noqa: F401

__all__ = ["config"]
