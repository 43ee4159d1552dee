"""imaged11_b200: ImageD11's grain-scoring hot path on NVIDIA B200 (sm_100a).

* ``imaged11_b200.cImageD11`` -- drop-in for compute_gv, compute_geometry,
  compute_xlylzl, score, score_and_refine, refine_assigned, score_and_assign
  and verify_rounding of ``ImageD11.cImageD11``;
* ``imaged11_b200.synth`` -- seeded synthetic peak sets for tests/benchmarks.

The CUDA library (``libimaged11_b200.so``) is built with
``python -m imaged11_b200.build``; importing ``cImageD11`` without it raises.
"""
__version__ = "0.1.0"
