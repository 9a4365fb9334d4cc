"""B200 (sm_100a) Monte Carlo form-factor path: Malley emission, nearest-hit
grid traversal and per-(source, hit) counting behind the reference's
ray_caster / emission / form_factors interfaces.

The compute path is libffb200.so (CUDA, built by form_factors_b200.build);
``native`` binds its C ABI, ``emission`` mirrors the reference's per-face ray
budgeting, ``scenes`` builds the seeded synthetic workloads.
"""
from . import emission, scenes  # noqa: F401
from .native import Context, FFBError, load  # noqa: F401
