"""B200-native Behler-Parrinello NNP energy/force path (sm_100a).

The compute path is libnnp_b200.so (CUDA, built in this directory); this
package is its Python front end (``ace_b200.nnp``), the potential text
format (``ace_b200.potential``) and seeded synthetic workloads
(``ace_b200.synth``).
"""
from . import potential, synth  # noqa: F401
from .nnp import NNP, NNPError, lib  # noqa: F401

__all__ = ["NNP", "NNPError", "lib", "potential", "synth"]
