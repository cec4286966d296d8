"""B200 (sm_100a) hot path of the gliding-collective-rotation Brownian-dynamics step.

``updates.SRK2_force_calc`` is the drop-in for the reference's step
(updates.py:132-267); ``engine.Engine`` is one ``libgcr`` context that can
hold one or many systems; ``batch`` and ``serve`` build the batched sweep and
the continuous-batching request loop on top of it.
"""
from . import _lib  # noqa: F401

__all__ = ["engine", "updates", "config", "defaults", "batch", "serve"]
__version__ = "0.1.0"


def library_path():
    return _lib.LIB_PATH
