"""B200 streamline tracker with the ``cuslines`` API.

Drop-in names of ``cuslines/__init__.py:82-88``: ``Tracker`` (= ``GPUTracker``),
``BootDirectionGetter``, ``ProbDirectionGetter``, ``PttDirectionGetter`` and
``BACKEND``.  The only backend is hand-written sm_100a CUDA behind a C ABI
(``include/gpustreamlines_b200.h``); there is no CPU fallback.
"""

from .direction_getters import BootDirectionGetter, ProbDirectionGetter, PttDirectionGetter
from .tracker import GPUTracker

Tracker = GPUTracker
BACKEND = "cuda"

__all__ = [
    "Tracker",
    "GPUTracker",
    "ProbDirectionGetter",
    "PttDirectionGetter",
    "BootDirectionGetter",
    "BACKEND",
]
