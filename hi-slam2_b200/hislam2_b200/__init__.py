"""hislam2_b200: B200 (sm_100a) kernels for HI-SLAM2's dense BA + correlation path.

``hislam2_b200.backends`` holds the operators with the reference extension's
signatures; the sibling package ``droid_backends`` re-exports them under the
reference's module name so HI-SLAM2's ``factor_graph.py``, ``track_frontend.py``
and ``track_backend.py`` run unchanged with ``hi-slam2_b200`` on ``sys.path``.
"""

from . import _lib  # noqa: F401
from .backends import (ba, frame_distance, corr_index_forward, corr_index_backward,  # noqa: F401
                       altcorr_forward, altcorr_backward, ba_keys, ba_workspace_bytes)

__all__ = ["ba", "frame_distance", "corr_index_forward", "corr_index_backward", "altcorr_forward",
           "altcorr_backward", "ba_keys", "ba_workspace_bytes"]
