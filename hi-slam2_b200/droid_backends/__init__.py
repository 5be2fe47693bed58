"""Drop-in replacement for HI-SLAM2's compiled ``droid_backends`` extension.

Exposes the operators of the dense-BA + correlation path with the reference's
names and positional signatures (``src/droid.cpp:325-341``): ``ba``,
``frame_distance``, ``corr_index_forward``, ``corr_index_backward``,
``altcorr_forward`` and ``altcorr_backward``, plus the keyframe / point-cloud
helpers ``covis_distance``, ``depth_filter`` and ``iproj``, the two operators of
the mono-depth-prior alignment ``proj_trans`` and ``bi_inter``, and the Sim3
pose-graph bundle adjustment ``pgba``.  They run on the B200 kernels of
``hislam2_b200``; there is no CPU fallback.
"""

from hislam2_b200.backends import (ba, frame_distance, corr_index_forward, corr_index_backward,  # noqa: F401
                                   altcorr_forward, altcorr_backward, covis_distance, depth_filter, iproj,
                                   proj_trans, bi_inter, pgba)
