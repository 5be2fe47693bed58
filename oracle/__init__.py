"""CPU oracle for the dense-BA + correlation path (TEST INFRASTRUCTURE ONLY).

This package is a float64 numpy restatement of the reference operators that the
drop-in replaces (HI-SLAM2 ``src/droid_kernels.cu``, ``src/correlation_kernels.cu``,
``src/altcorr_kernel.cu``).  Every function cites the reference file:line it
follows.

It is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.
The product path (``hislam2_b200`` / ``droid_backends``) never imports it and fails
loudly when its CUDA library is missing.

Pinning status (how far the oracle itself is checked against the reference):
  * corr_index_forward/backward, altcorr_forward/backward: pinned against the
    reference's own CUDA sources (``src/correlation_kernels.cu``,
    ``src/altcorr_kernel.cu``) compiled unmodified into ``oracle/_ref`` and run on
    a GPU (golden fixtures under ``tests/golden`` plus the live GPU tests).
  * ba, pgba, frame_distance, iproj, covis_distance, depth_filter: parity unpinned.  ``src/droid_kernels.cu`` cannot be
    built here (it includes Eigen, which is absent), the reference has no tests
    or golden vectors, and its Python path needs lietorch/torch_scatter (absent).
    These oracle functions are instead checked by independent mathematical
    identities (finite-difference Jacobians, the damped normal equations, the
    Schur complement against a direct joint solve).
"""

from . import se3, ba, corr, frame_distance, geometry, pgba  # noqa: F401
