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
    ``src/altcorr_kernel.cu``) compiled unmodified into ``oracle/_ref`` (golden
    fixtures under ``tests/golden`` plus live GPU tests).
  * ba, pgba, frame_distance, iproj, covis_distance, depth_filter, proj_trans,
    bi_inter: pinned against ``src/droid_kernels.cu`` compiled unmodified into
    ``oracle/_ref`` with a self-written dense stand-in for the Eigen facilities it
    includes (``oracle/eigen_standin``): fixtures ``ba_*``, ``pgba_*``, ``geo_*`` and
    live GPU tests.  Beyond that they are checked by independent identities
    (finite-difference Jacobians, the damped normal equations, the Schur complement
    against a direct joint solve).
  * jdsa (``jdsa.py``): pinned against the reference's own Python ``JDSA`` run here on
    the CPU with stand-ins for its uninstalled imports (fixtures ``jdsa_*``).
  * pgo (``pgo.py``): the procedure is pinned against the reference's own
    ``num_jacobi`` / ``global_relative_posesim3_constraints`` run on a Sim3 stand-in
    (fixtures ``pgo_*``); the Sim3 algebra by group identities; against lietorch
    itself (not installed) parity is unpinned.
  * lm_step (the float64 PyTorch LM step the adjoint tests differentiate): its forward
    equals one iteration of ``ba.py`` and its closed-form adjoint equals autograd through
    it (``tests/test_oracle_lm_step.py``).  torch_path (the CPU baseline's port of the
    reference's Python BA): its Jacobians against finite differences of its own
    reprojection (``tests/test_torch_path.py``).
"""

from . import se3, ba, corr, frame_distance, geometry, pgba  # noqa: F401
