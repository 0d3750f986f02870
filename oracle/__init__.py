"""CPU oracle for the UVLM hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl
reference`` legs of bench.py may import this package, and only as the checker of
the CUDA path.  The product (``pyvl_b200``) never imports it and has no CPU
fallback.

* ``oracle.c`` restates the reference's C kernels (induction, ring reductions,
  centroids, normals, topology, line forces) operation by operation.
* ``oracle.solver`` restates the reference's Python solver loop and free-wake model
  (python/pyvl/solver.py:175-263, python/pyvl/wake_models.py:17-330) with numpy and
  scipy LAPACK.
* ``oracle.ref`` loads the reference's own compiled extension from ``oracle/_ref``
  (built by ``oracle/build_ref.sh``) when it is present.

Parity of this restatement with the reference is pinned by the golden vectors in
tests/golden/ (generated from the compiled reference by tests/golden/make_golden.py).
"""
