"""CPU oracle for the voxel hex8 GMG-PCG solve -- TEST INFRASTRUCTURE ONLY.

This package is a plain-numpy restatement of the reference solver's algorithm
(VoxelSim-FEA ``core/fea.py`` and ``core/multigrid.py``), written from the
published algorithm and cited function by function.  It exists to check the
CUDA path, never to stand in for it:

* only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
  ``--impl reference`` legs of ``bench.py`` may import it;
* the product package (``voxelsim_fea_b200``) never imports it, and its solve
  path fails loudly when the CUDA library is missing.

Parity pin: the restatement is checked against golden vectors generated from
the reference's own code (``tests/golden/make_golden.py`` imports the
reference read-only and writes ``tests/golden/*.npz``); see
``tests/test_oracle_golden.py``.

Modules
-------
hex8      element stiffness / stress matrices and connectivity (fea.py:27-148)
islands   support-connectivity flood fill (fea.py:151-227)
mg        geometric-multigrid PCG on the full grid (multigrid.py:38-583)
fea       VoxelFEA facade: active compression, Jacobi-PCG, von Mises (fea.py:234-626)
galerkin  sparse Galerkin (R A P) coarse operators -- oracle for the
          project's own robust coarse hierarchy (not a reference algorithm)
"""
