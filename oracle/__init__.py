"""ORACLE — test infrastructure only.

CPU restatements of the reference's hot-path algorithms, used as the checker by
tests/, by ``__graft_entry__.smoke()`` and by bench.py's CPU-baseline leg (and its
``--impl reference`` arm).  The product package (laqphysics_b200) never imports
anything from here.

* ``cpu.tensor_apply``: the C/OpenMP restatement of src/kernels.f90:119-176
  (oracle/tensor_apply.c), pinned to the reference's Kronecker assembly;
* ``arnoldi``: numpy restatement of python/propagate.py:6-50;
* ``implicit``: numpy/scipy restatement of python/implicit.py:13-109;
* ``surface``: numpy restatement of the flux, contraction and Volkov integral of
  python/helium3d.py:69-77, python/surface_contract.py:41-56 and
  python/streaming_surface.py:39-64.
Each is pinned against goldens produced by the reference itself
(tests/golden/make_golden.py).
"""
