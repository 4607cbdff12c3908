"""B200-native discrete natural-neighbour interpolation engine.

The product is the native library ``libdnni.so`` (CUDA kernels for sm_100a
behind the C ABI in ``include/dnni.h`` and the C++ ``nni::`` shim in
``include/nni/nni.h``).  This package holds its sources (``csrc/``), the
in-tree build recipe (``build.py``) and thin Python bindings used by the tests
and the benchmark (``engine.py``, ``synth.py``).
"""
__all__ = ["build", "engine", "synth"]
