"""PDHCG-B200: a B200-native restarted Halpern PDHG / PDHCG solver behind the
reference's C interface (include/pdhcg.h).  The solver is libpdhcg_b200.so
(C++ host + sm_100a CUDA kernels); this package holds its Python host side:
ctypes bindings (capi, native), seeded instance generators (instances) and
the build recipe (build)."""
__version__ = "0.1.0"
