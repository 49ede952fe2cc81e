"""B200-native implementation of DNDSR's implicit residual path.

Variational reconstruction, Euler/NS right-hand side, local time step and
LU-SGS, as CUDA kernels for sm_100a behind the C-ABI of include/dndsb.h.
"""
from . import mesh  # noqa: F401  (synthetic mesh generation, host side)


def __getattr__(name):
    # the CUDA-backed classes load libdndsb.so lazily, so `import dndsr_b200` works on build hosts
    if name in ("VariationalReconstruction", "EulerEvaluator", "DeviceMesh"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
