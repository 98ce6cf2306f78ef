"""
mom25d_b200 - the per-frequency hot path of the 2.5-D MoM PCB solver mom25d (dense impedance-matrix fill with
layered-media Green tables, near-field singularity corrections and via kernels; complex dense LU and solves) as
hand-written CUDA for one B200 (sm_100a), behind the reference's own call signatures:

    from mom25d_b200.sim import Simulation          # Simulation(...).sparams(f)
    from mom25d_b200.run import solve_band          # solve_band(sim, fmin, fmax, linear=N)
    from mom25d_b200 import core                    # the compiled-core module's functions (fill_far, ...)
    from mom25d_b200.backend import CudaBackend     # the GPU LU backend seam (gpu.py)

The kernels live in libmom25d_b200.so (include/mom25d_b200.h); there is no CPU path.
"""
__version__ = '0.1.0'


def umma_available():
    """Whether the library carries the tensor-core (tcgen05, 3xTF32) trailing update of the complex64 LU."""
    from . import _lib
    try:
        f = getattr(_lib.lib(), 'm25_umma_available')
    except AttributeError:
        return False
    return bool(f())
