"""
mom25d_b200.backend - the reference's GPU LU backend seam (mom25d gpu.py:28-110, the `_Backend` interface and its
registry gpu._BACKENDS / get_backend) on the B200: the complex dense LU of Z^T in place with LAPACK's pivots, its
triangular solves on the device, the factor's download in scipy.linalg.lu_factor's form.

    import mom25d.gpu as gpu
    from mom25d_b200.backend import CudaBackend
    gpu._BACKENDS['cuda'] = CudaBackend          # then MOM25D_GPU=cuda, or get_backend('cuda')

The factorisation is libmom25d_b200's m25_getrf (blocked right-looking LU with partial pivoting; for complex64 the
trailing updates run on the tensor cores as 3xTF32 products) and the solves m25_getrs_aux (diagonal-block inverses
prepared once per factor). Unlike the reference's CuPy backend, solve() keeps the factor's precision on the device
and returns complex128 as it does.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import P, check, lib, stream_ptr


class GPUUnavailable(RuntimeError):
    """No CUDA device, or libmom25d_b200.so is not built (the reference's gpu.GPUUnavailable)."""


class CudaBackend:
    """The `_Backend` interface (gpu.py:28-48): name, device, inplace, hip, api, lu, piv; mem_free(), mem_total(),
    vram_needed(N), fits(N, extra), factor(Z), solve(R), download(), release()."""
    name, inplace, hip = 'cuda', True, False
    api = 'CUDA'

    def __init__(self, device=0, tf32=None):
        if not torch.cuda.is_available():
            raise GPUUnavailable("cuda: no CUDA device")
        try:
            lib()
        except _lib.M25Error as e:
            raise GPUUnavailable(f"cuda: {e}")
        self.dev_index = device
        self.device = torch.cuda.get_device_name(device)
        from . import umma_available
        self.tf32 = umma_available() if tf32 is None else bool(tf32)
        self.lu = self.piv = None
        self._aux = self._work = None
        self._n = 0
        self._single = True

    # ---- memory (gpu.py:36-40) --------------------------------------------------------------------------------
    def _info(self):
        sms, free, total = ctypes.c_int(), ctypes.c_size_t(), ctypes.c_size_t()
        with torch.cuda.device(self.dev_index):
            check(lib().m25_device_info(ctypes.byref(sms), ctypes.byref(free), ctypes.byref(total)),
                  'm25_device_info')
        return free.value, total.value

    def mem_free(self):
        return float(self._info()[0])

    def mem_total(self):
        return float(self._info()[1])

    def vram_needed(self, N, single=True):
        """The factor in place (8 N^2 bytes complex64, 16 N^2 complex128) plus the LU's workspace and the
        solves' diagonal-block inverses."""
        es = 8 if single else 16
        return float(es * N * N + lib().m25_getrf_workspace(int(N), int(single))
                     + lib().m25_getrs_aux_bytes(int(N), int(single)) + 64e6)

    def fits(self, N, extra=0.0):
        return self.vram_needed(N) <= 0.9 * (self.mem_free() + extra)

    # ---- factor / solve / download ----------------------------------------------------------------------------
    def factor(self, Z):
        """Z: host complex64 (or complex128), C-contiguous, square, equilibrated. Factors A = Z^T in place on the
        device (the row-major Z's memory read column-major), LAPACK getrf semantics."""
        Z = np.asarray(Z)
        if Z.ndim != 2 or Z.shape[0] != Z.shape[1] or Z.dtype not in (np.complex64, np.complex128):
            raise ValueError("factor: a square complex64 or complex128 matrix")
        self.release()
        n, single = Z.shape[0], Z.dtype == np.complex64
        with torch.cuda.device(self.dev_index):
            s = stream_ptr()
            A = _lib.dev(Z)
            ipiv = torch.empty(max(n, 1), dtype=torch.int32, device='cuda')
            nb = int(lib().m25_getrf_workspace(n, int(single)))
            work = torch.empty(max(nb, 1), dtype=torch.uint8, device='cuda')
            check(lib().m25_getrf(P(A), ctypes.c_long(n), n, P(ipiv), int(single), int(single and self.tf32),
                                  P(work), ctypes.c_size_t(nb), s), 'm25_getrf')
            na = int(lib().m25_getrs_aux_bytes(n, int(single)))
            aux = torch.empty(max(na, 1), dtype=torch.uint8, device='cuda')
            check(lib().m25_getrs_prepare(P(A), ctypes.c_long(n), n, P(ipiv), int(single), P(aux),
                                          ctypes.c_size_t(na), s), 'm25_getrs_prepare')
            _lib.sync_check(what='factor')
        self.lu, self.piv, self._aux, self._n, self._single = A, ipiv, aux, n, single

    def solve(self, R):
        """Z^-1 R for R (N or N x k, host), in the factor's precision on the device; returned complex128."""
        if self.lu is None:
            raise RuntimeError("solve: no factor (call factor first)")
        R = np.asarray(R)
        vec = R.ndim == 1
        R2 = R.reshape(-1, 1) if vec else R
        if R2.shape[0] != self._n:
            raise ValueError(f"solve: R must have {self._n} rows")
        k = R2.shape[1]
        with torch.cuda.device(self.dev_index):
            B = _lib.dev(R2, np.complex64 if self._single else np.complex128)
            if k:
                check(lib().m25_getrs_aux(P(self.lu), ctypes.c_long(self._n), self._n, int(self._single),
                                          P(self._aux), P(B), k, stream_ptr()), 'm25_getrs_aux')
            _lib.sync_check(what='solve')
            X = B.cpu().numpy().astype(complex)
        return X[:, 0] if vec else X

    def download(self):
        """The factor on the host as scipy.linalg.lu_factor's of A = Z^T: (lu Fortran-ordered, piv 0-based)."""
        if self.lu is None:
            raise RuntimeError("download: no factor")
        M = self.lu.cpu().numpy()                         # row-major memory = A column-major
        return M.T, self.piv[:self._n].cpu().numpy().astype(np.int32)

    def release(self):
        self.lu = self.piv = self._aux = None
        self._n = 0


def register(gpu_module):
    """Adds the backend to the reference's registry (gpu._BACKENDS['cuda']): get_backend('cuda') and
    MOM25D_GPU=cuda then select it."""
    gpu_module._BACKENDS['cuda'] = CudaBackend
    return CudaBackend
