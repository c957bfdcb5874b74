"""Device-resident cross-pass reuse store (reference option ``reuse="warm"``).

The reference keeps, per time step of a forward run, the converged load increment and ocean
function in a caller-owned dict (``reuse_store``, SLEvolve python/slevolve/solver_opt.py:
400-403, 514-528, 932-947) so that the next outer iteration over the same ice history
(run_outer.py) starts every step from them.  Here the store is two device arrays that outlive the
solvers of the successive passes: ``[capacity][ncoef]`` complex128 increments (packed) and
``[capacity][nlat*nlon]`` bytes of ocean function.  Entries ``0 .. recorded-1`` hold the steps a
pass has completed; a new pass reads step k's entry before the step and overwrites it after.
"""

from __future__ import annotations

import ctypes as C


class ReuseStore:
    """Grows on demand; ``recorded`` = steps completed by the latest pass."""

    def __init__(self, ncoef, ngrid, capacity=64):
        import torch

        self.ncoef, self.ngrid = int(ncoef), int(ngrid)
        self.recorded = 0
        self.ds = torch.zeros((max(1, int(capacity)), self.ncoef), dtype=torch.complex128, device="cuda")
        self.mask = torch.zeros((max(1, int(capacity)), self.ngrid), dtype=torch.uint8, device="cuda")

    @property
    def capacity(self) -> int:
        return int(self.ds.shape[0])

    @property
    def nbytes(self) -> int:
        return int(self.ds.numel() * 16 + self.mask.numel())

    def ensure(self, steps):
        """Capacity for `steps` entries (reallocates and keeps the recorded ones)."""
        import torch

        if steps <= self.capacity:
            return False
        cap = max(int(steps), 2 * self.capacity)
        ds = torch.zeros((cap, self.ncoef), dtype=torch.complex128, device="cuda")
        mask = torch.zeros((cap, self.ngrid), dtype=torch.uint8, device="cuda")
        ds[: self.capacity].copy_(self.ds)
        mask[: self.capacity].copy_(self.mask)
        self.ds, self.mask = ds, mask
        return True

    def pointers(self):
        return C.c_void_p(self.ds.data_ptr()), C.c_void_p(self.mask.data_ptr())
