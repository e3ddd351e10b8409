"""Solver: one periodic solve driven through liboux's C ABI.

Device memory is PyTorch-owned (torch is the allocator and stream provider, the
library never calls cudaMalloc for a solve).  The hot path is entirely inside
liboux; this class only carries pointers and sizes across the boundary.
"""
from __future__ import annotations

import ctypes as C
import numpy as np
import torch

from . import _lib
from ._lib import LIB, check
from .config import SolverConfig  # noqa: F401  (re-exported)


class Solver:
    """A bound liboux handle with its device state and scratch.

    `device` must be a CUDA device; the CUDA library is the only implementation.
    """

    def __init__(self, cfg: SolverConfig, device: str | torch.device = "cuda:0"):
        self.cfg = cfg
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("liboux runs on a CUDA device only (no CPU fallback)")
        c, keep = cfg.to_c()
        h = C.c_void_p()
        check(LIB.oux_create(C.byref(c), C.byref(h)))
        self._h = h
        sb, kb = C.c_size_t(), C.c_size_t()
        check(LIB.oux_state_bytes(C.byref(c), C.byref(sb)))
        check(LIB.oux_scratch_bytes(C.byref(c), C.byref(kb)))
        del keep
        self.state = torch.empty(sb.value // 8, dtype=torch.float64, device=self.device)
        self.scratch = torch.empty((kb.value + 7) // 8, dtype=torch.float64, device=self.device)
        self.stream = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            check(LIB.oux_bind(self._h, C.c_void_p(self.state.data_ptr()), C.c_void_p(self.scratch.data_ptr()),
                               C.c_size_t(self.scratch.numel() * 8), C.c_void_p(self.stream.cuda_stream)))
        lay = _lib.OuxLayout()
        check(LIB.oux_layout_of(self._h, C.byref(lay)))
        self.layout = lay
        self._bfix = {}  # device copies of boundary values / kinds (the library reads them every fill)
        for r in cfg.boundary_rules():
            face = r["face"]
            if r["farfield"] is not None:
                check(LIB.oux_set_boundary_farfield(self._h, face, *r["farfield"]))
            else:
                ptr = None
                if r["fixed"] is not None:
                    t = torch.from_numpy(r["fixed"].ravel()).to(self.device)
                    self._bfix[face] = t
                    ptr = C.c_void_p(t.data_ptr())
                check(LIB.oux_set_boundary(self._h, face, r["kind"], ptr))
            if r["cells"] is not None:
                t = torch.from_numpy(r["cells"]).to(self.device)
                self._bfix[("cells", face)] = t
                check(LIB.oux_set_boundary_cells(self._h, face, C.c_void_p(t.data_ptr())))
        check(LIB.oux_set_boundary_order(self._h, 1 if cfg.boundary_order == "y_last" else 0))

    # -- lifetime --
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            LIB.oux_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _s(self) -> C.c_void_p:
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    # -- state transfer (reference layout QJ(nx,nv,ny[,nz]), Fortran order) --
    def set_state(self, qj: np.ndarray) -> None:
        a = np.asfortranarray(qj, dtype=np.float64)
        self._keep = a  # the copy is asynchronous: keep the host buffer alive
        with torch.cuda.device(self.device):
            check(LIB.oux_set_state(self._h, a.ctypes.data_as(C.POINTER(C.c_double)), self._s()))
            torch.cuda.current_stream(self.device).synchronize()
        self._keep = None

    def get_state(self) -> np.ndarray:
        c = self.cfg
        shape = (c.nx, c.nv, c.ny, c.nz) if c.dim == 3 else (c.nx, c.nv, c.ny)
        out = np.empty(shape, dtype=np.float64, order="F")
        with torch.cuda.device(self.device):
            check(LIB.oux_get_state(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), self._s()))
        return out

    # -- hot path --
    def step(self, nsteps: int = 1) -> None:
        with torch.cuda.device(self.device):
            check(LIB.oux_step(self._h, int(nsteps), self._s()))

    def fill_ghosts(self) -> None:
        with torch.cuda.device(self.device):
            check(LIB.oux_fill_ghosts(self._h, self._s()))

    def rhs(self) -> np.ndarray:
        """The stage residual of the current state in the reference's Rs order."""
        c = self.cfg
        n = c.nv * (c.nx - 2) * (c.ny - 2) * ((c.nz - 2) if c.dim == 3 else 1)
        out = torch.zeros(n, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            check(LIB.oux_rhs(self._h, C.c_void_p(out.data_ptr()), self._s()))
        shape = (c.nx - 2, c.nv, c.ny - 2, c.nz - 2) if c.dim == 3 else (c.nx - 2, c.nv, c.ny - 2)
        return out.cpu().numpy().reshape(shape[::-1]).transpose(tuple(range(len(shape)))[::-1])

    def diagnostics(self) -> tuple[float, float, float]:
        out = (C.c_double * 3)()
        with torch.cuda.device(self.device):
            check(LIB.oux_diagnostics(self._h, out, self._s()))
        return out[0], out[1], out[2]

    def check_state(self) -> int:
        bits = C.c_int32()
        with torch.cuda.device(self.device):
            rc = LIB.oux_check_state(self._h, C.byref(bits), self._s())
        if rc not in (_lib.OUX_OK, _lib.OUX_E_DEVICE_FAULT):
            check(rc)
        return bits.value

    def launches(self) -> int:
        n = C.c_int64()
        check(LIB.oux_launch_count(self._h, C.byref(n)))
        return n.value
