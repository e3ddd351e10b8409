"""Z-slab decomposition of one 3D solve over ranks: the reference's COMMZ path
(3D_solver/src/calc_para.f90:343-384, exchanged after every RK stage in
3D_solver/src/calc_time_dev.f90.fypp:465-498).

The global grid's Nz interior planes are split evenly over `world` ranks. Each rank
holds its Nz / world planes plus g ghost planes at each z end (`bc_z = 2`: the library
leaves those planes to the caller). After every stage the rank sends the g lowest
interior planes of the array the stage wrote to the rank below and the g highest to
the rank above (periodic in rank), and writes what it receives into its ghost
planes. x and y stay periodic within the slab.

Two exchanges are provided: `halo_exchange` over a torch.distributed process group
(NCCL between GPUs, gloo for host tensors), and `LocalSlabs`, which runs all slabs
of a grid in one process on one device and exchanges by device copies, one slab
after the other (no kernel waits on another slab's).
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np
import torch
import torch.distributed as dist

from ._lib import LIB, check
from .solver import Solver, SolverConfig

# message tags: a rank's highest planes go up (received as the lower halo), its
# lowest planes go down (received as the upper halo)
TAG_UP, TAG_DOWN = 1, 2


def slab_bounds(nz: int, g: int, rank: int, world: int) -> tuple[int, int]:
    """(k0, nz_local): the slab's first global plane (ghosts included) and its plane count."""
    Nz = nz - 2 * g
    if world < 1 or Nz % world:
        raise ValueError(f"{Nz} interior z planes do not split evenly over {world} ranks")
    n = Nz // world
    if n < g:
        raise ValueError(f"a slab of {n} planes is thinner than the halo ({g} planes)")
    return rank * n, n + 2 * g


def slab_bc_z(periodic: bool, rank: int, world: int) -> int:
    """The slab's bc_z (enum oux_bc_z): halo planes at both ends, or, on a grid with a
    non-periodic z, the grid's boundary at the first slab's lower / the last slab's
    upper end."""
    if periodic:
        return 2
    if world == 1:
        return 1
    if rank == 0:
        return 3
    return 4 if rank == world - 1 else 2


def slab_config(cfg: SolverConfig, rank: int, world: int) -> tuple[SolverConfig, int]:
    """The rank's local configuration (its bc_z, z spacings and boundary rules) and its k0."""
    if cfg.dim != 3:
        raise ValueError("z slabs need a 3D configuration")
    if cfg.bc_z not in (0, 1):
        raise ValueError("split a periodic (bc_z = 0) or non-periodic (bc_z = 1) grid")
    k0, n = slab_bounds(cfg.nz, cfg.g, rank, world)
    dz = np.asarray(cfg.dz, dtype=np.float64)[k0:k0 + n - 1].copy()
    bc_z = slab_bc_z(cfg.bc_z == 0, rank, world)
    boundary = None
    if cfg.boundary:
        boundary = {}
        for face, rule in cfg.boundary.items():
            if face == "z_lo" and bc_z not in (1, 3):
                continue
            if face == "z_hi" and bc_z not in (1, 4):
                continue
            if not isinstance(rule, str) and rule[0] == "fixed" and face in ("x_lo", "x_hi", "y_lo", "y_hi"):
                # 3D fixed values are indexed (l, k, position in the plane): keep the slab's planes
                v = np.asarray(rule[1])
                other = cfg.ny if face.startswith("x") else cfg.nx
                v = v.reshape(v.shape[0], cfg.nz, other)[:, k0:k0 + n].reshape(v.shape[0], -1)
                rule = ("fixed", v)
            boundary[face] = rule
    return dataclasses.replace(cfg, nz=n, dz=dz, bc_z=bc_z, boundary=boundary), k0


def slab_state(qj: np.ndarray, cfg: SolverConfig, rank: int, world: int) -> np.ndarray:
    """The rank's part of a global state in the reference layout QJ(nx, nv, ny, nz)."""
    k0, n = slab_bounds(cfg.nz, cfg.g, rank, world)
    return np.asfortranarray(qj[:, :, :, k0:k0 + n])


def halo_exchange(send_lo: torch.Tensor, send_hi: torch.Tensor, recv_lo: torch.Tensor, recv_hi: torch.Tensor,
                  rank: int, world: int, group=None, periodic: bool = True) -> None:
    """Send `send_lo` down and `send_hi` up; receive the lower halo from below into
    `recv_lo` and the upper halo from above into `recv_hi` (periodic in rank; with a
    non-periodic z the first rank has no rank below and the last none above).

    Sends and receives are posted in the same order on every rank (up first, then
    down) and tagged, so two ranks that are each other's upper and lower neighbour
    match them correctly."""
    for req in post_halo_exchange(send_lo, send_hi, recv_lo, recv_hi, rank, world, group, periodic):
        req.wait()


def post_halo_exchange(send_lo: torch.Tensor, send_hi: torch.Tensor, recv_lo: torch.Tensor, recv_hi: torch.Tensor,
                       rank: int, world: int, group=None, periodic: bool = True) -> list:
    """halo_exchange without the wait: the posted requests (NCCL: waiting on one makes
    the current CUDA stream wait for it, so the caller can queue work in between)."""
    if world == 1:
        if periodic:
            recv_lo.copy_(send_hi)
            recv_hi.copy_(send_lo)
        return []
    up, down = (rank + 1) % world, (rank - 1) % world
    has_up = periodic or rank < world - 1
    has_down = periodic or rank > 0
    ops = []
    if has_up:
        ops.append(dist.P2POp(dist.isend, send_hi, up, group, TAG_UP))
    if has_down:
        ops.append(dist.P2POp(dist.irecv, recv_lo, down, group, TAG_UP))
        ops.append(dist.P2POp(dist.isend, send_lo, down, group, TAG_DOWN))
    if has_up:
        ops.append(dist.P2POp(dist.irecv, recv_hi, up, group, TAG_DOWN))
    return dist.batch_isend_irecv(ops) if ops else []


class SlabSolver:
    """One rank's slab of a global 3D solve, driven stage by stage with halo exchanges."""

    def __init__(self, cfg: SolverConfig, rank: int, world: int, device, group=None):
        self.global_cfg = cfg
        self.rank, self.world, self.group = rank, world, group
        self.cfg, self.k0 = slab_config(cfg, rank, world)
        self.solver = Solver(self.cfg, device)
        self.device = self.solver.device
        self.stages = 3 if cfg.rk == 3 else 4
        nbytes = max(self._halo_bytes(st) for st in range(self.stages))
        self.bufs = [torch.empty(nbytes, dtype=torch.uint8, device=self.device) for _ in range(4)]

    def _halo_bytes(self, stage: int) -> int:
        b = C.c_size_t()
        check(LIB.oux_halo_bytes(self.solver._h, stage, C.byref(b)))
        return b.value

    def set_global_state(self, qj: np.ndarray) -> None:
        self.solver.set_state(slab_state(qj, self.global_cfg, self.rank, self.world))

    def get_state(self) -> np.ndarray:
        return self.solver.get_state()

    # the steps of one stage, split so that a group of slabs in one process can
    # interleave them
    def run_stage(self, st: int, part: int = 0) -> None:
        """Stage st whole (part 0), or its interior planes (1) / its end planes and the
        ghost fill (2): oux_stage_part."""
        with torch.cuda.device(self.device):
            check(LIB.oux_stage_part(self.solver._h, st, part, self.solver._s()))

    def pack(self, st: int) -> tuple[torch.Tensor, torch.Tensor]:
        n = self._halo_bytes(st)
        lo, hi = self.bufs[0][:n], self.bufs[1][:n]
        with torch.cuda.device(self.device):
            check(LIB.oux_halo_pack(self.solver._h, st, C.c_void_p(lo.data_ptr()), C.c_void_p(hi.data_ptr()),
                                    self.solver._s()))
        return lo, hi

    def recv_buffers(self, st: int) -> tuple[torch.Tensor, torch.Tensor]:
        n = self._halo_bytes(st)
        return self.bufs[2][:n], self.bufs[3][:n]

    def unpack(self, st: int) -> None:
        lo, hi = self.recv_buffers(st)
        with torch.cuda.device(self.device):
            check(LIB.oux_halo_unpack(self.solver._h, st, C.c_void_p(lo.data_ptr()), C.c_void_p(hi.data_ptr()),
                                      self.solver._s()))

    def step(self, nsteps: int = 1) -> None:
        """nsteps time steps, exchanging halos with the neighbouring ranks after each stage.

        Each exchange overlaps the next stage's interior part: the stage's end planes are
        packed and posted, the next stage updates its interior planes (which do not read
        the ghost planes), then waits for the halo, unpacks it and updates its end
        planes (calc_time_dev.f90.fypp:465-470).  The last exchange completes before
        returning."""
        if self.world == 1:  # a slab exchanging with itself has nothing to overlap
            for _ in range(nsteps):
                for st in range(self.stages):
                    self.run_stage(st)
                    self._finish(self._post(st))
            return
        pending = None
        for _ in range(nsteps):
            for st in range(self.stages):
                self.run_stage(st, 1)
                pending = self._finish(pending)
                self.run_stage(st, 2)
                pending = self._post(st)
        self._finish(pending)

    def _post(self, st: int):
        send_lo, send_hi = self.pack(st)
        recv_lo, recv_hi = self.recv_buffers(st)
        with torch.cuda.device(self.device):
            reqs = post_halo_exchange(send_lo, send_hi, recv_lo, recv_hi, self.rank, self.world, self.group,
                                      periodic=self.global_cfg.bc_z == 0)
        return reqs, st

    def _finish(self, pending):
        if pending is not None:
            reqs, st = pending
            with torch.cuda.device(self.device):
                for req in reqs:
                    req.wait()
            self.unpack(st)
        return None

    def close(self) -> None:
        self.solver.close()


class LocalSlabs:
    """All `world` slabs of a global 3D solve in one process on one device: the
    decomposition without a process group (halo exchange by device copies)."""

    def __init__(self, cfg: SolverConfig, world: int, device="cuda:0"):
        self.cfg = cfg
        self.world = world
        self.slabs = [SlabSolver(cfg, r, world, device) for r in range(world)]

    def set_state(self, qj: np.ndarray) -> None:
        for s in self.slabs:
            s.set_global_state(qj)

    def step(self, nsteps: int = 1) -> None:
        """As SlabSolver.step, every slab's part at a time: interior parts, then the
        previous stage's halo copies and unpacks, then the end parts and packs."""
        W = self.world
        periodic = self.cfg.bc_z == 0
        sent = prev = None
        for _ in range(nsteps):
            for st in range(self.slabs[0].stages):
                for s in self.slabs:
                    s.run_stage(st, 1)
                if sent is not None:
                    self._deliver(sent, prev, periodic)
                for s in self.slabs:
                    s.run_stage(st, 2)
                sent, prev = [s.pack(st) for s in self.slabs], st
        if sent is not None:
            self._deliver(sent, prev, periodic)

    def _deliver(self, sent, st: int, periodic: bool) -> None:
        W = self.world
        for r, s in enumerate(self.slabs):
            recv_lo, recv_hi = s.recv_buffers(st)
            if periodic or r > 0:
                recv_lo.copy_(sent[(r - 1) % W][1])  # the highest planes of the slab below
            if periodic or r < W - 1:
                recv_hi.copy_(sent[(r + 1) % W][0])  # the lowest planes of the slab above
        for s in self.slabs:
            s.unpack(st)

    def get_state(self) -> np.ndarray:
        """The global state reassembled (ghost planes from the first and last slab)."""
        g = self.cfg.g
        parts = [s.get_state() for s in self.slabs]
        inner = [p[:, :, :, g:-g] for p in parts]
        return np.asfortranarray(np.concatenate([parts[0][:, :, :, :g], *inner, parts[-1][:, :, :, -g:]], axis=3))

    def check_state(self) -> int:
        """The OR of the slabs' fault bits (NaN / non-positive density or pressure)."""
        bits = 0
        for s in self.slabs:
            bits |= s.solver.check_state()
        return bits

    def diagnostics(self) -> tuple[float, float, float]:
        """KE, entropy and enstrophy averaged over the whole grid (the slabs hold equal
        numbers of cells)."""
        d = np.array([s.solver.diagnostics() for s in self.slabs])
        return tuple(float(x) for x in d.mean(axis=0))

    def close(self) -> None:
        for s in self.slabs:
            s.close()
