"""Output files of a run, byte-compatible with the reference writer.

* ``data/Q%05d.vtr`` -- VTK XML RectilinearGrid with raw appended Float32 data
  (src/print.f90:125-189 print_xml, :337-382 print_vtk_{2D,3D}).  The reference
  writes each appended block's header word as 4 + 4*N (the offset increment)
  instead of the byte count; that quirk is reproduced.
* ``data/kinetic_energy.d`` (t, ke, ke/ke0; Fortran 3e12.4) and
  ``data/entropy.d`` (t, (s0-s)/s0; 2e12.4) from float32 fields with a float32
  running sum (src/print.f90:42-122).
* ``recal/Q00001.dat`` -- raw stream of J*QJ, FP64, Q(nx, nv, ny[, nz]) order
  (3D_solver/src/main.f90:82-93).
"""
from __future__ import annotations

import ctypes as C
import math
import pathlib
import re
import struct

import numpy as np


def make_1d_for_print(qj: np.ndarray, J: np.ndarray, gamma: float):
    """float32 rho, p (N) and velocity (3N) of make_1d_for_print{2,3} (src/print.f90:192-243)."""
    if qj.ndim == 4:
        Jb = J[:, :, None]
        q1, q2, q3, q4, q5 = (qj[:, l] for l in range(5))
        rho = Jb * q1
        u, v, w = q2 / q1, q3 / q1, q4 / q1
        p = (gamma - 1.0) * (Jb * q5 - 0.5 * rho * (u ** 2 + v ** 2 + w ** 2))
    else:
        q1, q2, q3, q4 = (qj[:, l] for l in range(4))
        rho = J * q1
        u, v = q2 / q1, q3 / q1
        w = np.zeros_like(u)
        p = (gamma - 1.0) * (J * q4 - 0.5 * rho * (u ** 2 + v ** 2))
    rho_f = rho.astype(np.float32).ravel(order="F")
    p_f = p.astype(np.float32).ravel(order="F")
    vel = np.stack([u.astype(np.float32).ravel(order="F"), v.astype(np.float32).ravel(order="F"),
                    w.astype(np.float32).ravel(order="F")], axis=1).ravel()
    return rho_f, p_f, vel


def _i(v: int, w: int) -> str:
    s = str(int(v))
    return s.rjust(w) if len(s) <= w else "*" * w


def write_vtr(path, x, y, z, rho, p, vel, dimension: int = 3) -> None:
    """print_xml (src/print.f90:125-189) with io = 4 (Float32)."""
    io = 4
    ni, nj, nk = len(x), len(y), len(z)
    n = ni * nj * nk
    byte_x, byte_y, byte_z = 4 + io * ni, 4 + io * nj, 4 + io * nk
    byte_rho = 4 + io * n
    byte_p = byte_rho
    byte_v = 4 + io * dimension * n
    o1 = byte_x
    o2 = o1 + byte_y
    o3 = o2 + byte_z
    o4 = o3 + byte_rho
    o5 = o4 + byte_p
    s1, s2, s3, s4 = _i(ni - 1, 4), _i(nj - 1, 4), _i(nk - 1, 4), _i(dimension, 1)
    lf = "\n"
    head = [
        '<?xml version="1.0"?>',
        '<VTKFile type="RectilinearGrid" version="1.0" byte_order="LittleEndian">',
        f'  <RectilinearGrid WholeExtent="0 {s1} 0 {s2} 0 {s3}">',
        f'    <Piece Extent="0 {s1} 0 {s2} 0 {s3}">',
        '      <Coordinates>',
        '      <DataArray type="Float32" format="appended" offset="0"/>',
        f'      <DataArray type="Float32" format="appended" offset="{_i(o1, 12)}"/>',
        f'      <DataArray type="Float32" format="appended" offset="{_i(o2, 12)}"/>',
        '    </Coordinates>',
        '    <PointData>',
        f'      <DataArray type="Float32" format="appended" offset="{_i(o3, 12)}" Name="rho" NumberOfComponents="1"/>',
        f'      <DataArray type="Float32" format="appended" offset="{_i(o4, 12)}" Name="p" NumberOfComponents="1"/>',
        f'      <DataArray type="Float32" format="appended" offset="{_i(o5, 12)}" Name="velocity" NumberOfComponents="{s4}"/>',
        '      </PointData>',
        '    </Piece>',
        '  </RectilinearGrid>',
        '  <AppendedData encoding="raw">',
    ]
    f32 = lambda a: np.ascontiguousarray(a, dtype="<f4").tobytes()
    i32 = lambda v: struct.pack("<i", v)
    with open(path, "wb") as fh:
        fh.write((lf.join(head) + lf).encode())
        fh.write(b"  _")
        fh.write(i32(byte_x) + f32(x) + i32(byte_y) + f32(y) + i32(byte_z) + f32(z))
        fh.write(i32(byte_rho) + f32(rho) + i32(byte_p) + f32(p) + i32(byte_v) + f32(vel))
        fh.write(lf.encode())
        fh.write(("  </AppendedData>" + lf + "</VTKFile>" + lf).encode())


def read_vtr(path):
    """Parse a file written by write_vtr: returns (x, y, z, {rho, p, velocity})."""
    raw = pathlib.Path(path).read_bytes()
    i0 = raw.index(b"  _") + 3
    head = raw[:i0].decode()
    ext = re.search(r'WholeExtent="0\s+(\d+) 0\s+(\d+) 0\s+(\d+)"', head)
    ni, nj, nk = (int(ext.group(a)) + 1 for a in (1, 2, 3))
    ncomp = int(re.search(r'Name="velocity" NumberOfComponents="(\d)"', head).group(1))
    pos = i0
    out = []
    for cnt in (ni, nj, nk, ni * nj * nk, ni * nj * nk, ncomp * ni * nj * nk):
        pos += 4  # header word
        out.append(np.frombuffer(raw, dtype="<f4", count=cnt, offset=pos).copy())
        pos += 4 * cnt
    x, y, z, rho, p, vel = out
    shp = (nk, nj, ni)
    return x, y, z, {"rho": rho.reshape(shp), "p": p.reshape(shp), "velocity": vel.reshape(shp + (ncomp,))}


def fortran_e(v: float, w: int = 12, d: int = 4) -> str:
    """Fortran Ew.d edit descriptor: [-]0.<d digits>E<sign><2 digits>, right-justified in w."""
    if not math.isfinite(v):
        return ("NaN" if math.isnan(v) else ("Infinity" if v > 0 else "-Infinity")).rjust(w)
    if v == 0.0:
        return ("0." + "0" * d + "E+00").rjust(w)
    mant, ex = f"{abs(v):.{d - 1}e}".split("e")
    digits = mant.replace(".", "")
    e = int(ex) + 1
    exp = f"{'+' if e >= 0 else '-'}{abs(e):02d}"
    s = ("-" if v < 0 else "") + "0." + digits + ("E" + exp if abs(e) <= 99 else exp)
    return s.rjust(w)


def ref_diagnostics(nx, ny, nz, order, gamma, rho, p, vel) -> tuple[float, float]:
    """print_KE / print_entropy arithmetic (float32 sum, double terms) via liboux's host helper."""
    from ._lib import LIB
    r = np.ascontiguousarray(rho, dtype=np.float32)
    pp = np.ascontiguousarray(p, dtype=np.float32)
    v = np.ascontiguousarray(vel, dtype=np.float32)
    out = (C.c_double * 2)()
    fp = C.POINTER(C.c_float)
    rc = LIB.oux_host_ref_diagnostics(nx, ny, nz, order, C.c_double(gamma), r.ctypes.data_as(fp),
                                      pp.ctypes.data_as(fp), v.ctypes.data_as(fp), out)
    if rc != 0:
        raise RuntimeError("oux_host_ref_diagnostics failed")
    return out[0], out[1]


class HistoryWriter:
    """Appends data/kinetic_energy.d and data/entropy.d like print_KE / print_entropy."""

    def __init__(self, data_dir: pathlib.Path):
        self.dir = pathlib.Path(data_dir)
        self.ke0 = None
        self.s0 = None

    def record(self, t: float, ke: float, ent: float, step: int) -> None:
        if step == 0:
            self.ke0, self.s0 = np.float32(ke), np.float32(ent)
        ke32, s32 = np.float32(ke), np.float32(ent)
        # a flow that starts at rest has ke0 = 0: the ratio is written as the reference
        # writes it, Infinity / NaN
        with np.errstate(divide="ignore", invalid="ignore"):
            ds = np.float32((self.s0 - s32) / self.s0)
            kr = np.float32(ke32 / self.ke0)
        with open(self.dir / "entropy.d", "a") as f:
            f.write(fortran_e(float(np.float32(t))) + fortran_e(float(ds)) + "\n")
        with open(self.dir / "kinetic_energy.d", "a") as f:
            f.write(fortran_e(float(np.float32(t))) + fortran_e(float(ke32)) + fortran_e(float(kr)) + "\n")


def write_restart(path, q: np.ndarray) -> None:
    """Raw stream write of Q (Fortran order, FP64) -- recal/Q%05d.dat."""
    np.asfortranarray(q, dtype=np.float64).ravel(order="F").tofile(str(path))


def read_restart(path, shape) -> np.ndarray:
    """Raw stream or SEQFMT01 sequential restart (3D_solver/src/main.f90:38-60)."""
    raw = pathlib.Path(path).read_bytes()
    n = int(np.prod(shape))
    if len(raw) >= 4 + 8 + 4 and raw[4:12] == b"SEQFMT01":
        # sequential: [4B len][8B header][4B len][4B len][data][4B len]
        rec2 = 4 + 8 + 4
        data = np.frombuffer(raw, dtype="<f8", count=n, offset=rec2 + 4)
    else:
        data = np.frombuffer(raw, dtype="<f8", count=n)
    return data.reshape(shape, order="F").copy(order="F")
