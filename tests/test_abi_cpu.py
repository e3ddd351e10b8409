"""C-ABI checks that need no GPU: exports, configuration validation, sizes, layout."""
import ctypes as C
import pathlib
import re

import numpy as np
import pytest

from ouxsbli_b200 import _lib
from ouxsbli_b200.solver import SolverConfig

HEADER = pathlib.Path(__file__).resolve().parents[1] / "include" / "oux.h"


def header_functions():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(oux_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    names = header_functions()
    assert len(names) >= 19
    for n in names:
        assert hasattr(_lib.LIB, n), f"liboux.so does not export {n}"
    assert set(_lib.SYMBOLS) <= set(names)
    assert _lib.LIB.oux_abi_version() == 1


def small_cfg(**kw):
    n = 10 + 6
    d = np.full(n - 1, 0.1)
    base = dict(dim=3, nx=n, ny=n, nz=n, order=6, dx=d, dy=d, dz=d, dt=1e-4)
    base.update(kw)
    return SolverConfig(**base)


def create(cfg):
    c, keep = cfg.to_c()
    h = C.c_void_p()
    rc = _lib.LIB.oux_create(C.byref(c), C.byref(h))
    return rc, h


@pytest.mark.parametrize("kw,msg", [
    (dict(order=5), "order"),
    (dict(dim=4), "dim"),
    (dict(nx=6), "too small"),
    (dict(order=4, visc="Euler", bc_z=3), "order 2"),
    (dict(bc_z=5), "bc_z"),
    (dict(bc_x=2), "boundaries"),
    (dict(dim=2, nz=1, order=2, ny=3, dy=np.full(2, 0.1), bc_y=1), "too small"),
    (dict(rk=2), "rk"),
    (dict(dim=2, nz=1, scheme="Roe"), "Roe"),
    (dict(visc="NS", visc_order=2), "calc_Ev2_in"),
    (dict(order=4, nx=14, ny=14, nz=14, visc="NS", visc_order=6), "order 6"),
    (dict(dt=0.0), "dt"),
])
def test_create_rejects_invalid(kw, msg):
    rc, h = create(small_cfg(**kw))
    assert rc == _lib.OUX_E_INVALID
    assert msg in _lib.LIB.oux_last_error().decode()


@pytest.mark.parametrize("kw", [
    dict(bc_x=1, bc_y=1, visc="NS"),                                    # SBLI: Central-6, x / y walls
    dict(bc_y=1, visc="NS", visc_stencil="ME4Base"),
    dict(bc_x=1, bc_y=1, bc_z=1, visc="NS", visc_order=4),
    dict(order=4, nx=14, ny=14, nz=14, bc_z=1, visc="NS", visc_order=2),
    dict(order=2, nx=12, ny=12, nz=12, bc_x=1, bc_y=1, bc_z=1, visc="NS"),
    dict(bc_x=1, bc_y=1, visc="LES"),
    dict(order=2, nx=12, ny=12, nz=12, bc_y=1, bc_z=1, visc="LES"),
])
def test_create_accepts_3d_viscous_walls(kw):
    """3D Navier-Stokes and LES grids with non-periodic directions are accepted (the
    walled sweep variants)."""
    rc, h = create(small_cfg(**kw))
    assert rc == 0, _lib.LIB.oux_last_error().decode()
    _lib.LIB.oux_destroy(h)


def test_create_sizes_and_layout():
    cfg = small_cfg(scheme="Hybrid", visc="NS")
    rc, h = create(cfg)
    assert rc == 0
    lay = _lib.OuxLayout()
    assert _lib.LIB.oux_layout_of(h, C.byref(lay)) == 0
    assert lay.nv == 5 and lay.row_stride >= cfg.nx and lay.row_stride % 4 == 0
    assert lay.plane_stride == lay.row_stride * cfg.ny
    assert lay.var_stride >= lay.plane_stride * cfg.nz and lay.var_stride % 32 == 0
    c, keep = cfg.to_c()
    sb, kb = C.c_size_t(), C.c_size_t()
    assert _lib.LIB.oux_state_bytes(C.byref(c), C.byref(sb)) == 0
    assert _lib.LIB.oux_scratch_bytes(C.byref(c), C.byref(kb)) == 0
    assert sb.value == 5 * lay.var_stride * 8
    assert kb.value > sb.value
    # unbound handles refuse device work without touching CUDA
    assert _lib.LIB.oux_step(h, 1, None) == _lib.OUX_E_UNBOUND
    assert _lib.LIB.oux_fill_ghosts(h, None) == _lib.OUX_E_UNBOUND
    assert _lib.LIB.oux_destroy(h) == 0


def test_pack_unpack_roundtrip_host():
    cfg = small_cfg(dim=3, nx=13, ny=17, nz=11, order=2)
    cfg.dx, cfg.dy, cfg.dz = np.ones(12), np.ones(16), np.ones(10)
    rc, h = create(cfg)
    assert rc == 0
    lay = _lib.OuxLayout()
    _lib.LIB.oux_layout_of(h, C.byref(lay))
    ref = np.asfortranarray(np.random.default_rng(0).standard_normal((13, 5, 17, 11)))
    dev = np.zeros(5 * lay.var_stride)
    assert _lib.LIB.oux_pack_state(h, ref.ctypes.data_as(C.POINTER(C.c_double)), dev.ctypes.data_as(C.c_void_p)) == 0
    back = np.zeros_like(ref, order="F")
    assert _lib.LIB.oux_unpack_state(h, dev.ctypes.data_as(C.c_void_p), back.ctypes.data_as(C.POINTER(C.c_double))) == 0
    np.testing.assert_array_equal(back, ref)
    # SoA: variable l of cell (i,j,k) at l*vs + k*plane + j*row + i
    i, j, k, l = 4, 7, 3, 2
    assert dev[l * lay.var_stride + k * lay.plane_stride + j * lay.row_stride + i] == ref[i, l, j, k]
    _lib.LIB.oux_destroy(h)


def test_set_boundary_checks_without_a_device():
    """oux_set_boundary validates on the host: the face's direction must be
    non-periodic, the rule known, and a fixed rule needs its values."""
    n = 12
    d = np.full(n - 1, 0.1)
    cfg = SolverConfig(dim=2, nx=n, ny=n, nz=1, order=4, visc="NS", bc_y=1, dx=d, dy=d, dz=None, dt=1e-4)
    rc, h = create(cfg)
    assert rc == 0
    L = _lib.LIB
    assert L.oux_set_boundary(h, _lib.FACES["x_lo"], 0, None) == _lib.OUX_E_INVALID  # x is periodic
    assert "periodic" in L.oux_last_error().decode()
    assert L.oux_set_boundary(h, _lib.FACES["y_lo"], 9, None) == _lib.OUX_E_INVALID
    assert L.oux_set_boundary(h, _lib.FACES["y_hi"], _lib.BC_KINDS["fixed"], None) == _lib.OUX_E_INVALID
    assert L.oux_set_boundary(h, 7, 0, None) == _lib.OUX_E_INVALID
    assert L.oux_set_boundary(h, _lib.FACES["y_lo"], _lib.BC_KINDS["noslip_wall"], None) == 0
    assert L.oux_set_boundary(h, _lib.FACES["y_hi"], _lib.BC_KINDS["slip_wall"], None) == 0
    L.oux_destroy(h)


def test_3d_boundary_setters_without_a_device():
    """3D order-2 boundaries: z faces open only on non-periodic ends; the far field on
    a non-periodic high face and the Neumann rule are taken, far field through its own
    setter only; per-position kinds (2D only) are refused."""
    n = 10
    d = np.full(n - 1, 0.1)
    cfg = SolverConfig(dim=3, nx=n, ny=n, nz=n, order=2, visc="Euler", bc_x=1, bc_z=3, dx=d, dy=d, dz=d, dt=1e-4)
    rc, h = create(cfg)
    assert rc == 0, _lib.LIB.oux_last_error()
    L = _lib.LIB
    assert L.oux_set_boundary(h, _lib.FACES["z_lo"], _lib.BC_KINDS["slip_wall"], None) == 0  # the grid's end
    assert L.oux_set_boundary(h, _lib.FACES["z_hi"], 0, None) == _lib.OUX_E_INVALID       # a halo end
    assert L.oux_set_boundary(h, _lib.FACES["y_lo"], 0, None) == _lib.OUX_E_INVALID       # periodic y
    assert L.oux_set_boundary(h, _lib.FACES["x_hi"], _lib.BC_KINDS["noslip_wall"], None) == 0
    assert L.oux_set_boundary_farfield(h, _lib.FACES["x_hi"], 1.0, 1.0, 0.0, 1.0) == 0
    assert L.oux_set_boundary_farfield(h, _lib.FACES["x_lo"], 1.0, 1.0, 0.0, 1.0) == _lib.OUX_E_INVALID
    assert L.oux_set_boundary_farfield(h, _lib.FACES["y_hi"], 1.0, 1.0, 0.0, 1.0) == _lib.OUX_E_INVALID
    assert L.oux_set_boundary(h, _lib.FACES["x_hi"], _lib.BC_KINDS["farfield"], None) == _lib.OUX_E_INVALID
    assert L.oux_set_boundary(h, _lib.FACES["x_lo"], _lib.BC_KINDS["neumann"], None) == 0
    assert L.oux_set_boundary(h, _lib.FACES["x_lo"], 6, None) == _lib.OUX_E_INVALID
    assert L.oux_set_boundary_cells(h, _lib.FACES["x_lo"], None) == _lib.OUX_E_INVALID
    L.oux_destroy(h)


def test_bench_walls_grids_are_accepted():
    """bench.py --workload walls256: each of its grids (periodic; y; x and y; x, y and z
    walls) makes a valid configuration with the face rules its walls need."""
    import bench
    for which in bench.WALL_GRIDS:
        cfg, qj = bench.walled_workload(12, which)
        assert qj.shape == (cfg.nx, 5, cfg.ny, cfg.nz)
        assert cfg.interior_cells() == 12 ** 3
        rc, h = create(cfg)
        assert rc == 0, _lib.LIB.oux_last_error().decode()
        _lib.LIB.oux_destroy(h)


def test_stage_part_argument_checks_without_a_device():
    """oux_stage_part: part 0..2 only; the split parts are built for 3D Euler /
    Navier-Stokes (not LES, not 2D); the checks come before any device work."""
    rc, h = create(small_cfg(bc_z=2))
    assert rc == 0
    assert _lib.LIB.oux_stage_part(h, 0, 3, None) == _lib.OUX_E_INVALID
    assert _lib.LIB.oux_stage_part(h, 3, 1, None) == _lib.OUX_E_INVALID  # RK3 has stages 0..2
    assert _lib.LIB.oux_stage_part(h, 0, 1, None) == _lib.OUX_E_UNBOUND  # valid arguments, nothing bound
    _lib.LIB.oux_destroy(h)
    rc, h = create(small_cfg(visc="LES"))
    assert rc == 0
    assert _lib.LIB.oux_stage_part(h, 0, 1, None) == _lib.OUX_E_INVALID
    assert "Navier-Stokes" in _lib.LIB.oux_last_error().decode()
    _lib.LIB.oux_destroy(h)


def test_tma_tile_geometry_meets_the_tensor_copy_rules():
    """The x / y sweep tiles staged by tensor copies (oux_sweep.cuh): every box starts
    on a 16-byte boundary (x origin 32 b - 4 in the x sweep, 32 b in the y sweep), its
    rows are a multiple of 16 bytes for 4- and 8-byte elements, every cell the tile
    needs lies inside the row for each x ghost width (1 to 3), and each field's slab
    is a multiple of 128 bytes.  Constants read from the header."""
    import pathlib
    import re
    src = (pathlib.Path(__file__).resolve().parents[1] / "ouxsbli_b200" / "csrc" / "oux_sweep.cuh").read_text()
    const = {k: int(re.search(rf"constexpr int {k} = (\d+);", src).group(1))
             for k in ("TMA_ROW", "TMA_ROW_X", "TILE_HALO", "TMA_MAP_BYTES")}
    rows_y = int(re.search(r"#define OUX_SWEEP_BF (\d+)", src).group(1))
    rows_x = int(re.search(r"#define OUX_SWEEP_BR (\d+)", src).group(1))
    halo = const["TILE_HALO"]
    assert const["TMA_MAP_BYTES"] == 128
    for elem in (4, 8):
        for row, box_rows in ((const["TMA_ROW_X"], rows_x), (const["TMA_ROW"], rows_y + 2 * halo)):
            assert row * elem % 16 == 0
            slab = -(-row * box_rows * elem // 128) * 128
            assert slab % 128 == 0 and slab >= row * box_rows * elem
        for gx in (1, 2, 3):
            for b0 in range(64):
                bx0 = gx + 32 * b0
                # x sweep: cells bx0 - halo .. bx0 + 31 + halo, row from 32 b - 4, column gx + 1 + t
                x0 = bx0 - gx - 4
                assert x0 * elem % 16 == 0
                assert 0 <= (bx0 - halo) - x0 and (bx0 + 31 + halo) - x0 < const["TMA_ROW_X"]
                assert (bx0 - halo) - x0 == gx + 1
                # y sweep: owned cells bx0 .. bx0 + 31, row from 32 b, column gx + x
                y0 = bx0 - gx
                assert y0 * elem % 16 == 0 and y0 >= 0
                assert bx0 - y0 == gx and (bx0 + 31) - y0 < const["TMA_ROW"]
