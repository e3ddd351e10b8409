/*
 * liboux -- C ABI of the B200 (sm_100a) explicit compressible-flow time step.
 *
 * This is the drop-in boundary for OUxSBLI's GPU hot path.  Each entry point
 * names the reference interface it replaces (paths relative to the
 * OUxSBLI repository).  The reference has no C ABI of its own: its Python
 * layer (ouxsbli/case.py) drives a CUDA-Fortran executable, whose device
 * work is `RungeKutta` (3D_solver/src/calc_time_dev.f90.fypp:30-114) calling
 * `calc_EFG` (3D_solver/src/calc_flux_base.f90.fypp:109-198) once per stage.
 *
 * Conventions
 *   - Every call returns an int status: OUX_OK (0) or a negative OUX_E_*.
 *     oux_last_error() returns a thread-local message for the last failure.
 *   - Device memory is owned by the caller (e.g. PyTorch tensors): the library
 *     never allocates device memory for a solve.  oux_state_bytes() and
 *     oux_scratch_bytes() report the sizes to allocate; oux_bind() attaches them.
 *   - Calls that take a cudaStream_t (passed as void*) are asynchronous on that
 *     stream.  A handle is not thread-safe; several handles may share a stream.
 *   - Device-side faults (NaN / non-positive density or pressure found by the
 *     status check) set a device status word read by oux_status().
 *   - No C++ exception crosses this boundary.
 *
 * Device state layout ("SoA padded"): for each conservative variable v
 * (rho, rho u, rho v, [rho w], E, all divided by the cell Jacobian, i.e. the
 * reference's QJ), a block of nz * ny * row_stride doubles, x fastest, ghost
 * cells included (g = order/2 per side).  row_stride and var_stride are
 * reported by oux_layout().  The host-side converters oux_pack_state() /
 * oux_unpack_state() translate from/to the reference's Q(nx,nv,ny,nz) order.
 */
#ifndef OUX_H
#define OUX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OUX_ABI_VERSION 1

enum oux_status_code {
  OUX_OK = 0,
  OUX_E_INVALID = -1,      /* bad argument / unsupported configuration */
  OUX_E_CUDA = -2,         /* a CUDA runtime call failed */
  OUX_E_UNBOUND = -3,      /* handle has no device buffers bound */
  OUX_E_TOO_SMALL = -4,    /* a caller buffer is smaller than required */
  OUX_E_DEVICE_FAULT = -5  /* the device status word reports a fault */
};

/* Scheme, physics and option enums; the names follow config.fypp macros. */
enum oux_scheme { OUX_KEEP = 0, OUX_SLAU = 1, OUX_ROE = 2, OUX_HYBRID = 3 };
enum oux_visc { OUX_EULER = 0, OUX_NS = 1, OUX_LES = 2 };
enum oux_visc_stencil { OUX_CENTRAL = 0, OUX_ME4 = 1 };
enum oux_tvd { OUX_TVD_NONE = 0, OUX_TVD_TVD = 1, OUX_TVD_HYBRID = 2 };
enum oux_slau_variant { OUX_SLAU1 = 0, OUX_HRSLAU2 = 1 };
enum oux_precision { OUX_FP64 = 0, OUX_MIXED = 1 };
/* device status bits (oux_status).  OUX_FAULT_TIMEOUT: a bounded device wait gave up
 * (a batched step's dependency wait, or a sweep block whose tensor-copied tile never
 * arrived; that block skipped its faces, so the step's result is void). */
enum oux_fault_bits { OUX_FAULT_NAN = 1, OUX_FAULT_NONPOSITIVE = 2, OUX_FAULT_TIMEOUT = 4 };

/*
 * Solve configuration.  Replaces the compile-time configuration of the
 * reference: config.fypp macros (VISC, SCHEME, ORDER, TVD, SLAU_VARIANT, RK,
 * BC_X/Y/Z; VISC_ORDER, VISC_STENCIL) and mod_globals.f90 parameters
 * (nx, ny, nz incl. ghosts, gamma, R, Pr, Prt, threshold, dt).
 * dx/dy/dz are the host cell spacings of length n-1 (set_coordinate.f90).
 */
typedef struct oux_config {
  int32_t dim;          /* 2 or 3 */
  int32_t nx, ny, nz;   /* points incl. ghosts; nz = 1 for dim 2 */
  int32_t order;        /* convective order 2, 4, 6 */
  int32_t scheme;       /* enum oux_scheme */
  int32_t visc;         /* enum oux_visc */
  int32_t visc_order;   /* 2, 4, 6; 0: the order in 3D, 4 (order >= 4) or 2 in 2D */
  int32_t visc_stencil; /* enum oux_visc_stencil (ME4 only with visc_order 6) */
  int32_t tvd;          /* enum oux_tvd */
  int32_t slau;         /* enum oux_slau_variant */
  int32_t rk;           /* 3 (TVD-RK3) or 4 (classical RK4) */
  int32_t bc_x, bc_y, bc_z; /* 0 = periodic.  bc_x = 1 (2D): non-periodic x -- every x
                               face with the order lowered next to the boundary, as the
                               reference's calc_{slau,keep,hybrid}_x boundary kernels do
                               (2D_solver/src/calc_*_kernel.f90.fypp), and one boundary
                               cell on each side, zero-gradient unless oux_set_boundary
                               gives its face another rule (2D_solver/ST/set.f90 set_bc).
                               bc_y = 1 (2D): the same for y (calc_*_y), as the
                               BC_X = BC_Y = True cases build them (2D_solver/OS, BL).
                               Euler or NS.  3D non-periodic x / y / z (bc_z = 1):
                               Euler, NS and LES at orders 2 / 4 / 6, one boundary
                               cell a side; viscous faces outside the reference's
                               high-order guard take its 2nd-order fallback
                               (3D_solver/src/calc_visc_high.f90.fypp), as the SBLI /
                               TBL cases' BC_X = BC_Y = True builds do; the SGS
                               viscosity is 0 on no-slip walls.  bc_z = 2, 3, 4 (3D,
                               not LES): a z slab of a
                               larger grid (COMMZ, 3D_solver/src/calc_para.f90:343-384):
                               its g ghost planes at the halo ends (enum oux_bc_z) are
                               written by the caller's halo exchange (oux_halo_pack /
                               _unpack) after every stage, not by the fill. */
  int32_t precision;    /* enum oux_precision */
  double gamma, R, Pr, Prt, threshold, dt;
  const double *dx, *dy, *dz; /* host arrays, n-1 entries each (dz unused in 2D) */
} oux_config;

typedef struct oux_handle oux_handle;

typedef struct oux_layout {
  int32_t nv;          /* conservative variables: dim + 2 */
  int64_t row_stride;  /* elements between consecutive y rows */
  int64_t plane_stride;/* elements between consecutive z planes */
  int64_t var_stride;  /* elements between variables */
  int64_t elem_bytes;  /* 8 for FP64 state, 4 for the mixed form's state */
} oux_layout;

/* --- lifetime ----------------------------------------------------------- */
/* Replaces allocate_device_mem + pre_calc metrics (3D_solver/src/preprocess.f90.fypp:21-103).
 * Validates the configuration and computes the metric tables on the host. */
int oux_create(const oux_config* cfg, oux_handle** out);
int oux_destroy(oux_handle* h);
const char* oux_last_error(void);
int oux_abi_version(void);

/* Buffer sizes for a configuration (bytes) and the device layout. */
int oux_state_bytes(const oux_config* cfg, size_t* bytes);
int oux_scratch_bytes(const oux_config* cfg, size_t* bytes);
int oux_layout_of(const oux_handle* h, oux_layout* out);

/* Attach caller-owned device buffers (state = QJ of oux_state_bytes; scratch
 * of oux_scratch_bytes).  Uploads the metric tables into scratch on `stream`, and
 * for 3D grids with a Central-4/6 or ME4 viscous stencil encodes (on the host) the
 * tensor maps through which the x and y sweeps stage their tiles by TMA; they hold the
 * scratch's field addresses, so the buffers must stay where they were bound. */
int oux_bind(oux_handle* h, void* state_dev, void* scratch_dev, size_t scratch_bytes,
             void* stream);

/* --- host <-> device state (pre_calc H2D :88-95, send_recv_for_print_even D2H) --- */
/* Copy a host array in the reference order QJ(nx,nv,ny,nz) (Fortran, FP64) to
 * the bound device state, transposing on the device.  host may be pageable or
 * pinned; staging uses the scratch buffer. */
int oux_set_state(oux_handle* h, const double* host_qj, void* stream);
int oux_get_state(oux_handle* h, double* host_qj, void* stream);
/* oux_get_state without the final synchronisation: the copy into host_qj (pinned
 * memory for real asynchrony) completes when `stream` reaches it.  The handle's
 * scratch stages the copy, so further work on the handle must be ordered after it
 * (the same stream does that).  Same reference counterpart as oux_get_state. */
int oux_get_state_async(oux_handle* h, double* host_qj, void* stream);
/* Pure host converters between the reference order and the device layout. */
int oux_pack_state(const oux_handle* h, const double* ref_qj, void* dev_layout_host);
int oux_unpack_state(const oux_handle* h, const void* dev_layout_host, double* ref_qj);

/* --- stages and halo planes (z slabs, bc_z = 2) ----------------------------- */
/* One RK stage (0..2 for RK3, 0..3 for RK4) of a time step with the ghost /
 * boundary fill of the array it writes; oux_step(h, 1) is the stages in order.
 * A z slab exchanges halos between stages, as the reference's COMMZ path does
 * after each stage (3D_solver/src/calc_time_dev.f90.fypp:465-498, calc_para.f90:
 * 343-384): oux_halo_pack copies the g lowest and g highest interior planes of
 * every variable of the array the stage wrote into lo_dev / hi_dev ([nv][g][plane],
 * oux_halo_bytes each; elements FP64, or FP32 stage increments in the mixed form);
 * the caller sends lo to the rank below and hi to the rank above (periodic in
 * rank), and oux_halo_unpack writes the buffer received from the rank below (its
 * hi) into the lower ghost planes and the one from the rank above (its lo) into
 * the upper ones. */
int oux_stage(oux_handle* h, int32_t stage, void* stream);
/* One stage in two parts, so that a z slab's halo exchange overlaps the stage, as
 * the reference posts its COMMZ exchange, computes the faces of the interior planes
 * and then finishes the halo (3D_solver/src/calc_time_dev.f90.fypp:465-470,
 * calc_para.f90:343-384).  part 1 updates the cells of planes [2g, nz-2g), which do
 * not read the ghost planes, so the halo of the stage's source may still be in
 * flight; part 2, after oux_halo_unpack, updates the planes next to both ends and
 * fills the ghost cells.  Parts 1 then 2 give the bits of oux_stage; part 0 is
 * oux_stage.  3D Euler / Navier-Stokes grids (not LES). */
int oux_stage_part(oux_handle* h, int32_t stage, int32_t part, void* stream);
int oux_halo_bytes(const oux_handle* h, int32_t stage, size_t* bytes);
int oux_halo_pack(oux_handle* h, int32_t stage, void* lo_dev, void* hi_dev, void* stream);
int oux_halo_unpack(oux_handle* h, int32_t stage, const void* lo_dev, const void* hi_dev, void* stream);

/* --- boundary cells of non-periodic directions --------------------------- */
/* Replaces the case's own set_bc subroutine (2D_solver/OS/set.f90:50-90,
 * 2D_solver/ST/set.f90 set_bc), which the reference compiles into each case.
 * Faces: x low, x high, y low, y high (z low, z high in 3D).  Rules, applied to the
 * one boundary cell of every row (x faces) or column (y faces) from the adjacent
 * interior cell (3D: every line of cells normal to the face):
 *   ZERO_GRADIENT  the neighbour's Q/J (the default of every non-periodic face)
 *   SLIP_WALL      the neighbour's Q/J with the normal momentum negated
 *   NOSLIP_WALL    the neighbour's density and pressure with zero momentum:
 *                  p_wall = (gamma-1) (E - (m1^2 + m2^2) / (2 rho)) of the neighbour's
 *                  Q/J, E_wall = p_wall / (gamma-1) (the wall rows of
 *                  2D_solver/ST/set.f90 and 2D_solver/BL0/set.f90)
 *   FIXED          caller values: fixed_dev holds nv x len doubles of Q/J, variable-
 *                  major ([l * len + pos]; len = ny for x faces, nx for y faces;
 *                  3D: pos = j + ny k, i + nx k, i + nx j for x, y, z faces),
 *                  device memory owned by the caller and read at every fill until
 *                  the face is set again.  In the mixed form the stage increments
 *                  of FIXED cells are 0 (Q^n holds the values).
 * By default y faces are applied first over every column, then x faces over every
 * row, so a corner takes its x rule applied to the y-boundary cell next to it (the
 * order of 2D_solver/OS/set.f90; oux_set_boundary_order reverses it).  In 3D the
 * x, y and z faces are applied in that order (3D_solver/STZ/set.f90).  The face's
 * direction must be non-periodic.  Set rules before oux_batch_create when the
 * handle joins a batch. */
enum oux_face { OUX_FACE_X_LO = 0, OUX_FACE_X_HI = 1, OUX_FACE_Y_LO = 2, OUX_FACE_Y_HI = 3,
                OUX_FACE_Z_LO = 4, OUX_FACE_Z_HI = 5 };
/* bc_z (3D): periodic, non-periodic, or a z slab of a larger grid whose ghost planes
 * at both ends / the upper end only / the lower end only come from the halo exchange
 * (the other end being the grid's boundary, with the rules of its face). */
enum oux_bc_z { OUX_Z_PERIODIC = 0, OUX_Z_WALLS = 1, OUX_Z_SLAB = 2, OUX_Z_SLAB_LO_WALL = 3,
                OUX_Z_SLAB_HI_WALL = 4 };
/* NEUMANN: the neighbour's primitive state (rho, velocity, p) carried through the
 * two cells' Jacobians, Q/J(b) = Q(n) / J(b) (3D_solver/src/set_bc_tbl_sbli.f90
 * set_bc_Neumann_tbl_top_down, the TBL / SBLI top); ZERO_GRADIENT copies Q/J. */
enum oux_bc_kind { OUX_BC_ZERO_GRADIENT = 0, OUX_BC_SLIP_WALL = 1, OUX_BC_FIXED = 2, OUX_BC_NOSLIP_WALL = 3,
                   OUX_BC_FARFIELD = 4, OUX_BC_NEUMANN = 5 };
int oux_set_boundary(oux_handle* h, int32_t face, int32_t kind, const double* fixed_dev);
/* FARFIELD (x high or y high): the boundary state from the Riemann invariants along
 * the outward normal, R+ = u_n + 2c/(gamma-1) of the neighbour and R- = u_normal -
 * 2 c_inf/(gamma-1) of the far field; u_n = (R+ + R-)/2, c = (gamma-1)(R+ - R-)/4,
 * rho = rho_inf (c / c_inf)^(2/(gamma-1)), p = rho c^2 / gamma, tangential velocity
 * u_tangential (the top row of 2D_solver/BL0/set.f90).  In 3D the tangential
 * velocity is the first tangential axis's (u on y high, v on x high) and the other is
 * 0 (3D_solver/src/set_bc_tbl_sbli.f90 set_bc_Riemann_tbl_top_down). */
int oux_set_boundary_farfield(oux_handle* h, int32_t face, double rho_inf, double u_tangential,
                              double u_normal, double c_inf);
/* A rule per position along the face: kinds_dev holds one enum oux_bc_kind per
 * boundary cell (ny for x faces, nx for y faces), device memory owned by the caller
 * and read at every fill; FIXED positions take the face's values of
 * oux_set_boundary, FARFIELD positions its far-field state.  NULL restores the
 * face's single rule.  (2D_solver/BL0/set.f90: a slip-like copy ahead of the plate,
 * a no-slip wall along it.)  2D solves. */
int oux_set_boundary_cells(oux_handle* h, int32_t face, const int8_t* kinds_dev);
/* y_last = 1: the y faces are applied after the x faces, so a corner takes its y
 * rule of the x-boundary value beside it (2D_solver/BL0/set.f90); 0 (default): the
 * reverse (2D_solver/OS/set.f90). */
int oux_set_boundary_order(oux_handle* h, int32_t y_last);

/* --- hot path ----------------------------------------------------------- */
/* Ghost / boundary-cell fill: periodic images, set_bc_cyclic{2,4,6}
 * (3D_solver/src/set_bc_common.f90:101-273), and the rules of oux_set_boundary on
 * non-periodic faces. */
int oux_fill_ghosts(oux_handle* h, void* stream);
/* Stage residual R = dt*S*(flux differences) of the current state (coef 1), the
 * quantity calc_R forms (3D_solver/src/calc_steps.f90:8-38) after calc_EFG.
 * rhs_dev receives nv * (nz-2)*(ny-2)*(nx-2) doubles (3D) in the reference's
 * Rs(nx-2,nv,ny-2,nz-2) order, interior cells only (ghost entries are 0). */
int oux_rhs(oux_handle* h, double* rhs_dev, void* stream);
/* nsteps full time steps: the `do t1 = 1, nt` body of RungeKutta
 * (3D_solver/src/calc_time_dev.f90.fypp:81-101 RK3, :264-287 RK4;
 *  2D_solver/src/calc_time_dev.f90.fypp:26-108). */
int oux_step(oux_handle* h, int32_t nsteps, void* stream);
/* FP64 domain integrals over interior cells (replaces print_KE / print_entropy,
 * src/print.f90:42-122, computed on the device in FP64):
 * out[0] = mean 0.5 rho |u|^2, out[1] = mean rho log(p rho^-gamma),
 * out[2] = mean 0.5 rho |omega|^2 (enstrophy; no reference counterpart).
 * Blocking: synchronizes `stream` and copies 3 doubles to the host. */
int oux_diagnostics(oux_handle* h, double out[3], void* stream);
/* Device status word (OR of oux_fault_bits).  oux_check_state clears it, scans
 * the current state's interior for NaN / non-positive rho or p on `stream`,
 * synchronizes and returns OUX_E_DEVICE_FAULT when a bit is set.  The reference
 * has no counterpart (it only NaN-checks its rescaling profile,
 * 3D_solver/src/preprocess.f90.fypp:143-147). */
int oux_check_state(oux_handle* h, int32_t* fault_bits, void* stream);
int oux_status(oux_handle* h, int32_t* fault_bits);

/* Per-kernel timing for measurement tools: while enabled, every launch is
 * bracketed by CUDA events on its stream; oux_profile_read synchronizes and
 * returns, per kernel kind (0 prim, 1 sensor, 2 sgs, 3 sgs edges, 4 x sweep,
 * 5 y sweep, 6 z sweep, 7 ghost fill), the summed milliseconds and launch
 * counts since the last oux_profile call.  No reference counterpart (the
 * reference is profiled externally with ncu/nsys scripts). */
int oux_profile(oux_handle* h, int32_t enable);
int oux_profile_read(oux_handle* h, double* ms, int64_t* count, int32_t nkinds);

/* Host helper for the history files: the reference's KE / entropy arithmetic
 * (src/print.f90:42-122) on the float32 fields of make_1d_for_print: per-cell
 * terms in FP64, running sum rounded to float32 after every cell, mean over
 * (nx-order)(ny-order)(nz-order).  out[0] = ke, out[1] = entropy.  For 2D pass
 * nz = 1 with order 0 in the z extent handled by the caller (the reference
 * writes no 2D history). */
int oux_host_ref_diagnostics(int32_t nx, int32_t ny, int32_t nz, int32_t order, double gamma,
                             const float* rho_flat, const float* p_flat, const float* vel_flat,
                             double out[2]);

/* Number of kernel launches the last oux_step call issued (for reporting). */
int oux_launch_count(const oux_handle* h, int64_t* launches);

/* --- batched solves ---------------------------------------------------------
 * No reference counterpart: the reference runs one solve per executable.  A
 * batch advances many bound handles (independent periodic solves of any grid
 * sizes) with ONE persistent kernel launch per time step over a phase-major
 * tile work list; each solve computes what oux_step computes for it (bit for
 * bit in FP64).
 *
 * Members must share dim, order, visc, visc_order / visc_stencil, precision and
 * rk; scheme, tvd, slau, gamma, R, Pr, Prt, threshold, dt and the grid may
 * differ.  The batch snapshots each member's bound buffers and constants at
 * oux_batch_bind (for the mixed form: the pressure / temperature references of
 * the member's last oux_set_state), so set the states before binding. */
typedef struct oux_batch oux_batch;

typedef struct oux_batch_tuning {
  int32_t pencil;        /* sweep tiles per work item, >= 1 (consecutive along the sweep) */
  int32_t chunk;         /* cells per point-wise work item, >= 1 */
  int32_t blocks_per_sm; /* persistent blocks per SM; 0 = as many as fit */
  int32_t use_graph;     /* 1: each step replays one captured CUDA graph */
  int32_t mode;          /* enum oux_batch_mode */
} oux_batch_tuning;

/* OUX_BATCH_PERSISTENT: one persistent kernel per step over the tile work list
 * (pencil / chunk / blocks_per_sm apply).  OUX_BATCH_GRAPH: one CUDA graph per
 * step in which every solve's own stage kernels (those of oux_step) run on a
 * branch of their own, so the solves overlap on the device (always graphed). */
enum oux_batch_mode { OUX_BATCH_PERSISTENT = 0, OUX_BATCH_GRAPH = 1 };

/* tuning may be NULL (persistent, pencil 4, chunk 1152, all resident blocks, graphs on). */
int oux_batch_create(oux_handle* const* members, int32_t n, const oux_batch_tuning* tuning,
                     oux_batch** out);
/* Device workspace (step arguments, work list, counters) the batch needs. */
int oux_batch_workspace_bytes(const oux_batch* b, size_t* bytes);
/* Attach a caller-owned, 256-byte aligned workspace and upload the work list on
 * `stream` (synchronises it). */
int oux_batch_bind(oux_batch* b, void* workspace_dev, size_t bytes, void* stream);
/* nsteps time steps of every member: per step a counter reset and one kernel
 * launch (or one CUDA-graph replay); asynchronous on `stream`, no allocation. */
int oux_batch_step(oux_batch* b, int32_t nsteps, void* stream);
/* Batch status word: OUX_FAULT_TIMEOUT if a dependency wait gave up. */
int oux_batch_status(oux_batch* b, int32_t* fault_bits);
/* Work-list size, phases per step and the persistent grid. */
int oux_batch_info(const oux_batch* b, int64_t* items, int32_t* phases, int32_t* grid);
/* Polls a dependency wait of the persistent kernel makes before it gives up,
 * sets OUX_FAULT_TIMEOUT in the batch status word and ends its block (default
 * OUX_BATCH_SPIN_LIMIT, 2^22 polls of >= 64 ns).  A captured step is released and
 * captured anew at the next oux_batch_step.  No counterpart in the reference,
 * whose kernels never wait on each other. */
int oux_batch_set_spin_limit(oux_batch* b, int32_t polls);
/* Byte offset, within the bound workspace, of the dependency record of
 * (member, phase): two int32, the phase it waits for (-1: none) and the number of
 * that phase's items it waits for.  For failure-injection tests, which make a wait
 * run out by raising the count out of reach from the host.  No counterpart in the
 * reference. */
int oux_batch_dep_offset(const oux_batch* b, int32_t member, int32_t phase, size_t* offset);
int oux_batch_destroy(oux_batch* b);

/* --- allocation-free residual ---------------------------------------------
 * No counterpart in the reference.  The same stage residual as oux_rhs, for
 * callers that cannot allocate device memory when they call: a host program
 * that has no device allocator of its own and does not want to size, own and
 * bind a scratch buffer (a Fortran or C driver holding only plain pointers), or
 * code running where every free byte is already reserved by another allocator
 * (a caching allocator's pool) or where an allocation's implicit device
 * synchronisation is not acceptable.  It needs no handle and calls no
 * cudaMalloc / cudaFree or other allocating routine.
 *
 * Scratch: a fixed device array of OUX_NOALLOC_SCRATCH_BYTES inside the library,
 * created on every GPU where the library's device code is loaded and held until
 * the process exits.  A grid whose oux_scratch_bytes() exceeds that size is
 * rejected with OUX_E_TOO_SMALL and a message giving both sizes; that is about
 * 200 000 cells (59^3 with ghosts) in 3D FP64.
 *
 * The call has no handle, so it carries no boundary rules (oux_set_boundary):
 * LES on a grid with a non-periodic direction is refused with OUX_E_INVALID, since
 * the SGS viscosity of its wall cells depends on those rules.  Euler and
 * Navier-Stokes grids with non-periodic directions give oux_rhs's result (their
 * residual reads the boundary cells the caller filled, not the rules).
 *
 * Inputs: cfg (precision must be OUX_FP64); state_dev, a 256-byte aligned
 * device array in the layout oux_layout_of() reports for cfg (the state buffer
 * of oux_bind, ghost cells already filled), only read.  Output: rhs_dev as for
 * oux_rhs.  Asynchronous on `stream`; dx/dy/dz are copied on `stream`, so when
 * they are page-locked they must stay valid until the stream reaches the call.
 *
 * The first call on a device looks up the array's device address on that
 * device (cudaGetSymbolAddress, with that device current), and looks it up again
 * only if the device's context has been made anew since (after cudaDeviceReset).
 * With lazy module loading (CUDA_MODULE_LOADING=LAZY, the default since CUDA
 * 12.2) that first call is also when the library's device code is loaded on the
 * device and the array is created; if another allocator's pool already holds all
 * free device memory then, it fails with OUX_E_CUDA (out of memory).  So make the
 * first call on each device at start-up, before such pools fill the device and
 * before any stream capture.  Every call on a device
 * shares the one array, which keeps the previous call's contents (the call
 * clears what must start at zero), so calls whose GPU work overlaps (other
 * streams, other host threads) race and give wrong results: order them on one
 * stream or synchronise between them. */
#define OUX_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
int oux_rhs_noalloc(const oux_config* cfg, const double* state_dev, double* rhs_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* OUX_H */
