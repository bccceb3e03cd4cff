"""Python binding of libcmg.so (the C ABI in include/cmg.h).

Mirrors the reference's solver interface (src/AMGSolver.h, src/HAGrid.h) so
that a caller written against Cirrus-amg reads the same:

    grid = HADeviceGrid(1/8, 10)                 # HADeviceGrid(h0, log2hash per level)
    grid.set_tile_host(0, (0, 0, 0), LEAF)       # setTileHost
    grid.rebuild()
    grid.iterative_refine(level_target)          # or grid.refine_case(...)
    solver = AMGSolver(coeff_channel, 0.5, 1, 1)
    solver.prepareTypesAndCoeffs(grid)
    iters, rel = solver.solve(grid, False, 100, 1e-6, 2, 10, 1, False)

The library is required: there is no CPU path.  Importing this module on a
machine without libcmg.so raises; calling a device function without a CUDA
device returns the CUDA error as an exception.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcmg.so")

LEAF, NONLEAF, GHOST = 1, 2, 4
DIRICHLET, INTERIOR, NEUMANN = 1, 2, 4
STORAGE = {"fp32": 0, "bf16": 1, "fp16": 2}  # operator storage of the smoothing sweeps
CASE_UNIFORM, CASE_CENTER_POINT, CASE_SPHERE_EMPTY, CASE_SPHERE_SOLID = 0, 1, 2, 3
CASE_STAR_EMPTY, CASE_STAR_SOLID, CASE_SHELL, CASE_MULTI_SPHERE = 4, 5, 6, 7

# names of every entry point include/cmg.h declares
EXPORTS = [
    "cmg_last_error", "cmg_version", "cmg_check_division",
    "cmg_grid_create", "cmg_grid_destroy", "cmg_grid_set_tile", "cmg_grid_rebuild", "cmg_grid_iterative_refine",
    "cmg_grid_refine_case", "cmg_grid_refine_case_device", "cmg_grid_info", "cmg_grid_tiles", "cmg_grid_tables", "cmg_grid_channel_ptr",
    "cmg_grid_cell_type_ptr", "cmg_grid_upload_channel", "cmg_grid_download_channel", "cmg_grid_upload_cell_types",
    "cmg_grid_download_cell_types", "cmg_grid_fill_channel", "cmg_grid_copy_channel", "cmg_grid_set_leaf_cell_types_case", "cmg_grid_set_stream",
    "cmg_grid_calc_cell_types_from_leafs", "cmg_grid_load_hagr", "cmg_grid_dump_hagr", "cmg_ref_record_layout",
    "cmg_grid_synchronize",
    "cmg_amg_prepare_types_and_coeffs", "cmg_amg_prepare_system", "cmg_amg_cutcell_sphere_coeffs",
    "cmg_amg_face_velocity_fourier", "cmg_amg_divergence", "cmg_amg_add_gradient_to_face", "cmg_amg_full_neg_lap",
    "cmg_amg_dot", "cmg_amg_dot_noalloc",
    "cmg_amg_solver_create", "cmg_amg_solver_destroy", "cmg_amg_solver_set_smoother", "cmg_amg_solver_set_launch_mode",
    "cmg_gmg_solver_create", "cmg_cmg_solver_create", "cmg_mg_vcycle", "cmg_mg_gauss_seidel", "cmg_mg_full_neg_lap",
    "cmg_amg_fas_mu_cycle_solve", "cmg_gmg_damped_jacobi_solve",
    "cmg_amg_solve",
    "cmg_amg_solve_host", "cmg_amg_gauss_seidel", "cmg_amg_gauss_seidel_masked", "cmg_amg_fas_mu_cycle", "cmg_amg_last_solve_ms",
    "cmg_amg_last_solve_launches", "cmg_amg_solve_batch", "cmg_amg_solver_set_storage", "cmg_amg_divergence_without_coeff",
    "cmg_grid_gather_device_tiles", "cmg_grid_scatter_device_tiles",
    "cmg_learned_create", "cmg_learned_destroy", "cmg_learned_num_params", "cmg_learned_get_params",
    "cmg_learned_set_params", "cmg_learned_set_samples", "cmg_learned_forward", "cmg_learned_gradient", "cmg_learned_apply_grid",
    "cmg_learned_train", "cmg_learned_set_loss", "cmg_learned_set_inference", "cmg_amg_solver_set_learned",
    "cmg_amg_solver_autotune", "cmg_amg_solver_set_finest_iters", "cmg_amg_solver_learned_status",
    "cmg_amg_solver_set_residual_replacement", "cmg_amg_solver_residual_replacements", "cmg_amg_solver_set_coarsest_direct", "cmg_amg_solver_set_cycle_bf16",
    "cmg_batch_create", "cmg_batch_destroy", "cmg_batch_set_schedule", "cmg_batch_schedule", "cmg_batch_solve", "cmg_batch_autotune",
    "cmg_amg_vcycle", "cmg_amg_mu_cycle", "cmg_amg_fas_f_cycle", "cmg_set_dependent_launch",
]

TARGET_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "-j4"], check=True)


def lib():
    """The loaded library.  Raises if libcmg.so has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` (there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        P, I, F, D, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_size_t
        PP = ctypes.POINTER(ctypes.c_void_p)
        sig = {
            "cmg_last_error": (ctypes.c_char_p, []),
            "cmg_version": (I, []),
            "cmg_check_division": (I, [ctypes.c_longlong, ctypes.c_ulonglong, P, P]),
            "cmg_grid_create": (I, [F, I, I, PP]),
            "cmg_grid_destroy": (I, [P]),
            "cmg_grid_set_tile": (I, [P, I, I, I, I, I]),
            "cmg_grid_rebuild": (I, [P]),
            "cmg_grid_iterative_refine": (I, [P, TARGET_FN, P, P]),
            "cmg_grid_refine_case": (I, [P, I, P, I, P]),
            "cmg_grid_refine_case_device": (I, [P, I, P, I, P]),
            "cmg_grid_info": (I, [P, P, P, P]),
            "cmg_grid_tiles": (I, [P, P, P, P]),
            "cmg_grid_tables": (I, [P, P, P]),
            "cmg_grid_channel_ptr": (I, [P, I, PP]),
            "cmg_grid_cell_type_ptr": (I, [P, PP]),
            "cmg_grid_upload_channel": (I, [P, I, P, S]),
            "cmg_grid_download_channel": (I, [P, I, P, S]),
            "cmg_grid_upload_cell_types": (I, [P, P, S]),
            "cmg_grid_download_cell_types": (I, [P, P, S]),
            "cmg_grid_fill_channel": (I, [P, I, F]),
            "cmg_grid_copy_channel": (I, [P, I, I]),
            "cmg_grid_set_leaf_cell_types_case": (I, [P, I, P, I]),
            "cmg_grid_set_stream": (I, [P, P]),
            "cmg_grid_calc_cell_types_from_leafs": (I, [P]),
            "cmg_grid_load_hagr": (I, [P, S, I, PP]),
            "cmg_ref_record_layout": (I, [P, I]),
            "cmg_grid_dump_hagr": (I, [P, P, S, ctypes.POINTER(ctypes.c_size_t)]),
            "cmg_grid_synchronize": (I, [P]),
            "cmg_amg_prepare_types_and_coeffs": (I, [P, I, F]),
            "cmg_amg_prepare_system": (I, [P, I, F]),
            "cmg_amg_cutcell_sphere_coeffs": (I, [P, I, F, I, P]),
            "cmg_amg_face_velocity_fourier": (I, [P, I, I, P, P, P]),
            "cmg_amg_divergence": (I, [P, I, I, I]),
            "cmg_amg_add_gradient_to_face": (I, [P, I, I, I]),
            "cmg_amg_full_neg_lap": (I, [P, I, I, I]),
            "cmg_amg_dot": (I, [P, I, I, P]),
            "cmg_amg_dot_noalloc": (I, [P, I, I, P]),
            "cmg_amg_solver_create": (I, [I, F, F, F, PP]),
            "cmg_amg_solver_destroy": (I, [P]),
            "cmg_amg_solver_set_smoother": (I, [P, D, I]),
            "cmg_amg_solver_set_launch_mode": (I, [P, I]),
            "cmg_gmg_solver_create": (I, [F, F, PP]),
            "cmg_cmg_solver_create": (I, [F, F, PP]),
            "cmg_mg_vcycle": (I, [P, P, I, I, I, I, I]),
            "cmg_mg_gauss_seidel": (I, [P, P, I, I, I, I, I]),
            "cmg_mg_full_neg_lap": (I, [P, P, I, I]),
            "cmg_amg_fas_mu_cycle_solve": (I, [P, P, I, I, I, D, I, I, P, P]),
            "cmg_gmg_damped_jacobi_solve": (I, [P, P, I, I, D, F, P, P]),
            "cmg_amg_solve": (I, [P, P, I, I, D, I, I, I, I, P, P]),
            "cmg_amg_solve_host": (I, [P, P, P, P, S, I, D, I, I, I, I, P, P]),
            "cmg_amg_gauss_seidel": (I, [P, P, I, I, I, I, I]),
            "cmg_amg_gauss_seidel_masked": (I, [P, P, I, I, I, I, I]),
            "cmg_amg_fas_mu_cycle": (I, [P, P, I, I, I, I, I]),
            "cmg_amg_last_solve_ms": (I, [P, P]),
            "cmg_amg_last_solve_launches": (I, [P, P]),
            "cmg_amg_solve_batch": (I, [P, P, I, P, P, I, D, I, I, I, I, P, P, P]),
            "cmg_amg_vcycle": (I, [P, P, I, I, I, I, I]),
            "cmg_set_dependent_launch": (I, [I]),
            "cmg_amg_mu_cycle": (I, [P, P, I, I, I, I, I, I]),
            "cmg_amg_fas_f_cycle": (I, [P, P, I, I, I, I, I]),
            "cmg_batch_create": (I, [P, P, I, P]),
            "cmg_batch_destroy": (I, [P]),
            "cmg_batch_set_schedule": (I, [P, I, I, D]),
            "cmg_batch_schedule": (I, [P, P, P, P, P, P]),
            "cmg_batch_solve": (I, [P, P, P, I, D, I, I, I, I, P, P, P, P]),
            "cmg_batch_autotune": (I, [P, P, P, P, I, I, D, I, I, I, P, P]),
            "cmg_amg_solver_set_storage": (I, [P, I]),
            "cmg_amg_divergence_without_coeff": (I, [P, I, I]),
            "cmg_grid_gather_device_tiles": (I, [P, P, S, I, I, I]),
            "cmg_grid_scatter_device_tiles": (I, [P, P, S, I, I]),
            "cmg_learned_create": (I, [I, ctypes.c_ulonglong, P]),
            "cmg_learned_destroy": (I, [P]),
            "cmg_learned_num_params": (I, [P, P]),
            "cmg_learned_get_params": (I, [P, P, I]),
            "cmg_learned_set_params": (I, [P, P, I]),
            "cmg_learned_set_samples": (I, [P, I, P, P, P, P, P, P]),
            "cmg_learned_apply_grid": (I, [P, P, I, I, I, I, I, I]),
            "cmg_learned_forward": (I, [P, I, I, P]),
            "cmg_learned_gradient": (I, [P, I, I, P, P]),
            "cmg_learned_train": (I, [P, I, I, F, ctypes.c_ulonglong, P]),
            "cmg_learned_set_loss": (I, [P, I]),
            "cmg_learned_set_inference": (I, [I]),
            "cmg_amg_solver_autotune": (I, [P, P, I, P, I, D, I, P, P, P]),
            "cmg_amg_solver_set_finest_iters": (I, [P, I]),
            "cmg_amg_solver_set_residual_replacement": (I, [P, I]),
            "cmg_amg_solver_set_coarsest_direct": (I, [P, I]),
            "cmg_amg_solver_set_cycle_bf16": (I, [P, I]),
            "cmg_amg_solver_residual_replacements": (I, [P, ctypes.POINTER(I)]),
            "cmg_amg_solver_set_learned": (I, [P, P]),
            "cmg_amg_solver_learned_status": (I, [P, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class CmgError(RuntimeError):
    pass


def ref_record_layout():
    """The 'HAGR' header and PoissonTile<float,15> record layout the library assumes
    (see cmg_ref_record_layout in include/cmg.h), as a dict."""
    L = lib()
    m = L.cmg_ref_record_layout(None, 0)
    out = (ctypes.c_longlong * m)()
    L.cmg_ref_record_layout(out, m)
    keys = ["header_bytes", "off_magic", "off_version", "off_num_levels", "off_max_level", "off_tile_size",
            "off_coord_size", "off_h0", "off_tile_count", "coord_bytes", "tile_bytes", "types_offset",
            "channels", "channel_stride"]
    return dict(zip(keys, list(out)))


def check_division(n, seed=0):
    """Count of pairs on which the coarse-level division differs from IEEE division,
    and the first differing (a, d) as float bit patterns."""
    m = ctypes.c_longlong(0)
    first = (ctypes.c_uint * 2)()
    _check(lib().cmg_check_division(int(n), int(seed), ctypes.byref(m), first), "check_division")
    return m.value, (first[0], first[1])


def solve_batch(solvers, grids, max_iters, relative_tolerance, level_iters, coarsest_iters, sync_stride, is_pure_neumann,
                b_host=None, x_host=None):
    """n independent solves, each on its own grid's stream, enqueued together (cmg_amg_solve_batch).
    b_host / x_host: None, or lists of n host buffer addresses (num_tiles*512 floats each).
    Returns lists (iters, rel_res, ms)."""
    n = len(solvers)
    if len(grids) != n or (b_host is None) != (x_host is None):
        raise CmgError("solve_batch: solvers, grids and host buffers must match")
    for s_ in solvers:
        s_._sync_params()
    sv = (ctypes.c_void_p * max(n, 1))(*[s_.h for s_ in solvers])
    gv = (ctypes.c_void_p * max(n, 1))(*[g.h for g in grids])
    bv = (ctypes.c_void_p * max(n, 1))(*b_host) if b_host is not None else None
    xv = (ctypes.c_void_p * max(n, 1))(*x_host) if x_host is not None else None
    it = (ctypes.c_int * max(n, 1))()
    rel = (ctypes.c_double * max(n, 1))()
    ms = (ctypes.c_float * max(n, 1))()
    _check(lib().cmg_amg_solve_batch(sv, gv, n, bv, xv, max_iters, relative_tolerance, level_iters, coarsest_iters, sync_stride,
                                     int(is_pure_neumann), it, rel, ms), "solve_batch")
    return list(it[:n]), list(rel[:n]), list(ms[:n])


class PersistentBatch:
    """n octrees solved by ONE persistent launch inside a CUDA graph (cmg_batch_*): groups of
    resident blocks take the octrees largest first from a device queue and run each one's
    whole solve.  solvers[i] gives grid i its settings (one solver may serve several grids);
    results equal solver.solve(grid, ...) bit for bit.  Solvers and grids must outlive it."""

    def __init__(self, solvers, grids):
        if len(solvers) != len(grids):
            raise CmgError("PersistentBatch: one solver per grid")
        self.L = lib()
        self.solvers, self.grids = list(solvers), list(grids)
        self.n = len(grids)
        sv = (ctypes.c_void_p * max(self.n, 1))(*[s_.h for s_ in self.solvers])
        gv = (ctypes.c_void_p * max(self.n, 1))(*[g.h for g in self.grids])
        h = ctypes.c_void_p()
        _check(self.L.cmg_batch_create(sv, gv, self.n, ctypes.byref(h)), "cmg_batch_create")
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.L.cmg_batch_destroy(self.h)
            self.h = None

    def set_schedule(self, group_blocks=0, split=0.0, slots=4):
        """blocks of `slots` 128-thread slots (4, 6, 8); groups of `group_blocks` blocks on the
        shared queue (0: the resident blocks spread over the octrees); split > 0: octrees too
        large for such a group within split x (total work / resident blocks) get a group of
        their own"""
        _check(self.L.cmg_batch_set_schedule(self.h, int(slots), int(group_blocks), float(split)), "set_schedule")

    def set_group_blocks(self, group_blocks):
        self.set_schedule(group_blocks, 0.0, self.schedule()[0])

    def schedule(self):
        """(slots, small groups' blocks, groups, dedicated groups, resident blocks) of the next solve"""
        v = [ctypes.c_int(0) for _ in range(5)]
        _check(self.L.cmg_batch_schedule(self.h, *[ctypes.byref(x) for x in v]), "schedule")
        return tuple(x.value for x in v)

    def _sync(self):
        for s_ in {id(s_): s_ for s_ in self.solvers}.values():
            s_._sync_params()

    def solve(self, max_iters, relative_tolerance, level_iters, coarsest_iters, sync_stride, is_pure_neumann, b_host=None, x_host=None):
        """Returns (iters, rel_res, per-octree ms inside the launch, launch ms).  b_host / x_host:
        None (b, x in channels 1, 0) or lists of n host buffer addresses."""
        if (b_host is None) != (x_host is None):
            raise CmgError("PersistentBatch.solve: b_host and x_host go together")
        self._sync()
        n = max(self.n, 1)
        bv = (ctypes.c_void_p * n)(*b_host) if b_host is not None else None
        xv = (ctypes.c_void_p * n)(*x_host) if x_host is not None else None
        it, rel, ims = (ctypes.c_int * n)(), (ctypes.c_double * n)(), (ctypes.c_float * n)()
        bms = ctypes.c_float(0)
        _check(self.L.cmg_batch_solve(self.h, bv, xv, max_iters, relative_tolerance, level_iters, coarsest_iters, sync_stride,
                                      int(is_pure_neumann), it, rel, ims, ctypes.byref(bms)), "batch solve")
        return list(it[:self.n]), list(rel[:self.n]), list(ims[:self.n]), bms.value

    def autotune(self, candidates, max_iters, relative_tolerance, level_iters, coarsest_iters, repeats=2):
        """candidates: (group_blocks, split, slots) tuples (shorter tuples or a bare int: split 0,
        4 slots).  Times each schedule after one calibration run; keeps and returns the fastest
        (None if none converged) with the list of times (-1: not converged)."""
        self._sync()

        def norm(c):
            c = (c,) if isinstance(c, int) else tuple(c)
            return (int(c[0]), float(c[1]) if len(c) > 1 else 0.0, int(c[2]) if len(c) > 2 else 4)

        cand = [norm(c) for c in candidates]
        m = len(cand)
        gv = (ctypes.c_int * m)(*[c[0] for c in cand])
        sv = (ctypes.c_double * m)(*[c[1] for c in cand])
        nv = (ctypes.c_int * m)(*[c[2] for c in cand])
        ms = (ctypes.c_float * m)()
        best = ctypes.c_int(-1)
        _check(self.L.cmg_batch_autotune(self.h, nv, gv, sv, m, max_iters, relative_tolerance, level_iters, coarsest_iters, repeats, ms,
                                         ctypes.byref(best)), "batch autotune")
        return (candidates[best.value] if best.value >= 0 else None), list(ms[:m])


def _check(rc, what):
    if rc != 0:
        msg = lib().cmg_last_error()
        raise CmgError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class HADeviceGrid:
    """Octree of 8^3 tiles on the device (src/HAGrid.h:357)."""

    def __init__(self, h0=0.125, num_levels=10, num_channels=16):
        self.L = lib()
        h = ctypes.c_void_p()
        _check(self.L.cmg_grid_create(h0, num_levels, num_channels, ctypes.byref(h)), "cmg_grid_create")
        self.h = h
        self.h0 = h0
        self.num_channels = num_channels
        self._cb = None

    def _adopt(self, h, num_channels):
        self.L = lib()
        self.h = h
        self.num_channels = num_channels
        self._cb = None
        self.h0 = None  # held by the library

    def __del__(self):
        try:
            if self.h:
                self.L.cmg_grid_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def set_tile_host(self, level, coord, ttype):
        _check(self.L.cmg_grid_set_tile(self.h, level, int(coord[0]), int(coord[1]), int(coord[2]), ttype), "set_tile")

    def rebuild(self):
        _check(self.L.cmg_grid_rebuild(self.h), "rebuild")

    def iterative_refine(self, level_target):
        """level_target(level, i, j, k) -> target level of that tile."""
        cb = TARGET_FN(lambda user, l, i, j, k: int(level_target(l, i, j, k)))
        self._cb = cb
        steps = ctypes.c_int(0)
        _check(self.L.cmg_grid_iterative_refine(self.h, cb, None, ctypes.byref(steps)), "iterative_refine")
        return steps.value

    def refine_case(self, case_id, params, on_device=False):
        """iterativeRefine with a built-in target; on_device: the whole build (refinement,
        ghost layer, canonical order, tables) in device memory (cmg_grid_refine_case_device)."""
        prm = np.asarray(params, dtype=np.float64)
        steps = ctypes.c_int(0)
        fn = self.L.cmg_grid_refine_case_device if on_device else self.L.cmg_grid_refine_case
        _check(fn(self.h, case_id, _p(prm), len(prm), ctypes.byref(steps)), "refine_case")
        return steps.value

    def info(self):
        n, ml, nl = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        _check(self.L.cmg_grid_info(self.h, ctypes.byref(n), ctypes.byref(ml), ctypes.byref(nl)), "info")
        return n.value, ml.value, nl.value

    @property
    def num_tiles(self):
        return self.info()[0]

    @property
    def max_level(self):
        return self.info()[1]

    def tiles(self):
        n = self.num_tiles
        lv = np.zeros(n, np.int32)
        ijk = np.zeros((n, 3), np.int32)
        ty = np.zeros(n, np.uint8)
        _check(self.L.cmg_grid_tiles(self.h, _p(lv), _p(ijk), _p(ty)), "tiles")
        return lv, ijk, ty

    def tables(self):
        n = self.num_tiles
        nb = np.zeros((n, 8), np.int32)
        ch = np.zeros((n, 8), np.int32)
        _check(self.L.cmg_grid_tables(self.h, _p(nb), _p(ch)), "tables")
        return nb, ch

    def channel_ptr(self, ch):
        p = ctypes.c_void_p()
        _check(self.L.cmg_grid_channel_ptr(self.h, ch, ctypes.byref(p)), "channel_ptr")
        return p.value

    def upload(self, ch, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32).reshape(-1)
        _check(self.L.cmg_grid_upload_channel(self.h, ch, _p(a), a.size), "upload_channel")

    def download(self, ch):
        a = np.zeros((self.num_tiles, 512), np.float32)
        _check(self.L.cmg_grid_download_channel(self.h, ch, _p(a), a.size), "download_channel")
        return a

    def upload_cell_types(self, arr):
        a = np.ascontiguousarray(arr, dtype=np.uint8).reshape(-1)
        _check(self.L.cmg_grid_upload_cell_types(self.h, _p(a), a.size), "upload_cell_types")

    def download_cell_types(self):
        a = np.zeros((self.num_tiles, 512), np.uint8)
        _check(self.L.cmg_grid_download_cell_types(self.h, _p(a), a.size), "download_cell_types")
        return a

    def fill(self, ch, value):
        _check(self.L.cmg_grid_fill_channel(self.h, ch, value), "fill_channel")

    def copy(self, src_ch, dst_ch):
        _check(self.L.cmg_grid_copy_channel(self.h, src_ch, dst_ch), "copy_channel")

    @classmethod
    def loadBinaryBlob(cls, blob, num_channels=16):
        """HADeviceGrid::loadBinaryBlob (src/HAGrid.h:788): a grid from an 'HAGR' v1 blob."""
        L = lib()
        buf = (ctypes.c_uint8 * len(blob)).from_buffer_copy(bytes(blob))
        h = ctypes.c_void_p()
        _check(L.cmg_grid_load_hagr(buf, len(blob), num_channels, ctypes.byref(h)), "loadBinaryBlob")
        self = cls.__new__(cls)
        self._adopt(h, num_channels)
        return self

    def dumpBinaryBlob(self):
        """HADeviceGrid::dumpBinaryBlob (src/HAGrid.h:687): the grid as an 'HAGR' v1 blob (bytes)."""
        n = ctypes.c_size_t(0)
        _check(self.L.cmg_grid_dump_hagr(self.h, None, 0, ctypes.byref(n)), "dumpBinaryBlob")
        buf = (ctypes.c_uint8 * n.value)()
        _check(self.L.cmg_grid_dump_hagr(self.h, buf, n.value, ctypes.byref(n)), "dumpBinaryBlob")
        return bytes(buf)

    def gather_device_tiles(self, tile_ptrs, first_ch, num_ch, with_types=True):
        """Channels (and cell types) from the reference's own device tiles (PoissonTile<float,15>),
        tile_ptrs[t] = device address of the tile that is tile t of this grid."""
        arr = (ctypes.c_void_p * max(len(tile_ptrs), 1))(*tile_ptrs)
        _check(self.L.cmg_grid_gather_device_tiles(self.h, arr, 44880, first_ch, num_ch, int(with_types)), "gather_device_tiles")

    def scatter_device_tiles(self, tile_ptrs, first_ch, num_ch):
        """Channels of this grid written back into the reference's device tiles."""
        arr = (ctypes.c_void_p * max(len(tile_ptrs), 1))(*tile_ptrs)
        _check(self.L.cmg_grid_scatter_device_tiles(self.h, arr, 44880, first_ch, num_ch), "scatter_device_tiles")

    def calc_cell_types_from_leafs(self):
        """CalcCellTypesFromLeafs (src/PoissonGrid.cu:923): NONLEAF and GHOST cell types from the LEAF ones."""
        _check(self.L.cmg_grid_calc_cell_types_from_leafs(self.h), "calc_cell_types_from_leafs")

    def set_leaf_cell_types_case(self, case_id, params=(0, 0)):
        prm = np.asarray(params, dtype=np.float64)
        _check(self.L.cmg_grid_set_leaf_cell_types_case(self.h, case_id, _p(prm), len(prm)), "set_leaf_cell_types")

    def set_stream(self, stream_ptr):
        _check(self.L.cmg_grid_set_stream(self.h, ctypes.c_void_p(stream_ptr)), "set_stream")

    def synchronize(self):
        _check(self.L.cmg_grid_synchronize(self.h), "synchronize")

    # operator set-up and rhs (src/AMGSolver.cu, cirrus_cutcell/MeshCutCell.cu)
    def prepare_system(self, coeff_ch, R_matrix):
        _check(self.L.cmg_amg_prepare_system(self.h, coeff_ch, R_matrix), "prepare_system")

    def cutcell_sphere_coeffs(self, coeff_ch, spheres, R_matrix=0.5):
        s = np.ascontiguousarray(np.asarray(spheres, dtype=np.float32).reshape(-1, 4))
        _check(self.L.cmg_amg_cutcell_sphere_coeffs(self.h, coeff_ch, R_matrix, s.shape[0], _p(s)), "cutcell_sphere_coeffs")

    def face_velocity_fourier(self, u_ch, k, amp, phase):
        k = np.ascontiguousarray(k, dtype=np.float64)
        amp = np.ascontiguousarray(amp, dtype=np.float64)
        phase = np.ascontiguousarray(phase, dtype=np.float64)
        _check(self.L.cmg_amg_face_velocity_fourier(self.h, u_ch, len(phase), _p(k), _p(amp), _p(phase)), "face_velocity")

    def divergence(self, u_ch, coeff_ch, out_ch):
        _check(self.L.cmg_amg_divergence(self.h, u_ch, coeff_ch, out_ch), "divergence")

    def divergence_without_coeff(self, u_ch, out_ch):
        """AMGVolumeWeightedDivergenceWithoutCoeffOnLeafs (src/AMGSolver.cu:750)."""
        _check(self.L.cmg_amg_divergence_without_coeff(self.h, u_ch, out_ch), "divergence_without_coeff")

    def add_gradient_to_face(self, x_ch, coeff_ch, u_ch):
        _check(self.L.cmg_amg_add_gradient_to_face(self.h, x_ch, coeff_ch, u_ch), "add_gradient_to_face")

    def full_neg_lap(self, x_ch, coeff_ch, ax_ch):
        _check(self.L.cmg_amg_full_neg_lap(self.h, x_ch, coeff_ch, ax_ch), "full_neg_lap")

    def dot(self, a_ch, b_ch):
        out = ctypes.c_double(0)
        _check(self.L.cmg_amg_dot(self.h, a_ch, b_ch, ctypes.byref(out)), "dot")
        return out.value


class AMGSolver:
    """AMGSolver (src/AMGSolver.h:19-75): FAS mu-cycle preconditioned CG."""

    def __init__(self, coeff_channel, R_matrix_coeff=1.0, R_restrict_coeff=1.0, P_coeff=1.0):
        self.L = lib()
        h = ctypes.c_void_p()
        _check(self.L.cmg_amg_solver_create(coeff_channel, R_matrix_coeff, R_restrict_coeff, P_coeff, ctypes.byref(h)),
               "cmg_amg_solver_create")
        self.h = h
        self.coeff_channel = coeff_channel
        self.R_matrix_coeff = R_matrix_coeff
        self.omega = 1.5
        self.mu_cycle_repeat_times = 2
        self.finest_iters = -1  # sweeps on the finest level; -1: level_iters (the reference)

    def __del__(self):
        try:
            if self.h:
                self.L.cmg_amg_solver_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def set_launch_mode(self, use_graph=True, persistent=False, cluster=True, pipeline=True):
        """use_graph: one CUDA graph per solve (default) or kernel-by-kernel launches;
        persistent: levels 2-3 of each cycle in one cooperative kernel (off by default);
        cluster: each visit of level 2 in one 9-CTA cluster launch when levels 0-2 are complete;
        pipeline: the cycle's smoothing sweeps as a persistent kernel that prefetches the next tile."""
        flags = (1 if use_graph else 0) | (2 if persistent else 0) | (0 if cluster else 4) | (0 if pipeline else 8)
        _check(self.L.cmg_amg_solver_set_launch_mode(self.h, flags), "set_launch_mode")

    def set_residual_replacement(self, every):
        """Replace the recurrence residual by b - A x (stencil in FP64) every `every` PCG
        iterations; 0 (default) never, as the reference."""
        _check(self.L.cmg_amg_solver_set_residual_replacement(self.h, int(every)), "set_residual_replacement")

    def set_coarsest_direct(self, on=True):
        """Level 0 solved exactly (FP64 Cholesky-based inverse) when the cluster step runs
        levels 0-2, instead of the reference's coarsest sweeps."""
        _check(self.L.cmg_amg_solver_set_coarsest_direct(self.h, int(bool(on))), "set_coarsest_direct")

    def set_cycle_bf16(self, on=True):
        """x, rhs and saved x of the cycle's levels >= 3 stored in BF16 (FP32 arithmetic)."""
        _check(self.L.cmg_amg_solver_set_cycle_bf16(self.h, int(bool(on))), "set_cycle_bf16")

    def last_replacements(self):
        n = ctypes.c_int(0)
        _check(self.L.cmg_amg_solver_residual_replacements(self.h, ctypes.byref(n)), "residual_replacements")
        return n.value

    def set_storage(self, storage):
        """Operator storage of the mu-cycle's smoothing sweeps: "fp32" (default, the
        reference's arithmetic), "bf16" or "fp16" (mixed precision)."""
        _check(self.L.cmg_amg_solver_set_storage(self.h, STORAGE[storage]), "set_storage")

    def set_learned(self, net=None):
        """Use `net` (a LearnedNet, its current parameters) as the finest-level smoother:
        flexible PCG judged by the true residual, plain fallback.  None: the plain solve."""
        _check(self.L.cmg_amg_solver_set_learned(self.h, net.h if net is not None else None), "set_learned")

    def learned_status(self):
        """(true relative residual, fell back to the plain solve, learned iterations) of the last solve."""
        tr, fb, it = ctypes.c_double(0), ctypes.c_int(0), ctypes.c_int(0)
        _check(self.L.cmg_amg_solver_learned_status(self.h, ctypes.byref(tr), ctypes.byref(fb), ctypes.byref(it)),
               "learned_status")
        return tr.value, bool(fb.value), it.value

    def autotune(self, grid, candidates=None, max_iters=100, relative_tolerance=1e-6, repeats=2):
        """Time solves of the grid's current rhs (channel 1) under each candidate
        (omega, mu, level_iters, coarsest_iters[, finest_iters]) and keep the fastest that
        converges (among those within 3 % of the fastest, the one with the fewest
        iterations, then the smallest final residual).  Sets omega, mu_cycle_repeat_times and finest_iters; returns (best candidate
        as a 5-tuple or None, table of (candidate, ms or None, iters))."""
        if candidates is None:
            candidates = default_tune_candidates()
        candidates = [tuple(c) + (-1,) * (5 - len(c)) for c in candidates]
        n = len(candidates)
        arr = (TuneCandidate * n)(*[TuneCandidate(float(c[0]), int(c[1]), int(c[2]), int(c[3]), int(c[4])) for c in candidates])
        ms = np.zeros(n, np.float32)
        its = np.zeros(n, np.int32)
        best = ctypes.c_int(-1)
        self._sync_params()
        _check(self.L.cmg_amg_solver_autotune(self.h, grid.h, n, ctypes.cast(arr, ctypes.c_void_p), max_iters, relative_tolerance,
                                               repeats, _p(ms), _p(its), ctypes.byref(best)), "autotune")
        table = [(candidates[i], float(ms[i]) if ms[i] >= 0 else None, int(its[i])) for i in range(n)]
        if best.value < 0:
            return None, table
        b = candidates[best.value]
        self.omega, self.mu_cycle_repeat_times = float(b[0]), int(b[1])
        self.finest_iters = int(b[4])
        return b, table

    def _sync_params(self):
        _check(self.L.cmg_amg_solver_set_smoother(self.h, float(self.omega), int(self.mu_cycle_repeat_times)), "set_smoother")
        if hasattr(self, "finest_iters"):
            _check(self.L.cmg_amg_solver_set_finest_iters(self.h, int(self.finest_iters)), "set_finest_iters")

    def prepareTypesAndCoeffs(self, grid):
        _check(self.L.cmg_amg_prepare_types_and_coeffs(grid.h, self.coeff_channel, self.R_matrix_coeff), "prepareTypesAndCoeffs")

    def solve(self, grid, verbose, max_iters, relative_tolerance, level_iters, coarsest_iters, sync_stride, is_pure_neumann):
        self._sync_params()
        it, rel = ctypes.c_int(0), ctypes.c_double(0)
        _check(self.L.cmg_amg_solve(self.h, grid.h, int(verbose), max_iters, relative_tolerance, level_iters, coarsest_iters,
                                    sync_stride, int(is_pure_neumann), ctypes.byref(it), ctypes.byref(rel)), "solve")
        return it.value, rel.value

    def solve_host(self, grid, b_host_ptr, x_host_ptr, count, max_iters, relative_tolerance, level_iters, coarsest_iters,
                   sync_stride=1, is_pure_neumann=False):
        """Solve with host buffers (pointers, e.g. pinned memory): b copied in, x copied out."""
        self._sync_params()
        it, rel = ctypes.c_int(0), ctypes.c_double(0)
        _check(self.L.cmg_amg_solve_host(self.h, grid.h, ctypes.c_void_p(b_host_ptr), ctypes.c_void_p(x_host_ptr), count,
                                         max_iters, relative_tolerance, level_iters, coarsest_iters, sync_stride,
                                         int(is_pure_neumann), ctypes.byref(it), ctypes.byref(rel)), "solve_host")
        return it.value, rel.value

    def gauss_seidel(self, grid, iters, order, level, x_ch, rhs_ch):
        self._sync_params()
        _check(self.L.cmg_amg_gauss_seidel(self.h, grid.h, iters, order, level, x_ch, rhs_ch), "gauss_seidel")

    def gauss_seidel_masked(self, grid, iters, order, level, x_ch, rhs_ch):
        """The sweeps as the cycle runs them; x must be 0 on cells that are not INTERIOR."""
        self._sync_params()
        _check(self.L.cmg_amg_gauss_seidel_masked(self.h, grid.h, iters, order, level, x_ch, rhs_ch), "gauss_seidel_masked")

    def fas_mu_cycle(self, grid, x_ch, rhs_ch, x0_ch, level_iters, coarsest_iters):
        self._sync_params()
        _check(self.L.cmg_amg_fas_mu_cycle(self.h, grid.h, x_ch, rhs_ch, x0_ch, level_iters, coarsest_iters), "fas_mu_cycle")

    def VCycle(self, grid, x_ch, f_ch, rhs_ch, level_iters, coarsest_iters):
        """AMGSolver::VCycle (src/AMGSolver.cu:1060): correction-scheme V-cycle from x = 0 for rhs f."""
        self._sync_params()
        _check(self.L.cmg_amg_vcycle(self.h, grid.h, x_ch, f_ch, rhs_ch, level_iters, coarsest_iters), "VCycle")

    def muCycle(self, repeat_times, grid, x_ch, f_ch, rhs_ch, level_iters, coarsest_iters):
        """AMGSolver::muCycle (src/AMGSolver.cu:1151): correction-scheme mu-cycle from x = 0 for rhs f."""
        self._sync_params()
        _check(self.L.cmg_amg_mu_cycle(self.h, grid.h, repeat_times, x_ch, f_ch, rhs_ch, level_iters, coarsest_iters), "muCycle")

    def FASFCycle(self, grid, x_ch, rhs_ch, x0_ch, level_iters, coarsest_iters):
        """AMGSolver::FASFCycle (src/AMGSolver.cu:1358): the FAS full-multigrid cycle."""
        self._sync_params()
        _check(self.L.cmg_amg_fas_f_cycle(self.h, grid.h, x_ch, rhs_ch, x0_ch, level_iters, coarsest_iters), "FASFCycle")

    def FASMuCycleSolve(self, repeat_times, grid, verbose, max_iters, relative_tolerance, level_iters, coarsest_iters):
        """AMGSolver::FASMuCycleSolve (src/AMGSolver.cu:1311): mu-cycles as a stand-alone iteration."""
        self._sync_params()
        it, rel = ctypes.c_int(0), ctypes.c_double(0)
        _check(self.L.cmg_amg_fas_mu_cycle_solve(self.h, grid.h, repeat_times, int(verbose), max_iters, relative_tolerance,
                                                 level_iters, coarsest_iters, ctypes.byref(it), ctypes.byref(rel)),
               "FASMuCycleSolve")
        return it.value, rel.value

    def last_solve_ms(self):
        ms = ctypes.c_float(0)
        _check(self.L.cmg_amg_last_solve_ms(self.h, ctypes.byref(ms)), "last_solve_ms")
        return ms.value

    def last_solve_launches(self):
        n = ctypes.c_longlong(0)
        _check(self.L.cmg_amg_last_solve_launches(self.h, ctypes.byref(n)), "last_solve_launches")
        return n.value


class TuneCandidate(ctypes.Structure):
    """cmg_tune_candidate of include/cmg.h."""
    _fields_ = [("omega", ctypes.c_double), ("mu", ctypes.c_int), ("level_iters", ctypes.c_int),
                ("coarsest_iters", ctypes.c_int), ("finest_iters", ctypes.c_int)]


def default_tune_candidates():
    """The autotuner's default search: omega x mu x level_iters x coarsest_iters (finest level
    as the others), and for V-cycles a finest level with fewer sweeps than the others."""
    grid = [(om, mu, li, ci, -1) for om in (0.8, 0.9, 1.0, 1.1, 1.2, 1.3, 1.5) for mu in (1, 2) for li in (1, 2, 3)
            for ci in (2, 5, 10)]
    grid += [(om, 1, li, ci, fi) for om in (1.0, 1.2, 1.3) for li in (2, 3, 4) for ci in (5, 10) for fi in (1, 2) if fi < li]
    return grid


def set_dependent_launch(on):
    """Launch the pipelined smoothing passes as programmatic dependents of the kernel before
    them (default on; same results either way).  Takes effect for graphs built afterwards."""
    _check(lib().cmg_set_dependent_launch(int(bool(on))), "set_dependent_launch")


def set_learned_inference(kind):
    """Inference kernel of the learned smoother: "mma.sync" (default) or "tcgen05"."""
    _check(lib().cmg_learned_set_inference({"mma.sync": 0, "tcgen05": 1}[kind]), "set_learned_inference")


class LearnedNet:
    """The learned finest-level smoother's per-tile network (BF16 tensor cores), its
    parameters, Adam state and training samples on the device (no reference counterpart)."""

    def __init__(self, hidden=16, seed=0):
        self.L = lib()
        h = ctypes.c_void_p()
        _check(self.L.cmg_learned_create(int(hidden), ctypes.c_ulonglong(seed), ctypes.byref(h)), "cmg_learned_create")
        self.h = h
        self.hidden = hidden
        n = ctypes.c_int(0)
        _check(self.L.cmg_learned_num_params(self.h, ctypes.byref(n)), "num_params")
        self.num_params = n.value
        self.num_samples = 0

    def __del__(self):
        try:
            if self.h:
                self.L.cmg_learned_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def params(self):
        p = np.zeros(self.num_params, np.float32)
        _check(self.L.cmg_learned_get_params(self.h, _p(p), p.size), "get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(self.L.cmg_learned_set_params(self.h, _p(p), p.size), "set_params")

    def set_samples(self, rho, diag, types, target=None, faces=None, halo=None):
        """Tiles of 512 cells: rho, diag (float32), types (uint8), target (float32 or None);
        faces [n, 3, 512] (the -x/-y/-z face coefficients) and halo [n, 768] (the residual
        across the six faces, then 1/0 flags), each optional."""
        rho = np.ascontiguousarray(rho, dtype=np.float32).reshape(-1, 512)
        diag = np.ascontiguousarray(diag, dtype=np.float32).reshape(-1, 512)
        types = np.ascontiguousarray(types, dtype=np.uint8).reshape(-1, 512)
        n = rho.shape[0]
        tg = None if target is None else np.ascontiguousarray(target, dtype=np.float32).reshape(-1, 512)
        fc = None if faces is None else np.ascontiguousarray(faces, dtype=np.float32).reshape(n, 3, 512)
        hl = None if halo is None else np.ascontiguousarray(halo, dtype=np.float32).reshape(n, 768)
        _check(self.L.cmg_learned_set_samples(self.h, n, _p(rho), _p(diag), _p(types), _p(tg) if tg is not None else None,
                                              _p(fc) if fc is not None else None, _p(hl) if hl is not None else None), "set_samples")
        self.num_samples = rho.shape[0]

    def apply_grid(self, grid, level, r_ch, az_ch, coeff_ch, out_ch, overwrite=True):
        """The net on the grid's LEAF tiles of `level` (cmg_learned_apply_grid)."""
        _check(self.L.cmg_learned_apply_grid(self.h, grid.h, level, r_ch, az_ch, coeff_ch, out_ch, int(overwrite)), "apply_grid")

    def set_loss(self, kind):
        """"mse" (squared error, default) or "energy" (tile Laplacian-weighted)."""
        _check(self.L.cmg_learned_set_loss(self.h, {"mse": 0, "energy": 1}[kind]), "set_loss")

    def forward(self, first=0, n=None):
        n = self.num_samples - first if n is None else n
        out = np.zeros((n, 512), np.float32)
        _check(self.L.cmg_learned_forward(self.h, first, n, _p(out)), "forward")
        return out

    def gradient(self, first=0, n=None):
        n = self.num_samples - first if n is None else n
        loss = ctypes.c_double(0)
        g = np.zeros(self.num_params, np.float32)
        _check(self.L.cmg_learned_gradient(self.h, first, n, ctypes.byref(loss), _p(g)), "gradient")
        return loss.value, g

    def train(self, epochs, batch=256, lr=1e-3, seed=0):
        losses = np.zeros(max(epochs, 1), np.float32)
        _check(self.L.cmg_learned_train(self.h, epochs, batch, float(lr), ctypes.c_ulonglong(seed), _p(losses)), "train")
        return losses[:epochs]


class _GeometricSolver(AMGSolver):
    """Common part of GMGSolver and CMGSolver: PCG preconditioned by one V-cycle."""

    _create = None

    def __init__(self, one_over_alpha=1.0, prolong_coeff=1.0):
        self.L = lib()
        h = ctypes.c_void_p()
        _check(getattr(self.L, self._create)(one_over_alpha, prolong_coeff, ctypes.byref(h)), self._create)
        self.h = h
        self.one_over_alpha = one_over_alpha
        self.prolong_coeff = prolong_coeff
        self.omega = 1.5  # unused by the V-cycle smoother; kept for the shared launch plumbing
        self.mu_cycle_repeat_times = 1

    def prepareTypesAndCoeffs(self, grid):
        raise CmgError("geometric solvers derive their operator from tile and cell types: set the LEAF cell types, "
                       "then HADeviceGrid.calc_cell_types_from_leafs()")

    def VCycle(self, grid, x_channel, f_channel, rhs_channel, level_iters, coarsest_iters):
        _check(self.L.cmg_mg_vcycle(self.h, grid.h, x_channel, f_channel, rhs_channel, level_iters, coarsest_iters), "VCycle")

    def gauss_seidel(self, grid, iters, order, level, x_ch, rhs_ch):
        _check(self.L.cmg_mg_gauss_seidel(self.h, grid.h, iters, order, level, x_ch, rhs_ch), "gauss_seidel")

    def full_neg_lap(self, grid, x_channel, ax_channel):
        _check(self.L.cmg_mg_full_neg_lap(self.h, grid.h, x_channel, ax_channel), "full_neg_lap")

    def fas_mu_cycle(self, *args, **kwargs):
        raise CmgError("fas_mu_cycle belongs to AMGSolver; geometric solvers use VCycle")


class GMGSolver(_GeometricSolver):
    """GMGSolver(one_over_alpha, prolong_coeff) (src/GMGSolver.h:17-52)."""

    _create = "cmg_gmg_solver_create"


def _gmg_damped_jacobi(self, grid, verbose, max_iters, relative_tolerance, omega):
    """GMGSolver::dampedJacobiSolve (src/GMGSolver.cu:390)."""
    it, rel = ctypes.c_int(0), ctypes.c_double(0)
    _check(self.L.cmg_gmg_damped_jacobi_solve(self.h, grid.h, int(verbose), max_iters, relative_tolerance, omega,
                                              ctypes.byref(it), ctypes.byref(rel)), "dampedJacobiSolve")
    return it.value, rel.value


GMGSolver.dampedJacobiSolve = _gmg_damped_jacobi


class CMGSolver(_GeometricSolver):
    """CMGSolver(one_over_alpha, prolong_coeff) (src/CMGSolver.h:17-50)."""

    _create = "cmg_cmg_solver_create"
