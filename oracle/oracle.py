"""ctypes binding of the CPU oracle (test infrastructure only).

Imported by tests/, by the smoke check and by the CPU-baseline leg of the
benchmark -- never by the product.  The C source, cmg_oracle.c, restates the
reference solver; see its header for the reference files it follows.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

LEAF, NONLEAF, GHOST = 1, 2, 4
DIRICHLET, INTERIOR, NEUMANN = 1, 2, 4
CASE_UNIFORM, CASE_CENTER_POINT, CASE_SPHERE_EMPTY, CASE_SPHERE_SOLID = 0, 1, 2, 3
CASE_STAR_EMPTY, CASE_STAR_SOLID, CASE_SHELL, CASE_MULTI_SPHERE = 4, 5, 6, 7
GMG, CMG = 1, 2

TARGET_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P, I, F, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
        LL = ctypes.c_longlong
        sig = {
            "og_grid_new": (P, [F, I]),
            "og_grid_free": (None, [P]),
            "og_set_tile": (I, [P, I, I, I, I, I]),
            "og_rebuild": (I, [P]),
            "og_refine_case": (I, [P, I, P, I]),
            "og_num_tiles": (I, [P]),
            "og_max_level": (I, [P]),
            "og_get_tiles": (None, [P, P, P, P]),
            "og_get_tables": (None, [P, P, P, P]),
            "og_alloc_channels": (I, [P, I]),
            "og_channel": (P, [P, I]),
            "og_cell_types": (P, [P]),
            "og_set_leaf_cell_types_case": (None, [P, I, P, I]),
            "og_coarsen_types_and_coeffs": (None, [P, I, F]),
            "og_cutcell_sphere_coeffs": (None, [P, I, F, I, P]),
            "og_prepare_system": (None, [P, I, F]),
            "og_full_neg_lap_leafs": (None, [P, I, I, I]),
            "og_gauss_seidel": (None, [P, I, I, I, I, I, I, D]),
            "og_residual_restrict": (None, [P, I, I, I, I, F]),
            "og_fas_save": (None, [P, I, I, I, I, I]),
            "og_fas_prolong": (None, [P, I, I, I, F]),
            "og_fas_mu_cycle": (None, [P, I, I, I, I, I, I, I, D, F, F]),
            "og_vcycle": (None, [P, I, I, I, I, I, I, D, F, F]),
            "og_mu_cycle": (None, [P, I, I, I, I, I, I, I, D, F, F]),
            "og_fas_f_cycle": (None, [P, I, I, I, I, I, I, I, D, F, F]),
            "og_dot": (D, [P, I, I]),
            "og_amg_solve": (I, [P, I, D, I, F, F, I, D, I, I, I, I, P]),
            "og_face_velocity_fourier": (None, [P, I, I, P, P, P]),
            "og_divergence": (None, [P, I, I, I]),
            "og_add_gradient_to_face": (None, [P, I, I, I]),
            "og_calc_cell_types_from_leafs": (None, [P]),
            "og_geo_full_neg_lap": (None, [P, I, I, I]),
            "og_geo_gauss_seidel": (None, [P, I, I, I, I, I, I]),
            "og_geo_vcycle": (None, [P, I, I, I, I, I, I, F, F]),
            "og_geo_solve": (I, [P, I, F, F, I, D, I, I, I, I, P]),
            "og_fas_mu_cycle_solve": (I, [P, I, I, D, F, F, I, D, I, I, P]),
            "og_gmg_damped_jacobi_solve": (I, [P, I, D, F, P]),
            "og_assemble_count": (I, [P, I, P, P]),
            "og_assemble": (I, [P, I, P, P, P, P, P]),
            "og_csr_solve": (I, [I, P, P, P, P, P, D, I, I, P, P]),
            "og_csr_matvec": (I, [I, P, P, P, P, P]),
            "og_frac_inside": (F, [F, F]),
            "og_face_fluid_ratio": (None, [P, I, P]),
            "og_cell_corner_inside_count": (None, [P, F, P]),
            "og_case_target_at": (I, [F, I, P, I, I, I, I, I]),
            "og_case_types_at": (None, [F, I, I, I, I, I, P]),
            "og_set_reference_mask": (None, [P, I]),
            "og_set_x_bf16": (None, [P, I]),
            "og_refine_fn": (I, [P, TARGET_FN, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Grid:
    """Oracle octree: tiles in canonical order (level, tile type, Morton)."""

    def __init__(self, h0=0.125, num_levels=10):
        self.L = lib()
        self.g = self.L.og_grid_new(h0, num_levels)
        self.h0 = h0
        self.nch = 0

    def __del__(self):
        try:
            self.L.og_grid_free(self.g)
        except Exception:
            pass

    def set_tile(self, level, i, j, k, ttype):
        return self.L.og_set_tile(self.g, level, i, j, k, ttype)

    def rebuild(self):
        self.L.og_rebuild(self.g)

    def refine_case(self, case_id, params):
        prm = np.asarray(params, dtype=np.float64)
        return self.L.og_refine_case(self.g, case_id, _p(prm), len(prm))

    def iterative_refine(self, level_target):
        """level_target(level, i, j, k) -> target level of that tile (HADeviceGrid::iterativeRefine)."""
        cb = TARGET_FN(lambda user, level, i, j, k: int(level_target(level, i, j, k)))
        return self.L.og_refine_fn(self.g, cb, None)

    def set_reference_mask(self, on):
        self.L.og_set_reference_mask(self.g, int(bool(on)))

    def set_x_bf16(self, on):
        self.L.og_set_x_bf16(self.g, int(bool(on)))

    @property
    def n(self):
        return self.L.og_num_tiles(self.g)

    @property
    def max_level(self):
        return self.L.og_max_level(self.g)

    def tiles(self):
        n = self.n
        lv = np.zeros(n, np.int32)
        ijk = np.zeros((n, 3), np.int32)
        ty = np.zeros(n, np.uint8)
        self.L.og_get_tiles(self.g, _p(lv), _p(ijk), _p(ty))
        return lv, ijk, ty

    def tables(self):
        n = self.n
        nbr = np.zeros((n, 6), np.int32)
        par = np.zeros(n, np.int32)
        ch = np.zeros((n, 8), np.int32)
        self.L.og_get_tables(self.g, _p(nbr), _p(par), _p(ch))
        return nbr, par, ch

    def alloc(self, nch=16):
        self.nch = nch
        self.L.og_alloc_channels(self.g, nch)

    def channel(self, ch):
        """A writable numpy view (n, 512) of channel `ch`."""
        ptr = self.L.og_channel(self.g, ch)
        buf = (ctypes.c_float * (self.n * 512)).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float32).reshape(self.n, 512)

    def cell_types(self):
        ptr = self.L.og_cell_types(self.g)
        buf = (ctypes.c_uint8 * (self.n * 512)).from_address(ptr)
        return np.frombuffer(buf, dtype=np.uint8).reshape(self.n, 512)

    def set_leaf_cell_types_case(self, case_id, params=(0, 0)):
        prm = np.asarray(params, dtype=np.float64)
        self.L.og_set_leaf_cell_types_case(self.g, case_id, _p(prm), len(prm))

    def coarsen_types_and_coeffs(self, coeff_ch, R=0.5):
        self.L.og_coarsen_types_and_coeffs(self.g, coeff_ch, R)

    def cutcell_sphere_coeffs(self, coeff_ch, spheres, R=0.5):
        s = np.ascontiguousarray(np.asarray(spheres, dtype=np.float32).reshape(-1, 4))
        self.L.og_cutcell_sphere_coeffs(self.g, coeff_ch, R, s.shape[0], _p(s))

    def full_neg_lap_leafs(self, x_ch, coeff_ch, ax_ch):
        self.L.og_full_neg_lap_leafs(self.g, x_ch, coeff_ch, ax_ch)

    def gauss_seidel(self, iters, order, level, x_ch, coeff_ch, rhs_ch, omega):
        self.L.og_gauss_seidel(self.g, iters, order, level, x_ch, coeff_ch, rhs_ch, omega)

    def fas_mu_cycle(self, mu, x_ch, rhs_ch, x0_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict=1.0, P=1.0):
        self.L.og_fas_mu_cycle(self.g, mu, x_ch, rhs_ch, x0_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict, P)

    def vcycle(self, x_ch, f_ch, rhs_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict=1.0, P=1.0):
        """AMGSolver::VCycle (src/AMGSolver.cu:1060)"""
        self.L.og_vcycle(self.g, x_ch, f_ch, rhs_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict, P)

    def mu_cycle(self, repeat_times, x_ch, f_ch, rhs_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict=1.0, P=1.0):
        """AMGSolver::muCycle (src/AMGSolver.cu:1151)"""
        self.L.og_mu_cycle(self.g, repeat_times, x_ch, f_ch, rhs_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict, P)

    def fas_f_cycle(self, mu, x_ch, rhs_ch, x0_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict=1.0, P=1.0):
        """AMGSolver::FASFCycle (src/AMGSolver.cu:1358)"""
        self.L.og_fas_f_cycle(self.g, mu, x_ch, rhs_ch, x0_ch, coeff_ch, level_iters, coarsest_iters, omega, R_restrict, P)

    def dot(self, a, b):
        return self.L.og_dot(self.g, a, b)

    def amg_solve(self, coeff_ch, omega=1.5, mu=2, R_restrict=1.0, P=1.0, max_iters=100, tol=1e-6,
                  level_iters=2, coarsest_iters=10, sync_stride=1, pure_neumann=False):
        rel = ctypes.c_double(0)
        it = self.L.og_amg_solve(self.g, coeff_ch, omega, mu, R_restrict, P, max_iters, tol, level_iters,
                                 coarsest_iters, sync_stride, int(pure_neumann), ctypes.byref(rel))
        return it, rel.value

    def calc_cell_types_from_leafs(self):
        self.L.og_calc_cell_types_from_leafs(self.g)

    def geo_full_neg_lap(self, kind, x_ch, ax_ch):
        self.L.og_geo_full_neg_lap(self.g, kind, x_ch, ax_ch)

    def geo_gauss_seidel(self, kind, iters, order, level, x_ch, rhs_ch):
        self.L.og_geo_gauss_seidel(self.g, kind, iters, order, level, x_ch, rhs_ch)

    def geo_vcycle(self, kind, x_ch, f_ch, rhs_ch, level_iters, coarsest_iters, one_over_alpha=1.0, P=1.0):
        self.L.og_geo_vcycle(self.g, kind, x_ch, f_ch, rhs_ch, level_iters, coarsest_iters, one_over_alpha, P)

    def geo_solve(self, kind, one_over_alpha=1.0, P=1.0, max_iters=100, tol=1e-6, level_iters=2, coarsest_iters=10,
                  sync_stride=1, pure_neumann=False):
        """GMGSolver / CMGSolver::solve: PCG preconditioned by one V-cycle."""
        rel = ctypes.c_double(0)
        it = self.L.og_geo_solve(self.g, kind, one_over_alpha, P, max_iters, tol, level_iters, coarsest_iters, sync_stride,
                                 int(pure_neumann), ctypes.byref(rel))
        return it, rel.value

    def fas_mu_cycle_solve(self, coeff_ch, repeat_times=1, omega=1.5, R_restrict=1.0, P=1.0, max_iters=100, tol=1e-6,
                           level_iters=2, coarsest_iters=10):
        rel = ctypes.c_double(0)
        it = self.L.og_fas_mu_cycle_solve(self.g, coeff_ch, repeat_times, omega, R_restrict, P, max_iters, tol, level_iters,
                                          coarsest_iters, ctypes.byref(rel))
        return it, rel.value

    def gmg_damped_jacobi_solve(self, max_iters=100, tol=1e-6, omega=1.0):
        rel = ctypes.c_double(0)
        it = self.L.og_gmg_damped_jacobi_solve(self.g, max_iters, tol, omega, ctypes.byref(rel))
        return it, rel.value

    def face_velocity_fourier(self, u_ch, k, amp, phase):
        k = np.ascontiguousarray(k, dtype=np.float64)
        amp = np.ascontiguousarray(amp, dtype=np.float64)
        phase = np.ascontiguousarray(phase, dtype=np.float64)
        self.L.og_face_velocity_fourier(self.g, u_ch, len(phase), _p(k), _p(amp), _p(phase))

    def divergence(self, u_ch, coeff_ch, out_ch):
        self.L.og_divergence(self.g, u_ch, coeff_ch, out_ch)

    def divergence_without_coeff(self, u_ch, out_ch):
        self.L.og_divergence(self.g, u_ch, -1, out_ch)

    def add_gradient_to_face(self, x_ch, coeff_ch, u_ch):
        self.L.og_add_gradient_to_face(self.g, x_ch, coeff_ch, u_ch)

    def assemble(self, coeff_ch):
        """FP64 CSR of the leaf operator; rows/cols are INTERIOR cells of LEAF tiles."""
        nr = ctypes.c_int(0)
        nnz = ctypes.c_longlong(0)
        self.L.og_assemble_count(self.g, coeff_ch, ctypes.byref(nr), ctypes.byref(nnz))
        n, z = nr.value, nnz.value
        rp = np.zeros(n + 1, np.int64)
        ci = np.zeros(z, np.int32)
        va = np.zeros(z, np.float64)
        rt = np.zeros(n, np.int32)
        rc = np.zeros(n, np.int32)
        self.L.og_assemble(self.g, coeff_ch, _p(rp), _p(ci), _p(va), _p(rt), _p(rc))
        return rp, ci, va, rt, rc


def csr_solve(rp, ci, va, b, tol=1e-12, max_iters=20000, method=0):
    """Jacobi-preconditioned FP64 CG (method 0) or BiCGSTAB (method 1)."""
    n = len(rp) - 1
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n, np.float64)
    it = ctypes.c_int(0)
    rel = ctypes.c_double(0)
    lib().og_csr_solve(n, _p(rp), _p(ci), _p(va), _p(b), _p(x), tol, max_iters, method, ctypes.byref(it), ctypes.byref(rel))
    return x, it.value, rel.value


def csr_matvec(rp, ci, va, x):
    n = len(rp) - 1
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(n, np.float64)
    lib().og_csr_matvec(n, _p(rp), _p(ci), _p(va), _p(x), _p(y))
    return y


def frac_inside(a, b):
    return lib().og_frac_inside(a, b)


def face_fluid_ratio(phi4):
    phi4 = np.ascontiguousarray(phi4, np.float32).reshape(-1, 4)
    out = np.zeros(len(phi4), np.float32)
    lib().og_face_fluid_ratio(_p(phi4), len(phi4), _p(out))
    return out


def cell_corner_inside_count(nodes729, iso):
    nodes = np.ascontiguousarray(nodes729, np.float32).reshape(729)
    out = np.zeros(512, np.int32)
    lib().og_cell_corner_inside_count(_p(nodes), iso, _p(out))
    return out


def case_target_at(h0, case_id, params, level, ijk):
    prm = np.asarray(params, dtype=np.float64)
    return lib().og_case_target_at(h0, case_id, _p(prm), len(prm), level, int(ijk[0]), int(ijk[1]), int(ijk[2]))


def case_types_at(h0, case_id, level, ijk):
    out = np.zeros(512, np.uint8)
    lib().og_case_types_at(h0, case_id, level, int(ijk[0]), int(ijk[1]), int(ijk[2]), _p(out))
    return out
