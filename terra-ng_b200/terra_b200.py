"""Python mirror of the terra_b200 C ABI (include/terra_b200.h) over ctypes.

The product is the CUDA library ``libterra_b200.so`` built in-tree by
``build.py``; this module only marshals torch CUDA tensors to its entry points.
It raises when the library is missing: there is no CPU fallback.

Vectors are torch tensors on the GPU: a nodal scalar ``(10, nl, nl, nr)``, a
velocity a ``(3, 10, nl, nl, nr)`` tensor (components are passed as three
pointers, so a list of three tensors works too).
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libterra_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "terra_b200.h")

TN_OK = 0
TN_F64, TN_F32 = 0, 1
NEUMANN, DIRICHLET, FREESLIP = 0, 1, 2
REPLACE, ADD = 0, 1
SKIP_COMMUNICATION, COMMUNICATE_ADDITIVELY = 0, 1

_lib = None
STORED_OFF, STORED_FULL = 0, 1


SMOOTHER_CHEBYSHEV, SMOOTHER_JACOBI = 0, 1
COARSE_PCG, COARSE_DENSE = 0, 1
TRANSFER_CONSTANT, TRANSFER_LINEAR = 0, 1


class SolverOptions(ctypes.Structure):
    """tn_solver_options."""

    _fields_ = [
        ("restart", ctypes.c_int),
        ("max_iterations", ctypes.c_int),
        ("relative_tolerance", ctypes.c_double),
        ("absolute_tolerance", ctypes.c_double),
        ("chebyshev_order", ctypes.c_int),
        ("chebyshev_iterations", ctypes.c_int),
        ("power_iterations", ctypes.c_int),
        ("num_vcycles", ctypes.c_int),
        ("coarse_max_iterations", ctypes.c_int),
        ("coarse_relative_tolerance", ctypes.c_double),
        ("coarse_absolute_tolerance", ctypes.c_double),
        ("gca", ctypes.c_int),
        ("mixed_precision", ctypes.c_int),
        ("seed", ctypes.c_uint64),
        ("normalize_pressure", ctypes.c_int),
        ("project_pressure_mean", ctypes.c_int),
        ("cuda_graphs", ctypes.c_int),
        ("smoother", ctypes.c_int),
        ("jacobi_omega", ctypes.c_double),
        ("coarse_solver", ctypes.c_int),
        ("transfer", ctypes.c_int),
    ]


class TerraError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"terra_b200 error {code}: {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not found: build it with `python terra-ng_b200/build.py`")
    L = ctypes.CDLL(path)
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    vpp = ctypes.POINTER(ctypes.c_void_p)
    dp = ctypes.POINTER(ctypes.c_double)
    sig = {
        "tn_last_error": ([], ctypes.c_char_p),
        "tn_version": ([], ctypes.c_char_p),
        "tn_kernel_launch_count": ([], ctypes.c_uint64),
        "tn_shell_create": ([i, i, i, d, d, ctypes.POINTER(vp)], i),
        "tn_shell_destroy": ([vp], None),
        "tn_shell_num_levels": ([vp, ctypes.POINTER(i)], i),
        "tn_shell_level_dims": ([vp, i, ctypes.POINTER(i), ctypes.POINTER(i)], i),
        "tn_shell_copy_coords": ([vp, i, vp], i),
        "tn_shell_copy_radii": ([vp, i, vp], i),
        "tn_shell_copy_ownership": ([vp, i, vp], i),
        "tn_shell_copy_boundary_mask": ([vp, i, vp], i),
        "tn_shell_duplicate_classes": ([vp, i, vp, ctypes.POINTER(i)], i),
        "tn_mesh_generate_host": ([i, i, d, d, vp, vp, vp, vp, ctypes.POINTER(i)], i),
        "tn_shell_check_device_error": ([vp, ctypes.POINTER(i)], i),
        "tn_epsdivdiv_create": ([vp, i, i, vp, vp, i, i, i, ctypes.POINTER(vp)], i),
        "tn_operator_destroy": ([vp], None),
        "tn_operator_set_modes": ([vp, i, i], i),
        "tn_operator_set_diagonal": ([vp, i], i),
        "tn_operator_set_boundary_conditions": ([vp, i, i], i),
        "tn_operator_set_tile": ([vp, i, i], i),
        "tn_operator_apply": ([vp, vpp, vpp, vp], i),
        "tn_divergence_create": ([vp, i, i, i, i, ctypes.POINTER(vp)], i),
        "tn_gradient_create": ([vp, i, i, i, i, ctypes.POINTER(vp)], i),
        "tn_stokes_create": ([vp, i, i, vp, vp, i, i, ctypes.POINTER(vp)], i),
        "tn_operator_components": ([vp, ctypes.POINTER(i), ctypes.POINTER(i)], i),
        "tn_kmass_lumped_diagonal": ([vp, i, i, vp, vp, vp], i),
        "tn_vector_mass_apply": ([vp, i, i, vpp, vpp, vp], i),
        "tn_prolongate_add": ([vp, i, i, i, vpp, vpp, vp], i),
        "tn_restrict": ([vp, i, i, i, vpp, vpp, vp], i),
        "tn_prolongate_linear_add": ([vp, i, i, i, vpp, vpp, vp], i),
        "tn_restrict_linear": ([vp, i, i, i, vpp, vpp, vp], i),
        "tn_gca_build_interpolated": ([vp, vp, i, i, vp], i),
        "tn_interface_sum": ([vp, i, i, i, vpp, vp], i),
        "tn_vec_lincomb": ([vp, i, i, i, vpp, d, i, dp, vpp, vpp, vpp, vp], i),
        "tn_vec_dot": ([vp, i, i, i, vpp, vpp, dp, vp], i),
        "tn_vec_random": ([vp, i, i, i, ctypes.c_uint64, vpp, vp], i),
        "tn_vec_alloc": ([vp, i, i, i, vpp], i),
        "tn_vec_free": ([i, vpp], None),
        "tn_sync": ([vp], i),
        "tn_operator_set_stored_matrix_mode": ([vp, i, vp], i),
        "tn_gca_build": ([vp, vp, vp], i),
        "tn_operator_copy_local_matrices": ([vp, vp], i),
        "tn_solver_options_default": ([ctypes.POINTER(SolverOptions)], None),
        "tn_stokes_solver_create": ([vp, i, vp, vp, vp, i, i, ctypes.POINTER(SolverOptions), vp,
                                     ctypes.POINTER(vp)], i),
        "tn_velocity_solver_create": ([vp, i, vp, vp, i, i, ctypes.POINTER(SolverOptions), vp, ctypes.POINTER(vp)],
                                      i),
        "tn_multigrid_solver_create": ([vp, i, vp, vp, i, i, ctypes.POINTER(SolverOptions), vp, ctypes.POINTER(vp)],
                                       i),
        "tn_solver_destroy": ([vp], None),
        "tn_solver_solve": ([vp, vpp, vpp, vp], i),
        "tn_solver_result": ([vp, ctypes.POINTER(i), dp, ctypes.POINTER(i)], i),
        "tn_solver_history": ([vp, dp, i, ctypes.POINTER(i)], i),
        "tn_solver_full_residual": ([vp, dp], i),
        "tn_epsdivdiv_vjp": ([vp, vpp, vpp, vp, vpp, vp], i),
        "tn_stokes_misfit_gradient": ([vp, vpp, vpp, vp, vpp, vp], i),
        "tn_divergence_apply_noalloc": ([vp, i, i, i, i, vpp, vp, vp], i),
        "tn_solver_precondition": ([vp, vpp, vpp, vp], i),
        "tn_solver_vcycle": ([vp, i, vpp, vpp, vp], i),
        "tn_solver_level_lambda": ([vp, i, dp], i),
        "tn_solver_inverse_diagonal": ([vp, i, vpp, vp], i),
        "tn_solver_coarse_stats": ([vp, dp], i),
        "tn_solver_level_matrices": ([vp, i, vp], i),
        "tn_xdmf_create": ([vp, i, ctypes.c_char_p, i, ctypes.POINTER(vp)], i),
        "tn_xdmf_add": ([vp, ctypes.c_char_p, i, i, vpp, i], i),
        "tn_xdmf_write": ([vp, vp], i),
        "tn_xdmf_destroy": ([vp], None),
        "tn_xdmf_read": ([vp, i, ctypes.c_char_p, ctypes.c_char_p, i, i, i, vpp], i),
        "tn_vec_invert": ([vp, i, i, i, vpp, vp], i),
        "tn_vec_scale": ([vp, i, i, i, vpp, vpp, vp], i),
        "tn_vec_max_abs": ([vp, i, i, i, vpp, dp, vp], i),
        "tn_vec_has_nan_or_inf": ([vp, i, i, i, vpp, ctypes.POINTER(i), vp], i),
        "tn_vec_swap": ([vp, i, i, i, vpp, vpp, vp], i),
        "tn_vec_cast": ([ctypes.c_int64, i, vp, vp, vp], i),
        "tn_vec_assign_masked": ([vp, i, i, i, vpp, i, d, vp], i),
        "tn_vec_rotate_normal_tangential": ([vp, i, i, vpp, i, i, vp], i),
        "tn_vec_freeslip_project": ([vp, i, i, vpp, i, vp], i),
        "tn_stokes_rhs_enforce": ([vp, i, i, i, i, vpp, vp], i),
        "tn_gca_mark_elements": ([vp, i, i, vp, vp, vp], i),
        "tn_operator_set_selective_matrices": ([vp, i, vp, vp], i),
        "tn_operator_stored_cells": ([vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)], i),
        "tn_solver_level_storage": ([vp, i, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def kernel_launch_count() -> int:
    """Kernel launches issued by the library so far (tn_kernel_launch_count)."""
    return int(load().tn_kernel_launch_count())


def declared_symbols(header: str = HEADER_PATH):
    """Names of all functions declared in the public header."""
    import re

    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tn_[a-z0-9_]+)\s*\(", text)))


def _check(rc):
    if rc != TN_OK:
        raise TerraError(rc, load().tn_last_error().decode())


def _ptrs(arrs):
    return (ctypes.c_void_p * len(arrs))(*[int(a.data_ptr()) for a in arrs])


def _comps(v):
    if isinstance(v, (list, tuple)):
        return list(v)
    if v.dim() == 5:
        return [v[c] for c in range(v.shape[0])]
    return [v]


def _stream(stream):
    if stream is None:
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(int(stream))


def _prec(dtype):
    import torch

    if dtype == torch.float64:
        return TN_F64
    if dtype == torch.float32:
        return TN_F32
    raise TypeError(f"unsupported dtype {dtype}")


class Shell:
    """Mesh hierarchy on the device (tn_shell_*)."""

    def __init__(self, lat_level: int, rad_level: int | None = None, num_levels: int = 1, r_min=0.55, r_max=1.0):
        L = load()
        if rad_level is None:
            rad_level = lat_level
        h = ctypes.c_void_p()
        _check(L.tn_shell_create(lat_level, rad_level, num_levels, r_min, r_max, ctypes.byref(h)))
        self._h = h
        self.num_levels = num_levels
        self.lat_level, self.rad_level = lat_level, rad_level

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tn_shell_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def dims(self, level: int = -1):
        level = level % self.num_levels
        nl, nr = ctypes.c_int(), ctypes.c_int()
        _check(load().tn_shell_level_dims(self._h, level, ctypes.byref(nl), ctypes.byref(nr)))
        return nl.value, nr.value

    def coords(self, level: int = -1):
        import numpy as np

        nl, _ = self.dims(level)
        out = np.zeros((10, nl, nl, 3))
        _check(load().tn_shell_copy_coords(self._h, level % self.num_levels, out.ctypes.data))
        return out

    def radii(self, level: int = -1):
        import numpy as np

        _, nr = self.dims(level)
        out = np.zeros(nr)
        _check(load().tn_shell_copy_radii(self._h, level % self.num_levels, out.ctypes.data))
        return out

    def ownership(self, level: int = -1):
        import numpy as np

        nl, nr = self.dims(level)
        out = np.zeros((10, nl, nl, nr), np.uint8)
        _check(load().tn_shell_copy_ownership(self._h, level % self.num_levels, out.ctypes.data))
        return out

    def boundary_mask(self, level: int = -1):
        import numpy as np

        nl, nr = self.dims(level)
        out = np.zeros((10, nl, nl, nr), np.uint8)
        _check(load().tn_shell_copy_boundary_mask(self._h, level % self.num_levels, out.ctypes.data))
        return out

    def duplicate_classes(self, level: int = -1):
        import numpy as np

        nl, _ = self.dims(level)
        out = np.zeros((10, nl, nl), np.int32)
        n = ctypes.c_int()
        _check(load().tn_shell_duplicate_classes(self._h, level % self.num_levels, out.ctypes.data, ctypes.byref(n)))
        return out, n.value

    def check_device_error(self):
        c = ctypes.c_int()
        _check(load().tn_shell_check_device_error(self._h, ctypes.byref(c)))
        return c.value

    def interface_sum(self, v, level: int = -1, stream=None):
        comps = _comps(v)
        _check(load().tn_interface_sum(self._h, level % self.num_levels, _prec(comps[0].dtype), len(comps),
                                       _ptrs(comps), _stream(stream)))
        return v

    def dot(self, a, b, level: int = -1, stream=None):
        ca, cb = _comps(a), _comps(b)
        out = ctypes.c_double()
        _check(load().tn_vec_dot(self._h, level % self.num_levels, _prec(ca[0].dtype), len(ca), _ptrs(ca), _ptrs(cb),
                                 ctypes.byref(out), _stream(stream)))
        return out.value

    def lincomb(self, y, c0, coeffs=(), xs=(), level: int = -1, stream=None):
        cy = _comps(y)
        n = len(coeffs)
        cc = (ctypes.c_double * max(n, 1))(*coeffs) if n else None
        xp = [_ptrs(_comps(x)) for x in xs] + [None] * (3 - n)
        _check(load().tn_vec_lincomb(self._h, level % self.num_levels, _prec(cy[0].dtype), len(cy), _ptrs(cy),
                                     float(c0), n, cc, xp[0], xp[1], xp[2], _stream(stream)))
        return y


def mesh_generate_host(lat_level: int, rad_level: int, r_min=0.55, r_max=1.0):
    """Host-only mesh of one level: (coords, radii, owned_lat, class_of_lat, num_classes)."""
    import numpy as np

    nl, nr = (1 << lat_level) + 1, (1 << rad_level) + 1
    coords = np.zeros((10, nl, nl, 3))
    radii = np.zeros(nr)
    owned = np.zeros((10, nl, nl), np.uint8)
    cls = np.zeros((10, nl, nl), np.int32)
    n = ctypes.c_int()
    _check(load().tn_mesh_generate_host(lat_level, rad_level, r_min, r_max, coords.ctypes.data, radii.ctypes.data,
                                        owned.ctypes.data, cls.ctypes.data, ctypes.byref(n)))
    return coords, radii, owned, cls, n.value


class Operator:
    """Common part of the operator handles (tn_operator_*)."""

    _h = None

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tn_operator_destroy(self._h)
            self._h = None

    def _adopt(self, h):
        self._h = h
        si, di = ctypes.c_int(), ctypes.c_int()
        _check(load().tn_operator_components(h, ctypes.byref(si), ctypes.byref(di)))
        self.src_components, self.dst_components = si.value, di.value

    def set_modes(self, apply_mode=REPLACE, comm_mode=COMMUNICATE_ADDITIVELY):
        _check(load().tn_operator_set_modes(self._h, apply_mode, comm_mode))

    def set_boundary_conditions(self, bc_cmb, bc_surface):
        _check(load().tn_operator_set_boundary_conditions(self._h, bc_cmb, bc_surface))

    def apply(self, src, dst, stream=None):
        cs, cd = _comps(src), _comps(dst)
        if len(cs) != self.src_components or len(cd) != self.dst_components:
            raise ValueError(f"operator takes {self.src_components} -> {self.dst_components} components")
        _check(load().tn_operator_apply(self._h, _ptrs(cs), _ptrs(cd), _stream(stream)))
        return dst


class EpsDivDiv(Operator):
    """epsilon-div-div operator (tn_epsdivdiv_create)."""

    def __init__(self, shell: Shell, level: int = -1, k=None, k_cell=None, bc_cmb=DIRICHLET, bc_surface=DIRICHLET,
                 diagonal=False):
        L = load()
        if (k is None) == (k_cell is None):
            raise ValueError("give exactly one of k (nodal) or k_cell (Q0)")
        ref = k if k is not None else k_cell
        self.shell, self.level = shell, level % shell.num_levels
        self.dtype = ref.dtype
        h = ctypes.c_void_p()
        kp = ctypes.c_void_p(k.data_ptr()) if k is not None else None
        kc = ctypes.c_void_p(k_cell.data_ptr()) if k_cell is not None else None
        _check(L.tn_epsdivdiv_create(shell.handle, self.level, _prec(self.dtype), kp, kc, bc_cmb, bc_surface,
                                     int(diagonal), ctypes.byref(h)))
        self._adopt(h)

    def set_diagonal(self, flag: bool):
        _check(load().tn_operator_set_diagonal(self._h, int(flag)))

    def set_tile(self, tile_y=0, chunk_x=0):
        _check(load().tn_operator_set_tile(self._h, tile_y, chunk_x))

    def vjp(self, u, lam, grad_cell, grad_u=None, stream=None):
        """Backward of apply: grad_cell = d(lam^T A u)/d log(eta_cell); grad_u = A lam (tn_epsdivdiv_vjp)."""
        gu = None if grad_u is None else _ptrs(_comps(grad_u))
        _check(load().tn_epsdivdiv_vjp(self._h, _ptrs(_comps(u)), _ptrs(_comps(lam)),
                                       ctypes.c_void_p(grad_cell.data_ptr()), gu, _stream(stream)))
        return grad_cell

    def set_stored_matrix_mode(self, mode=STORED_FULL, stream=None):
        _check(load().tn_operator_set_stored_matrix_mode(self._h, mode, _stream(stream)))

    def set_selective_matrices(self, level_range: int, marks, stream=None):
        """Selective storage (tn_operator_set_selective_matrices): marks is a uint8 device tensor over the cells of
        the level level_range levels coarser, as gca_mark_elements returns it."""
        _check(load().tn_operator_set_selective_matrices(self._h, level_range, ctypes.c_void_p(marks.data_ptr()),
                                                         _stream(stream)))

    def stored_cells(self):
        """(cells with stored matrices, device bytes of the stored matrices)."""
        n, b = ctypes.c_int64(), ctypes.c_int64()
        _check(load().tn_operator_stored_cells(self._h, ctypes.byref(n), ctypes.byref(b)))
        return n.value, b.value

    def local_matrices(self):
        """(10, nl-1, nl-1, nr-1, 2, 18, 18) stored matrices (host)."""
        import numpy as np

        nl, nr = self.shell.dims(self.level)
        out = np.zeros((10, nl - 1, nl - 1, nr - 1, 2, 18, 18))
        _check(load().tn_operator_copy_local_matrices(self._h, out.ctypes.data))
        return out


def gca_build(fine: EpsDivDiv, coarse: EpsDivDiv, stream=None, interpolation=0, tensor_cores=True):
    """TwoGridGCA: coarse receives sum P^T A_fine P (tn_gca_build_interpolated)."""
    _check(load().tn_gca_build_interpolated(fine._h, coarse._h, interpolation, int(tensor_cores), _stream(stream)))


def gca_mark_elements(shell: Shell, level: int, level_range: int, k, stream=None):
    """GCAElementsCollector on the nodal coefficient k of `level`: a uint8 tensor over the cells of level
    level - level_range, 1 where a descendant wedge's reference-coordinate gradient of k exceeds 10."""
    import torch

    level = level % shell.num_levels
    nl, nr = shell.dims(level - level_range)
    marks = torch.empty((10, nl - 1, nl - 1, nr - 1), dtype=torch.uint8, device=k.device)
    _check(load().tn_gca_mark_elements(shell.handle, level, level_range, ctypes.c_void_p(k.data_ptr()),
                                       ctypes.c_void_p(marks.data_ptr()), _stream(stream)))
    return marks


def random_vector(shell: Shell, level: int, ncomp: int, seed: int, dtype=None, stream=None):
    """tn_vec_random into new tensors of shape (ncomp, 10, nl, nl, nr)."""
    import torch

    dtype = dtype or torch.float64
    nl, nr = shell.dims(level)
    v = torch.empty((ncomp, 10, nl, nl, nr), dtype=dtype, device="cuda")
    comps = [v[c] for c in range(ncomp)]
    _check(load().tn_vec_random(shell.handle, level % shell.num_levels, _prec(dtype), ncomp, ctypes.c_uint64(seed),
                                _ptrs(comps), _stream(stream)))
    return v


class Divergence(Operator):
    """B: velocity on `level` -> pressure on `level - 1` (tn_divergence_create)."""

    def __init__(self, shell: Shell, level: int = -1, dtype=None, bc_cmb=DIRICHLET, bc_surface=DIRICHLET):
        import torch

        self.shell, self.level = shell, level % shell.num_levels
        h = ctypes.c_void_p()
        _check(load().tn_divergence_create(shell.handle, self.level, _prec(dtype or torch.float64), bc_cmb,
                                           bc_surface, ctypes.byref(h)))
        self._adopt(h)


class Gradient(Operator):
    """B^T: pressure on `level - 1` -> velocity on `level` (tn_gradient_create)."""

    def __init__(self, shell: Shell, level: int = -1, dtype=None, bc_cmb=DIRICHLET, bc_surface=DIRICHLET):
        import torch

        self.shell, self.level = shell, level % shell.num_levels
        h = ctypes.c_void_p()
        _check(load().tn_gradient_create(shell.handle, self.level, _prec(dtype or torch.float64), bc_cmb, bc_surface,
                                         ctypes.byref(h)))
        self._adopt(h)


class Stokes(Operator):
    """[A B^T; B 0] on (velocity level, level - 1) (tn_stokes_create); vectors are 4 components."""

    def __init__(self, shell: Shell, level: int = -1, k=None, k_cell=None, bc_cmb=DIRICHLET, bc_surface=DIRICHLET):
        if (k is None) == (k_cell is None):
            raise ValueError("give exactly one of k (nodal) or k_cell (Q0)")
        ref = k if k is not None else k_cell
        self.shell, self.level = shell, level % shell.num_levels
        h = ctypes.c_void_p()
        kp = ctypes.c_void_p(k.data_ptr()) if k is not None else None
        kc = ctypes.c_void_p(k_cell.data_ptr()) if k_cell is not None else None
        _check(load().tn_stokes_create(shell.handle, self.level, _prec(ref.dtype), kp, kc, bc_cmb, bc_surface,
                                       ctypes.byref(h)))
        self._adopt(h)


def divergence_apply_noalloc(shell: Shell, velocity_level: int, u, p_out, bc_cmb=DIRICHLET, bc_surface=DIRICHLET,
                             stream=None):
    """p_out = B u with the static-scratch entry point (tn_divergence_apply_noalloc)."""
    cu = _comps(u)
    _check(load().tn_divergence_apply_noalloc(shell.handle, velocity_level % shell.num_levels, _prec(cu[0].dtype),
                                              bc_cmb, bc_surface, _ptrs(cu), ctypes.c_void_p(p_out.data_ptr()),
                                              _stream(stream)))
    return p_out


def kmass_lumped_diagonal(shell: Shell, level: int, k, out, stream=None):
    _check(load().tn_kmass_lumped_diagonal(shell.handle, level % shell.num_levels, _prec(k.dtype),
                                           ctypes.c_void_p(k.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                           _stream(stream)))
    return out


def vector_mass_apply(shell: Shell, level: int, src, dst, stream=None):
    cs, cd = _comps(src), _comps(dst)
    _check(load().tn_vector_mass_apply(shell.handle, level % shell.num_levels, _prec(cs[0].dtype), _ptrs(cs),
                                       _ptrs(cd), _stream(stream)))
    return dst


def prolongate_add(shell: Shell, fine_level: int, coarse, fine, stream=None):
    cc, cf = _comps(coarse), _comps(fine)
    _check(load().tn_prolongate_add(shell.handle, fine_level % shell.num_levels, _prec(cc[0].dtype), len(cc),
                                    _ptrs(cc), _ptrs(cf), _stream(stream)))
    return fine


def restrict(shell: Shell, fine_level: int, fine, coarse, stream=None):
    cf, cc = _comps(fine), _comps(coarse)
    _check(load().tn_restrict(shell.handle, fine_level % shell.num_levels, _prec(cf[0].dtype), len(cf), _ptrs(cf),
                              _ptrs(cc), _stream(stream)))
    return coarse


FLAG_INNER, FLAG_BOUNDARY, FLAG_CMB, FLAG_SURFACE = 1, 2, 6, 10


def vec_invert(shell: Shell, level: int, y, stream=None):
    cy = _comps(y)
    _check(load().tn_vec_invert(shell.handle, level % shell.num_levels, _prec(cy[0].dtype), len(cy), _ptrs(cy),
                                _stream(stream)))
    return y


def vec_scale(shell: Shell, level: int, y, x, stream=None):
    cy, cx = _comps(y), _comps(x)
    _check(load().tn_vec_scale(shell.handle, level % shell.num_levels, _prec(cy[0].dtype), len(cy), _ptrs(cy),
                               _ptrs(cx), _stream(stream)))
    return y


class DeviceVector:
    """ncomp arrays of a level's nodes allocated by the library (tn_vec_alloc, zero-filled); `pointers` holds the
    device addresses, released by tn_vec_free when the object goes away."""

    def __init__(self, shell: Shell, level: int, ncomp: int, dtype=None):
        import torch

        self.shell, self.level, self.ncomp = shell, level % shell.num_levels, ncomp
        self.dtype = dtype or torch.float64
        arr = (ctypes.c_void_p * ncomp)()
        _check(load().tn_vec_alloc(shell.handle, self.level, _prec(self.dtype), ncomp, arr))
        self._arr = arr
        self.pointers = [arr[c] for c in range(ncomp)]

    def __del__(self):
        if getattr(self, "_arr", None) is not None and _lib is not None:
            _lib.tn_vec_free(self.ncomp, self._arr)
            self._arr = None


def sync(stream=None):
    """tn_sync: wait for the stream's work."""
    _check(load().tn_sync(_stream(stream)))


def vec_max_abs(shell: Shell, level: int, a, stream=None) -> float:
    ca = _comps(a)
    out = ctypes.c_double()
    _check(load().tn_vec_max_abs(shell.handle, level % shell.num_levels, _prec(ca[0].dtype), len(ca), _ptrs(ca),
                                 ctypes.byref(out), _stream(stream)))
    return out.value


def vec_has_nan_or_inf(shell: Shell, level: int, a, stream=None) -> bool:
    ca = _comps(a)
    out = ctypes.c_int()
    _check(load().tn_vec_has_nan_or_inf(shell.handle, level % shell.num_levels, _prec(ca[0].dtype), len(ca),
                                        _ptrs(ca), ctypes.byref(out), _stream(stream)))
    return bool(out.value)


def vec_swap(shell: Shell, level: int, a, b, stream=None):
    ca, cb = _comps(a), _comps(b)
    _check(load().tn_vec_swap(shell.handle, level % shell.num_levels, _prec(ca[0].dtype), len(ca), _ptrs(ca),
                              _ptrs(cb), _stream(stream)))


def vec_cast(src, out, stream=None):
    """FP64 -> FP32 or FP32 -> FP64 copy of a contiguous tensor (tn_vec_cast)."""
    _check(load().tn_vec_cast(src.numel(), _prec(src.dtype), ctypes.c_void_p(src.data_ptr()),
                              ctypes.c_void_p(out.data_ptr()), _stream(stream)))
    return out


def vec_assign_masked(shell: Shell, level: int, v, flag: int, value: float = 0.0, stream=None):
    cv = _comps(v)
    _check(load().tn_vec_assign_masked(shell.handle, level % shell.num_levels, _prec(cv[0].dtype), len(cv),
                                       _ptrs(cv), flag, value, _stream(stream)))
    return v


def vec_rotate_normal_tangential(shell: Shell, level: int, v, flag: int, direction: int, stream=None):
    cv = _comps(v)
    _check(load().tn_vec_rotate_normal_tangential(shell.handle, level % shell.num_levels, _prec(cv[0].dtype),
                                                  _ptrs(cv), flag, direction, _stream(stream)))
    return v


def vec_freeslip_project(shell: Shell, level: int, v, flag: int, stream=None):
    cv = _comps(v)
    _check(load().tn_vec_freeslip_project(shell.handle, level % shell.num_levels, _prec(cv[0].dtype), _ptrs(cv),
                                          flag, _stream(stream)))
    return v


def stokes_rhs_enforce(shell: Shell, level: int, u, bc_cmb: int, bc_surface: int, stream=None):
    """The application's right-hand-side boundary treatment on the 3 velocity components (tn_stokes_rhs_enforce)."""
    cu = _comps(u)
    _check(load().tn_stokes_rhs_enforce(shell.handle, level % shell.num_levels, _prec(cu[0].dtype), bc_cmb,
                                        bc_surface, _ptrs(cu), _stream(stream)))
    return u


def prolongate_linear_add(shell: Shell, fine_level: int, coarse, fine, stream=None):
    cc, cf = _comps(coarse), _comps(fine)
    _check(load().tn_prolongate_linear_add(shell.handle, fine_level % shell.num_levels, _prec(cc[0].dtype), len(cc),
                                           _ptrs(cc), _ptrs(cf), _stream(stream)))
    return fine


def restrict_linear(shell: Shell, fine_level: int, fine, coarse, stream=None):
    cf, cc = _comps(fine), _comps(coarse)
    _check(load().tn_restrict_linear(shell.handle, fine_level % shell.num_levels, _prec(cf[0].dtype), len(cf),
                                     _ptrs(cf), _ptrs(cc), _stream(stream)))
    return coarse


def solver_options(**kw) -> SolverOptions:
    o = SolverOptions()
    load().tn_solver_options_default(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class _Solver:
    _h = None

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tn_solver_destroy(self._h)
            self._h = None

    def solve(self, x, b, stream=None):
        """x (initial guess, overwritten), b: component lists. Returns True when converged."""
        cx, cb = _comps(x), _comps(b)
        rc = load().tn_solver_solve(self._h, _ptrs(cx), _ptrs(cb), _stream(stream))
        if rc == -7:
            return False
        _check(rc)
        return True

    def result(self):
        it, rr, cv = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        _check(load().tn_solver_result(self._h, ctypes.byref(it), ctypes.byref(rr), ctypes.byref(cv)))
        return it.value, rr.value, bool(cv.value)

    def full_residual(self):
        out = ctypes.c_double()
        _check(load().tn_solver_full_residual(self._h, ctypes.byref(out)))
        return out.value

    def history(self):
        n = ctypes.c_int()
        _check(load().tn_solver_history(self._h, None, 0, ctypes.byref(n)))
        buf = (ctypes.c_double * max(n.value, 1))()
        _check(load().tn_solver_history(self._h, buf, n.value, ctypes.byref(n)))
        return list(buf[: n.value])

    def precondition(self, v, z, stream=None):
        _check(load().tn_solver_precondition(self._h, _ptrs(_comps(v)), _ptrs(_comps(z)), _stream(stream)))
        return z

    def vcycle(self, x, b, stream=None):
        cx, cb = _comps(x), _comps(b)
        _check(load().tn_solver_vcycle(self._h, _prec(cx[0].dtype), _ptrs(cx), _ptrs(cb), _stream(stream)))
        return x

    def level_lambda(self, level):
        out = ctypes.c_double()
        _check(load().tn_solver_level_lambda(self._h, level, ctypes.byref(out)))
        return out.value

    def inverse_diagonal(self, level):
        import torch

        nl, nr = self.shell.dims(level)
        out = torch.zeros((3, 10, nl, nl, nr), dtype=torch.float64, device="cuda")
        _check(load().tn_solver_inverse_diagonal(self._h, level, _ptrs([out[c] for c in range(3)]), _stream(None)))
        return out

    def coarse_stats(self):
        out = (ctypes.c_double * 3)()
        _check(load().tn_solver_coarse_stats(self._h, out))
        return list(out)

    def level_matrices(self, level):
        import numpy as np

        nl, nr = self.shell.dims(level)
        out = np.zeros((10, nl - 1, nl - 1, nr - 1, 2, 18, 18))
        _check(load().tn_solver_level_matrices(self._h, level, out.ctypes.data))
        return out

    def level_storage(self, level):
        """(cells with stored matrices, device bytes of the stored matrices) of hierarchy level `level`."""
        n, b = ctypes.c_int64(), ctypes.c_int64()
        _check(load().tn_solver_level_storage(self._h, level, ctypes.byref(n), ctypes.byref(b)))
        return n.value, b.value


def _opt_ptr(eta):
    return None if eta is None else ctypes.c_void_p(eta.data_ptr())


class StokesSolver(_Solver):
    """FGMRES + block-triangular GMG preconditioner (tn_stokes_solver_create).
    Vectors are 4 components (u_x, u_y, u_z on `level`, p on `level - 1`)."""

    def __init__(self, shell: Shell, level: int = -1, eta=None, eta_cell=None, k_schur=None, bc_cmb=DIRICHLET,
                 bc_surface=FREESLIP, stream=None, **options):
        self.shell, self.level = shell, level % shell.num_levels
        self.options = solver_options(**options)
        h = ctypes.c_void_p()
        _check(load().tn_stokes_solver_create(shell.handle, self.level, _opt_ptr(eta), _opt_ptr(eta_cell),
                                              _opt_ptr(k_schur), bc_cmb, bc_surface, ctypes.byref(self.options),
                                              _stream(stream), ctypes.byref(h)))
        self._h = h

    def misfit_gradient(self, x, u_obs, grad_cell, lam=None, stream=None):
        """dJ/dlog(eta_cell), J = 1/2 sum_owned |u - u_obs|^2 at the forward solution x (tn_stokes_misfit_gradient).
        Returns whether the adjoint solve converged."""
        lp = None if lam is None else _ptrs(_comps(lam))
        rc = load().tn_stokes_misfit_gradient(self._h, _ptrs(_comps(x)), _ptrs(_comps(u_obs)),
                                              ctypes.c_void_p(grad_cell.data_ptr()), lp, _stream(stream))
        if rc == -7:
            return False
        _check(rc)
        return True


class VelocitySolver(_Solver):
    """CG on the epsilon-div-div operator with the GMG preconditioner (tn_velocity_solver_create)."""

    def __init__(self, shell: Shell, level: int = -1, eta=None, eta_cell=None, bc_cmb=DIRICHLET,
                 bc_surface=DIRICHLET, stream=None, **options):
        self.shell, self.level = shell, level % shell.num_levels
        self.options = solver_options(**options)
        h = ctypes.c_void_p()
        _check(load().tn_velocity_solver_create(shell.handle, self.level, _opt_ptr(eta), _opt_ptr(eta_cell), bc_cmb,
                                                bc_surface, ctypes.byref(self.options), _stream(stream),
                                                ctypes.byref(h)))
        self._h = h


class MultigridSolver(VelocitySolver):
    """The velocity multigrid used as the solver (tn_multigrid_solver_create): repeated V-cycles."""

    def __init__(self, shell: Shell, level: int = -1, eta=None, eta_cell=None, bc_cmb=DIRICHLET,
                 bc_surface=DIRICHLET, stream=None, **options):
        self.shell, self.level = shell, level % shell.num_levels
        self.options = solver_options(**options)
        h = ctypes.c_void_p()
        _check(load().tn_multigrid_solver_create(shell.handle, self.level, _opt_ptr(eta), _opt_ptr(eta_cell), bc_cmb,
                                                 bc_surface, ctypes.byref(self.options), _stream(stream),
                                                 ctypes.byref(h)))
        self._h = h


class XdmfWriter:
    """XDMF output / checkpoint of one shell level in the reference's file format (tn_xdmf_*). Fields are added
    before the first write; every write() stores their current values as a new step."""

    def __init__(self, shell: Shell, level: int, directory: str, geometry_bytes: int = 4):
        self.shell, self.level = shell, level % shell.num_levels
        self._keep = []
        h = ctypes.c_void_p()
        _check(load().tn_xdmf_create(shell.handle, self.level, directory.encode(), geometry_bytes, ctypes.byref(h)))
        self._h = h

    def add(self, name: str, field, output_bytes: int = 4):
        cs = _comps(field)
        self._keep.append(cs)
        _check(load().tn_xdmf_add(self._h, name.encode(), _prec(cs[0].dtype), len(cs), _ptrs(cs), output_bytes))

    def write(self, stream=None):
        _check(load().tn_xdmf_write(self._h, _stream(stream)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tn_xdmf_destroy(self._h)
            self._h = None


def xdmf_read(shell: Shell, level: int, directory: str, name: str, step: int, out):
    """Restore field `name` of `step` from an XDMF checkpoint directory into `out` (tn_xdmf_read)."""
    cs = _comps(out)
    _check(load().tn_xdmf_read(shell.handle, level % shell.num_levels, directory.encode(), name.encode(), step,
                               _prec(cs[0].dtype), len(cs), _ptrs(cs)))
    return out
