"""CPU oracle for the TERRA-NG Stokes hot path -- TEST INFRASTRUCTURE ONLY.

Python bindings to ``tn_oracle.c`` plus numpy restatements of the reference's
solvers. Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg import this module; the product never does.

Vector shapes: velocity ``(3, 10, nl, nl, nr)``, scalar ``(10, nl, nl, nr)``,
cell fields ``(10, nl-1, nl-1, nr-1)``, all float64, r fastest.

Reference citations are paths inside the reference project (src/terra/...).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtn_oracle.so")
_lib = None

NEUMANN, DIRICHLET, FREESLIP = 0, 1, 2


def build():
    """Compile the oracle library (make, gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        dpp = ctypes.POINTER(dp)
        L.tno_unit_sphere_coords.argtypes = [ctypes.c_int, dp]
        L.tno_uniform_radii.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, dp]
        L.tno_duplicate_classes.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int32)]
        L.tno_ownership.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_uint8)]
        L.tno_boundary_mask.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint8)]
        for name in ("tno_epsdivdiv_slow", "tno_epsdivdiv_fast"):
            getattr(L, name).argtypes = [ctypes.c_void_p, dpp, dpp]
        L.tno_epsdivdiv_local_matrix.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 5 + [dp]
        L.tno_epsdivdiv_stored.argtypes = [ctypes.c_void_p, dp, dpp, dpp]
        L.tno_divergence.argtypes = [ctypes.c_void_p, dpp, dp]
        L.tno_gradient.argtypes = [ctypes.c_void_p, dp, dpp]
        L.tno_kmass_lumped.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp, dp]
        L.tno_vector_mass.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dpp, dpp]
        L.tno_interface_sum.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dpp]
        L.tno_prolongate_add.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dpp, dpp]
        L.tno_restrict.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dpp, dpp]
        L.tno_gca_coarsen.argtypes = [ctypes.c_void_p, dp, dp]
        L.tno_gca_coarsen_w.argtypes = [ctypes.c_void_p, dp, dp, dp]
        L.tno_masked_dot.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dpp, dpp]
        L.tno_masked_dot.restype = ctypes.c_double
        L.tno_epsdivdiv_vjp_logeta.argtypes = [ctypes.c_void_p, dpp, dpp, dp]
        L.tno_set_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return lib().tno_set_threads(int(n))


def _dp(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _dpp(arrs):
    ptrs = (ctypes.POINTER(ctypes.c_double) * len(arrs))(*[_dp(a) for a in arrs])
    return ptrs


class _OpStruct(ctypes.Structure):
    _fields_ = [
        ("nl", ctypes.c_int),
        ("nr", ctypes.c_int),
        ("coords", ctypes.c_void_p),
        ("radii", ctypes.c_void_p),
        ("k", ctypes.c_void_p),
        ("k_q0", ctypes.c_void_p),
        ("bc_cmb", ctypes.c_int),
        ("bc_surface", ctypes.c_int),
        ("diagonal", ctypes.c_int),
    ]


# --------------------------------------------------------------------------
# Mesh
# --------------------------------------------------------------------------
class Shell:
    """One level of the thick spherical shell (grid/shell/spherical_shell.hpp)."""

    def __init__(self, lat_level: int, rad_level: int | None = None, r_min=0.55, r_max=1.0):
        if rad_level is None:
            rad_level = lat_level
        self.lat_level, self.rad_level = lat_level, rad_level
        self.nl = (1 << lat_level) + 1
        self.nr = (1 << rad_level) + 1
        self.r_min, self.r_max = float(r_min), float(r_max)
        L = lib()
        self.coords = np.zeros((10, self.nl, self.nl, 3))
        L.tno_unit_sphere_coords(lat_level, _dp(self.coords))
        self.radii = np.zeros(self.nr)
        L.tno_uniform_radii(self.r_min, self.r_max, self.nr, _dp(self.radii))
        self.classes = np.zeros((10, self.nl, self.nl), np.int32)
        self.num_classes = L.tno_duplicate_classes(lat_level, self.classes.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        self.owned_lat = np.zeros((10, self.nl, self.nl), np.uint8)
        L.tno_ownership(lat_level, self.owned_lat.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        self.boundary_mask = np.zeros((10, self.nl, self.nl, self.nr), np.uint8)
        L.tno_boundary_mask(self.nl, self.nr, self.boundary_mask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        self.owned = np.broadcast_to(self.owned_lat[..., None], (10, self.nl, self.nl, self.nr)).astype(bool)

    @property
    def scalar_shape(self):
        return (10, self.nl, self.nl, self.nr)

    @property
    def vec_shape(self):
        return (3, 10, self.nl, self.nl, self.nr)

    @property
    def cell_shape(self):
        return (10, self.nl - 1, self.nl - 1, self.nr - 1)

    def coarser(self) -> "Shell":
        return Shell(self.lat_level - 1, self.rad_level - 1, self.r_min, self.r_max)

    def physical_coords(self):
        """(10, nl, nl, nr, 3) node positions."""
        return self.coords[:, :, :, None, :] * self.radii[None, None, None, :, None]

    def interface_sum(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        comps = [v] if v.ndim == 4 else [v[i] for i in range(v.shape[0])]
        comps = [np.ascontiguousarray(c) for c in comps]
        lib().tno_interface_sum(self.lat_level, self.nr, len(comps), _dpp(comps))
        return comps[0] if v.ndim == 4 else np.stack(comps)

    def dot(self, a, b):
        """Owned-masked dot (kernels/common/grid_operations.hpp:630-673)."""
        m = self.owned
        if a.ndim == 4:
            return float(np.sum(a[m] * b[m]))
        return float(sum(np.sum(a[i][m] * b[i][m]) for i in range(a.shape[0])))


# --------------------------------------------------------------------------
# Operators
# --------------------------------------------------------------------------
class EpsDivDiv:
    """epsilon-div-div operator (epsilon_divdiv_kerngen.hpp), Replace mode,
    interface sum included unless comm=False."""

    def __init__(self, shell: Shell, k=None, k_q0=None, bc_cmb=DIRICHLET, bc_surface=DIRICHLET, diagonal=False,
                 stored=None):
        self.shell = shell
        self.k = None if k is None else np.ascontiguousarray(k, np.float64)
        self.k_q0 = None if k_q0 is None else np.ascontiguousarray(k_q0, np.float64)
        if self.k is None and self.k_q0 is None:
            raise ValueError("need k or k_q0")
        self.bc_cmb, self.bc_surface = bc_cmb, bc_surface
        self.diagonal = bool(diagonal)
        self.stored = None if stored is None else np.ascontiguousarray(stored, np.float64)

    def _struct(self, diagonal=None):
        s = _OpStruct()
        s.nl, s.nr = self.shell.nl, self.shell.nr
        s.coords = self.shell.coords.ctypes.data
        s.radii = self.shell.radii.ctypes.data
        s.k = None if self.k is None else self.k.ctypes.data
        s.k_q0 = None if self.k_q0 is None else self.k_q0.ctypes.data
        s.bc_cmb, s.bc_surface = self.bc_cmb, self.bc_surface
        s.diagonal = int(self.diagonal if diagonal is None else diagonal)
        return s

    def apply(self, src, path="fast", comm=True, diagonal=None):
        src = [np.ascontiguousarray(src[i], np.float64) for i in range(3)]
        dst = [np.zeros(self.shell.scalar_shape) for _ in range(3)]
        s = self._struct(diagonal)
        if self.stored is not None:
            lib().tno_epsdivdiv_stored(ctypes.byref(s), _dp(self.stored), _dpp(src), _dpp(dst))
        elif path == "slow":
            lib().tno_epsdivdiv_slow(ctypes.byref(s), _dpp(src), _dpp(dst))
        else:
            lib().tno_epsdivdiv_fast(ctypes.byref(s), _dpp(src), _dpp(dst))
        if self.bc_cmb == FREESLIP and self.bc_surface == FREESLIP and not s.diagonal:
            # added to every copy before the interface sum, as the reference does (:711-785)
            modes = null_space_modes(self.shell)
            alpha = [PENALTY_EPSILON * self.shell.dot(m, np.stack(src)) for m in modes]
            for c in range(3):
                dst[c] += alpha[0] * modes[0][c] + alpha[1] * modes[1][c] + alpha[2] * modes[2][c]
        if comm:
            lib().tno_interface_sum(self.shell.lat_level, self.shell.nr, 3, _dpp(dst))
        return np.stack(dst)

    def diag(self):
        """diag(A) via diagonal mode applied to ones (stokes_solver.hpp:390-417)."""
        return self.apply(np.ones(self.shell.vec_shape), diagonal=True, path="slow" if self.stored is None else "fast")

    def local_matrix(self, d, x, y, r, w):
        A = np.zeros(324)
        s = self._struct(False)
        lib().tno_epsdivdiv_local_matrix(ctypes.byref(s), d, x, y, r, w, _dp(A))
        return A.reshape(18, 18)

    def vjp_logeta(self, u, lam):
        """cell gradient of lambda^T A u with respect to log(eta_cell) (Q0 only)."""
        g = np.zeros(self.shell.cell_shape)
        s = self._struct(False)
        uu = [np.ascontiguousarray(u[i]) for i in range(3)]
        ll = [np.ascontiguousarray(lam[i]) for i in range(3)]
        rc = lib().tno_epsdivdiv_vjp_logeta(ctypes.byref(s), _dpp(uu), _dpp(ll), _dp(g))
        if rc != 0:
            raise ValueError("vjp needs a per-cell (Q0) coefficient")
        return g


PENALTY_EPSILON = 1e-7  # epsilon_divdiv_kerngen.hpp:168
_MODES_CACHE: dict = {}


def null_space_modes(shell: Shell):
    """Orthonormal rotation modes of the free-slip/free-slip shell (epsilon_divdiv_kerngen.hpp:324-445):
    e_i x X for the three axes, then modified Gram-Schmidt with owned-node dots. The reference also runs a
    free-slip pass over the modes, but on nodes flagged CMB | SURFACE together, which no node is, so it leaves
    them unchanged (the rotation modes are tangential on every sphere anyway)."""
    key = (shell.lat_level, shell.rad_level, shell.r_min, shell.r_max)
    if key in _MODES_CACHE:
        return _MODES_CACHE[key]
    X = shell.physical_coords()
    modes = []
    for axis in range(3):
        a1, a2 = (axis + 1) % 3, (axis + 2) % 3
        m = np.zeros(shell.vec_shape)
        m[a1] = X[..., a2]
        m[a2] = -X[..., a1]
        modes.append(m)
    for i in range(3):
        for j in range(i):
            modes[i] = modes[i] - shell.dot(modes[i], modes[j]) * modes[j]
        modes[i] = modes[i] * (1.0 / math.sqrt(shell.dot(modes[i], modes[i])))
    _MODES_CACHE[key] = modes
    return modes


def gca_coarsen(fine_op: EpsDivDiv, fine_mats=None, linear=False):
    """Two-grid GCA (gca.hpp) of a Neumann fine operator or stored fine matrices; InterpolationMode::Linear
    (the linear-transfer weights of the fine level) when linear, else Constant."""
    sh = fine_op.shell
    nlc, nrc = (sh.nl + 1) // 2, (sh.nr + 1) // 2
    out = np.zeros((10, nlc - 1, nlc - 1, nrc - 1, 2, 18, 18))
    s = fine_op._struct(False)
    fm = None if fine_mats is None else _dp(np.ascontiguousarray(fine_mats))
    lw = _dp(np.ascontiguousarray(linear_weights(sh))) if linear else None
    lib().tno_gca_coarsen_w(ctypes.byref(s), fm, lw, _dp(out))
    return out


def _linear_parents(x, y, r, nrf):
    """Coarse parents of a fine node for the linear transfers (prolongation_linear.hpp operator())."""
    if x % 2 == 0 and y % 2 == 0 and r % 2 == 0:
        return 0, (x // 2, y // 2), (x // 2, y // 2), r // 2, r // 2
    rb = r // 2 if r < nrf - 1 else r // 2 - 1
    if x % 2 == 0 and y % 2 == 0:
        return 1, (x // 2, y // 2), (x // 2, y // 2), rb, rb + 1
    if x % 2 == 0:
        return 2, (x // 2, y // 2), (x // 2, y // 2 + 1), rb, rb + 1
    if y % 2 == 0:
        return 2, (x // 2, y // 2), (x // 2 + 1, y // 2), rb, rb + 1
    return 2, (x // 2 + 1, y // 2), (x // 2, y // 2 + 1), rb, rb + 1


_LINW_CACHE: dict = {}


def linear_weights(fine: Shell):
    """(10, nl, nl, nr, 2) weights of prolongation_linear_weights (grid_transfer_linear.hpp:13-157) per fine
    node: (1 - nu, nu) for radially aligned nodes, (0.5 (1 - nu), 0.5 nu) for nodes on a facet, nu measured
    along the radius from the (chord midpoint of the) bottom coarse pair to the top pair; (1, 0) on coarse
    nodes."""
    key = (fine.lat_level, fine.rad_level, fine.r_min, fine.r_max)
    if key in _LINW_CACHE:
        return _LINW_CACHE[key]
    nl, nr = fine.nl, fine.nr
    w = np.zeros((10, nl, nl, nr, 2))
    w[..., 0] = 1.0
    C, R = fine.coords, fine.radii
    for d in range(10):
        for x in range(nl):
            for y in range(nl):
                for r in range(nr):
                    kind, p0, p1, rb, rt = _linear_parents(x, y, r, nr)
                    if kind == 0:
                        continue
                    nf = np.linalg.norm(C[d, x, y] * R[r])
                    if kind == 1:
                        nb = np.linalg.norm(C[d, x, y] * R[2 * rb])
                        nt = np.linalg.norm(C[d, x, y] * R[2 * rt])
                    else:
                        u0, u1 = C[d, 2 * p0[0], 2 * p0[1]], C[d, 2 * p1[0], 2 * p1[1]]
                        nb = np.linalg.norm(0.5 * (u0 * R[2 * rb] + u1 * R[2 * rb]))
                        nt = np.linalg.norm(0.5 * (u0 * R[2 * rt] + u1 * R[2 * rt]))
                    nu = (nf - nb) / (nt - nb)
                    w[d, x, y, r] = (1.0 - nu, nu) if kind == 1 else (0.5 * (1.0 - nu), 0.5 * nu)
    _LINW_CACHE[key] = w
    return w


def prolongate_linear_add(fine: Shell, coarse_v, fine_v):
    """fine_v += P coarse_v with the linear prolongation per component (ProlongationLinear)."""
    w = linear_weights(fine)
    nr = fine.nr
    out = np.array(fine_v, dtype=np.float64, copy=True)
    for d in range(10):
        for x in range(fine.nl):
            for y in range(fine.nl):
                for r in range(nr):
                    kind, p0, p1, rb, rt = _linear_parents(x, y, r, nr)
                    for c in range(coarse_v.shape[0]):
                        cv = coarse_v[c, d]
                        if kind == 0:
                            v = cv[p0[0], p0[1], rb]
                        elif kind == 1:
                            v = w[d, x, y, r, 0] * cv[p0[0], p0[1], rb] + w[d, x, y, r, 1] * cv[p0[0], p0[1], rt]
                        else:
                            v = (w[d, x, y, r, 0] * (cv[p0[0], p0[1], rb] + cv[p1[0], p1[1], rb]) +
                                 w[d, x, y, r, 1] * (cv[p0[0], p0[1], rt] + cv[p1[0], p1[1], rt]))
                        out[c, d, x, y, r] += v
    return out


def restrict_linear(fine: Shell, fine_v):
    """P^T over owned fine nodes, then the coarse interface sum (RestrictionLinear per component)."""
    w = linear_weights(fine)
    coarse = fine.coarser()
    nr = fine.nr
    out = np.zeros((fine_v.shape[0],) + coarse.scalar_shape)
    for d in range(10):
        for x in range(fine.nl):
            for y in range(fine.nl):
                if not fine.owned_lat[d, x, y]:
                    continue
                for r in range(nr):
                    kind, p0, p1, rb, rt = _linear_parents(x, y, r, nr)
                    for c in range(fine_v.shape[0]):
                        f = fine_v[c, d, x, y, r]
                        if kind == 0:
                            out[c, d, p0[0], p0[1], rb] += f
                        elif kind == 1:
                            out[c, d, p0[0], p0[1], rb] += w[d, x, y, r, 0] * f
                            out[c, d, p0[0], p0[1], rt] += w[d, x, y, r, 1] * f
                        else:
                            for p in (p0, p1):
                                out[c, d, p[0], p[1], rb] += w[d, x, y, r, 0] * f
                                out[c, d, p[0], p[1], rt] += w[d, x, y, r, 1] * f
    return coarse.interface_sum(out)


class Divergence:
    """B: velocity (level L) -> pressure (level L-1) (divergence_kerngen.hpp)."""

    def __init__(self, shell: Shell, bc_cmb=DIRICHLET, bc_surface=DIRICHLET):
        self.shell, self.bc_cmb, self.bc_surface = shell, bc_cmb, bc_surface
        self.coarse = shell.coarser()

    def _struct(self):
        s = _OpStruct()
        s.nl, s.nr = self.shell.nl, self.shell.nr
        s.coords = self.shell.coords.ctypes.data
        s.radii = self.shell.radii.ctypes.data
        s.bc_cmb, s.bc_surface = self.bc_cmb, self.bc_surface
        return s

    def apply(self, u, comm=True):
        uu = [np.ascontiguousarray(u[i], np.float64) for i in range(3)]
        p = np.zeros(self.coarse.scalar_shape)
        s = self._struct()
        lib().tno_divergence(ctypes.byref(s), _dpp(uu), _dp(p))
        if comm:
            p = self.coarse.interface_sum(p)
        return p

    def apply_transpose(self, p, comm=True):
        p = np.ascontiguousarray(p, np.float64)
        dst = [np.zeros(self.shell.scalar_shape) for _ in range(3)]
        s = self._struct()
        lib().tno_gradient(ctypes.byref(s), _dp(p), _dpp(dst))
        if comm:
            lib().tno_interface_sum(self.shell.lat_level, self.shell.nr, 3, _dpp(dst))
        return np.stack(dst)


def kmass_lumped(shell: Shell, k):
    d = np.zeros(shell.scalar_shape)
    k = np.ascontiguousarray(k, np.float64)
    lib().tno_kmass_lumped(shell.nl, shell.nr, _dp(shell.coords), _dp(shell.radii), _dp(k), _dp(d))
    return shell.interface_sum(d)


def vector_mass(shell: Shell, v):
    vv = [np.ascontiguousarray(v[i], np.float64) for i in range(3)]
    dst = [np.zeros(shell.scalar_shape) for _ in range(3)]
    lib().tno_vector_mass(shell.nl, shell.nr, _dp(shell.coords), _dp(shell.radii), _dpp(vv), _dpp(dst))
    lib().tno_interface_sum(shell.lat_level, shell.nr, 3, _dpp(dst))
    return np.stack(dst)


def prolongate_add(fine: Shell, coarse_v, fine_v):
    """fine_v += P coarse_v (in place), any number of components."""
    cv = [np.ascontiguousarray(coarse_v[i]) for i in range(coarse_v.shape[0])]
    fv = [np.ascontiguousarray(fine_v[i]) for i in range(fine_v.shape[0])]
    lib().tno_prolongate_add(fine.lat_level, fine.rad_level, len(cv), _dpp(cv), _dpp(fv))
    fine_v[...] = np.stack(fv)
    return fine_v


def restrict(fine: Shell, fine_v):
    coarse = fine.coarser()
    fv = [np.ascontiguousarray(fine_v[i]) for i in range(fine_v.shape[0])]
    cv = [np.zeros(coarse.scalar_shape) for _ in range(len(fv))]
    lib().tno_restrict(fine.lat_level, fine.rad_level, len(fv), _dpp(fv), _dpp(cv))
    return np.stack(cv)


# --------------------------------------------------------------------------
# Boundary-condition helpers for right-hand sides
# --------------------------------------------------------------------------
def trafo_nt(n):
    """Rows (n, t1, t2) (local_basis_trafo_normal_tangential.hpp:34-76)."""
    n = np.asarray(n, np.float64)
    nn = n / np.linalg.norm(n)
    a = np.abs(nn)
    if a[0] <= a[1] and a[0] <= a[2]:
        ref = np.array([1.0, 0, 0])
    elif a[1] <= a[0] and a[1] <= a[2]:
        ref = np.array([0, 1.0, 0])
    else:
        ref = np.array([0, 0, 1.0])
    t1 = np.cross(ref, nn)
    t1 /= np.linalg.norm(t1)
    t2 = np.cross(nn, t1)
    t2 /= np.linalg.norm(t2)
    return np.stack([nn, t1, t2])


def enforce_rhs_bcs(shell: Shell, f, bc_cmb, bc_surface):
    """Zero Dirichlet rows and the normal component on free-slip boundaries
    (strong_algebraic_dirichlet_enforcement.hpp:114-123,
    strong_algebraic_freeslip_enforcement.hpp:22-38)."""
    f = f.copy()
    for r, bc in ((0, bc_cmb), (shell.nr - 1, bc_surface)):
        if bc == DIRICHLET:
            f[:, :, :, :, r] = 0.0
        elif bc == FREESLIP:
            n = shell.coords  # radial direction
            un = np.einsum("cdxy,dxyc->dxy", f[:, :, :, :, r], n) / np.sum(n * n, axis=-1)
            f[:, :, :, :, r] -= np.moveaxis(un[..., None] * n, -1, 0)
    return f


INNER_FLAG, BOUNDARY_FLAG, CMB_FLAG, SURFACE_FLAG = 1, 2, 6, 10  # grid/shell/bit_masks.hpp:11-19


def has_flag(mask, flag):
    """util/bit_masking.hpp:43-53: all bits of flag set; NO_FLAG matches only unflagged nodes."""
    mask = np.asarray(mask)
    if flag == 0:
        return mask == 0
    return (mask & flag) == flag


def shell_boundary_flag(bc_cmb, bc_surface, bcf):
    """get_shell_boundary_flag (grid/shell/bit_masks.hpp:68-77): the FIRST boundary carrying condition bcf
    (CMB before SURFACE), or NO_FLAG."""
    for sbf, bc in ((CMB_FLAG, bc_cmb), (SURFACE_FLAG, bc_surface)):
        if bc == bcf:
            return sbf
    return 0


def assign_masked(shell: Shell, f, flag, value=0.0):
    """assign_masked_else_keep_old on every component (kernels/common/grid_operations.hpp:54-101)."""
    f = np.array(f, dtype=np.float64, copy=True)
    m = has_flag(shell.boundary_mask, flag)
    f[:, m] = value
    return f


def freeslip_project(shell: Shell, f, flag):
    """strong_algebraic_freeslip_enforcement_in_place (strong_algebraic_freeslip_enforcement.hpp:22-38): at
    nodes carrying flag, rotate to (n, t1, t2), zero the normal part, rotate back."""
    f = np.array(f, dtype=np.float64, copy=True)
    idx = np.argwhere(has_flag(shell.boundary_mask, flag))
    for d, x, y, r in idx:
        Rm = trafo_nt(shell.coords[d, x, y])
        nt = Rm @ f[:, d, x, y, r]
        nt[0] = 0.0
        f[:, d, x, y, r] = Rm.T @ nt
    return f


def rhs_enforce_app(shell: Shell, f, bc_cmb, bc_surface):
    """The application's right-hand-side treatment (stokes_solver.hpp:662-671): zero the velocity on the
    boundary get_shell_boundary_flag returns for DIRICHLET, then remove the normal component on the one it
    returns for FREESLIP. With Dirichlet on both boundaries only the CMB is zeroed (the lookup stops at the
    first match)."""
    f = assign_masked(shell, f, shell_boundary_flag(bc_cmb, bc_surface, DIRICHLET))
    return freeslip_project(shell, f, shell_boundary_flag(bc_cmb, bc_surface, FREESLIP))


# --------------------------------------------------------------------------
# Solvers (numpy restatements of linalg/solvers/*.hpp)
# --------------------------------------------------------------------------
def power_iteration(apply_scaled, start, dot, iterations):
    """power_iteration.hpp:15-57 with a caller-provided start vector."""
    it = start.copy()
    norm = math.sqrt(dot(it, it))
    if norm < np.finfo(np.float64).tiny:
        return 1.0
    it = it / norm
    aux = apply_scaled(it)
    radius = 0.0
    for _ in range(iterations):
        norm = math.sqrt(dot(aux, aux))
        if norm < np.finfo(np.float64).tiny:
            return radius if radius > 0.0 else 1.0
        it = aux / norm
        aux = apply_scaled(it)
        radius = dot(it, aux)
    return radius


@dataclass
class Chebyshev:
    """Chebyshev-Jacobi smoother (chebyshev.hpp:102-176)."""

    order: int
    inv_diag: np.ndarray
    iterations: int = 1
    lambda_max_est: float | None = None

    def solve(self, A, x, b):
        ev = self.lambda_max_est
        if ev is None or not np.isfinite(ev) or ev <= 0:
            ev = 1.0
        lmax, lmin = 1.5 * ev, 0.1 * ev
        theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
        sigma = theta / delta
        rho = 1.0 / sigma
        d = None
        for _ in range(self.iterations):
            z = (b - A(x)) * self.inv_diag
            d = z / theta
            x = x + d
            for _i in range(2, self.order + 1):
                rho_new = 1.0 / (2.0 * sigma - rho)
                beta = rho_new * rho
                alpha = 2.0 * rho_new / delta
                z = (b - A(x)) * self.inv_diag
                d = alpha * z + beta * d
                x = x + d
                rho = rho_new
        return x


@dataclass
class Jacobi:
    """Damped Jacobi smoother (jacobi.hpp:51-60): x += omega D^-1 (b - A x),
    `iterations` times."""

    inv_diag: np.ndarray
    iterations: int = 1
    omega: float = 1.0

    def solve(self, A, x, b):
        for _ in range(self.iterations):
            x = x + self.omega * ((b - A(x)) * self.inv_diag)
        return x


def pcg(A, x, b, dot, max_iter, rtol, atol=1e-16, precond=None, history=None):
    """pcg.hpp:81-169. ``precond(z, r)`` returns the new z; like the
    reference's solve(preconditioner_, A, z_, r_) it receives the previous z
    (zeros at the start), which only matters for preconditioners that use it
    as an initial guess (multigrid)."""
    r = b - A(x)
    z = np.zeros_like(r)
    z = r.copy() if precond is None else precond(z, r)
    p = z.copy()
    init = math.sqrt(dot(r, r))
    if history is not None:
        history.append(1.0)
    if init < atol:
        return x
    for it in range(1, max_iter + 1):
        an = dot(z, r)
        ap = A(p)
        ad = dot(ap, p)
        if abs(ad) < np.finfo(np.float64).tiny:
            return x
        alpha = an / ad
        x = x + alpha * p
        r = r - alpha * ap
        res = math.sqrt(dot(r, r))
        if history is not None:
            history.append(res / init)
        if res / init <= rtol or res < atol:
            return x
        z = r.copy() if precond is None else precond(z, r)
        bn = dot(z, r)
        if abs(an) < np.finfo(np.float64).tiny:
            return x
        p = z + (bn / an) * p
    return x


class Multigrid:
    """V-cycle (multigrid.hpp:216-432); levels[0] is the coarsest. transfer: "constant" (the application's
    ProlongationVecConstant / RestrictionVecConstant) or "linear" (ProlongationLinear / RestrictionLinear per
    component)."""

    def __init__(self, ops, shells, smoothers, coarse_solve, num_cycles=1, transfer="constant"):
        self.ops, self.shells, self.smoothers = ops, shells, smoothers
        self.coarse_solve, self.num_cycles = coarse_solve, num_cycles
        self.transfer = transfer

    def _rec(self, level, x, b):
        if level == 0:
            return self.coarse_solve(self.ops[0], x, b)
        A = self.ops[level]
        x = self.smoothers[level].solve(A, x, b)
        res = b - A(x)
        lin = self.transfer == "linear"
        rc = restrict_linear(self.shells[level], res) if lin else restrict(self.shells[level], res)
        ec = np.zeros_like(rc)
        ec = self._rec(level - 1, ec, rc)
        if lin:
            x = prolongate_linear_add(self.shells[level], ec, x)
        else:
            prolongate_add(self.shells[level], ec, x)
        x = self.smoothers[level].solve(A, x, b)
        return x

    def solve(self, x, b):
        for _ in range(self.num_cycles):
            x = self._rec(len(self.ops) - 1, x, b)
        return x


def fgmres(A, x, b, dot, precond, restart, rtol, atol, max_iter, history=None):
    """fgmres.hpp:109-373 (modified Gram-Schmidt, Givens rotations)."""
    eps = np.finfo(np.float64).eps
    r = b - A(x)
    beta0 = math.sqrt(dot(r, r))
    init = beta0
    if history is not None:
        history.append(1.0)
    if beta0 <= atol:
        return x, 0
    total = 0
    m = restart
    while total < max_iter:
        V = [r / beta0]
        Z = []
        H = np.zeros((m + 1, m))
        g = np.zeros(m + 1)
        cs = np.zeros(m + 1)
        sn = np.zeros(m + 1)
        g[0] = beta0
        inner = 0
        j = 0
        while j < m and total < max_iter:
            # each step counts toward max_iter when it starts, so a cycle that
            # ends early (tolerance met by the estimate only, breakdown) still
            # lets the loop end (the product's FGMRES counts the same way)
            total += 1
            z = precond(V[j])
            if not np.all(np.isfinite(z)):
                z = V[j].copy()
            Z.append(z)
            w = A(z)
            for i in range(j + 1):
                hij = dot(w, V[i])
                H[i, j] = hij
                w = w - hij * V[i]
            h = math.sqrt(dot(w, w))
            if h < eps * init:
                H[j + 1, j] = 0
                inner = j + 1
                break
            H[j + 1, j] = h
            V.append(w / h)
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            a, bb = H[j, j], H[j + 1, j]
            rab = math.hypot(a, bb)
            cs[j] = 1.0 if rab == 0 else a / rab
            sn[j] = 0.0 if rab == 0 else bb / rab
            H[j, j] = rab
            H[j + 1, j] = 0
            if abs(H[j, j]) < eps:
                inner = j
                break
            gj, gj1 = g[j], g[j + 1]
            g[j] = cs[j] * gj + sn[j] * gj1
            g[j + 1] = -sn[j] * gj + cs[j] * gj1
            abs_res = abs(g[j + 1])
            if history is not None:
                history.append(abs_res / init)
            if not np.isfinite(abs_res):
                inner = j
                break
            inner = j + 1
            if abs_res / init <= rtol or abs_res < atol:
                break
            j += 1
        y = np.zeros(inner)
        for row in range(inner - 1, -1, -1):
            s = g[row] - sum(H[row, c] * y[c] for c in range(row + 1, inner))
            y[row] = s / H[row, row]
        for i in range(inner):
            x = x + y[i] * Z[i]
        r = b - A(x)
        beta0 = math.sqrt(dot(r, r))
        if not np.isfinite(beta0):
            return x, total
        if beta0 <= atol or beta0 / init <= rtol:
            return x, total
    return x, total


# --------------------------------------------------------------------------
# Seeded synthetic inputs (shared definition with the product's generators is
# NOT assumed: tests create inputs here and hand them to both sides).
# --------------------------------------------------------------------------
def seeded_normal(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape)


def seeded_uniform(shell: Shell, ncomp: int, seed: int):
    """Uniform(-1, 1) per (seed, canonical node, component) from SplitMix64,
    the canonical node being the lowest lateral index of the node's duplicate
    class times nr plus r (duplicates get equal values)."""
    nl, nr = shell.nl, shell.nr
    nlat = 10 * nl * nl
    canon = np.arange(nlat, dtype=np.int64)
    cls = shell.classes.reshape(-1)
    for k in range(shell.num_classes):
        m = np.where(cls == k)[0]
        canon[m] = m.min()
    u64 = np.uint64
    gid_node = canon[:, None].astype(u64) * u64(nr) + np.arange(nr, dtype=u64)[None, :]
    out = np.empty((ncomp, nlat, nr))
    with np.errstate(over="ignore"):
        for c in range(ncomp):
            gid = gid_node * u64(ncomp) + u64(c)
            z = u64(seed) + (gid + u64(1)) * u64(0x9E3779B97F4A7C15)
            z = (z ^ (z >> u64(30))) * u64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> u64(27))) * u64(0x94D049BB133111EB)
            z = z ^ (z >> u64(31))
            out[c] = 2.0 * ((z >> u64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)) - 1.0
    return out.reshape(ncomp, 10, nl, nl, nr)


def inject(coarse: Shell, fine_field):
    """coarse(d, x, y, r) = fine(d, 2x, 2y, 2r)."""
    return np.ascontiguousarray(fine_field[:, ::2, ::2, ::2])


def gca_marks(fine: Shell, k, level_range):
    """GCAElementsCollector (gca_elements_collector.hpp:49-103): per wedge of every fine cell the gradient of the
    nodal k in reference coordinates at (1/3, 1/3, 0) (grad_shape, integrands.hpp:228-235, summed over the six
    nodes in order with separate roundings); where its norm exceeds 10 the ancestor cell level_range halvings
    coarser (map_to_coarse_element) is marked. Returns a bool array over the coarse cells."""
    k = np.asarray(k, np.float64)
    nl, nr = fine.nl, fine.nr
    nlc, nrc = ((nl - 1) >> level_range) + 1, ((nr - 1) >> level_range) + 1
    marks = np.zeros((10, nlc - 1, nlc - 1, nrc - 1), bool)
    offs = [[(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1)],
            [(1, 1, 0), (0, 1, 0), (1, 0, 0), (1, 1, 1), (0, 1, 1), (1, 0, 1)]]
    third = 1.0 / 3.0
    slat = [1.0 - third - third, third, third]
    gxi, geta = [-1.0, 1.0, 0.0], [-1.0, 0.0, 1.0]
    hit = np.zeros((10, nl - 1, nl - 1, nr - 1), bool)
    for w in range(2):
        g = [np.zeros((10, nl - 1, nl - 1, nr - 1)) for _ in range(3)]
        for n, (ox, oy, orr) in enumerate(offs[w]):
            kn = k[:, ox:ox + nl - 1, oy:oy + nl - 1, orr:orr + nr - 1]
            m, grad = n % 3, (-0.5 if n < 3 else 0.5)
            g[0] = g[0] + (gxi[m] * 0.5) * kn
            g[1] = g[1] + (geta[m] * 0.5) * kn
            g[2] = g[2] + (slat[m] * grad) * kn
        hit |= np.sqrt(((0.0 + g[0] * g[0]) + g[1] * g[1]) + g[2] * g[2]) > 10.0
    d, x, y, r = np.nonzero(hit)
    marks[d, x >> level_range, y >> level_range, r >> level_range] = True
    return marks


def expand_marks(marks, levels):
    """marks of coarse cells -> marks of their descendants `levels` levels finer."""
    m = marks
    for _ in range(levels):
        m = m.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)
    return m


def element_matrices(op: "EpsDivDiv"):
    """get_local_matrix of every cell of an operator without stored matrices: (10, nl-1, nl-1, nr-1, 2, 18, 18)."""
    sh = op.shell
    out = np.zeros(sh.cell_shape + (2, 18, 18))
    for d, x, y, r in np.ndindex(*sh.cell_shape):
        for w in range(2):
            out[d, x, y, r, w] = op.local_matrix(d, x, y, r, w)
    return out


class VelocityHierarchy:
    """Multigrid hierarchy as the product builds it (levels[0] coarsest):
    GCA coarse operators (TwoGridGCA top-down, stokes_solver.hpp:375-389) or
    rediscretised ones (injected nodal coefficient), inverse diagonals from
    the diagonal mode, and Chebyshev smoothers with given lambda_max values."""

    def __init__(self, fine: Shell, k, bc_cmb, bc_surface, num_levels, gca=True, lambdas=None, cheb_order=2,
                 cheb_iters=2, coarse_max_iter=50, coarse_rtol=1e-6, coarse_atol=1e-16, transfer="constant"):
        self.transfer = transfer
        shells = [fine]
        for _ in range(num_levels - 1):
            shells.insert(0, shells[0].coarser())
        self.shells = shells
        ops = [None] * num_levels
        ops[-1] = EpsDivDiv(fine, k=k, bc_cmb=bc_cmb, bc_surface=bc_surface)
        self.mats = [None] * num_levels
        self.marks = None
        if gca == 2:
            # adaptive GCA (stokes_solver.hpp:278-287, :360-366): the Galerkin matrices of the full chain on the
            # cells below marked coarsest cells (their fine children are marked too, so the selective chain
            # reproduces the full one there), the rediscretised operator's element matrices elsewhere
            self.marks = gca_marks(fine, k, num_levels - 1)
            full = VelocityHierarchy(fine, k, bc_cmb, bc_surface, num_levels, gca=1, lambdas=lambdas,
                                     cheb_order=cheb_order, cheb_iters=cheb_iters, coarse_max_iter=coarse_max_iter,
                                     coarse_rtol=coarse_rtol, coarse_atol=coarse_atol, transfer=transfer)
        kk = k
        for l in range(num_levels - 2, -1, -1):
            if gca == 2:
                kk = inject(shells[l], kk)
                ml = expand_marks(self.marks, l)[..., None, None, None]
                rediscretised = element_matrices(EpsDivDiv(shells[l], k=kk, bc_cmb=bc_cmb, bc_surface=bc_surface))
                self.mats[l] = np.where(ml, full.mats[l], rediscretised)
                ops[l] = EpsDivDiv(shells[l], k=kk, bc_cmb=bc_cmb, bc_surface=bc_surface, stored=self.mats[l])
            elif gca:
                lin = transfer == "linear"
                if l == num_levels - 2:
                    src = EpsDivDiv(shells[l + 1], k=k, bc_cmb=NEUMANN, bc_surface=NEUMANN)
                    m = gca_coarsen(src, linear=lin)
                else:
                    src = EpsDivDiv(shells[l + 1], k=np.ones(shells[l + 1].scalar_shape), stored=self.mats[l + 1])
                    m = gca_coarsen(src, fine_mats=self.mats[l + 1], linear=lin)
                self.mats[l] = m
                ops[l] = EpsDivDiv(shells[l], k=np.ones(shells[l].scalar_shape), bc_cmb=bc_cmb, bc_surface=bc_surface,
                                   stored=m)
            else:
                kk = inject(shells[l], kk)
                ops[l] = EpsDivDiv(shells[l], k=kk, bc_cmb=bc_cmb, bc_surface=bc_surface)
        self.ops = ops
        self.inv_diag = [None] + [1.0 / ops[l].diag() for l in range(1, num_levels)]
        self.lambdas = lambdas
        self.cheb_order, self.cheb_iters = cheb_order, cheb_iters
        self.coarse = (coarse_max_iter, coarse_rtol, coarse_atol)

    def apply(self, l, u):
        return self.ops[l].apply(u, path="slow" if self.ops[l].stored is None else "fast")

    def power_iteration(self, l, start, iterations):
        return power_iteration(lambda v: self.apply(l, v) * self.inv_diag[l], start, self.shells[l].dot, iterations)

    def multigrid(self, num_cycles=1, smoother="chebyshev", omega=1.0):
        n = len(self.shells)
        if smoother == "jacobi":
            smoothers = [None] + [Jacobi(self.inv_diag[l], self.cheb_iters, omega) for l in range(1, n)]
        else:
            smoothers = [None] + [Chebyshev(self.cheb_order, self.inv_diag[l], self.cheb_iters, self.lambdas[l])
                                  for l in range(1, n)]
        ops = [(lambda v, l=l: self.apply(l, v)) for l in range(n)]
        it, rtol, atol = self.coarse
        coarse = lambda A, x, b: pcg(A, x, b, self.shells[0].dot, it, rtol, atol)
        return Multigrid(ops, self.shells, smoothers, coarse, num_cycles, transfer=self.transfer)


class StokesSystem:
    """[A B^T; B 0] on flat block vectors (u raveled, then p) with the
    block-triangular preconditioner (block_preconditioner_2x2.hpp:205-221)."""

    def __init__(self, fine: Shell, k, bc_cmb, bc_surface, hierarchy: VelocityHierarchy, k_schur=None):
        self.sh, self.shp = fine, fine.coarser()
        self.A = EpsDivDiv(fine, k=k, bc_cmb=bc_cmb, bc_surface=bc_surface)
        self.B = Divergence(fine, bc_cmb=bc_cmb, bc_surface=bc_surface)
        self.nu = int(np.prod(fine.vec_shape))
        kp = k_schur if k_schur is not None else 1.0 / inject(self.shp, k)
        self.inv_schur = 1.0 / kmass_lumped(self.shp, kp)
        self.mg = hierarchy.multigrid()

    def split(self, v):
        return v[: self.nu].reshape(self.sh.vec_shape), v[self.nu:].reshape(self.shp.scalar_shape)

    def join(self, u, p):
        return np.concatenate([np.ravel(u), np.ravel(p)])

    def apply(self, v):
        u, p = self.split(v)
        return self.join(self.A.apply(u) + self.B.apply_transpose(p), self.B.apply(u))

    def dot(self, a, b):
        ua, pa = self.split(a)
        ub, pb = self.split(b)
        return self.sh.dot(ua, ub) + self.shp.dot(pa, pb)

    def precondition(self, v):
        vu, vp = self.split(v)
        zp = self.inv_schur * vp
        t = self.B.apply_transpose(zp) + vu
        zu = self.mg.solve(np.zeros_like(vu), t)
        return self.join(zu, -zp)
