"""Python bindings to the reference's own FP64 Stokes path -- TEST INFRASTRUCTURE ONLY.

``oracle/_ref/libterra_ref.so`` is compiled from the reference sources by ``oracle/ref/Makefile`` (vendored
Kokkos 4.6.01 with the Serial and OpenMP host backends, a single-rank MPI stand-in, and the C entry points of
``oracle/ref/terra_ref.cpp``). Only ``tests/``, ``__graft_entry__`` and ``bench.py``'s reference arm use it,
to check the restatement in ``oracle.py`` and the product against the reference itself and to time the
reference on the host cores. The library is built here from ``/root/reference``; where that tree is absent
(the GPU host) the prebuilt library is used if it travelled with the repository, and ``available()`` says
whether it is there.

Shapes follow ``oracle.py``: velocity ``(3, 10, nl, nl, nr)``, scalar ``(10, nl, nl, nr)``, cells
``(10, nl-1, nl-1, nr-1)``, all float64.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "libterra_ref.so")
_REF_TREE = "/root/reference"
_lib = None

NEUMANN, DIRICHLET, FREESLIP = 0, 1, 2


def build() -> bool:
    """Build the library from the reference tree when that tree is present. Returns whether it exists."""
    if os.path.isdir(_REF_TREE):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(_HERE, "ref"), "REF=" + _REF_TREE], check=True)
    return os.path.exists(_LIB_PATH)


def available() -> bool:
    return os.path.exists(_LIB_PATH)


class RefError(RuntimeError):
    pass


def lib(threads: int = 0):
    """Load and initialise the library (OpenMP threads: the host's cores unless given). With fewer than 16
    threads the reference's fast gradient path is wrong (1x1x1 team tiles, gradient_kerngen.hpp:154-166), so
    the library then runs the gradient's own slow path instead (terra_ref.cpp, guard_small_teams)."""
    global _lib
    if _lib is None:
        if not available():
            raise RefError("oracle/_ref/libterra_ref.so is not built")
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        dpp = ctypes.POINTER(dp)
        u8 = ctypes.POINTER(ctypes.c_uint8)
        i64 = ctypes.POINTER(ctypes.c_int64)
        I, D = ctypes.c_int, ctypes.c_double
        L.tnr_last_error.restype = ctypes.c_char_p
        L.tnr_init.argtypes = [I]
        L.tnr_mesh.argtypes = [I, I, D, D, dp, dp, u8, u8, i64]
        L.tnr_epsdivdiv.argtypes = [I, D, D, dp, dp, I, I, I, I, I, I, dp, dp]
        L.tnr_divergence.argtypes = [I, D, D, I, I, dp, dp]
        L.tnr_gradient.argtypes = [I, D, D, I, I, dp, dp]
        L.tnr_kmass_lumped.argtypes = [I, D, D, dp, dp]
        L.tnr_vector_mass.argtypes = [I, D, D, dp, dp]
        L.tnr_prolongate_add.argtypes = [I, D, D, dp, dp]
        L.tnr_restrict.argtypes = [I, D, D, dp, dp]
        L.tnr_gca.argtypes = [I, I, D, D, dp, I, dp]
        L.tnr_prolongate_linear_add.argtypes = [I, D, D, I, dp, dp]
        L.tnr_restrict_linear.argtypes = [I, D, D, I, dp, dp]
        L.tnr_stokes_create.argtypes = [I, I, D, D, I, I, dp, dpp, dp, dpp, I, I, I, I, I, I,
                                        ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(D)]
        L.tnr_stokes_solve.argtypes = [ctypes.c_void_p, D, D, I, dp, dp, dp, I, ctypes.POINTER(I), ctypes.POINTER(D)]
        L.tnr_stokes_destroy.argtypes = [ctypes.c_void_p]
        L.tnr_stokes_destroy.restype = None
        L.tnr_epsdivdiv_time.argtypes = [I, D, D, dp, I, I, dp, I, dp]
        L.tnr_rhs_enforce.argtypes = [I, D, D, I, I, dp]
        L.tnr_xdmf_write.argtypes = [I, D, D, ctypes.c_char_p, I, dp, dp, I]
        L.tnr_gca_marks.argtypes = [I, I, D, D, dp, dp]
        L.tnr_stokes_level_apply.argtypes = [ctypes.c_void_p, I, I, dp, dp]
        _check(L, L.tnr_init(int(threads) if threads > 0 else (os.cpu_count() or 1)))
        _lib = L
    return _lib


def _check(L, rc):
    if rc != 0:
        raise RefError(L.tnr_last_error().decode())


def num_threads() -> int:
    return lib().tnr_num_threads()


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _sizes(lat):
    return (1 << lat) + 1


def mesh(lat, rad=None, r_min=0.55, r_max=1.0):
    """coords (10,nl,nl,3), radii (10,nr), boundary flags and ownership (10,nl,nl,nr) u8, and per node the
    smallest global index among its interface duplicates (int64)."""
    rad = lat if rad is None else rad
    nl, nr = _sizes(lat), _sizes(rad)
    coords = np.zeros((10, nl, nl, 3))
    radii = np.zeros((10, nr))
    bmask = np.zeros((10, nl, nl, nr), np.uint8)
    owned = np.zeros((10, nl, nl, nr), np.uint8)
    rep = np.zeros((10, nl, nl, nr), np.int64)
    L = lib()
    _check(L, L.tnr_mesh(lat, rad, r_min, r_max, _dp(coords), _dp(radii),
                         bmask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                         owned.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                         rep.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
    return dict(coords=coords, radii=radii, boundary=bmask, owned=owned, class_rep=rep)


def epsdivdiv(lat, src, k=None, k_q0=None, bc_cmb=DIRICHLET, bc_surface=DIRICHLET, diagonal=False, slow=False,
              add_to=None, comm=True, r_min=0.55, r_max=1.0):
    nl = _sizes(lat)
    if k is None:
        k = np.ones((10, nl, nl, nl))
    dst = np.zeros((3, 10, nl, nl, nl)) if add_to is None else _c(add_to).copy()
    L = lib()
    _check(L, L.tnr_epsdivdiv(lat, r_min, r_max, _dp(_c(k)), _dp(None if k_q0 is None else _c(k_q0)), bc_cmb,
                              bc_surface, int(diagonal), int(slow), int(add_to is not None), int(comm),
                              _dp(_c(src)), _dp(dst)))
    return dst


def divergence(lat, u, bc_cmb=DIRICHLET, bc_surface=DIRICHLET, r_min=0.55, r_max=1.0):
    nc = _sizes(lat - 1)
    p = np.zeros((10, nc, nc, nc))
    L = lib()
    _check(L, L.tnr_divergence(lat, r_min, r_max, bc_cmb, bc_surface, _dp(_c(u)), _dp(p)))
    return p


def gradient(lat, p, bc_cmb=DIRICHLET, bc_surface=DIRICHLET, r_min=0.55, r_max=1.0):
    nl = _sizes(lat)
    u = np.zeros((3, 10, nl, nl, nl))
    L = lib()
    _check(L, L.tnr_gradient(lat, r_min, r_max, bc_cmb, bc_surface, _dp(_c(p)), _dp(u)))
    return u


def kmass_lumped(lat, k, r_min=0.55, r_max=1.0):
    nl = _sizes(lat)
    d = np.zeros((10, nl, nl, nl))
    L = lib()
    _check(L, L.tnr_kmass_lumped(lat, r_min, r_max, _dp(_c(k)), _dp(d)))
    return d


def vector_mass(lat, v, r_min=0.55, r_max=1.0):
    out = np.zeros_like(_c(v))
    L = lib()
    _check(L, L.tnr_vector_mass(lat, r_min, r_max, _dp(_c(v)), _dp(out)))
    return out


def prolongate_add(fine_lat, coarse_v, fine_v, r_min=0.55, r_max=1.0):
    out = _c(fine_v).copy()
    L = lib()
    _check(L, L.tnr_prolongate_add(fine_lat, r_min, r_max, _dp(_c(coarse_v)), _dp(out)))
    return out


def restrict(fine_lat, fine_v, r_min=0.55, r_max=1.0):
    nc = _sizes(fine_lat - 1)
    out = np.zeros((3, 10, nc, nc, nc))
    L = lib()
    _check(L, L.tnr_restrict(fine_lat, r_min, r_max, _dp(_c(fine_v)), _dp(out)))
    return out


def gca(fine_lat, coarse_lat, k, linear=False, r_min=0.55, r_max=1.0):
    """Element matrices of level coarse_lat from TwoGridGCA chained down from the Neumann operator of fine_lat
    (InterpolationMode::Linear when linear, else Constant)."""
    nc = _sizes(coarse_lat)
    out = np.zeros((10, nc - 1, nc - 1, nc - 1, 2, 18, 18))
    L = lib()
    _check(L, L.tnr_gca(fine_lat, coarse_lat, r_min, r_max, _dp(_c(k)), int(linear), _dp(out)))
    return out


def gca_marks(lat, level_range, k, r_min=0.55, r_max=1.0):
    """GCAElementsCollector on level lat: bool marks of the cells of level lat - level_range."""
    nc = _sizes(lat - level_range)
    out = np.zeros((10, nc - 1, nc - 1, nc - 1))
    L = lib()
    _check(L, L.tnr_gca_marks(lat, level_range, r_min, r_max, _dp(_c(k)), _dp(out)))
    return out > 0.5


def prolongate_linear_add(fine_lat, coarse_v, fine_v, r_min=0.55, r_max=1.0):
    """fine += P coarse with ProlongationLinear per component."""
    out = _c(fine_v).copy()
    cv = _c(coarse_v)
    L = lib()
    _check(L, L.tnr_prolongate_linear_add(fine_lat, r_min, r_max, cv.shape[0], _dp(cv), _dp(out)))
    return out


def restrict_linear(fine_lat, fine_v, r_min=0.55, r_max=1.0):
    """coarse = R fine with RestrictionLinear per component (interface sum included)."""
    fv = _c(fine_v)
    nc = _sizes(fine_lat - 1)
    out = np.zeros((fv.shape[0], 10, nc, nc, nc))
    L = lib()
    _check(L, L.tnr_restrict_linear(fine_lat, r_min, r_max, fv.shape[0], _dp(fv), _dp(out)))
    return out


def xdmf_write(lat, directory, scalar, vec, geometry_bytes=4, out_bytes=4, r_min=0.55, r_max=1.0):
    """The reference's XDMFOutput: one step with the scalar field "temperature" and the vector "velocity"."""
    L = lib()
    _check(L, L.tnr_xdmf_write(lat, r_min, r_max, directory.encode(), geometry_bytes, _dp(_c(scalar)), _dp(_c(vec)),
                               out_bytes))


def rhs_enforce(lat, f, bc_cmb, bc_surface, r_min=0.55, r_max=1.0):
    """f: flat Stokes vector (3 velocity components on lat, pressure on lat-1); returns the enforced copy."""
    out = _c(f).copy()
    L = lib()
    _check(L, L.tnr_rhs_enforce(lat, r_min, r_max, bc_cmb, bc_surface, _dp(out)))
    return out


class StokesRef:
    """The reference application's Stokes solver (FGMRES + block-triangular GMG), built once."""

    def __init__(self, lat, num_levels, k, k_schur, k_levels=None, start=None, bc_cmb=DIRICHLET, bc_surface=FREESLIP,
                 gca=True, restart=30, cheb_order=2, cheb_iterations=2, power_iterations=10, vcycles=1, r_min=0.55,
                 r_max=1.0):
        dp = ctypes.POINTER(ctypes.c_double)
        self._keep = []

        def arr(lst):
            if lst is None:
                return None
            cs = [None if a is None else _c(a) for a in lst]
            self._keep.append(cs)
            return (dp * len(cs))(*[_dp(a) if a is not None else None for a in cs])

        k, k_schur = _c(k), _c(k_schur)
        self._keep.append((k, k_schur))
        h, t = ctypes.c_void_p(), ctypes.c_double()
        L = lib()
        _check(L, L.tnr_stokes_create(lat, num_levels, r_min, r_max, bc_cmb, bc_surface, _dp(k), arr(k_levels),
                                      _dp(k_schur), arr(start), int(gca), restart, cheb_order, cheb_iterations,
                                      power_iterations, vcycles, ctypes.byref(h), ctypes.byref(t)))
        self._h, self.setup_seconds = h, t.value

    def solve(self, b, x0=None, rtol=1e-8, atol=1e-30, max_it=100):
        """Returns (x, relative residual history, wall seconds of the solve)."""
        b = _c(b)
        x = np.zeros_like(b) if x0 is None else _c(x0).copy()
        hist = np.zeros(max_it + 64)
        n, t = ctypes.c_int(0), ctypes.c_double()
        L = lib()
        _check(L, L.tnr_stokes_solve(self._h, rtol, atol, max_it, _dp(b), _dp(x), _dp(hist), len(hist),
                                     ctypes.byref(n), ctypes.byref(t)))
        return x, hist[: n.value].copy(), t.value

    def level_apply(self, level, src, diagonal=False):
        """A_l src of hierarchy level `level` (0 = coarsest; the fine block at the top), Replace mode with the
        interface sum; src is (3, 10, n, n, nr)."""
        src = _c(src)
        out = np.zeros_like(src)
        L = lib()
        _check(L, L.tnr_stokes_level_apply(self._h, level, int(diagonal), _dp(src), _dp(out)))
        return out

    def close(self):
        if self._h:
            lib().tnr_stokes_destroy(self._h)
            self._h = None

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tnr_stokes_destroy(self._h)
            self._h = None


def stokes_fgmres(lat, num_levels, k, k_schur, b, x0=None, k_levels=None, start=None, bc_cmb=DIRICHLET,
                  bc_surface=FREESLIP, gca=True, restart=30, rtol=1e-8, atol=1e-30, max_it=100, cheb_order=2,
                  cheb_iterations=2, power_iterations=10, vcycles=1, r_min=0.55, r_max=1.0):
    """The reference application's Stokes solve; returns (x, relative residual history)."""
    S = StokesRef(lat, num_levels, k, k_schur, k_levels=k_levels, start=start, bc_cmb=bc_cmb, bc_surface=bc_surface,
                  gca=gca, restart=restart, cheb_order=cheb_order, cheb_iterations=cheb_iterations,
                  power_iterations=power_iterations, vcycles=vcycles, r_min=r_min, r_max=r_max)
    x, hist, _ = S.solve(b, x0=x0, rtol=rtol, atol=atol, max_it=max_it)
    S.close()
    return x, hist


def epsdivdiv_time(lat, k, src, reps=5, bc_cmb=DIRICHLET, bc_surface=FREESLIP, r_min=0.55, r_max=1.0):
    """Seconds of each of `reps` reference applies after one warm-up (fast path, with the interface sum)."""
    out = np.zeros(reps)
    L = lib()
    _check(L, L.tnr_epsdivdiv_time(lat, r_min, r_max, _dp(_c(k)), bc_cmb, bc_surface, _dp(_c(src)), reps, _dp(out)))
    return out
