"""ORACLE — test infrastructure only.  ctypes bindings for the CPU checkers.

* ``Oracle``      — the C++ restatement of Apollo's nodal-DG RHS and SSPRK(5,2)
                    stepper (dg_oracle.cpp, built to _build/liboracle.so).
* ``RefPlugins``  — Apollo's own equation plugins and exprFunc compiled
                    unmodified (ref_adapter.cpp, built to _ref/libapollo_ref.so
                    where the Apollo source tree exists).
* ``RefLimiter``  — Apollo's own eulerLimiterHW and grid boundary conditions
                    compiled unmodified (ref_limiter.cpp, built to
                    _ref/libapollo_reflim.so where the Apollo source tree exists).
* ``RefDriver``   — Apollo's own nodal-DG right-hand side with its geometry
                    and cubature code compiled unmodified (ref_driver.cpp, built
                    to _ref/libapollo_refdrv.so where the Apollo source tree
                    exists).

Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py``
import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libapollo_ref.so")
REFLIM_PATH = os.path.join(HERE, "_ref", "libapollo_reflim.so")
REFDRV_PATH = os.path.join(HERE, "_ref", "libapollo_refdrv.so")

EQ_ADVECTION, EQ_EULER, EQ_MAXWELL = 0, 1, 2
# source plugins (Apollo kind names tranverseMagneticSrc, pointCurrentSrc)
SRC_TM, SRC_POINT = 1, 2
BC_FIXED, BC_VORTEX, BC_TM, BC_PEC = 0, 1, 2, 3
BC_EULER_WALL, BC_EULER_INFLOW, BC_EULER_ZEROGRAD, BC_EULER_DIRICHLET = 4, 5, 6, 7
# Euler numerical fluxes (eqp[3]), Apollo's Numerical_Flux codes
NF_LF, NF_HLL, NF_ROE, NF_WAVE = 0, 1, 2, 4
NF_UPWIND = 8  # an extension (not in Apollo): advection, and the Maxwell TM fields with chi = gamma = 0

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def reference_src() -> str:
    """Apollo's source tree (its ``src`` directory): ``$APOLLO_SRC`` where set,
    else the default of the build recipe (oracle/Makefile, ``make print-src``).
    The tree is only read to build the reference plugins and by the tests that
    parse Apollo's example inputs; nothing needs it at run time."""
    src = os.environ.get("APOLLO_SRC")
    if src:
        return src
    out = subprocess.run(["make", "-s", "-C", HERE, "print-src"], capture_output=True, text=True)
    return out.stdout.strip()


def have_reference() -> bool:
    return os.path.isdir(reference_src())


def build(with_ref: bool = True) -> None:
    """Compile the oracle (and the reference plugins where the source exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    src = reference_src()
    if with_ref and os.path.isdir(src):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "reflim", "refdrv", f"APOLLO_SRC={src}"], check=True)


def _lib():
    if not os.path.exists(LIB_PATH):
        build(with_ref=False)
    lib = C.CDLL(LIB_PATH)
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip, C.c_int, _ip,
                               _dp, C.c_double]
    for name in ("orc_destroy",):
        getattr(lib, name).argtypes = [C.c_void_p]
    for name in ("orc_meqn", "orc_np", "orc_nc", "orc_ng", "orc_error"):
        getattr(lib, name).argtypes = [C.c_void_p]
        getattr(lib, name).restype = C.c_int
    for name in ("orc_dtscale", "orc_rmin"):
        getattr(lib, name).argtypes = [C.c_void_p]
        getattr(lib, name).restype = C.c_double
    lib.orc_set_threads.argtypes = [C.c_void_p, C.c_int]
    lib.orc_set_ref_plugins.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.orc_node_coords.argtypes = [C.c_void_p, _dp, _dp]
    lib.orc_connectivity.argtypes = [C.c_void_p, _ip]
    lib.orc_operator.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.orc_fmask.argtypes = [C.c_void_p, _ip]
    lib.orc_apply_bc.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
    lib.orc_rhs.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, _dp]
    lib.orc_rhs.restype = C.c_double
    lib.orc_init_dt.argtypes = [C.c_void_p, _dp]
    lib.orc_init_dt.restype = C.c_double
    lib.orc_ssp_step.argtypes = [C.c_void_p, _dp, C.c_double, C.c_double]
    lib.orc_ssp_step.restype = C.c_double
    lib.orc_run.argtypes = [C.c_void_p, _dp, C.c_int, _dp, _dp, C.c_double]
    lib.orc_run.restype = C.c_int
    lib.orc_set_limiter.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
    lib.orc_set_limiter.restype = C.c_int
    lib.orc_limit.argtypes = [C.c_void_p, _dp]
    lib.orc_limit.restype = None
    lib.orc_add_source.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
    lib.orc_add_source.restype = C.c_int
    lib.orc_source_terms.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _dp]
    lib.orc_source_terms.restype = None
    lib.orc_set_limiter_ta.argtypes = [C.c_void_p]
    lib.orc_set_limiter_ta.restype = C.c_int
    lib.orc_ta_prim.argtypes = [C.c_void_p, _dp, _dp]
    lib.orc_ta_prim.restype = None
    lib.orc_ta_node.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
    lib.orc_ta_node.restype = C.c_int
    return lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class Oracle:
    """CPU oracle for one mesh, order and equation (fields in Apollo's count:
    1 advection, 5 Euler, 8 Maxwell)."""

    def __init__(self, mesh, N: int, eq: int, eqp, bcs=(), cfl: float = 0.5):
        self.lib = _lib()
        self.N = N
        eqp = np.zeros(4) if eqp is None else np.asarray(list(eqp) + [0.0] * (4 - len(eqp)), dtype=np.float64)
        kinds = np.asarray([b[0] for b in bcs] or [0], dtype=np.int32)
        pars = np.zeros((max(1, len(bcs)), 8))
        for i, b in enumerate(bcs):
            pars[i, :len(b[1])] = b[1]
        self._keep = [mesh, eqp, kinds, pars]
        self.h = self.lib.orc_create(N, eq, _p(eqp), mesh.nverts, _p(mesh.vx), _p(mesh.vy), mesh.K,
                                     _p(mesh.etov, _ip), _p(mesh.face_tag, _ip), _p(mesh.vert_canon, _ip),
                                     max(1, len(bcs)), _p(kinds, _ip), _p(pars), cfl)
        self.K = mesh.K
        self.meqn = self.lib.orc_meqn(self.h)
        self.Np = self.lib.orc_np(self.h)
        self.Nc = self.lib.orc_nc(self.h)
        self.Ng = self.lib.orc_ng(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @property
    def shape(self):
        return (self.K, self.Np, self.meqn)

    def set_threads(self, n: int) -> None:
        self.lib.orc_set_threads(self.h, int(n))

    def use_ref_plugins(self, ref: "RefPlugins", eqn_handle) -> None:
        self._ref_keep = (ref, eqn_handle)
        self.lib.orc_set_ref_plugins(self.h, C.cast(ref.lib.ref_flux, C.c_void_p),
                                     C.cast(ref.lib.ref_numflux, C.c_void_p), eqn_handle)

    def node_coords(self):
        x = np.empty((self.K, self.Np))
        y = np.empty((self.K, self.Np))
        self.lib.orc_node_coords(self.h, _p(x), _p(y))
        return x, y

    def connectivity(self):
        c = np.empty((self.K, 6), dtype=np.int32)
        self.lib.orc_connectivity(self.h, _p(c, _ip))
        return c

    def operator(self, which: int):
        shapes = {0: (self.Nc, self.Np), 1: (self.Nc, self.Np), 2: (self.Nc, self.Np), 3: (3 * self.Ng, self.Np),
                  4: (self.Np, self.Np), 5: (self.Nc,), 6: (self.Ng,), 7: (self.Np, self.Np)}
        out = np.empty(shapes[which])
        self.lib.orc_operator(self.h, which, _p(out))
        return out

    def fmask(self):
        out = np.empty(3 * (self.N + 1), dtype=np.int32)
        self.lib.orc_fmask(self.h, _p(out, _ip))
        return out

    def apply_bc(self, tag: int, xc, nx, q):
        """Boundary condition `tag` (1-based, in bcs order) at one point."""
        xc5 = np.zeros(5)
        xc5[:len(xc)] = xc
        q = np.ascontiguousarray(q, dtype=np.float64)
        qb = np.zeros(max(len(q), 8))
        self.lib.orc_apply_bc(self.h, int(tag), _p(xc5), _p(np.array(nx, dtype=np.float64)), _p(q), _p(qb))
        return qb[:len(q)]

    @property
    def error(self) -> int:
        return self.lib.orc_error(self.h)

    @property
    def dtscale(self) -> float:
        return self.lib.orc_dtscale(self.h)

    @property
    def rmin(self) -> float:
        return self.lib.orc_rmin(self.h)

    def rhs(self, u, t: float = 0.0, dt: float = 0.0):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.shape)
        out = np.empty_like(u)
        sugg = self.lib.orc_rhs(self.h, t, dt, _p(u), _p(out))
        return out, sugg

    def init_dt(self, u) -> float:
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.shape)
        return self.lib.orc_init_dt(self.h, _p(u))

    def ssp_step(self, u, t0: float, dt: float) -> float:
        assert u.flags.c_contiguous and u.dtype == np.float64
        return self.lib.orc_ssp_step(self.h, _p(u), t0, dt)

    def add_source(self, kind: int, out: int, params=()) -> None:
        """A source plugin adding into Apollo field `out` (SRC_TM; SRC_POINT
        with xLocation, yLocation, radius, currentDensity, frequency, phase,
        charge, mass, epsilon0)."""
        p = np.zeros(9)
        p[:len(params)] = params
        if self.lib.orc_add_source(self.h, kind, out, _p(p)) != 0:
            raise ValueError("bad source")

    def source_terms(self, t: float, x: float, y: float):
        out = np.zeros(self.meqn)
        self.lib.orc_source_terms(self.h, t, x, y, _p(out))
        return out

    def set_limiter(self, gamma: float, min_pressure: float, min_density: float) -> None:
        """Apollo's eulerLimiterHW on every stage input (5 fields, N <= 4)."""
        if self.lib.orc_set_limiter(self.h, gamma, min_pressure, min_density) != 0:
            raise ValueError("the limiter needs eulerEqn at order <= 4")

    def set_limiter_ta(self) -> None:
        """Apollo's tuAliabadiLimiter on every stage input (eulerEqn with the
        equation's own gas_gamma, minPressure, minDensity; phMaxwellEqn as
        element averaging; N <= 4)."""
        if self.lib.orc_set_limiter_ta(self.h) != 0:
            raise ValueError("tuAliabadiLimiter needs eulerEqn or phMaxwellEqn at order <= 4")

    def ta_prim(self, qc):
        """(floored conserved, primitive) of one Euler state, as the limiter computes them."""
        c = np.array(qc, dtype=np.float64, copy=True)
        p = np.zeros(5)
        self.lib.orc_ta_prim(self.h, _p(c), _p(p))
        return c, p

    def ta_node(self, cc, cp, dq):
        """(limited conserved state, error bits) of one node."""
        out = np.zeros(5)
        a, b, d = (np.ascontiguousarray(v, dtype=np.float64) for v in (cc, cp, dq))
        err = self.lib.orc_ta_node(self.h, _p(a), _p(b), _p(d), _p(out))
        return out, err

    def limit(self, u):
        """The limiter applied to a copy of u."""
        v = np.array(u, dtype=np.float64, order="C", copy=True)
        self.lib.orc_limit(self.h, _p(v))
        return v

    def run(self, u, nsteps: int, t: float, dt: float, tend: float = -1.0):
        """Advance u in place; returns (steps taken, t, dt for the next step)."""
        assert u.flags.c_contiguous and u.dtype == np.float64
        tt = C.c_double(t)
        dd = C.c_double(dt)
        n = self.lib.orc_run(self.h, _p(u), nsteps, C.byref(tt), C.byref(dd), tend)
        return n, tt.value, dd.value


class RefPlugins:
    """Apollo's own equation plugins and exprFunc (compiled unmodified)."""

    def __init__(self):
        if not os.path.exists(REF_PATH):
            raise FileNotFoundError(REF_PATH)
        lib = C.CDLL(REF_PATH)
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_eqn_create.restype = C.c_void_p
        lib.ref_eqn_create.argtypes = [C.c_char_p]
        lib.ref_eqn_destroy.argtypes = [C.c_void_p]
        lib.ref_eqn_meqn.argtypes = [C.c_void_p]
        lib.ref_eqn_meqn.restype = C.c_int
        lib.ref_flux.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        lib.ref_numflux.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        lib.ref_speed2.argtypes = [C.c_void_p, _dp]
        lib.ref_speed2.restype = C.c_double
        lib.ref_exprfunc_create.restype = C.c_void_p
        lib.ref_exprfunc_create.argtypes = [C.c_char_p]
        lib.ref_exprfunc_size.argtypes = [C.c_void_p]
        lib.ref_exprfunc_size.restype = C.c_int
        lib.ref_exprfunc_eval.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _dp]
        lib.ref_exprfunc_destroy.argtypes = [C.c_void_p]
        lib.ref_primitive.argtypes = [C.c_void_p, _dp, _dp]
        lib.ref_ta_limit.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        lib.ref_src_create.restype = C.c_void_p
        lib.ref_src_create.argtypes = [C.c_char_p, C.c_int]
        lib.ref_src_eval.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _dp, _dp]
        lib.ref_src_destroy.argtypes = [C.c_void_p]
        self.lib = lib

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_PATH)

    def equation(self, kind: str, **params):
        body = "\n".join(f"  {k} = {v}" for k, v in params.items())
        text = f"<top>\n Equations = [eq]\n <eq>\n  Kind = {kind}\n{body}\n </eq>\n</top>\n"
        h = self.lib.ref_eqn_create(text.encode())
        if not h:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return h

    def flux(self, h, d: int, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        f = np.zeros_like(q)
        self.lib.ref_flux(h, d, _p(q), _p(f))
        return f

    def numflux(self, h, n, qM, qP):
        n = np.ascontiguousarray(n, dtype=np.float64)
        qM = np.array(qM, dtype=np.float64)
        qP = np.array(qP, dtype=np.float64)
        f = np.zeros_like(qM)
        lam = C.c_double(0.0)
        self.lib.ref_numflux(h, _p(n), _p(qM), _p(qP), _p(f), C.byref(lam))
        return f, lam.value

    def primitive(self, h, qc):
        """(conserved as rewritten by the equation, primitive) of one state."""
        c = np.array(qc, dtype=np.float64, copy=True)
        p = np.zeros_like(c)
        self.lib.ref_primitive(h, _p(c), _p(p))
        return c, p

    def ta_limit(self, h, cc, cp, dq):
        """One node of the equation's Tu-Aliabadi reconstruction."""
        a, b, d = (np.array(v, dtype=np.float64, copy=True) for v in (cc, cp, dq))
        out = np.zeros_like(a)
        self.lib.ref_ta_limit(h, _p(a), _p(b), _p(d), _p(out))
        return out

    def speed2(self, h, q) -> float:
        q = np.ascontiguousarray(q, dtype=np.float64)
        return self.lib.ref_speed2(h, _p(q))

    def sources(self, blocks: dict, meqn: int):
        """Apollo's source set from {name: (kind, {key: value})}."""
        body = "".join(f" <{n}>\n  Kind = {k}\n" + "".join(f"  {a} = {v}\n" for a, v in kv.items()) + f" </{n}>\n"
                       for n, (k, kv) in blocks.items())
        text = f"<top>\n Sources = [{', '.join(blocks)}]\n{body}</top>\n"
        h = self.lib.ref_src_create(text.encode(), meqn)
        if not h:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return h

    def source_terms(self, h, meqn: int, t: float, x: float, y: float, q=None):
        q = np.zeros(meqn) if q is None else np.array(q, dtype=np.float64)
        s = np.zeros(meqn)
        self.lib.ref_src_eval(h, t, x, y, _p(q), _p(s))
        return s

    def exprfunc(self, text: str):
        h = self.lib.ref_exprfunc_create(text.encode())
        if not h:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return h

    def exprfunc_eval(self, h, t: float, x: float, y: float):
        out = np.zeros(self.lib.ref_exprfunc_size(h))
        self.lib.ref_exprfunc_eval(h, t, x, y, _p(out))
        return out


class RefLimiter:
    """Apollo's own eulerLimiterHW and grid boundary-condition plugins
    (compiled unmodified) on the oracle's geometry: node coordinates, face
    masks, mass matrix and element-to-element-to-face table of an Oracle."""

    def __init__(self, o: "Oracle"):
        if not os.path.exists(REFLIM_PATH):
            raise FileNotFoundError(REFLIM_PATH)
        lib = C.CDLL(REFLIM_PATH)
        lib.reflim_last_error.restype = C.c_char_p
        lib.reflim_create.restype = C.c_void_p
        lib.reflim_create.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _ip, _ip, _dp]
        lib.reflim_destroy.argtypes = [C.c_void_p]
        lib.reflim_add_bc.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
        lib.reflim_add_bc.restype = C.c_int
        lib.reflim_apply_bc.argtypes = [C.c_void_p, C.c_char_p, _dp, _dp, _dp, C.c_int, _dp]
        lib.reflim_apply_bc.restype = C.c_int
        lib.reflim_set_limiter.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
        lib.reflim_set_limiter.restype = C.c_int
        lib.reflim_limit.argtypes = [C.c_void_p, _dp, _dp]
        lib.reflim_limit.restype = C.c_int
        self.lib = lib
        x, y = o.node_coords()
        self._keep = (np.ascontiguousarray(x), np.ascontiguousarray(y),
                      np.ascontiguousarray(o.connectivity(), dtype=np.int32), o.fmask(), o.operator(7))
        x, y, conn, fm, mass = self._keep
        self.K, self.Np = x.shape
        self.h = lib.reflim_create(int(self.K), int(o.N), int(o.lib.orc_meqn(o.h)), _p(x), _p(y), _p(conn, _ip),
                                   _p(fm, _ip), _p(mass))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.reflim_destroy(self.h)
            self.h = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REFLIM_PATH)

    @staticmethod
    def _block(name: str, params: dict) -> bytes:
        body = "".join(f"  {k} = {v}\n" for k, v in params.items())
        return f"<{name}>\n{body}</{name}>\n".encode()

    def add_bc(self, name: str, kind: str, **params) -> None:
        """Register Apollo's boundary condition of `kind` under `name`."""
        if self.lib.reflim_add_bc(self.h, kind.encode(), self._block(name, params)) != 0:
            raise RuntimeError(self.lib.reflim_last_error().decode())

    def apply_bc(self, name: str, xc, nx, q):
        xc5 = np.zeros(5)
        xc5[:len(xc)] = xc
        q = np.ascontiguousarray(q, dtype=np.float64)
        qb = np.zeros(max(len(q), 8))
        if self.lib.reflim_apply_bc(self.h, name.encode(), _p(xc5), _p(np.array(nx, dtype=np.float64)), _p(q),
                                    len(q), _p(qb)) != 0:
            raise RuntimeError(self.lib.reflim_last_error().decode())
        return qb[:len(q)]

    def set_limiter(self, boundary_conditions, gas_gamma: float, min_pressure: float, min_density: float) -> None:
        """eulerLimiterHW with the named boundary conditions in tag order."""
        text = self._block("eulerLimit", {"Kind": "eulerLimiterHW", "gas_gamma": gas_gamma,
                                          "min_pressure": min_pressure, "min_density": min_density,
                                          "boundaryConditions": "[" + ", ".join(boundary_conditions) + "]"})
        if self.lib.reflim_set_limiter(self.h, 0, text) != 0:
            raise RuntimeError(self.lib.reflim_last_error().decode())

    def set_limiter_ta(self, boundary_conditions, equation: str, **params) -> None:
        """tuAliabadiLimiter with the named boundary conditions in tag order,
        over Apollo's equation `equation` with its own keys."""
        eq = "".join(f"  {k} = {v}\n" for k, v in params.items())
        text = (f"<taLimit>\n  Kind = tuAliabadiLimiter\n  boundaryConditions = [{', '.join(boundary_conditions)}]\n"
                f"  Equations = [eq]\n <eq>\n  Kind = {equation}\n{eq} </eq>\n</taLimit>\n").encode()
        if self.lib.reflim_set_limiter(self.h, 1, text) != 0:
            raise RuntimeError(self.lib.reflim_last_error().decode())

    def limit(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(u)
        if self.lib.reflim_limit(self.h, _p(u), _p(out)) != 0:
            raise RuntimeError(self.lib.reflim_last_error().decode())
        return out


class RefDriver:
    """Apollo's own nodal-DG right-hand side (WxNodalDG2dMethod with its
    geometry, cubature, equation, source and boundary-condition code,
    compiled unmodified) on a triangle mesh through a minimal stand-in for
    PETSc's mesh, vector and dense-matrix calls."""

    def __init__(self, mesh):
        if not os.path.exists(REFDRV_PATH):
            raise FileNotFoundError(REFDRV_PATH)
        lib = C.CDLL(REFDRV_PATH)
        lib.refdrv_last_error.restype = C.c_char_p
        lib.refdrv_create.restype = C.c_void_p
        lib.refdrv_create.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip]
        lib.refdrv_destroy.argtypes = [C.c_void_p]
        lib.refdrv_add_bc.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
        lib.refdrv_add_bc.restype = C.c_int
        lib.refdrv_add_limiter.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
        lib.refdrv_add_limiter.restype = C.c_int
        lib.refdrv_setup.argtypes = [C.c_void_p, C.c_char_p]
        lib.refdrv_setup.restype = C.c_int
        for name in ("refdrv_np", "refdrv_meqn"):
            getattr(lib, name).argtypes = [C.c_void_p]
            getattr(lib, name).restype = C.c_int
        lib.refdrv_init.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
        lib.refdrv_init.restype = C.c_int
        lib.refdrv_rhs.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, _dp, _dp]
        lib.refdrv_rhs.restype = C.c_int
        self.lib = lib
        self._keep = (np.ascontiguousarray(mesh.vx, dtype=np.float64), np.ascontiguousarray(mesh.vy, dtype=np.float64),
                      np.ascontiguousarray(mesh.etov, dtype=np.int32),
                      np.ascontiguousarray(mesh.face_tag, dtype=np.int32))
        vx, vy, etov, tags = self._keep
        self.K = etov.shape[0]
        self.h = lib.refdrv_create(len(vx), _p(vx), _p(vy), self.K, _p(etov, _ip), _p(tags, _ip))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.refdrv_destroy(self.h)
            self.h = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REFDRV_PATH)

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.refdrv_last_error().decode())

    def add_bc(self, name: str, kind: str, **params) -> None:
        body = "".join(f"  {k} = {v}\n" for k, v in params.items())
        self._check(self.lib.refdrv_add_bc(self.h, kind.encode(), f"<{name}>\n{body}</{name}>\n".encode()))

    def add_limiter(self, name: str, kind: str, boundary_conditions, **params) -> None:
        """A limiter sub-solver (eulerLimiterHW with gas_gamma, min_pressure,
        min_density; or tuAliabadiLimiter with an `equation` kind and its keys)
        for the method's `Limiter = [name]`."""
        bcs = f"  boundaryConditions = [{', '.join(boundary_conditions)}]\n"
        if kind == "eulerLimiterHW":
            body = bcs + "".join(f"  {k} = {v}\n" for k, v in params.items())
            code = 0
        else:
            eq = params.pop("equation")
            body = bcs + f"  Equations = [eq]\n <eq>\n  Kind = {eq}\n" + "".join(
                f"  {k} = {v}\n" for k, v in params.items()) + " </eq>\n"
            code = 1
        self._check(self.lib.refdrv_add_limiter(self.h, code, f"<{name}>\n  Kind = {kind}\n{body}</{name}>\n".encode()))

    def setup(self, text: str) -> None:
        """The nodalDG2d sub-solver's cryptset block, as in an Apollo input
        (keys before sub-sets: Apollo's cryptset reader does not see a key
        written after a sub-set)."""
        self._check(self.lib.refdrv_setup(self.h, text.encode()))
        self.Np, self.meqn = self.lib.refdrv_np(self.h), self.lib.refdrv_meqn(self.h)

    def init(self, t: float = 0.0):
        u = np.zeros((self.K, self.Np, self.meqn))
        dt = C.c_double()
        self._check(self.lib.refdrv_init(self.h, t, _p(u), C.byref(dt)))
        return u, dt.value

    def rhs(self, u, t: float = 0.0, dt: float = 0.0):
        """(right-hand side, suggested dt) at u; u itself is left as it is."""
        return self.rhs_stage(np.array(u, dtype=np.float64, order="C", copy=True), t, dt)

    def rhs_stage(self, w, t: float = 0.0, dt: float = 0.0):
        """The right-hand side at the stage vector w (float64, C-contiguous),
        which a limiter in the method's Limiter list rewrites in place, as
        Apollo's step does to PETSc's stage vector."""
        assert w.dtype == np.float64 and w.flags.c_contiguous
        out = np.zeros_like(w)
        s = C.c_double()
        self._check(self.lib.refdrv_rhs(self.h, t, dt, _p(w), _p(out), C.byref(s)))
        return out, s.value

    def ssp_step(self, u, t0: float, dt: float):
        """One SSPRK(5,2) step through Apollo's right-hand side: PETSc's TSSSP
        `rks2` with 5 stages as documented (w = u; 4x w += dt/4 L(w) at
        t0 + dt i/4; u = 4/5 w + dt/5 L(w) + 1/5 u), the arithmetic of the
        oracle's orc_ssp_step.  Returns (u, suggested dt of the last stage)."""
        w = np.array(u, dtype=np.float64, order="C", copy=True)
        for i in range(4):
            F, _ = self.rhs_stage(w, t0 + dt * (i / 4.0), dt)
            w += (dt / 4.0) * F
        F, sugg = self.rhs_stage(w, t0 + dt, dt)
        return 0.8 * w + (dt / 5.0) * F + 0.2 * np.asarray(u), sugg

    def run(self, u, nsteps: int, t: float, dt: float):
        """nsteps steps with Apollo's dt policy (ApSolver::ComputeRHSforTS: the
        next dt is the smaller of this one and the last stage's suggestion)."""
        for _ in range(nsteps):
            u, sugg = self.ssp_step(u, t, dt)
            t += dt
            dt = min(sugg, dt)
        return u, t, dt


# Apollo's isentropicVortex example input (examples/unstructuredDG/euler/
# isentropicVortex/isentropicVortex.pin): the exprFunc program of its
# initial state
VORTEX_PROGN = ["r = sqrt((x-xo)*(x-xo)+(y-yo)*(y-yo))", "u = uo - beta*exp(1.-r*r)*(y-yo)/(2.*pi)",
                "v = vo + beta*exp(1.-r*r)*(x-xo)/(2.*pi)",
                "base = 1. - ( (gamma-1.)*beta*beta*exp(2.*(1.-r*r))/(16.*gamma*pi*pi) )",
                "rho = base^(1./(gamma-1.))", "p   = rho^gamma", "en = p/(gamma-1.) + 0.5*rho*(u*u + v*v)",
                "rhou = rho*u", "rhov = rho*v"]


def apollo_vortex_driver(mesh, N: int, cfl: float, x0: float = 5.0, y0: float = 5.0, beta: float = 5.0,
                         gamma: float = 1.4, u0: float = 1.0, v0: float = 0.0) -> RefDriver:
    """Apollo's isentropicVortex example on `mesh` through Apollo's own
    right-hand-side code: eulerEqn (Lax-Friedrichs), the exprFunc initial
    state, isentropicVortexBC (the exact vortex) on every boundary face."""
    r = RefDriver(mesh)
    r.add_bc("allSides", "isentropicVortexBC", u0=u0, v0=v0, x0=x0, y0=y0, gas_gamma=gamma, beta=beta)
    consts = "".join(f"  {k} = {v}\n" for k, v in (("xo", x0), ("yo", y0), ("beta", beta), ("gamma", gamma),
                                                    ("uo", u0), ("vo", v0), ("pi", 3.141592653589793)))
    progn = ", ".join(f'"{p}"' for p in VORTEX_PROGN)
    r.setup(f"<hyperbolic>\n Kind = nodalDG2d\n Equations = [euler]\n boundaryConditions = [allSides]\n"
            f" polynomialOrder = {N}\n cfl = {cfl!r}\n DataStructure = [0, dg, {5 * (N + 1) * (N + 2) // 2}]\n"
            f" <InitialCondition>\n  Kind = exprFunc\n{consts}"
            f'  exprList = ["rho", "rhou", "rhov", "0.0", "en"]\n  progn = [{progn}]\n </InitialCondition>\n'
            f" <euler>\n  Kind = eulerEqn\n  gas_gamma = {gamma!r}\n </euler>\n</hyperbolic>\n")
    return r


def _apollo_deck(N: int, cfl: float, eq: str, bcs, meqn: int, exprs, consts: str = "") -> str:
    return (f"<hyperbolic>\n Kind = nodalDG2d\n Equations = [eq]\n boundaryConditions = [{', '.join(bcs)}]\n"
            f" polynomialOrder = {N}\n cfl = {cfl!r}\n DataStructure = [0, dg, {meqn * (N + 1) * (N + 2) // 2}]\n"
            f" <InitialCondition>\n  Kind = exprFunc\n{consts}  exprList = ["
            + ", ".join(f'"{e}"' for e in exprs) + f"]\n </InitialCondition>\n <eq>\n{eq}\n </eq>\n</hyperbolic>\n")


def apollo_tm_driver(mesh, N: int, cfl: float) -> RefDriver:
    """Apollo's transverseMagnetic example on `mesh` through Apollo's own
    right-hand-side code: phMaxwellEqn (c0 = 1), Ez = sin(pi x) sin(pi y),
    maxwellTransverseMagneticBC on every boundary face."""
    r = RefDriver(mesh)
    r.add_bc("walls", "maxwellTransverseMagneticBC")
    r.setup(_apollo_deck(N, cfl, "  Kind = phMaxwellEqn\n  c0 = 1.0", ["walls"], 8,
                         ["0.0", "0.0", "sin(pi*x)*sin(pi*y)"] + ["0.0"] * 5, "  pi = 3.141592653589793\n"))
    return r


def apollo_advection_driver(mesh, N: int, cfl: float) -> RefDriver:
    """Advection of a Gaussian through Apollo's own right-hand-side code:
    advectionEqn (ux = 1, uy = 0.5), exp(-r^2/0.01) about (0.5, 0.5), a fixed
    zero value on every boundary face (gridFixedBC)."""
    r = RefDriver(mesh)
    r.add_bc("fixed", "gridFixedBC", value=0.0)
    r.setup(_apollo_deck(N, cfl, "  Kind = advectionEqn\n  ux = 1.0\n  uy = 0.5", ["fixed"], 1,
                         ["exp(-((x-0.5)*(x-0.5)+(y-0.5)*(y-0.5))/0.01)"]))
    return r
