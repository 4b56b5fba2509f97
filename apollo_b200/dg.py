"""Host-side mirror of Apollo's nodal-DG sub-solver over the C ABI (include/apollo_dg.h).

``NodalDG2d`` keeps the call shape of ``WxNodalDG2dMethod`` (setup from an
equation kind, boundary-condition kinds and a mesh; ``init`` for the first dt;
``step(t, dt, in, out)`` returning ``(status, suggested_dt)``) and adds the
resident-state stepper ``advance`` (PETSc TSSSP SSPRK(5,2) with Apollo's dt
policy).  Arrays are float64 ``[K][Np][m]``, numpy (host) or torch CUDA tensors
(device).  The CUDA library is required: import fails loudly without it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .mesh import Mesh

_HERE = os.path.dirname(os.path.abspath(__file__))
# APOLLO_DG_LIB selects another build of the library (e.g. an instrumented one)
LIB_PATH = os.environ.get("APOLLO_DG_LIB", os.path.join(_HERE, "lib", "libapollo_dg.so"))

APOLLO_HOST_PTR, APOLLO_DEVICE_PTR = 0, 1
PREC = {"fp64": 0, "mixed": 1}

STATUS = {
    0: "APOLLO_OK", 1: "APOLLO_ERR_CONFIG", 2: "APOLLO_ERR_MESH", 3: "APOLLO_ERR_NONPHYSICAL",
    4: "APOLLO_ERR_NAN", 5: "APOLLO_ERR_TIMEOUT", 6: "APOLLO_ERR_CUDA", 7: "APOLLO_ERR_STATE",
    8: "APOLLO_ERR_ARG", 9: "APOLLO_ERR_ALLOC",
}

# Apollo equation kinds -> fields per node
FIELDS = {"advectionEqn": 1, "eulerEqn": 5, "phMaxwellEqn": 8, "eulerEqn2d": 4, "maxwellTM": 3}


class ApolloError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class _Config(C.Structure):
    _fields_ = [("polynomial_order", C.c_int), ("cfl", C.c_double), ("device", C.c_int), ("stream", C.c_void_p)]


class HaloSizes(C.Structure):
    _fields_ = [("n_local", C.c_int), ("n_ghost", C.c_int), ("n_peers", C.c_int), ("n_send", C.c_int),
                ("n_recv", C.c_int)]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


def load_library(path: str = LIB_PATH):
    """Load libapollo_dg.so and declare its entry points (raises if missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} not built: run __graft_entry__.build() or make -C apollo_b200/csrc")
    lib = C.CDLL(path)
    H = C.c_void_p
    sig = {
        "apollo_dg_create": (C.c_int, [C.POINTER(_Config), C.POINTER(H)]),
        "apollo_dg_set_equation": (C.c_int, [H, C.c_char_p, _dp, C.c_int]),
        "apollo_dg_add_bc": (C.c_int, [H, C.c_char_p, _dp, C.c_int]),
        "apollo_dg_add_source": (C.c_int, [H, C.c_char_p, _ip, C.c_int, _dp, C.c_int]),
        "apollo_dg_set_numerical_flux": (C.c_int, [H, C.c_char_p]),
        "apollo_dg_set_limiter": (C.c_int, [H, C.c_char_p, _dp, C.c_int]),
        "apollo_dg_averaging_weights": (C.c_int, [H, _dp]),
        "apollo_dg_set_launch_shape": (C.c_int, [H, C.c_int, C.c_int]),
        "apollo_dg_set_mesh": (C.c_int, [H, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip]),
        "apollo_dg_num_fields": (C.c_int, [H]),
        "apollo_dg_num_nodes": (C.c_int, [H]),
        "apollo_dg_num_elements": (C.c_int, [H]),
        "apollo_dg_num_cubature": (C.c_int, [H]),
        "apollo_dg_num_gauss": (C.c_int, [H]),
        "apollo_dg_node_coords": (C.c_int, [H, _dp, _dp]),
        "apollo_dg_set_state": (C.c_int, [H, C.c_void_p, C.c_int]),
        "apollo_dg_get_state": (C.c_int, [H, C.c_void_p, C.c_int]),
        "apollo_dg_set_state_async": (C.c_int, [H, C.c_void_p, C.c_int]),
        "apollo_dg_get_state_async": (C.c_int, [H, C.c_void_p, C.c_int]),
        "apollo_dg_init_dt": (C.c_int, [H, _dp]),
        "apollo_dg_rhs": (C.c_int, [H, C.c_double, C.c_double, C.c_void_p, C.c_void_p, _dp, C.c_int, C.c_int]),
        "apollo_dg_step": (C.c_int, [H, C.c_int, _dp, _dp, C.c_double, C.c_int]),
        "apollo_dg_step_async": (C.c_int, [H, C.c_int, C.c_double, C.c_double, C.c_int]),
        "apollo_dg_get_time": (C.c_int, [H, _dp, _dp]),
        "apollo_dg_synchronize": (C.c_int, [H]),
        "apollo_dg_integrals": (C.c_int, [H, C.c_void_p, C.c_int, _dp]),
        "apollo_dg_energy": (C.c_int, [H, C.c_void_p, C.c_int, _dp]),
        "apollo_dg_kernel_times": (C.c_int, [H, C.c_int, C.c_int, _dp, _ip]),
        "apollo_dg_rhs_noalloc": (C.c_int, [H, C.c_double, C.c_double, C.c_void_p, C.c_void_p, _dp, C.c_void_p]),
        "apollo_dg_forward_fixed": (C.c_int, [H, C.c_int, C.c_double, C.c_double, C.c_int]),
        "apollo_dg_backward": (C.c_int, [H, C.c_void_p, C.c_void_p, C.c_int]),
        "apollo_dg_forward_revolve": (C.c_int, [H, C.c_int, C.c_double, C.c_double, C.c_int]),
        "apollo_dg_adjoint_stats": (C.c_int, [H, C.POINTER(C.c_longlong)]),
        "apollo_dg_set_fp64_kernels": (C.c_int, [H, C.c_int]),
        "apollo_dg_revolve_schedule": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
        "apollo_dg_tangent": (C.c_int, [H, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_int]),
        "apollo_dg_rhs_jvp": (C.c_int, [H, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
        "apollo_dg_rhs_vjp": (C.c_int, [H, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
        "apollo_dg_adjoint_memory": (C.c_int, [H, C.POINTER(C.c_size_t)]),
        "apollo_dg_batch_create": (C.c_int, [C.POINTER(_Config), C.c_char_p, _dp, C.c_int, C.POINTER(H)]),
        "apollo_dg_batch_add_bc": (C.c_int, [H, C.c_char_p, _dp, C.c_int]),
        "apollo_dg_batch_set_numerical_flux": (C.c_int, [H, C.c_char_p]),
        "apollo_dg_batch_add_mesh": (C.c_int, [H, C.c_int, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip, _ip]),
        "apollo_dg_batch_finalize": (C.c_int, [H]),
        "apollo_dg_batch_size": (C.c_int, [H]),
        "apollo_dg_batch_instance_info": (C.c_int, [H, C.c_int, _ip, _ip, _ip, _ip]),
        "apollo_dg_batch_node_coords": (C.c_int, [H, C.c_int, _dp, _dp]),
        "apollo_dg_batch_set_state": (C.c_int, [H, C.c_int, C.c_void_p, C.c_int]),
        "apollo_dg_batch_get_state": (C.c_int, [H, C.c_int, C.c_void_p, C.c_int]),
        "apollo_dg_batch_init_dt": (C.c_int, [H, _dp]),
        "apollo_dg_batch_step": (C.c_int, [H, C.c_int, _dp, _dp, C.c_int]),
        "apollo_dg_batch_autotune": (C.c_int, [H, C.c_int, _ip, _ip]),
        "apollo_dg_batch_last_error": (C.c_char_p, [H]),
        "apollo_dg_batch_destroy": (C.c_int, [H]),
        "apollo_dg_mesh_read_gmsh": (C.c_int, [C.c_char_p, C.POINTER(H), C.c_char_p, C.c_int]),
        "apollo_dg_mesh_info": (C.c_int, [H, _ip, _ip]),
        "apollo_dg_mesh_arrays": (C.c_int, [H, _dp, _dp, _ip, _ip]),
        "apollo_dg_mesh_destroy": (C.c_int, [H]),
        "apollo_dg_partition": (C.c_int, [C.c_int, _dp, _dp, C.c_int, _ip, C.c_int, _ip]),
        "apollo_dg_halo_plan": (C.c_int, [C.c_int, C.c_int, _ip, _ip, _ip, _ip, C.c_int, C.POINTER(HaloSizes),
                                          _ip, _ip, _ip, _ip, _ip, _ip, _ip]),
        "apollo_dg_set_mesh_partition": (C.c_int, [H, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip, _ip, C.c_int]),
        "apollo_dg_halo_info": (C.c_int, [H, C.c_int, _ip, _ip, _ip, _ip, _ip]),
        "apollo_dg_halo_bind": (C.c_int, [H, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p]),
        "apollo_dg_dist_start": (C.c_int, [H, C.c_double, C.c_double, C.c_int]),
        "apollo_dg_stage_begin": (C.c_int, [H, C.c_int, C.c_int]),
        "apollo_dg_stage_end": (C.c_int, [H, C.c_int, C.c_int]),
        "apollo_dg_step_end": (C.c_int, [H]),
        "apollo_dg_debug_set_waits": (C.c_int, [H, C.c_uint, C.c_int]),
        "apollo_dg_debug_fail_alloc": (None, [C.c_int]),
        "apollo_dg_deck_config": (C.c_int, [C.c_char_p, C.POINTER(_Config), C.c_char_p, C.c_int]),
        "apollo_dg_deck_equation": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, _dp, _ip, C.c_char_p,
                                              C.c_int, C.c_char_p, C.c_int]),
        "apollo_dg_deck_bc": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, _ip, C.c_char_p, C.c_int, _dp, _ip,
                                        C.c_char_p, C.c_int]),
        "apollo_dg_deck_limiter": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, _dp, _ip, C.c_char_p,
                                             C.c_int]),
        "apollo_dg_set_equation_text": (C.c_int, [H, C.c_char_p, C.c_char_p]),
        "apollo_dg_add_bc_text": (C.c_int, [H, C.c_char_p, C.c_char_p]),
        "apollo_dg_set_limiter_text": (C.c_int, [H, C.c_char_p, C.c_char_p]),
        "apollo_dg_deck_source": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, _ip, C.c_char_p, C.c_int, _ip, _ip,
                                            _dp, _ip, C.c_char_p, C.c_int]),
        "apollo_dg_add_source_text": (C.c_int, [H, C.c_char_p, C.c_char_p]),
        "apollo_dg_last_error": (C.c_char_p, [H]),
        "apollo_dg_destroy": (C.c_int, [H]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a, sync: bool = True):
    """(pointer, where) of a numpy array or a torch tensor.  With sync, torch's
    current stream is drained first when the tensor is on the device."""
    if isinstance(a, np.ndarray):
        assert a.dtype == np.float64 and a.flags.c_contiguous
        return C.c_void_p(a.ctypes.data), APOLLO_HOST_PTR
    # torch tensor
    assert a.dtype.__repr__().endswith("float64") and a.is_contiguous()
    if a.is_cuda:
        # the library works on its own stream: whatever torch queued that
        # produces or still reads this tensor must finish first (the library's
        # calls return with their own stream synchronised)
        if sync:
            import torch
            torch.cuda.current_stream(a.device).synchronize()
        return C.c_void_p(a.data_ptr()), APOLLO_DEVICE_PTR
    return C.c_void_p(a.data_ptr()), APOLLO_HOST_PTR


class NodalDG2d:
    """One nodal-DG discretisation on the GPU (Apollo ``Kind = nodalDG2d``)."""

    def __init__(self, N: int, cfl: float, equation: str | None, eq_params, mesh: Mesh, bcs=(), device: int = 0,
                 stream: int | None = None, part=None, rank: int = 0, numerical_flux: str = "LF",
                 deck: str | None = None, sources=()):
        """``part`` (int32 [K], optional): a partition of ``mesh``; the handle then
        holds the elements with ``part == rank`` (apollo_dg_set_mesh_partition)
        and steps through ``apollo_b200.distributed.DistNodalDG2d``.
        ``deck`` (with ``equation`` None): Apollo input-deck text whose
        equation block, boundary-condition list and sources configure the
        handle (apollo_dg_set_equation_text, apollo_dg_add_bc_text,
        apollo_dg_add_source_text).  ``sources``: (kind, out_range, params)
        triples (apollo_dg_add_source)."""
        self.lib = load_library()
        cfg = _Config(N, cfl, device, C.c_void_p(stream) if stream else None)
        h = C.c_void_p()
        self._check(self.lib.apollo_dg_create(C.byref(cfg), C.byref(h)), h=None)
        self.h = h
        if equation is None:
            self._check(self.lib.apollo_dg_set_equation_text(h, None, deck.encode()))
            self._check(self.lib.apollo_dg_add_bc_text(h, None, deck.encode()))
            self._check(self.lib.apollo_dg_add_source_text(h, None, deck.encode()))
        else:
            p = np.asarray(list(eq_params), dtype=np.float64)
            self._check(self.lib.apollo_dg_set_equation(h, equation.encode(), p.ctypes.data_as(_dp), len(p)))
            self._check(self.lib.apollo_dg_set_numerical_flux(h, numerical_flux.encode()))
        for kind, params in bcs:
            bp = np.asarray(list(params), dtype=np.float64)
            self._check(self.lib.apollo_dg_add_bc(h, kind.encode(), bp.ctypes.data_as(_dp), len(bp)))
        for kind, out, params in sources:
            o = np.asarray(list(out), dtype=np.int32)
            sp = np.asarray(list(params) or [0.0], dtype=np.float64)
            self._check(self.lib.apollo_dg_add_source(h, kind.encode(), o.ctypes.data_as(_ip), len(o),
                                                      sp.ctypes.data_as(_dp), len(params)))
        self.mesh = mesh
        if part is None:
            self._check(self.lib.apollo_dg_set_mesh(
                h, mesh.nverts, mesh.vx.ctypes.data_as(_dp), mesh.vy.ctypes.data_as(_dp), mesh.K,
                mesh.etov.ctypes.data_as(_ip), mesh.face_tag.ctypes.data_as(_ip), mesh.vert_canon.ctypes.data_as(_ip)))
        else:
            self.part = np.ascontiguousarray(part, dtype=np.int32)
            assert self.part.shape == (mesh.K,)
            self._check(self.lib.apollo_dg_set_mesh_partition(
                h, mesh.nverts, mesh.vx.ctypes.data_as(_dp), mesh.vy.ctypes.data_as(_dp), mesh.K,
                mesh.etov.ctypes.data_as(_ip), mesh.face_tag.ctypes.data_as(_ip), mesh.vert_canon.ctypes.data_as(_ip),
                self.part.ctypes.data_as(_ip), rank))
        self.rank = rank
        self.stream = stream
        self.N = N
        self.equation = equation
        self.K = self.lib.apollo_dg_num_elements(h)
        self.Np = self.lib.apollo_dg_num_nodes(h)
        self.m = self.lib.apollo_dg_num_fields(h)
        self.Nc = self.lib.apollo_dg_num_cubature(h)
        self.Ng = self.lib.apollo_dg_num_gauss(h)

    def _check(self, code, h=0):
        if code != 0:
            hh = self.h if h == 0 else h
            msg = self.lib.apollo_dg_last_error(hh).decode() if hh else ""
            raise ApolloError(code, msg)

    def close(self):
        if getattr(self, "h", None):
            self.lib.apollo_dg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_launch_shape(self, grid_share: int = 1, tile_shape: int = 0):
        """The persistent grids' share of the SMs and the mixed stage's operand chunking."""
        self._check(self.lib.apollo_dg_set_launch_shape(self.h, grid_share, tile_shape))

    def set_fp64_kernels(self, fused=True):
        """Float64 stage kernels: True (1) the fused stage kernel, False (0, the
        default) the volume, face and LIFT kernels, 2 the fused one on meshes
        of about one wave of tiles."""
        self._check(self.lib.apollo_dg_set_fp64_kernels(self.h, int(fused)))

    def averaging_weights(self):
        """w[Np]: an element's average of a nodal field is sum_n w[n] u[n]."""
        w = np.empty(self.Np)
        self._check(self.lib.apollo_dg_averaging_weights(self.h, w.ctypes.data_as(_dp)))
        return w

    def write_vtu(self, path: str, U=None, time: float | None = None):
        """The resident state (or U) as a VTK file (apollo_b200.vtk.write_vtu)."""
        from .vtk import write_vtu
        write_vtu(path, self.mesh, self.get_state() if U is None else U, averages=self.averaging_weights(), time=time)

    def set_limiter(self, kind: str | None, params=()):
        """Apollo's limiter on every stage input: kind "eulerLimiterHW" (params
        gas_gamma, min_pressure, min_density) or "tuAliabadiLimiter" (no
        params: the equation's own); None removes it."""
        p = np.asarray(list(params), dtype=np.float64)
        self._check(self.lib.apollo_dg_set_limiter(self.h, kind.encode() if kind else None,
                                                   p.ctypes.data_as(_dp) if len(p) else None, len(p)))

    @property
    def shape(self):
        return (self.K, self.Np, self.m)

    @property
    def dofs(self) -> int:
        return self.K * self.Np * self.m

    def node_coords(self):
        x = np.empty((self.K, self.Np))
        y = np.empty((self.K, self.Np))
        self._check(self.lib.apollo_dg_node_coords(self.h, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp)))
        return x, y

    def set_state(self, U):
        p, where = _ptr(U)
        self._check(self.lib.apollo_dg_set_state(self.h, p, where))

    def get_state(self, out=None):
        if out is None:
            out = np.empty(self.shape)
        p, where = _ptr(out)
        self._check(self.lib.apollo_dg_get_state(self.h, p, where))
        return out

    def set_state_async(self, U):
        """Queue the copy of U into the resident state on the handle's stream
        and return (apollo_dg_set_state_async): the caller orders it against
        the stream that produces U, and a host U should be page-locked."""
        p, where = _ptr(U, sync=False)
        self._check(self.lib.apollo_dg_set_state_async(self.h, p, where))

    def get_state_async(self, out):
        """Queue the copy of the resident state into ``out`` (a device tensor or
        page-locked host memory) on the handle's stream and return."""
        p, where = _ptr(out, sync=False)
        self._check(self.lib.apollo_dg_get_state_async(self.h, p, where))
        return out

    def init_dt(self) -> float:
        dt = C.c_double()
        self._check(self.lib.apollo_dg_init_dt(self.h, C.byref(dt)))
        return dt.value

    def step(self, t: float, dt: float, u, out=None, precision: str = "fp64"):
        """One RHS evaluation out = L(u) (WxNodalDG2dMethod::step); returns (out, suggested dt)."""
        if out is None:
            out = np.empty(self.shape) if isinstance(u, np.ndarray) else u.new_empty(u.shape)
        pi, wi = _ptr(u)
        po, wo = _ptr(out)
        assert wi == wo
        s = C.c_double()
        self._check(self.lib.apollo_dg_rhs(self.h, t, dt, pi, po, C.byref(s), wi, PREC[precision]))
        return out, s.value

    def advance(self, nsteps: int, t: float, dt: float, tend: float = -1.0, precision: str = "fp64"):
        """Advance the resident state; returns (t, dt for the next step)."""
        tt, dd = C.c_double(t), C.c_double(dt)
        self._check(self.lib.apollo_dg_step(self.h, nsteps, C.byref(tt), C.byref(dd), tend, PREC[precision]))
        return tt.value, dd.value

    def advance_async(self, nsteps: int, t: float, dt: float, precision: str = "fp64"):
        self._check(self.lib.apollo_dg_step_async(self.h, nsteps, t, dt, PREC[precision]))

    def synchronize(self):
        self._check(self.lib.apollo_dg_synchronize(self.h))

    def time(self):
        tt, dd = C.c_double(), C.c_double()
        self._check(self.lib.apollo_dg_get_time(self.h, C.byref(tt), C.byref(dd)))
        return tt.value, dd.value

    def kernel_times(self, iters: int = 10, precision: str = "fp64"):
        """Average ms per kernel of one RHS on the resident state."""
        ms = np.zeros(8)
        nk = C.c_int()
        self._check(self.lib.apollo_dg_kernel_times(self.h, PREC[precision], iters, ms.ctypes.data_as(_dp),
                                                    C.byref(nk)))
        return ms[:nk.value]

    def integrals(self, U=None):
        sums = np.zeros(self.m)
        if U is None:
            self._check(self.lib.apollo_dg_integrals(self.h, None, 0, sums.ctypes.data_as(_dp)))
        else:
            p, where = _ptr(U)
            self._check(self.lib.apollo_dg_integrals(self.h, p, where, sums.ctypes.data_as(_dp)))
        return sums

    def square_integrals(self, U=None):
        """Per-field integrals of U^2 over the mesh (apollo_dg_energy)."""
        sums = np.zeros(self.m)
        if U is None:
            self._check(self.lib.apollo_dg_energy(self.h, None, 0, sums.ctypes.data_as(_dp)))
        else:
            p, where = _ptr(U)
            self._check(self.lib.apollo_dg_energy(self.h, p, where, sums.ctypes.data_as(_dp)))
        return sums

    # ---- derivatives (float64; fixed step size dt) ------------------------------
    def _like(self, a, out):
        if out is not None:
            return out
        return np.empty(self.shape) if isinstance(a, np.ndarray) else a.new_empty(a.shape)

    def forward_fixed(self, nsteps: int, t0: float, dt: float, checkpoint_every: int):
        """Advance the resident state by nsteps fixed steps, keeping checkpoints for backward()."""
        self._check(self.lib.apollo_dg_forward_fixed(self.h, nsteps, t0, dt, checkpoint_every))

    def forward_revolve(self, nsteps: int, t0: float, dt: float, snapshots: int):
        """Advance the resident state by nsteps fixed steps with `snapshots`
        state slots (the initial state's included) for backward(), which then
        follows the binomial (revolve) schedule."""
        self._check(self.lib.apollo_dg_forward_revolve(self.h, nsteps, t0, dt, snapshots))

    @staticmethod
    def revolve_schedule(nsteps: int, snapshots: int):
        """(forward steps the revolve backward sweep runs, states the forward
        pass stores) for a trajectory of nsteps steps; host only."""
        lib = load_library()
        n, k = C.c_longlong(), C.c_int()
        rc = lib.apollo_dg_revolve_schedule(nsteps, snapshots, C.byref(n), C.byref(k))
        if rc:
            raise ApolloError(rc, "revolve schedule")
        return n.value, k.value

    def recomputed_steps(self) -> int:
        n = C.c_longlong()
        self._check(self.lib.apollo_dg_adjoint_stats(self.h, C.byref(n)))
        return n.value

    def backward(self, ubar_T, out=None):
        """dJ/dU(0) of the last forward_fixed trajectory, given dJ/dU(T)."""
        out = self._like(ubar_T, out)
        pi, wi = _ptr(ubar_T)
        po, wo = _ptr(out)
        assert wi == wo
        self._check(self.lib.apollo_dg_backward(self.h, pi, po, wi))
        return out

    def tangent(self, nsteps: int, t0: float, dt: float, du0, out=None):
        """Advance the resident state and return (dU(T)/dU(0)) du0."""
        out = self._like(du0, out)
        pi, wi = _ptr(du0)
        po, wo = _ptr(out)
        assert wi == wo
        self._check(self.lib.apollo_dg_tangent(self.h, nsteps, t0, dt, pi, po, wi))
        return out

    def rhs_jvp(self, t: float, x, v, out=None):
        out = self._like(x, out)
        (px, wx), (pv, _), (po, _) = _ptr(x), _ptr(v), _ptr(out)
        self._check(self.lib.apollo_dg_rhs_jvp(self.h, t, px, pv, po, wx))
        return out

    def rhs_vjp(self, t: float, x, w, out=None):
        out = self._like(x, out)
        (px, wx), (pw, _), (po, _) = _ptr(x), _ptr(w), _ptr(out)
        self._check(self.lib.apollo_dg_rhs_vjp(self.h, t, px, pw, po, wx))
        return out

    def adjoint_memory(self) -> int:
        b = C.c_size_t()
        self._check(self.lib.apollo_dg_adjoint_memory(self.h, C.byref(b)))
        return b.value


class NodalDG2dBatch:
    """Independent meshes of one equation (any sizes, orders 2..5) stepped
    together: each order's instances share one discretisation and every stage
    is one persistent launch; one CUDA graph per step (apollo_dg_batch_*)."""

    def __init__(self, cfl: float, equation: str, eq_params, bcs=(), device: int = 0, numerical_flux: str = "LF"):
        self.lib = load_library()
        cfg = _Config(0, cfl, device, None)
        h = C.c_void_p()
        p = np.asarray(list(eq_params), dtype=np.float64)
        self._check(self.lib.apollo_dg_batch_create(C.byref(cfg), equation.encode(), p.ctypes.data_as(_dp), len(p),
                                                    C.byref(h)), h=None)
        self.h = h
        if numerical_flux != "LF":
            self._check(self.lib.apollo_dg_batch_set_numerical_flux(h, numerical_flux.encode()))
        for kind, params in bcs:
            bp = np.asarray(list(params), dtype=np.float64)
            self._check(self.lib.apollo_dg_batch_add_bc(h, kind.encode(), bp.ctypes.data_as(_dp), len(bp)))
        self.info = []

    def _check(self, code, h=0):
        if code != 0:
            hh = self.h if h == 0 else h
            msg = self.lib.apollo_dg_batch_last_error(hh).decode() if hh else ""
            raise ApolloError(code, msg)

    def add_mesh(self, N: int, mesh: Mesh) -> int:
        inst = C.c_int()
        canon = mesh.vert_canon.ctypes.data_as(_ip) if mesh.vert_canon is not None else None
        tag = mesh.face_tag.ctypes.data_as(_ip) if mesh.face_tag is not None else None
        self._check(self.lib.apollo_dg_batch_add_mesh(self.h, N, mesh.nverts, mesh.vx.ctypes.data_as(_dp),
                                                      mesh.vy.ctypes.data_as(_dp), mesh.K, mesh.etov.ctypes.data_as(_ip),
                                                      tag, canon, C.byref(inst)))
        return inst.value

    def finalize(self):
        self._check(self.lib.apollo_dg_batch_finalize(self.h))
        self.info = []
        for i in range(self.lib.apollo_dg_batch_size(self.h)):
            N, K, Np, m = C.c_int(), C.c_int(), C.c_int(), C.c_int()
            self._check(self.lib.apollo_dg_batch_instance_info(self.h, i, C.byref(N), C.byref(K), C.byref(Np),
                                                               C.byref(m)))
            self.info.append({"N": N.value, "K": K.value, "Np": Np.value, "m": m.value})

    def __len__(self):
        return len(self.info)

    def shape(self, i):
        d = self.info[i]
        return (d["K"], d["Np"], d["m"])

    def node_coords(self, i):
        K, Np, _ = self.shape(i)
        x, y = np.empty((K, Np)), np.empty((K, Np))
        self._check(self.lib.apollo_dg_batch_node_coords(self.h, i, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp)))
        return x, y

    def set_state(self, i, U):
        p, where = _ptr(U)
        self._check(self.lib.apollo_dg_batch_set_state(self.h, i, p, where))

    def get_state(self, i, out=None):
        if out is None:
            out = np.empty(self.shape(i))
        p, where = _ptr(out)
        self._check(self.lib.apollo_dg_batch_get_state(self.h, i, p, where))
        return out

    def init_dt(self):
        dt = np.zeros(len(self))
        self._check(self.lib.apollo_dg_batch_init_dt(self.h, dt.ctypes.data_as(_dp)))
        return dt

    def step(self, nsteps: int, t, dt, precision: str = "fp64"):
        """Advance every instance nsteps steps from its (t[i], dt[i]); returns the new (t, dt) arrays."""
        t = np.ascontiguousarray(t, dtype=np.float64).copy()
        dt = np.ascontiguousarray(dt, dtype=np.float64).copy()
        self._check(self.lib.apollo_dg_batch_step(self.h, nsteps, t.ctypes.data_as(_dp), dt.ctypes.data_as(_dp),
                                                  PREC[precision]))
        return t, dt

    def autotune(self, precision: str = "mixed"):
        """Pick each order group's launch and tile shape by timing; returns
        {order: (grid share, tile shape)}."""
        share = np.zeros(4, dtype=np.int32)
        shape = np.zeros(4, dtype=np.int32)
        self._check(self.lib.apollo_dg_batch_autotune(self.h, PREC[precision], share.ctypes.data_as(_ip),
                                                      shape.ctypes.data_as(_ip)))
        return {N: (int(share[N - 2]), int(shape[N - 2])) for N in range(2, 6) if share[N - 2]}

    def close(self):
        if getattr(self, "h", None):
            self.lib.apollo_dg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
