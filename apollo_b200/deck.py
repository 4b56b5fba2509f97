"""Apollo input decks (.pin cryptset text) through the C ABI's deck calls.

Apollo's nodalDG2d sub-solver reads polynomialOrder, cfl and the lists
Equations, boundaryConditions and Limiter from its input deck
(src/subsolvers/wxnodaldg2dmethod.cc:50-152); each list names a block whose
Kind and keys configure one plugin.  ``deck_*`` return what the library reads
from such text; ``solver_from_deck`` builds a handle from it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .dg import ApolloError, NodalDG2d, _Config, load_library

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _enc(s):
    return None if s is None else s.encode()


def _raise(code, err):
    raise ApolloError(code, err.value.decode())


def deck_config(text: str):
    """(polynomialOrder, cfl) of the deck's nodalDG2d block."""
    lib = load_library()
    cfg = _Config(0, 0.0, 0, None)
    err = C.create_string_buffer(256)
    rc = lib.apollo_dg_deck_config(text.encode(), C.byref(cfg), err, 256)
    if rc:
        _raise(rc, err)
    return cfg.polynomial_order, cfg.cfl


def deck_equation(text: str, kind: str | None = None):
    """(kind, params, numerical flux) of the deck's equation block."""
    lib = load_library()
    k = C.create_string_buffer(64)
    nf = C.create_string_buffer(32)
    err = C.create_string_buffer(256)
    p = np.zeros(8)
    n = C.c_int()
    rc = lib.apollo_dg_deck_equation(_enc(kind), text.encode(), k, 64, p.ctypes.data_as(_dp), C.byref(n), nf, 32,
                                     err, 256)
    if rc:
        _raise(rc, err)
    return k.value.decode(), tuple(p[:n.value]), nf.value.decode()


def deck_bcs(text: str, kind: str | None = None):
    """[(kind, params)] of the deck's boundaryConditions, in order."""
    lib = load_library()
    err = C.create_string_buffer(256)
    count = C.c_int()
    rc = lib.apollo_dg_deck_bc(_enc(kind), text.encode(), 0, C.byref(count), None, 0, None, None, err, 256)
    if rc:
        _raise(rc, err)
    out = []
    for i in range(count.value):
        k = C.create_string_buffer(64)
        p = np.zeros(8)
        n = C.c_int()
        rc = lib.apollo_dg_deck_bc(_enc(kind), text.encode(), i, C.byref(count), k, 64, p.ctypes.data_as(_dp),
                                   C.byref(n), err, 256)
        if rc:
            _raise(rc, err)
        out.append((k.value.decode(), tuple(p[:n.value])))
    return out


def deck_limiter(text: str, kind: str | None = None):
    """(kind, params) of the deck's limiter, or None when it lists none."""
    lib = load_library()
    k = C.create_string_buffer(64)
    err = C.create_string_buffer(256)
    p = np.zeros(8)
    n = C.c_int()
    rc = lib.apollo_dg_deck_limiter(_enc(kind), text.encode(), k, 64, p.ctypes.data_as(_dp), C.byref(n), err, 256)
    if rc:
        _raise(rc, err)
    return (k.value.decode(), tuple(p[:n.value])) if k.value else None


def solver_from_deck(text: str, mesh, device: int = 0, stream: int | None = None) -> NodalDG2d:
    """A handle configured by the deck (order, cfl, equation with its numerical
    flux, boundary conditions, limiter) on ``mesh``."""
    N, cfl = deck_config(text)
    s = NodalDG2d(N, cfl, None, None, mesh, device=device, stream=stream, deck=text)
    s._check(s.lib.apollo_dg_set_limiter_text(s.h, None, text.encode()))
    return s
