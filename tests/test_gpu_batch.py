"""Batched ensembles (apollo_dg_batch_*): independent meshes of mixed orders
stepped together must give each instance exactly what a handle of its own gives."""
import numpy as np
import pytest

from apollo_b200 import ApolloError, NodalDG2d, NodalDG2dBatch, problems
from golden_cases import rel_l2

pytestmark = pytest.mark.gpu

# (vertex grid n, order N, vortex strength beta): sizes from a few elements to
# a few thousand, every order, two instances of one order in one group
CASES = [(9, 2, 1.5), (17, 4, 5.0), (5, 3, 2.0), (25, 5, 3.5), (13, 4, 1.0), (33, 3, 4.0)]


def _problems():
    return [problems.euler_vortex(n=n, N=N, seed=10 + i, beta=b) for i, (n, N, b) in enumerate(CASES)]


def _batch(ps):
    b = NodalDG2dBatch(ps[0].cfl, ps[0].equation, ps[0].eq_params)
    ids = [b.add_mesh(p.N, p.mesh) for p in ps]
    assert ids == list(range(len(ps)))
    b.finalize()
    return b


def _single(p):
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    s.set_state(U0)
    return s, U0


def test_batch_layout_and_coords():
    ps = _problems()
    b = _batch(ps)
    assert len(b) == len(ps)
    for i, p in enumerate(ps):
        s, _ = _single(p)
        assert b.shape(i) == s.shape
        x, y = b.node_coords(i)
        xs, ys = s.node_coords()
        np.testing.assert_array_equal(x, xs)
        np.testing.assert_array_equal(y, ys)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_single_handles(precision):
    ps = _problems()
    b = _batch(ps)
    singles = [_single(p) for p in ps]
    for i, (s, U0) in enumerate(singles):
        b.set_state(i, U0)
        np.testing.assert_array_equal(b.get_state(i), U0)
    dt_b = b.init_dt()
    dt_s = np.array([s.init_dt() for s, _ in singles])
    np.testing.assert_array_equal(dt_b, dt_s)
    nsteps = 7
    t_b, d_b = b.step(nsteps, np.zeros(len(ps)), dt_b, precision=precision)
    for i, (s, _) in enumerate(singles):
        t, d = s.advance(nsteps, 0.0, dt_s[i], precision=precision)
        Ub, Us = b.get_state(i), s.get_state()
        e = rel_l2(Ub, Us)
        print(i, precision, "rel", e, "t", t_b[i], t, "dt", d_b[i], d)
        # every element and face is computed exactly as its own handle computes
        # it, and the per-instance wave-speed maximum is order-independent: the
        # batch is bit-identical in both precisions
        assert e == 0.0
        assert t_b[i] == t and d_b[i] == d


def test_batch_continues_across_calls():
    """Two calls of n steps equal one call of 2n steps (t, dt and traces carried)."""
    ps = _problems()[:3]
    b1, b2 = _batch(ps), _batch(ps)
    for i, p in enumerate(ps):
        s, U0 = _single(p)
        b1.set_state(i, U0)
        b2.set_state(i, U0)
    dt0 = b1.init_dt()
    for prec in ("mixed", "fp64"):
        t1, d1 = b1.step(4, np.zeros(len(ps)), dt0, precision=prec)
        t1, d1 = b1.step(4, t1, d1, precision=prec)
        t2, d2 = b2.step(8, np.zeros(len(ps)), dt0, precision=prec)
        np.testing.assert_allclose(t1, t2, rtol=1e-14)
        for i in range(len(ps)):
            assert rel_l2(b1.get_state(i), b2.get_state(i)) <= 1e-13
        for i, p in enumerate(ps):
            s, U0 = _single(p)
            b1.set_state(i, U0)
            b2.set_state(i, U0)


def test_batch_autotune_keeps_state():
    ps = _problems()
    b = _batch(ps)
    U0 = []
    for i, p in enumerate(ps):
        _, u = _single(p)
        b.set_state(i, u)
        U0.append(u)
    choice = b.autotune("mixed")
    assert set(choice) == {p.N for p in ps}
    assert all(share in (1, 2, 4) and shape in (0, 1) for share, shape in choice.values())
    for i in range(len(ps)):
        np.testing.assert_array_equal(b.get_state(i), U0[i])
    # stepping after tuning still matches a single handle
    dt = b.init_dt()
    t, d = b.step(3, np.zeros(len(ps)), dt, precision="mixed")
    s, _ = _single(ps[1])
    s.set_launch_shape(*choice[ps[1].N])  # the kernel the batch picked for that order
    ts, _ = s.advance(3, 0.0, dt[1], precision="mixed")
    np.testing.assert_array_equal(b.get_state(1), s.get_state())
    assert t[1] == ts


def test_batch_vortex_errors_per_instance():
    """Each instance of a small ensemble tracks its exact vortex, and mixed
    tracks float64 to 1e-6 relative L2, instance by instance."""
    ps = problems.euler_ensemble(count=6, k_range=(1000, 4000), seed=3)
    b = _batch(ps)
    for i, p in enumerate(ps):
        x, y = b.node_coords(i)
        b.set_state(i, np.ascontiguousarray(p.ic(x, y)))
    dt = b.init_dt()
    t64, _ = b.step(20, np.zeros(len(ps)), dt, precision="fp64")
    U64 = [b.get_state(i) for i in range(len(ps))]
    for i, p in enumerate(ps):
        x, y = b.node_coords(i)
        b.set_state(i, np.ascontiguousarray(p.ic(x, y)))
    tmx, _ = b.step(20, np.zeros(len(ps)), dt, precision="mixed")
    # dt follows each run's own wave speeds (float32 in the mixed stage)
    np.testing.assert_allclose(tmx, t64, rtol=1e-6)
    for i, p in enumerate(ps):
        x, y = b.node_coords(i)
        ex = p.exact(x, y, t64[i])
        e_exact = rel_l2(U64[i], ex)
        e_mixed = rel_l2(b.get_state(i), U64[i])
        print(i, p.N, p.mesh.K, p.meta["beta"], "exact", e_exact, "mixed", e_mixed)
        assert e_exact <= 2e-2
        assert e_mixed <= 1e-6


def test_batch_errors():
    ps = _problems()[:2]
    b = NodalDG2dBatch(ps[0].cfl, ps[0].equation, ps[0].eq_params)
    with pytest.raises(ApolloError):
        b.add_mesh(6, ps[0].mesh)
    with pytest.raises(ApolloError):
        b.finalize()          # no meshes
    b.add_mesh(ps[0].N, ps[0].mesh)
    b.finalize()
    with pytest.raises(ApolloError):
        b.add_mesh(ps[1].N, ps[1].mesh)   # after finalize
    with pytest.raises(ApolloError):
        b.set_state(5, np.zeros(b.shape(0)))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_with_hll_flux_and_boundaries(precision):
    """A batch with Apollo's HLL flux and the channel's four boundary kinds
    steps every instance exactly as a handle of its own does."""
    from golden_cases import load
    g = load("euler_hll_N3")
    bcs = g["bcs"]
    b = NodalDG2dBatch(float(g["cfl"]), g["equation"], g["eqp"][:3], bcs=bcs, numerical_flux="HLL")
    for _ in range(2):
        b.add_mesh(int(g["N"]), g["mesh"])
    b.finalize()
    U = [g["U0"], g["U0"] * np.array([1.0, 1.02, 0.98, 0.0, 1.01])]
    for i, u in enumerate(U):
        b.set_state(i, np.ascontiguousarray(u))
    dt = b.init_dt()
    t, d = b.step(3, np.zeros(2), dt, precision=precision)
    for i, u in enumerate(U):
        s = NodalDG2d(int(g["N"]), float(g["cfl"]), g["equation"], g["eqp"][:3], g["mesh"], bcs=bcs,
                      numerical_flux="HLL")
        s.set_state(np.ascontiguousarray(u))
        ts, ds = s.advance(3, 0.0, dt[i], precision=precision)
        np.testing.assert_array_equal(b.get_state(i), s.get_state())
        assert t[i] == ts and d[i] == ds
        s.close()
