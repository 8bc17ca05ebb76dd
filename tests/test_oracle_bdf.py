"""The oracle integrator (oracle/zrk_bdf.c) against an independent stiff
integrator.

CVODE is not vendored in the reference (SUNDIALS 5.8.0 is a download), so
the oracle restates a published BDF; this cross-check integrates the same
reactors with SciPy's BDF (solve_ivp, the Shampine-Reichelt NDF family) on
the oracle's own right-hand side and Jacobian, both at tight tolerance, and
requires the end states to agree within a few times the requested tolerance.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import oracle_tables, synth


def _rhs_and_jac(ot, T0, P0, Y0):
    import zrk_oracle as zo
    L = ot.lib
    kin = zo.ZoKinetics()
    L.zo_kinetics_oracle(ot.ptr, C.byref(kin))
    L.zo_reactor_new.restype = C.c_void_p
    L.zo_reactor_new.argtypes = [C.c_void_p, C.POINTER(zo.ZoKinetics), C.c_double, C.c_double,
                                 C.c_double]
    L.zo_reactor_free.argtypes = [C.c_void_p]
    L.zo_reactor_set_density.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p]
    L.zo_reactor_rhs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.zo_jac_values.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p]
    r = L.zo_reactor_new(ot.ptr, C.byref(kin), 1.0, 1e-30, 1e22)
    Y0 = np.ascontiguousarray(Y0, dtype=np.float64)
    L.zo_reactor_set_density(r, T0, P0, Y0.ctypes.data)
    pat = ot.pat.contents
    n, nnz = pat.n, pat.nnz
    cp = np.ctypeslib.as_array(pat.col_ptr, (n + 1,)).copy()
    ri = np.ctypeslib.as_array(pat.row_idx, (nnz,)).copy()

    def f(t, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(n)
        assert L.zo_reactor_rhs(r, y.ctypes.data, out.ctypes.data) == 0
        return out

    def jac(t, y):
        from scipy.sparse import csc_matrix
        y = np.ascontiguousarray(y, dtype=np.float64)
        fy = f(t, y)
        v = np.zeros(nnz)
        L.zo_jac_values(r, ot.pat, y.ctypes.data, fy.ctypes.data, v.ctypes.data, None)
        return csc_matrix((v, ri, cp), shape=(n, n))

    return f, jac, lambda: L.zo_reactor_free(r)


@pytest.mark.parametrize("idx", [0, 3, 7])
def test_oracle_bdf_matches_scipy_bdf(idx, mech_dir):
    scipy_integrate = pytest.importorskip("scipy.integrate")
    import zerork_b200 as zb
    from zerork_b200 import mechgen
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 8, "c1", seed=11)
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    dt, rtol, atol = 1e-3, 1e-10, 1e-22
    To, Po, Yo, st = ot.solve(T[idx:idx + 1], P[idx:idx + 1], Y[idx:idx + 1], dt,
                              rtol=rtol, atol=atol, max_steps=200000)
    assert st["status"][0] == 0
    f, jac, free = _rhs_and_jac(ot, T[idx], P[idx], Y[idx])
    try:
        y0 = np.concatenate([Y[idx], [T[idx]]])
        sol = scipy_integrate.solve_ivp(f, (0.0, dt), y0, method="BDF", rtol=rtol, atol=atol,
                                        jac=jac)
    finally:
        free()
    assert sol.status == 0
    ys = sol.y[:, -1]
    assert abs(ys[-1] - To[0]) <= 1e-6 * To[0]
    assert np.max(np.abs(ys[:-1] - Yo[0])) <= 1e-7


@pytest.mark.parametrize("cv", [1, 0])
def test_oracle_bdf_sources_match_scipy_radau(cv, mech_dir):
    """The oracle BDF with pressure-rate and energy sources, at constant
    volume and at constant pressure, against SciPy's Radau on the oracle's
    own right-hand side (time-dependent through the sources): end
    temperature within 5e-3 K and mass fractions within 1e-6.  The
    right-hand side takes T from the reference's energy inversion, which
    stops at 1e-6 K, so neither integrator can be driven much tighter."""
    scipy_integrate = pytest.importorskip("scipy.integrate")
    import zerork_b200 as zb
    from zerork_b200 import mechgen
    g, (mf, tf) = synth("c1_h2", mech_dir)
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    T, P, Y = mechgen.reactor_states(g, 2, "c1", seed=23)
    T, P, Y = T[1:], P[1:], Y[1:]
    dpdt, esrc, dt = np.array([2.6e6]), np.array([7.6e7]), 5e-4
    To, Po, Yo, so = ot.solve(T, P, Y, dt, dpdt=dpdt, e_src=esrc, constant_volume=cv,
                              rtol=1e-10, atol=1e-22, max_steps=400000, fail_caps=0)
    assert so["status"][0] == 0

    def f(t, y):
        return ot.reactor_rhs(1 - cv, T, P, Y, np.array([t]), y[None, :], dpdt=dpdt, e_src=esrc)[0]

    y0 = np.concatenate([Y[0], T])
    sol = scipy_integrate.solve_ivp(f, (0.0, dt), y0, method="Radau", rtol=1e-9, atol=1e-20)
    assert sol.status == 0
    assert abs(sol.y[-1, -1] - To[0]) < 5e-3, (sol.y[-1, -1], To[0])
    assert np.max(np.abs(sol.y[:-1, -1] - Yo[0])) < 1e-6


def test_oracle_per_step_failure_limits(mech_dir):
    """CVODE's per-step limits (7 error-test, 10 convergence failures per
    step; order and step cut after the 3rd error-test failure) end an
    attempt that the energy inversion's 1e-6 K noise floor keeps rejecting
    at rtol 1e-10: with the limits the constant-pressure reactor with
    pressure-rate and energy sources needs retries (or fails), without them
    it grinds through in one attempt."""
    import zerork_b200 as zb
    from zerork_b200 import mechgen
    g, (mf, tf) = synth("c1_h2", mech_dir)
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    T, P, Y = mechgen.reactor_states(g, 2, "c1", seed=23)
    T, P, Y = T[1:], P[1:], Y[1:]
    src = dict(dpdt=np.array([2.6e6]), e_src=np.array([7.6e7]), constant_volume=0, rtol=1e-10,
               atol=1e-22, max_steps=400000)
    _, _, _, capped = ot.solve(T, P, Y, 5e-4, **src)
    _, _, _, free = ot.solve(T, P, Y, 5e-4, fail_caps=0, **src)
    assert free["status"][0] == 0 and free["retries"][0] == 0
    assert capped["status"][0] != 0 or capped["retries"][0] > 0
