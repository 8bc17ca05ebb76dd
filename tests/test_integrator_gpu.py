"""GPU batched integrator through the cfd_plugin C ABI, against the CPU oracle.

The oracle (oracle/zrk_bdf.c) integrates the same reactors with the same BDF
method but a dense LU with partial pivoting on the CPU; the GPU uses a
shared-memory Gauss-Jordan inverse (method 1) or a warp-level sparse LU with
static pivots (method 2), so step sequences differ and end states are
compared at the integration tolerance: both are also compared with a
tight-tolerance oracle run (rtol 1e-12), and the GPU error must be within
  |T_gpu - T_tight| <= 50 * |T_oracle - T_tight| + 1e-5 * T
  max_k |Y_gpu - Y_tight| <= 50 * max_k |Y_oracle - Y_tight| + 1e-8
per reactor: the oracle's own error at rtol 1e-8 sets the scale (two valid
integrations at the same tolerance with different step sequences differ by
a small multiple of it).  The per-reactor scale is floored at 10x the median
oracle error over the batch, since a reactor whose oracle run happens to be
far more accurate than the batch does not make a different valid
integration of it less accurate.
"""
import os

import numpy as np
import pytest

from conftest import have_gpu, oracle_tables, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    if not have_gpu():
        pytest.skip("no CUDA device")
    return True


def _solve(mf, tf, T, P, Y, dt, **opts):
    from zerork_b200.plugin import Plugin
    p = Plugin(mf, tf, **opts)
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    rc = p.solve(dt, Tg, Pg, Yg, raise_on_fail=False)
    return rc, Tg, Pg, Yg, p


def _check_against_tight(ot, T, P, Y, dt, Tg, Yg):
    nt = os.cpu_count() or 1
    To, Po, Yo, so = ot.solve(T, P, Y, dt, nthreads=nt)
    Tt, Pt, Yt, st = ot.solve(T, P, Y, dt, nthreads=nt, rtol=1e-12, atol=1e-24, max_steps=400000, fail_caps=0)
    ok = (so["status"] == 0) & (st["status"] == 0)
    assert ok.sum() >= max(1, len(T) // 2)
    eo_T = np.abs(To - Tt)[ok]
    eg_T = np.abs(Tg - Tt)[ok]
    eo_Y = np.max(np.abs(Yo - Yt), axis=1)[ok]
    eg_Y = np.max(np.abs(Yg - Yt), axis=1)[ok]
    fT, fY = 10 * np.median(eo_T), 10 * np.median(eo_Y)
    assert np.all(eg_T <= 50 * np.maximum(eo_T, fT) + 1e-5 * Tt[ok]), (eg_T, eo_T)
    assert np.all(eg_Y <= 50 * np.maximum(eo_Y, fY) + 1e-8), (eg_Y, eo_Y)
    return eg_T, eg_Y


@pytest.mark.parametrize("fp32,method", [(0, 1), (1, 1), (0, 2), (1, 2)])
def test_c1_end_states(gpu, fp32, method, mech_dir):
    from zerork_b200 import mechgen
    import zerork_b200 as zb
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 16, "c1", seed=11)
    rc, Tg, Pg, Yg, p = _solve(mf, tf, T, P, Y, 1e-3, lu_fp32=fp32, gpu_method=method)
    assert rc == 0
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    _check_against_tight(ot, T, P, Y, 1e-3, Tg, Yg)
    st = p.last_stats()
    assert st["nfailed"] == 0 and st["nsteps"] > 0
    # mass fractions stay normalised; pressure from the ideal gas at fixed density
    assert np.allclose(Yg.sum(axis=1), 1.0, atol=1e-8)


@pytest.mark.parametrize("fp32", [0, 1])
def test_c3_subset_end_states(gpu, fp32, mech_dir):
    from zerork_b200 import mechgen
    import zerork_b200 as zb
    g, (mf, tf) = synth("c3_160", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 6, "c3", seed=5)
    rc, Tg, Pg, Yg, p = _solve(mf, tf, T, P, Y, 2e-4, lu_fp32=fp32)
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    _check_against_tight(ot, T, P, Y, 2e-4, Tg, Yg)


@pytest.mark.parametrize("fp32", [0, 1])
def test_c4_subset_end_states(gpu, fp32, mech_dir):
    """650 species: the dense block does not fit, the warp-level sparse LU path
    runs (FP32: the factor preconditions an FP64 Krylov solve)."""
    from zerork_b200 import mechgen
    import zerork_b200 as zb
    g, (mf, tf) = synth("c4_650", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 6, "c4", seed=11)
    rc, Tg, Pg, Yg, p = _solve(mf, tf, T, P, Y, 5e-4, lu_fp32=fp32)
    assert rc == 0
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    _check_against_tight(ot, T, P, Y, 5e-4, Tg, Yg)


def test_mass_fraction_sources(gpu, mech_dir):
    """ZERORK_FIELD_Y_SRC: per-reactor mass-fraction sources added to the
    species equations and to the energy balance
    (reactor_constant_volume_cpu.cpp:108-113), against the oracle with the
    same sources."""
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    import zerork_b200 as zb
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 12, "c1", seed=11)
    pm = zb.Mechanism(mf, tf, device=False)
    ys = np.zeros_like(Y)
    ys[:, pm.species.index("N2")] = 10.0  # 1 % of mass added per ms as N2
    p = Plugin(mf, tf)
    p.set_aux_field("Y_SRC", ys)
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert p.solve(1e-3, Tg, Pg, Yg) == 0
    ot = oracle_tables(pm)
    nt = os.cpu_count() or 1
    To, Po, Yo, so = ot.solve(T, P, Y, 1e-3, nthreads=nt, y_src=ys)
    Tt, Pt, Yt, st = ot.solve(T, P, Y, 1e-3, nthreads=nt, y_src=ys, rtol=1e-12, atol=1e-24,
                              max_steps=400000, fail_caps=0)
    ok = (so["status"] == 0) & (st["status"] == 0)
    eo_T, eo_Y = np.abs(To - Tt)[ok], np.max(np.abs(Yo - Yt), axis=1)[ok]
    fT, fY = 10 * np.median(eo_T), 10 * np.median(eo_Y)
    assert np.all(np.abs(Tg - Tt)[ok] <= 50 * np.maximum(eo_T, fT) + 1e-5 * Tt[ok])
    assert np.all(np.max(np.abs(Yg - Yt), axis=1)[ok] <= 50 * np.maximum(eo_Y, fY) + 1e-8)
    # the sources were applied: about 1e-2 of mass added per reactor
    assert np.allclose(Yg.sum(axis=1), 1.01, atol=1e-6)


def test_ignition_time(gpu, mech_dir):
    """ZERORK_FIELD_IGNITION_TIME with delta_temperature_ignition: the first
    time T reaches T0 + delta (the root function of
    reactor_nvector_serial.cpp:774-784), located by linear interpolation
    between accepted steps, against the oracle and its tight-tolerance run."""
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    import zerork_b200 as zb
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 16, "c1", seed=11)
    p = Plugin(mf, tf, delta_temperature_ignition=400.0)
    ign = p.set_aux_field("IGNITION_TIME", np.full(16, -7.0))
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert p.solve(1e-3, Tg, Pg, Yg) == 0
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    nt = os.cpu_count() or 1
    _, _, _, so = ot.solve(T, P, Y, 1e-3, nthreads=nt, dT_ign=400.0)
    _, _, _, st = ot.solve(T, P, Y, 1e-3, nthreads=nt, dT_ign=400.0, rtol=1e-12, atol=1e-24,
                           max_steps=400000, fail_caps=0)
    to, tt = so["t_ign"], st["t_ign"]
    assert np.array_equal(ign < 0, tt < 0) and np.any(tt > 0)  # the same reactors ignite
    hit = tt > 0
    eo = np.abs(to - tt)[hit]
    eg = np.abs(ign - tt)[hit]
    assert np.all(eg <= 50 * np.maximum(eo, 10 * np.median(eo)) + 1e-3 * tt[hit]), (eg, eo)
    # reactors that did not reach T0 + 400 K keep the caller's value (the
    # reference sets the root time only when CVODE found one,
    # zerork_reactor_manager.cpp:1128-1131)
    assert np.all(ign[~hit] == -7.0)


@pytest.mark.parametrize("method", [1, 2])
def test_stop_after_ignition(gpu, method, mech_dir):
    """stop_after_ignition (solver_cvode.cpp:259-263): each reactor's call
    ends at its ignition time, with the state interpolated linearly between
    the accepted steps around the crossing, so T ends at T0 + 400 K; against
    the oracle with the same option."""
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    import zerork_b200 as zb
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 16, "c1", seed=11)
    p = Plugin(mf, tf, delta_temperature_ignition=400.0, stop_after_ignition=1, gpu_method=method)
    ign = p.set_aux_field("IGNITION_TIME", np.full(16, -1.0))
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert p.solve(1e-3, Tg, Pg, Yg) == 0
    hit = ign > 0
    assert np.any(hit) and np.any(~hit)
    np.testing.assert_allclose(Tg[hit], T[hit] + 400.0, rtol=0, atol=1e-6)
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    To, Po, Yo, so = ot.solve(T, P, Y, 1e-3, nthreads=os.cpu_count() or 1, dT_ign=400.0, stop_ign=1)
    assert np.array_equal(so["t_ign"] > 0, hit)
    np.testing.assert_allclose(To[hit], T[hit] + 400.0, rtol=0, atol=1e-6)
    # ignition times and stopped states agree at the integration tolerance
    assert np.all(np.abs(ign[hit] - so["t_ign"][hit]) <= 1e-4 * so["t_ign"][hit])
    assert np.max(np.abs(Yg[hit] - Yo[hit])) < 1e-4
    # the others ran the whole interval as without the option
    q = Plugin(mf, tf, delta_temperature_ignition=400.0, gpu_method=method)
    T2, P2, Y2 = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert q.solve(1e-3, T2, P2, Y2) == 0
    assert np.array_equal(T2[~hit], Tg[~hit]) and np.array_equal(Y2[~hit], Yg[~hit])


@pytest.mark.parametrize("method", [1, 2])
def test_abstol_dens(gpu, method, mech_dir):
    """abstol_dens = 1: species absolute tolerances abs_tol / (rho / W_k *
    1e-3) (reactor_nvector_serial.cpp:107-119), with abs_tol 1e-12 (a
    molar-concentration tolerance in mol/cm^3); against the oracle with the
    same option and its tight-tolerance run, and different from the run
    without the option."""
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    import zerork_b200 as zb
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 12, "c1", seed=11)
    rc, Tg, Pg, Yg, p = _solve(mf, tf, T, P, Y, 1e-3, abstol_dens=1, abs_tol=1e-12, gpu_method=method)
    assert rc == 0
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    nt = os.cpu_count() or 1
    To, Po, Yo, so = ot.solve(T, P, Y, 1e-3, nthreads=nt, abstol_dens=1, atol=1e-12)
    Tt, Pt, Yt, st = ot.solve(T, P, Y, 1e-3, nthreads=nt, rtol=1e-12, atol=1e-24, max_steps=400000, fail_caps=0)
    ok = (so["status"] == 0) & (st["status"] == 0)
    eo_T, eg_T = np.abs(To - Tt)[ok], np.abs(Tg - Tt)[ok]
    assert np.all(eg_T <= 50 * np.maximum(eo_T, 10 * np.median(eo_T)) + 1e-5 * Tt[ok])
    # the option changes the step sequence: steps differ from the default run
    rc2, T2, P2, Y2, p2 = _solve(mf, tf, T, P, Y, 1e-3, abs_tol=1e-12, gpu_method=method)
    assert p.last_stats()["nsteps"] != p2.last_stats()["nsteps"]


def test_hopeless_reactors_fail_cleanly(gpu, mech_dir):
    """At rtol 1e-30 no reactor can meet the error test in FP64: every
    attempt ends (max_steps, or CVODE's per-step failure limits of
    integrator.h), the call returns FAILED_SOLVE for each reactor and leaves
    its state unchanged (zerork_reactor_manager.cpp:1123-1137).  The limits
    themselves are shown on the oracle in tests/test_oracle_bdf.py."""
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 4, "c1", seed=3)
    for method in (1, 2):
        p = Plugin(mf, tf, rel_tol=1e-30, abs_tol=1e-40, cvode_num_retries=2, max_steps=500,
                   gpu_method=method)
        Tg, Pg, Yg = T.copy(), P.copy(), Y.copy()
        rc = p.solve(1e-3, Tg, Pg, Yg, raise_on_fail=False)
        assert rc == 7
        st = p.last_stats()
        assert st["nfailed"] == 4 and st["nsteps"] <= 4 * 2 * 500
        assert np.array_equal(Tg, T) and np.array_equal(Yg, Y)


def _src_case(g, pm, n, seed):
    """C1 reactors with pressure-rate, energy and mass-fraction sources; a
    quarter of the reactors have none."""
    from zerork_b200 import mechgen
    T, P, Y = mechgen.reactor_states(g, n, "c1", seed=seed)
    rng = np.random.default_rng(seed)
    on = rng.uniform(size=n) >= 0.25
    dpdt = np.where(on, rng.uniform(-1e6, 1e7, n), 0.0)       # up to 0.1 bar per ms
    esrc = np.where(on, rng.uniform(-1e8, 1e8, n), 0.0)       # up to ~100 K per ms
    ys = np.zeros_like(Y)
    ys[:, pm.species.index("N2")] = np.where(on, 5.0, 0.0)
    return T, P, Y, dpdt, esrc, ys


@pytest.mark.parametrize("cv,method,fp32,ysrc", [(1, 1, 0, False), (0, 1, 0, False),
                                                 (1, 2, 0, False), (0, 2, 0, False),
                                                 (0, 1, 0, True), (1, 1, 0, True),
                                                 (1, 1, 1, False), (0, 2, 1, False)])
def test_pressure_energy_sources_and_constant_pressure(gpu, cv, method, fp32, ysrc, mech_dir):
    """Constant-volume (constant_volume = 1) and constant-pressure
    (constant_volume = 0) reactors with ZERORK_FIELD_DPDT and ZERORK_FIELD_E_SRC
    sources (reactor_constant_volume_cpu.cpp:64-128,
    reactor_constant_pressure_cpu.cpp:71-135), optionally with Y_SRC, on both
    integrators and both precisions, against the oracle with the same
    sources: end T, P and Y within the integration-tolerance bound of the
    module docstring.  The reference run is at rtol 1e-10: with an energy
    source the right-hand side takes T from the reference's energy inversion,
    which stops at 1e-6 K, and tighter runs stall on that noise."""
    from zerork_b200.plugin import Plugin
    import zerork_b200 as zb
    g, (mf, tf) = synth("c1_h2", mech_dir)
    pm = zb.Mechanism(mf, tf, device=False)
    n, dt = 16, 1e-3
    T, P, Y, dpdt, esrc, ys = _src_case(g, pm, n, 21 + cv + 2 * method)
    p = Plugin(mf, tf, constant_volume=cv, gpu_method=method, lu_fp32=fp32)
    p.set_aux_field("DPDT", dpdt)
    p.set_aux_field("E_SRC", esrc)
    if ysrc:
        p.set_aux_field("Y_SRC", ys)
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert p.solve(dt, Tg, Pg, Yg) == 0
    ot = oracle_tables(pm)
    nt = os.cpu_count() or 1
    src = dict(dpdt=dpdt, e_src=esrc, y_src=ys if ysrc else None, constant_volume=cv)
    To, Po, Yo, so = ot.solve(T, P, Y, dt, nthreads=nt, **src)
    Tt, Pt, Yt, st = ot.solve(T, P, Y, dt, nthreads=nt, rtol=1e-10, atol=1e-22, max_steps=400000, fail_caps=0,
                              **src)
    ok = (so["status"] == 0) & (st["status"] == 0)
    assert ok.sum() >= n - 2
    for g_, o_, t_, rel in ((Tg, To, Tt, 1e-5), (Pg, Po, Pt, 1e-8)):
        eo, eg = np.abs(o_ - t_)[ok], np.abs(g_ - t_)[ok]
        assert np.all(eg <= 50 * np.maximum(eo, 10 * np.median(eo)) + rel * np.abs(t_[ok])), (eg, eo)
    eo_Y, eg_Y = np.max(np.abs(Yo - Yt), axis=1)[ok], np.max(np.abs(Yg - Yt), axis=1)[ok]
    assert np.all(eg_Y <= 50 * np.maximum(eo_Y, 10 * np.median(eo_Y)) + 1e-8)
    # at constant pressure without mass sources the end pressure is P0 + dpdt dt
    if cv == 0 and not ysrc:
        assert np.allclose(Pg, P + dpdt * dt, rtol=1e-14, atol=0.0)
    # the energy source acts: against a run without it, the end temperature
    # moves the way the source points
    Tn, Pn, Yn = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    q = Plugin(mf, tf, constant_volume=cv, gpu_method=method, lu_fp32=fp32)
    q.set_aux_field("DPDT", dpdt)
    if ysrc:
        q.set_aux_field("Y_SRC", ys)
    assert q.solve(dt, Tn, Pn, Yn) == 0
    big = np.abs(esrc) > 1e7
    assert np.all(np.sign(Tg - Tn)[big] == np.sign(esrc)[big])


@pytest.mark.parametrize("cv,method", [(1, 1), (0, 1), (1, 2)])
def test_fixed_temperature_reactors(gpu, cv, method, mech_dir):
    """always_solve_temperature = 0: reactors whose input TEMPERATURE_DELTA is
    not positive integrate at their initial temperature and report the
    temperature of their energy at the end composition; the others solve the
    temperature (zerork_reactor_manager.cpp:1107-1113,
    reactor_constant_volume_cpu.cpp:51-56).  Against the oracle with the same
    per-reactor choice."""
    from zerork_b200.plugin import Plugin
    import zerork_b200 as zb
    g, (mf, tf) = synth("c1_h2", mech_dir)
    pm = zb.Mechanism(mf, tf, device=False)
    from zerork_b200 import mechgen
    n, dt = 16, 1e-3
    T, P, Y = mechgen.reactor_states(g, n, "c1", seed=31)
    tdel_in = np.where(np.arange(n) % 2 == 0, 0.0, 50.0)
    esrc = np.where(np.arange(n) % 4 == 0, 3e7, 0.0)
    p = Plugin(mf, tf, constant_volume=cv, gpu_method=method, always_solve_temperature=0)
    tdel = p.set_aux_field("TEMPERATURE_DELTA", tdel_in.copy())
    p.set_aux_field("E_SRC", esrc)
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert p.solve(dt, Tg, Pg, Yg) == 0
    ot = oracle_tables(pm)
    nt = os.cpu_count() or 1
    fix = (tdel_in <= 0).astype(np.int32)
    src = dict(e_src=esrc, fix_T=fix, constant_volume=cv)
    To, Po, Yo, so = ot.solve(T, P, Y, dt, nthreads=nt, **src)
    Tt, Pt, Yt, st = ot.solve(T, P, Y, dt, nthreads=nt, rtol=1e-10, atol=1e-22, max_steps=400000, fail_caps=0,
                              **src)
    ok = (so["status"] == 0) & (st["status"] == 0)
    assert ok.sum() >= n - 2
    for g_, o_, t_, rel in ((Tg, To, Tt, 1e-5), (Pg, Po, Pt, 1e-8)):
        eo, eg = np.abs(o_ - t_)[ok], np.abs(g_ - t_)[ok]
        assert np.all(eg <= 50 * np.maximum(eo, 10 * np.median(eo)) + rel * np.abs(t_[ok])), (eg, eo)
    eo_Y, eg_Y = np.max(np.abs(Yo - Yt), axis=1)[ok], np.max(np.abs(Yg - Yt), axis=1)[ok]
    assert np.all(eg_Y <= 50 * np.maximum(eo_Y, 10 * np.median(eo_Y)) + 1e-8)
    # the fixed-temperature reactors differ from a run that solves every
    # temperature, and the output deltas feed the next call's choice
    q = Plugin(mf, tf, constant_volume=cv, gpu_method=method)
    q.set_aux_field("E_SRC", esrc)
    Ta, Pa, Ya = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert q.solve(dt, Ta, Pa, Ya) == 0
    assert np.all(np.abs(Ya - Yg).max(axis=1)[fix == 0] < 1e-6)
    assert np.any(np.abs(Ya - Yg).max(axis=1)[fix == 1] > 1e-6)
    d = Tg - T
    assert np.allclose(tdel, np.where(d < 2.0, 0.0, d))


def test_constant_pressure_c3_subset(gpu, mech_dir):
    """Constant-pressure C3 reactors (160 species, dense integrator) without
    sources: end state against the oracle, pressure unchanged."""
    from zerork_b200 import mechgen
    import zerork_b200 as zb
    g, (mf, tf) = synth("c3_160", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 6, "c3", seed=5)
    rc, Tg, Pg, Yg, p = _solve(mf, tf, T, P, Y, 2e-4, constant_volume=0)
    assert rc == 0
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    nt = os.cpu_count() or 1
    To, Po, Yo, so = ot.solve(T, P, Y, 2e-4, nthreads=nt, constant_volume=0)
    Tt, Pt, Yt, st = ot.solve(T, P, Y, 2e-4, nthreads=nt, constant_volume=0, rtol=1e-12, atol=1e-24,
                              max_steps=400000, fail_caps=0)
    ok = (so["status"] == 0) & (st["status"] == 0)
    assert ok.sum() >= 3
    eo_T, eg_T = np.abs(To - Tt)[ok], np.abs(Tg - Tt)[ok]
    assert np.all(eg_T <= 50 * np.maximum(eo_T, 10 * np.median(eo_T)) + 1e-5 * Tt[ok])
    eo_Y, eg_Y = np.max(np.abs(Yo - Yt), axis=1)[ok], np.max(np.abs(Yg - Yt), axis=1)[ok]
    assert np.all(eg_Y <= 50 * np.maximum(eo_Y, 10 * np.median(eo_Y)) + 1e-8)
    assert np.array_equal(Pg, P)


def test_failure_leaves_state_and_reports(gpu, mech_dir):
    """max_steps too small: FAILED_SOLVE, state unchanged, negative cost
    (zerork_reactor_manager.cpp:1123-1137)."""
    from zerork_b200 import mechgen
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 8, "c1", seed=3)
    from zerork_b200.plugin import Plugin
    p = Plugin(mf, tf, max_steps=3, cvode_num_retries=1)
    cost = p.set_aux_field("COST", np.zeros(8))
    Tg, Pg, Yg = T.copy(), P.copy(), Y.copy()
    rc = p.solve(1e-3, Tg, Pg, Yg, raise_on_fail=False)
    assert rc == 7  # FAILED_SOLVE
    assert np.array_equal(Tg, T) and np.array_equal(Yg, Y) and np.array_equal(Pg, P)
    assert np.all(cost < 0)


def test_cost_and_temperature_delta_fields(gpu, mech_dir):
    from zerork_b200 import mechgen
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 8, "c1", seed=4)
    from zerork_b200.plugin import Plugin
    p = Plugin(mf, tf)
    cost = p.set_aux_field("COST", np.ones(8))
    tdel = p.set_aux_field("TEMPERATURE_DELTA", np.zeros(8))
    Tg, Pg, Yg = T.copy(), P.copy(), Y.copy()
    assert p.solve(1e-3, Tg, Pg, Yg) == 0
    assert np.all(cost > 0)
    d = Tg - T
    assert np.allclose(tdel, np.where(d < 2.0, 0.0, d))
    # second call reuses the cost ordering and gives the same answer, replaying
    # the captured graph of the first call
    T2, P2, Y2 = T.copy(), P.copy(), Y.copy()
    assert p.solve(1e-3, T2, P2, Y2) == 0
    assert np.array_equal(T2, Tg) and np.array_equal(Y2, Yg)
    assert p.graph_stats() == {"captures": 1, "launches": 2}
    # a different interval is a different graph
    T3, P3, Y3 = T.copy(), P.copy(), Y.copy()
    assert p.solve(5e-4, T3, P3, Y3) == 0
    assert p.graph_stats() == {"captures": 2, "launches": 3}


def test_integrator_autotune(gpu, mech_dir):
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 64, "c1", seed=6)
    p = Plugin(mf, tf)
    T0, Y0 = T.copy(), Y.copy()
    best, ms = p.autotune(1e-3, T, P, Y)
    assert best in (128, 256, 512) and ms > 0
    assert p.get_int("gpu_threads") == best
    assert np.array_equal(T, T0) and np.array_equal(Y, Y0)
    assert p.solve(1e-3, T, P, Y) == 0
