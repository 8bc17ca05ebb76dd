"""The plain FP64 GPU path (gpu_method 3): one BDF integration per group of
n_reactors_max reactors with a shared step size, order and WRMS norm, driven
from the host kernel by kernel, as the reference's GPU branch of the
cfd_plugin integrates a batch with one CVODE instance
(applications/cfd_plugin/zerork_reactor_manager.cpp:909-1054,
solver_cvode.cpp:52).  End states against the CPU oracle's tight-tolerance
run at the bound the batched integrators meet (tests/test_integrator_gpu.py),
the group split, the failure semantics, and the options the path rejects.
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


def _tight_check(ot, T, P, Y, dt, Tg, Yg, **kw):
    nt = os.cpu_count() or 1
    To, Po, Yo, so = ot.solve(T, P, Y, dt, nthreads=nt, **kw)
    Tt, Pt, Yt, st = ot.solve(T, P, Y, dt, nthreads=nt, rtol=1e-12, atol=1e-24, max_steps=400000,
                              fail_caps=0, **kw)
    ok = (so["status"] == 0) & (st["status"] == 0)
    assert ok.sum() >= max(1, len(T) // 2)
    eo_T, eg_T = np.abs(To - Tt)[ok], np.abs(Tg - Tt)[ok]
    eo_Y = np.max(np.abs(Yo - Yt), axis=1)[ok]
    eg_Y = np.max(np.abs(Yg - Yt), axis=1)[ok]
    assert np.all(eg_T <= 50 * np.maximum(eo_T, 10 * np.median(eo_T)) + 1e-5 * Tt[ok]), (eg_T, eo_T)
    assert np.all(eg_Y <= 50 * np.maximum(eo_Y, 10 * np.median(eo_Y)) + 1e-8), (eg_Y, eo_Y)


@pytest.mark.parametrize("gmax", [16, 5])
def test_group_end_states(gpu, gmax, mech_dir):
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    import zerork_b200 as zb
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 16, "c1", seed=11)
    p = Plugin(mf, tf, gpu_method=3, n_reactors_max=gmax)
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert p.solve(1e-3, Tg, Pg, Yg) == 0
    st = p.last_stats()
    # 16 reactors in groups of at most 5: 5, 5, then the last two split 3 + 3
    assert st["groups"] == (1 if gmax == 16 else 4)
    assert st["nfailed"] == 0 and st["group_steps"] > 0
    # every norm costs a host synchronization: more syncs than group steps
    assert st["syncs"] > st["group_steps"] and st["launches"] > st["syncs"]
    _tight_check(oracle_tables(zb.Mechanism(mf, tf, device=False)), T, P, Y, 1e-3, Tg, Yg)


def test_group_shares_the_step_size(gpu, mech_dir):
    """A group takes one step sequence: the per-reactor statistics of all
    reactors of a group are the group's, and a group of reactors of uneven
    stiffness takes more steps than its least stiff reactor alone."""
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 8, "c1", seed=11)
    grp = Plugin(mf, tf, gpu_method=3, n_reactors_max=8)
    cost_g = grp.set_aux_field("COST", np.zeros(8))
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert grp.solve(1e-3, Tg, Pg, Yg) == 0
    assert np.all(cost_g == cost_g[0]) and grp.last_stats()["group_steps"] == cost_g[0]
    per = Plugin(mf, tf, gpu_method=1)
    cost_p = per.set_aux_field("COST", np.zeros(8))
    T1, P1, Y1 = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert per.solve(1e-3, T1, P1, Y1) == 0
    assert cost_g[0] > np.min(cost_p)


def test_group_sources_constant_pressure_ignition(gpu, mech_dir):
    """Constant pressure with pressure-rate and mass-fraction sources, and
    ignition times, against the oracle with the same sources."""
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    import zerork_b200 as zb
    g, (mf, tf) = synth("c1_h2", mech_dir)
    pm = zb.Mechanism(mf, tf, device=False)
    n = 12
    T, P, Y = mechgen.reactor_states(g, n, "c1", seed=5)
    rng = np.random.default_rng(5)
    dpdt = rng.uniform(-1e6, 1e7, n)
    ys = np.zeros_like(Y)
    ys[:, pm.species.index("N2")] = 5.0
    p = Plugin(mf, tf, gpu_method=3, n_reactors_max=6, constant_volume=0,
               delta_temperature_ignition=400.0)
    p.set_aux_field("DPDT", dpdt)
    p.set_aux_field("Y_SRC", ys)
    ign = p.set_aux_field("IGNITION_TIME", np.full(n, -1.0))
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert p.solve(1e-3, Tg, Pg, Yg) == 0
    ot = oracle_tables(pm)
    kw = dict(constant_volume=0, dpdt=dpdt, y_src=ys)
    _tight_check(ot, T, P, Y, 1e-3, Tg, Yg, **kw)
    _, _, _, so = ot.solve(T, P, Y, 1e-3, nthreads=os.cpu_count() or 1, dT_ign=400.0, **kw)
    hit = so["t_ign"] > 0
    assert np.array_equal(ign > 0, hit)
    if hit.any():
        assert np.all(np.abs(ign[hit] - so["t_ign"][hit]) <= 2e-2 * so["t_ign"][hit])


def test_group_failure_fails_the_group(gpu, mech_dir):
    """A group whose every attempt fails reports FAILED_SOLVE for each of its
    reactors and leaves their states unchanged."""
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 6, "c1", seed=3)
    p = Plugin(mf, tf, gpu_method=3, rel_tol=1e-30, abs_tol=1e-40, cvode_num_retries=2, max_steps=300)
    Tg, Pg, Yg = T.copy(), P.copy(), Y.copy()
    assert p.solve(1e-3, Tg, Pg, Yg, raise_on_fail=False) == 7
    assert p.last_stats()["nfailed"] == 6
    assert np.array_equal(Tg, T) and np.array_equal(Yg, Y)


@pytest.mark.parametrize("opt", [dict(lu_fp32=1), dict(delta_temperature_ignition=400.0, stop_after_ignition=1)])
def test_group_rejects_batched_only_options(gpu, opt, mech_dir):
    from zerork_b200 import mechgen
    from zerork_b200.plugin import Plugin, PluginError
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, 4, "c1", seed=3)
    p = Plugin(mf, tf, gpu_method=3, **opt)
    with pytest.raises(PluginError):
        p.solve(1e-4, T.copy(), P.copy(), Y.copy())
