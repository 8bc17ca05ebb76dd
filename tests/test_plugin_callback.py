"""The plugin's per-step callback (zerork_reactor_set_callback_fn,
zerork_cfd_plugin.h:44-46), called as the reference's CVODE loop calls it
(solver_cvode.cpp:225-262): after every accepted step of every reactor with
the reactor's id (zerork_reactor_set_reactor_ids, else its index), the call
counter, the time from the call's start, the step, y = [Y, T / Tref] and the
interpolant's derivative; at the first crossing of T0 +
delta_temperature_ignition one more call at the crossing (CVode's root
return); a nonzero return ends that reactor's integration there.

Checked on the GPU for both integrators:
* a callback that returns 0 changes no result (bit-identical to the run
  without it), is called once per accepted step (the solve's step total),
  with strictly increasing times whose differences are the dt argument, the
  call counter 1, 2, ... and the last state equal to the returned one;
* the first step is first order, so its derivative times its step is the
  state change (rounding of one difference);
* a nonzero return at a reactor's third call ends that reactor at that
  record's state and leaves the others bit-identical;
* with delta_temperature_ignition the crossing record sits at the reactor's
  IGNITION_TIME, and with stop_after_ignition it is the reactor's last call
  and its state the returned one.
"""
import numpy as np
import pytest

from conftest import have_gpu, synth

pytestmark = pytest.mark.gpu

DT = 1e-3
TREF = 1000.0


@pytest.fixture(scope="module")
def gpu():
    if not have_gpu():
        pytest.skip("no CUDA device")
    return True


def _case(mech_dir, n=8):
    from zerork_b200 import mechgen
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T, P, Y = mechgen.reactor_states(g, n, "c1", seed=11)
    return mf, tf, T, P, Y


def _run(mf, tf, T, P, Y, cb=None, ids=None, ign=False, **opts):
    from zerork_b200.plugin import Plugin
    p = Plugin(mf, tf, reference_temperature=TREF, **opts)
    if cb is not None:
        p.set_callback(cb)
    if ids is not None:
        p.set_reactor_ids(ids)
    t_ign = p.set_aux_field("IGNITION_TIME", np.full(len(T), -1.0)) if ign else None
    Tg, Pg, Yg = T.copy(), P.copy(), np.ascontiguousarray(Y.copy())
    assert p.solve(DT, Tg, Pg, Yg) == 0
    return Tg, Pg, Yg, p.last_stats(), t_ign


class Recorder:
    def __init__(self, stop_id=None, stop_at=None):
        self.rec = {}
        self.stop_id, self.stop_at = stop_id, stop_at

    def __call__(self, rid, steps, t, dt, y, dy):
        r = self.rec.setdefault(rid, [])
        r.append((steps, t, dt, y.copy(), dy.copy()))
        return int(rid == self.stop_id and len(r) == self.stop_at)


@pytest.mark.parametrize("method", [1, 2])
def test_callback_records_every_step(gpu, method, mech_dir):
    mf, tf, T, P, Y = _case(mech_dir)
    n, ns = len(T), Y.shape[1]
    T0, P0, Y0, s0, _ = _run(mf, tf, T, P, Y, gpu_method=method)
    ids = np.arange(n, dtype=np.int32) * 7 + 100
    rec = Recorder()
    T1, P1, Y1, s1, _ = _run(mf, tf, T, P, Y, cb=rec, ids=ids, gpu_method=method)
    assert np.array_equal(T0, T1) and np.array_equal(P0, P1) and np.array_equal(Y0, Y1)
    assert sorted(rec.rec) == sorted(ids.tolist())
    assert sum(len(v) for v in rec.rec.values()) == s1["nsteps"] == s0["nsteps"]
    for k, rid in enumerate(ids):
        r = rec.rec[int(rid)]
        steps = np.array([e[0] for e in r])
        t = np.array([e[1] for e in r])
        dt = np.array([e[2] for e in r])
        assert np.array_equal(steps, np.arange(1, len(r) + 1))
        assert np.all(np.diff(t) > 0) and abs(t[-1] - DT) <= 1e-15 * DT
        np.testing.assert_allclose(dt, np.diff(np.concatenate([[0.0], t])), rtol=0, atol=1e-18)
        y_last = r[-1][3]
        assert y_last.shape == (ns + 1,)
        assert np.array_equal(y_last[:ns], Y1[k])
        assert abs(y_last[ns] * TREF - T1[k]) <= 1e-12 * T1[k]
        # the first step is BDF order 1: y' h = y_1 - y_0
        y0 = np.concatenate([Y[k], [T[k] / TREF]])
        d1 = r[0][3] - y0
        sc = np.abs(y0) + np.abs(r[0][3])
        assert np.all(np.abs(r[0][4] * r[0][2] - d1) <= 1e-12 * sc + 1e-300)


@pytest.mark.parametrize("method", [1, 2])
def test_callback_nonzero_return_ends_reactor(gpu, method, mech_dir):
    mf, tf, T, P, Y = _case(mech_dir)
    ns = Y.shape[1]
    T0, P0, Y0, _, _ = _run(mf, tf, T, P, Y, gpu_method=method)
    full = Recorder()
    _run(mf, tf, T, P, Y, cb=full, gpu_method=method)
    k = 5
    assert len(full.rec[k]) > 3
    rec = Recorder(stop_id=k, stop_at=3)
    T1, P1, Y1, _, _ = _run(mf, tf, T, P, Y, cb=rec, gpu_method=method)
    assert len(rec.rec[k]) == 3
    y3 = full.rec[k][2][3]
    assert np.array_equal(Y1[k], y3[:ns])
    assert abs(T1[k] - y3[ns] * TREF) <= 1e-12 * T1[k]
    others = np.arange(len(T)) != k
    assert np.array_equal(T1[others], T0[others]) and np.array_equal(Y1[others], Y0[others])
    for j in np.nonzero(others)[0]:
        assert len(rec.rec[int(j)]) == len(full.rec[int(j)])


@pytest.mark.parametrize("method", [1, 2])
def test_callback_ignition_crossing(gpu, method, mech_dir):
    mf, tf, T, P, Y = _case(mech_dir, n=16)
    ns = Y.shape[1]
    rec = Recorder()
    _, _, _, st, ign = _run(mf, tf, T, P, Y, cb=rec, ign=True, gpu_method=method,
                            delta_temperature_ignition=400.0)
    hit = ign > 0
    assert np.any(hit) and np.any(~hit)
    assert sum(len(v) for v in rec.rec.values()) == st["nsteps"] + int(hit.sum())
    for k in np.nonzero(hit)[0]:
        t = np.array([e[1] for e in rec.rec[int(k)]])
        assert np.all(np.diff(t) > 0)
        j = int(np.nonzero(t == ign[k])[0][0])
        assert j + 1 < len(t)  # the step that crossed follows
        Tc = rec.rec[int(k)][j][3][ns] * TREF
        assert abs(Tc - (T[k] + 400.0)) < 25.0
    # stop_after_ignition: the crossing is the last call, its state returned
    rec2 = Recorder()
    T2, _, Y2, _, ign2 = _run(mf, tf, T, P, Y, cb=rec2, ign=True, gpu_method=method,
                              delta_temperature_ignition=400.0, stop_after_ignition=1)
    assert np.array_equal(ign2 > 0, hit)
    for k in np.nonzero(hit)[0]:
        last = rec2.rec[int(k)][-1]
        assert last[1] == ign2[k]
        assert np.array_equal(last[3][:ns], Y2[k])
        np.testing.assert_allclose(T2[k], T[k] + 400.0, rtol=0, atol=1e-6)
