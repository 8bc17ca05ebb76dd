"""The learned BDF predictor in the integrator (N3 form, no reference
counterpart): a network trained on the GPU, by the library's own kernels,
on (state, interval, next state) pairs that the integrator generated from
seeded initial states, attached to the cfd_plugin handle as the Newton
starting iterate.

Accuracy must be unchanged: the polynomial predictor still defines the
error estimate, every rejected learned start falls back to it, so end
states meet the same bound against the tight-tolerance oracle as the plain
integrator (tests/test_integrator_gpu.py).  The gain is measured, not
assumed: the test records Newton iterations per step, rejections, steps and
kernel time with and without the network.  At rtol 1e-8 the Newton
tolerance is a fraction of the error weights (about 1e-9 relative for
major species), far below what the network's regression error reaches, so
the learned start rarely converges and the gate turns it off: the measured
gain is near zero or negative, and the test bounds the loss.
"""
import json
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


def test_learned_predictor_accuracy_and_gain(gpu, mech_dir, tmp_path):
    import zerork_b200 as zb
    from zerork_b200 import mechgen, predictor as pr
    from zerork_b200.plugin import Plugin
    g, (mf, tf) = synth("c1_h2", mech_dir)
    T0, P0, Y0 = mechgen.reactor_states(g, 512, "c1", seed=1001)
    X, Tt = pr.generate_pairs(mf, tf, T0, P0, Y0, rounds=32, seed=5)
    assert X.shape[0] > 10000 and np.all(np.isfinite(X)) and np.all(np.isfinite(Tt))
    net, xs, ts, hist = pr.train(X, Tt, epochs=8, batch=1024, lr=1e-3)
    assert hist[-1] < 0.5 * hist[0], hist
    T, P, Y = mechgen.reactor_states(g, 32, "c1", seed=11)
    stats, ends = {}, {}
    for mode in ("plain", "learned"):
        p = Plugin(mf, tf)
        if mode == "learned":
            p.set_predictor(net, xs, ts)
        Tg, Pg, Yg = T.copy(), P.copy(), Y.copy()
        assert p.solve(1e-3, Tg, Pg, Yg) == 0
        stats[mode] = p.last_stats()
        ends[mode] = (Tg, Yg)
    s0, s1 = stats["plain"], stats["learned"]
    gain = {"newton_per_step": [s0["nnewt"] / s0["nsteps"], s1["nnewt"] / s1["nsteps"]],
            "rejected_per_step": [s0["nrej"] / s0["nsteps"], s1["nrej"] / s1["nsteps"]],
            "steps": [s0["nsteps"], s1["nsteps"]], "kernel_ms": [s0["kernel_ms"], s1["kernel_ms"]],
            "train_loss": hist}
    print("learned predictor (plain, learned):", json.dumps(gain))
    # the network was consulted: the learned starts change the Newton counts
    assert s1["nnewt"] != s0["nnewt"]
    # accuracy unchanged: same bound against the tight oracle as the plain path
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    nt = os.cpu_count() or 1
    To, Po, Yo, so = ot.solve(T, P, Y, 1e-3, nthreads=nt)
    Tw, Pw, Yw, sw = ot.solve(T, P, Y, 1e-3, nthreads=nt, rtol=1e-12, atol=1e-24, max_steps=400000, fail_caps=0)
    ok = (so["status"] == 0) & (sw["status"] == 0)
    eo_T, eo_Y = np.abs(To - Tw)[ok], np.max(np.abs(Yo - Yw), axis=1)[ok]
    fT, fY = 10 * np.median(eo_T), 10 * np.median(eo_Y)
    for mode in ("plain", "learned"):
        Tg, Yg = ends[mode]
        assert np.all(np.abs(Tg - Tw)[ok] <= 50 * np.maximum(eo_T, fT) + 1e-5 * Tw[ok]), mode
        assert np.all(np.max(np.abs(Yg - Yw), axis=1)[ok] <= 50 * np.maximum(eo_Y, fY) + 1e-8), mode
    # the fallback bounds the cost of a poor network
    assert s1["nnewt"] / s1["nsteps"] <= 2.0 * s0["nnewt"] / s0["nsteps"]
