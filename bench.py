#!/usr/bin/env python
"""Benchmark: FP64 net production rates + sparse reactor Jacobian (rate-eval states/s).

Workload: seeded synthetic CHEMKIN mechanism with 53 species (C,H,O,N,Ar) and
325 reactions (10% falloff, 15% third-body, 20% irreversible), 2^20
independent states (T U[300,3000] K, log10 P U[0,2] atm, Y ~ Dirichlet(0.5)).
One step = one fused pass over all states producing wdot [53] and the 1798
Jacobian values of the 54x54 reactor Jacobian per state.  Inputs (445 MB) and
outputs (15 GB) exceed the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU (torchrun): every rank integrates its own 2^20 states (weak
scaling, no collective on the data path); timing is the max over ranks.
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "c2_53"
METRIC = "rate-eval states/s"


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--states", type=int, default=1 << 20)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--launch", default="",
                   help="ts,v,warps,flags (bit 0 global workspace, bit 1 staged tables, bit 2 two "
                        "CTAs per SM): fixed rates-kernel mapping instead of the autotuner "
                        "(profiling captures of one known kernel)")
    p.add_argument("--reactors", type=int, default=4096,
                   help="reactors of the 160-species integration workload (0: skip)")
    p.add_argument("--no-learned", action="store_true",
                   help="skip the learned-predictor form of the integration leg")
    p.add_argument("--integration-suite", default="",
                   help="comma-separated integration configs (c1,c3,c4,c5) to run instead of the "
                        "rates headline: every form, with end-state tolerance verdicts")
    p.add_argument("--suite-scale", type=float, default=1.0,
                   help="fraction of each config's reactor count (bounded calibration runs)")
    p.add_argument("--suite-pairs", type=int, default=1 << 20,
                   help="training pairs of the learned predictor in the suite")
    p.add_argument("--integ-warm", type=int, default=1,
                   help="1: time each batched form on a second call in the first call's cost order; "
                        "0: one call per form, index order")
    p.add_argument("--plain-sample", type=int, default=256,
                   help="reactors the plain group path is timed on (a stratified sample)")
    p.add_argument("--integ-dt", type=float, default=2e-3,
                   help="integration interval per reactor in seconds (2 ms: the workload; "
                        "shorter only for bounded profiling captures)")
    return p.parse_args()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc, self.start = gpu, [], None, 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a while to start: wait (bounded) for its first
            # row and keep only the rows from the region itself
            deadline = time.time() + 5.0
            while not self.rows and time.time() < deadline:
                time.sleep(0.01)
            self.start = len(self.rows)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            # a short region may end between two samples: take the next one
            deadline = time.time() + 1.0
            while len(self.rows) <= self.start and time.time() < deadline:
                time.sleep(0.01)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = self.rows[self.start:]
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def traffic_per_state():
    """DRAM bytes per state of the rates+Jacobian kernel from the committed
    ncu summary (profiles/), or None."""
    p = os.path.join(ROOT, "profiles", "rates_jac_c2_ncu.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("dram_bytes_per_state")
    return None


def make_workload(directory, n, seed):
    from zerork_b200 import mechgen
    g = mechgen.generate(mechgen.SPECS[WORKLOAD])
    m, t = g.write(directory)
    T, P, Y = mechgen.rate_states(g, n, seed=seed)
    return g, (m, t), T, P, Y


def cpu_reference(files, T, P, Y, budget_s=12.0, nthreads=None):
    """The reference's own CPU mechanism library (oracle/_ref, default fmath exp
    build) with the restated plugin Jacobian assembly, OpenMP over states."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import zrk_oracle as zo
    kind = "fmath" if zo.ref_available("fmath") else "libc"
    if not zo.ref_available(kind):
        return None
    nthreads = nthreads or os.cpu_count()
    ref = zo.RefMechanism(files[0], files[1], kind=kind)
    ot = zo.OracleTables(ref.tables)
    # calibrate a bounded sample
    m = 64 * nthreads
    t0 = time.perf_counter()
    ref.batch_rates_jac(files, ot, T[:m], P[:m], Y[:m], nthreads=nthreads)
    dt = time.perf_counter() - t0
    m2 = int(min(len(T), max(m, m * budget_s / max(dt, 1e-6))))
    t0 = time.perf_counter()
    ref.batch_rates_jac(files, ot, T[:m2], P[:m2], Y[:m2], nthreads=nthreads)
    dt = time.perf_counter() - t0
    return {"value": m2 / dt, "unit": "states/s", "cores": nthreads, "kind": "reference",
            "sample": f"{m2} of the {len(T)} states, reference zerork::mechanism "
                      f"({kind} exp) + restated SetupJacobianSparse, {nthreads} OpenMP threads"}


def rates_tc_workload(files, T, P, Y, n_max=1 << 18):
    """The (T, C) states of the rates-only comparison: the rate workload's
    states as molar concentrations, species-major, in batches of n_max
    reactors (the reference GPU mechanism's nReactorsMax)."""
    import torch
    import zerork_b200 as zb
    pm = zb.Mechanism(*files, device=False)
    mw = pm.table("mw")
    rho = P / (8.314462618e3 * T * np.sum(Y / mw, axis=1))
    conc = rho[:, None] * Y / mw
    n = len(T)
    nb = min(n, n_max)
    dev = torch.device("cuda")
    batches = []
    for b0 in range(0, n - nb + 1, nb):
        Tb = torch.from_numpy(np.ascontiguousarray(T[b0:b0 + nb])).to(dev)
        Cb = torch.from_numpy(np.ascontiguousarray(conc[b0:b0 + nb].T)).to(dev)
        batches.append((Tb, Cb))
    return pm.nsp, pm.nstep, nb, batches


def _time_rates_tc(fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def rates_only_b200(files, T, P, Y, reps=5):
    """This repository's rates-from-concentrations kernel (zrk_rates_tc_dev:
    net, create, destroy and rates of progress, no Jacobian, no limiter) on
    the rates-only workload; the reference arm times the reference's own GPU
    path (mechanism_cuda::getReactionRates_CUDA_mr_dev) on the same states."""
    import torch
    import zerork_b200 as zb
    S, N, nb, batches = rates_tc_workload(files, T, P, Y)
    pm = zb.Mechanism(*files)
    kw = dict(dtype=torch.float64, device=torch.device("cuda"))
    outs = [torch.empty((S, nb), **kw) for _ in range(3)] + [torch.empty((N, nb), **kw)]
    L = zb.lib()

    def step():
        for Tb, Cb in batches:
            zb.check(L.zrk_rates_tc_dev(pm.handle, nb, nb, zb._ptr(Tb), zb._ptr(Cb), None,
                                        *[zb._ptr(o) for o in outs], None))
    ms = _time_rates_tc(step, reps)
    n = len(batches) * nb
    return {"workload": f"rates from (T, C), no Jacobian: {S} species / {N} steps, {n} states "
                        f"in batches of {nb}", "ms_per_step": ms, "states_per_s": n / (ms / 1e3),
            "bytes_per_state": 8 * (1 + S + 3 * S + N)}


def reference_gpu_rates(files, T, P, Y, reps=5):
    """The reference's own GPU rate path, mechanism_cuda::getReactionRates_CUDA_mr_dev
    (src/zerork/mechanism_cuda.cu:150-156), compiled unmodified for sm_100a into
    oracle/_ref/libzrk_ref_cuda.so, on the rates-only workload of
    rates_only_b200.  None when the library was not built or no GPU."""
    import ctypes as C
    import torch
    path = os.path.join(ROOT, "oracle", "_ref", "libzrk_ref_cuda.so")
    if not os.path.exists(path) or not torch.cuda.is_available():
        return None
    L = C.CDLL(path)
    vp = C.c_void_p
    L.zrkref_cuda_load.restype = vp
    L.zrkref_cuda_load.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]
    L.zrkref_cuda_free.argtypes = [vp]
    L.zrkref_cuda_rates.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp]
    S, N, nb, batches = rates_tc_workload(files, T, P, Y)
    h = L.zrkref_cuda_load(files[0].encode(), files[1].encode(), os.devnull.encode(), nb)
    if not h:
        return None
    kw = dict(dtype=torch.float64, device=torch.device("cuda"))
    outs = [torch.empty((S, nb), **kw) for _ in range(3)] + [torch.empty((N, nb), **kw)]
    ptrs = [o.data_ptr() for o in outs]

    def step():
        for Tb, Cb in batches:
            L.zrkref_cuda_rates(h, nb, Tb.data_ptr(), Cb.data_ptr(), *ptrs)
    ms = _time_rates_tc(step, reps)
    L.zrkref_cuda_free(h)
    n = len(batches) * nb
    return {"workload": f"rates from (T, C), no Jacobian: {S} species / {N} steps, {n} states "
                        f"in batches of {nb} (nReactorsMax)", "ms_per_step": ms,
            "states_per_s": n / (ms / 1e3),
            "source": "oracle/_ref/libzrk_ref_cuda.so (reference src/zerork CUDA sources, sm_100a)"}


def _run_form(mf, tf, T, P, Y, dt, opts, net=None, cost=None, warm=True):
    """A form through the cfd_plugin API with host arrays, as a CFD code calls
    it step after step: a first call (untimed, warm=True) fills the COST field
    and the timed call takes the reactors in that cost order (the plugin's
    sort_reactors); cost, if given, is the COST field to start from instead.
    Wall time around the timed call (host copies included).  Returns the
    form's record, the end states and the per-reactor cost (negative for a
    failed reactor)."""
    from zerork_b200.plugin import Plugin
    p = Plugin(mf, tf, **opts)
    if net is not None:
        p.set_predictor(*net)
    c = p.set_aux_field("COST", np.zeros(len(T)) if cost is None else np.array(cost, dtype=np.float64))
    if warm:
        Tg, Pg, Yg = T.copy(), P.copy(), Y.copy()
        p.solve(dt, Tg, Pg, Yg, raise_on_fail=False)
    Tg, Pg, Yg = T.copy(), P.copy(), Y.copy()
    t0 = time.perf_counter()
    rc = p.solve(dt, Tg, Pg, Yg, raise_on_fail=False)
    wall = time.perf_counter() - t0
    st = p.last_stats()
    cost_out = np.array(c)
    p.close()
    n = len(T)
    res = {"value": n / wall, "unit": "reactors/s", "reactors": n, "wall_s": wall,
           "kernel_ms": st["kernel_ms"], "status": rc, "failed": st["nfailed"],
           "steps": st["nsteps"], "newton_per_step": st["nnewt"] / max(1, st["nsteps"]),
           "rejected": st["nrej"], "factorizations": st["nlu"], "jacobians": st["njac"],
           "krylov_per_newton": st["nkry"] / max(1, st["nnewt"]),
           "h2d_bytes": int(T.nbytes + P.nbytes + Y.nbytes), "d2h_bytes": int(T.nbytes + P.nbytes + Y.nbytes)}
    if st.get("groups"):
        res.update(groups=st["groups"], group_steps=st["group_steps"], group_newton=st["group_newton"],
                   launches=st["launches"], host_syncs=st["syncs"], group_status=st["group_status"])
    return res, (Tg, Yg), cost_out


# The plain group path shares one step sequence among the reactors of a
# group, so a group of reactors of uneven stiffness needs far more steps than
# any of them alone: with the default 5000 steps per attempt every C3 group
# fails (measured: 5 attempts x 5000 steps, all 512 reactors of a group
# failed).  Its form runs with a step budget it can finish in.
PLAIN_MAX_STEPS = 200000

# The forms of the integration blocks.  "plain_fp64" is the plain FP64 GPU
# path: the reference's GPU algorithm (one BDF per group of n_reactors_max =
# 1024 reactors with a shared step size and WRMS norm, host-driven kernel by
# kernel, gpu_method 3).  The batched forms run every reactor with its own
# step control in one persistent graph-captured launch; "batched_fp32_learned"
# is the chosen form (batched + FP32 preconditioner + learned predictor).
FORMS = [("plain_fp64", dict(gpu_method=3, max_steps=PLAIN_MAX_STEPS), False),
         ("batched_fp64", dict(), False),
         ("batched_fp32", dict(lu_fp32=1), False),
         ("batched_fp64_learned", dict(), True),
         ("batched_fp32_learned", dict(lu_fp32=1), True)]


def _plain_sample(n, n_plain):
    """Reactor indices the plain group path is timed on: every k-th reactor
    (a stratified sample of the same states)."""
    if n_plain <= 0 or n_plain >= n:
        return np.arange(n)
    return np.arange(0, n, max(1, n // n_plain))[:n_plain]


def _plain_pick(n, n_plain, cost):
    """The plain path's reactors: a stratified sample of n_plain reactors
    without those the batched FP64 path failed (one failed reactor fails its
    whole group on the plain path), taken in the batched FP64 path's cost
    order (reactors of similar stiffness share a group: the order most
    favourable to a shared step size)."""
    ok = np.flatnonzero(cost > 0)
    idx = ok[_plain_sample(len(ok), n_plain)]
    note = (f"{len(idx)} reactors: every {max(1, len(ok) // len(idx))}th of the {len(ok)} reactors the "
            f"batched FP64 path integrated ({n - len(ok)} failed there), in its cost order")
    return np.sort(idx), note


def _ratios(res):
    """Throughput ratios over the plain path and over the batched FP64 form.
    When the plain path failed (its group's every attempt), its reactors/s is
    the sample over the time it ran before failing, an upper bound on its
    rate, and the ratios over it are lower bounds."""
    base = res["plain_fp64"]["value"]
    res["plain_fp64"]["finished"] = res["plain_fp64"]["failed"] == 0
    if not res["plain_fp64"]["finished"]:
        res["plain_fp64"]["note"] = ("the group integration failed after the steps shown; its value is "
                                     "an upper bound on the plain path's rate, the ratios over it lower bounds")
    for form, _, _ in FORMS[1:]:
        if form in res:
            res[form]["over_plain"] = res[form]["value"] / base
            res[form]["over_batched_fp64"] = res[form]["value"] / res["batched_fp64"]["value"]
    if "batched_fp32_learned" in res:
        res["chosen_over_plain"] = res["batched_fp32_learned"]["over_plain"]


def integration_bench(n_reactors, cpu=True, dt=2e-3, learned=True, n_plain=1024, warm=True):
    """Reactors integrated/s on the 160-species / 900-reaction mechanism (2 ms
    per reactor at rtol 1e-8, atol 1e-20) through the cfd_plugin API with host
    arrays, one solve call per form on the same states in index order: the
    plain FP64 GPU path (the reference's group algorithm, timed on a
    stratified sample of n_plain reactors, since it integrates group after
    group at the same cost per reactor), the batched FP64 and FP32 forms, and
    with the learned predictor (trained on the GPU on pairs the integrator
    generates from other seeded states).  The CPU oracle integrates a bounded
    sample of the same reactors on all host cores; its end states give the
    error of each GPU form on that sample."""
    from zerork_b200 import mechgen
    g = mechgen.generate(mechgen.SPECS["c3_160"])
    out = {"metric": "reactors integrated/s at rtol 1e-8", "unit": "reactors/s",
           "workload": f"160 species / 900 reactions, {n_reactors} constant-volume reactors "
                       "(T U[700,2500] K, P U[1,100] atm, 1-4 fuel-like species), "
                       f"{dt * 1e3:g} ms each, rtol 1e-8, atol 1e-20, one call per form, index order"}
    with tempfile.TemporaryDirectory() as d:
        mf, tf = g.write(d)
        T, P, Y = mechgen.reactor_states(g, n_reactors, "c3", seed=11)
        net = None
        if learned:
            from zerork_b200 import predictor as pr
            t0 = time.perf_counter()
            T0, P0, Y0 = mechgen.reactor_states(g, 2048, "c3", seed=1001)
            Xp, Tp = pr.generate_pairs(mf, tf, T0, P0, Y0, rounds=64, seed=5)
            t_gen = time.perf_counter() - t0
            t0 = time.perf_counter()
            mlp, xs, ts, hist = pr.train(Xp, Tp, epochs=12, batch=1024, lr=1e-3)
            net = (mlp, xs, ts)
            out["learned_predictor"] = {"pairs": int(Xp.shape[0]), "generate_s": t_gen,
                                        "train_s": time.perf_counter() - t0,
                                        "loss_first_last": [hist[0], hist[-1]],
                                        "network": "163 -> 3 x 256 SiLU -> 161, BF16 weights, "
                                                   "FP32 accumulation"}
        ends, cost = {}, None
        for form, opts, use_net in FORMS[1:] + FORMS[:1]:  # the plain path last
            if use_net and not learned:
                continue
            if form == "plain_fp64":
                idx, note = _plain_pick(n_reactors, n_plain, cost)
                out[form], e, _ = _run_form(mf, tf, T[idx], P[idx], Y[idx], dt, opts, cost=cost[idx], warm=False)
                out[form]["sample"] = note
                ends[form] = (idx, e)
            else:
                out[form], e, c = _run_form(mf, tf, T, P, Y, dt, opts, net if use_net else None, warm=warm)
                if form == "batched_fp64":
                    cost = c
                ends[form] = (np.arange(n_reactors), e)
            print(json.dumps({"progress": form, "reactors_per_s": out[form]["value"]}), file=sys.stderr,
                  flush=True)
        out["timing"] = ("second call in the first call's cost order" if warm
                         else "one call per form, index order")
        _ratios(out)
        if cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import zerork_b200 as zb
            import zrk_oracle as zo
            pm = zb.Mechanism(mf, tf, device=False)
            ot = _oracle_tables(pm, zo)
            nth = os.cpu_count() or 1
            m = min(n_reactors, 2 * nth)
            idx = ends["plain_fp64"][0][:m]  # reactors every form integrated
            t0 = time.perf_counter()
            To, Po, Yo, so = ot.solve(T[idx], P[idx], Y[idx], dt, nthreads=nth)
            elapsed = time.perf_counter() - t0
            ok = so["status"] == 0
            out["cpu_oracle"] = {"value": m / elapsed, "unit": "reactors/s", "cores": nth, "kind": "port",
                                 "sample": f"{m} reactors of the plain path's sample, restated "
                                           "BDF/Newton with dense LU (FP64), one reactor per thread",
                                 "failed": int((~ok).sum())}
            for form, (ix, (Tg, Yg)) in ends.items():
                pos = np.searchsorted(ix, idx)
                out[form]["max_abs_dT_vs_oracle"] = float(np.abs(Tg[pos] - To)[ok].max())
                out[form]["max_abs_dY_vs_oracle"] = float(np.abs(Yg[pos] - Yo)[ok].max())
    return out


INTEG_CONFIGS = {
    # name: (mechanism spec, state workload, reactors, interval s, CPU oracle sample)
    "c1": ("c1_h2", "c1", 64, 1e-3, 64),
    "c3": ("c3_160", "c3", 16384, 2e-3, 32),
    "c4": ("c4_650", "c4", 4096, 5e-3, 8),
    "c5": ("c3_160", "c5", 16384, 2e-3, 32),
}


def integration_suite(names, scale=1.0, pairs=1 << 20, threads=None, n_plain=1024, warm=False):
    """Every integration config through the cfd_plugin API (host arrays, one
    solve call per form, reactors in index order): the plain FP64 GPU path
    (the reference's group algorithm, on a stratified sample of n_plain
    reactors; dense-block mechanisms only, so not C4), the batched FP64 and
    FP32 forms, and with the learned predictor (C1, C3, C5), the batched
    FP32 + learned form being the chosen one.  Per form: reactors/s, solver
    counters, failed reactors, and the end-state error on a sample against
    the CPU oracle (rtol 1e-8) and its tight-tolerance run (rtol 1e-12, no
    per-step failure limits): the verdict passes when every sampled
    reactor's |T - T_tight| is within 50 x the oracle's own error (floored at
    10 x the sample median) + 1e-5 T, and its max |Y - Y_tight| within 50 x
    (same floor) + 1e-8, the bound of the test suite
    (tests/test_integrator_gpu.py).  C5 trains the predictor network on about
    `pairs` (state, interval, next state) pairs that the integrator generates
    from other seeded states of the same mechanism."""
    from zerork_b200 import mechgen
    import zerork_b200 as zb
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import zrk_oracle as zo
    out = {}
    nth = threads or os.cpu_count() or 1
    for name in names:
        spec, wl, nr, dt, msamp = INTEG_CONFIGS[name]
        nr = max(8, int(nr * scale))
        g = mechgen.generate(mechgen.SPECS[spec])
        res = {"workload": f"{spec}: {len(g.species)} species, {nr} reactors ({wl} states), "
                           f"{dt * 1e3:g} ms each, rtol 1e-8, atol 1e-20, "
                           + ("cost order from a first call" if warm else "one call per form, index order")}
        with tempfile.TemporaryDirectory() as d:
            mf, tf = g.write(d)
            T, P, Y = mechgen.reactor_states(g, nr, "c3" if wl == "c5" else wl, seed=11)
            net = None
            learned = name in ("c1", "c3", "c5")
            if learned:
                from zerork_b200 import predictor as pr
                t0 = time.perf_counter()
                ng = max(64, min(16384, pairs // 64))  # 64 intervals of ng reactors
                T0, P0, Y0 = mechgen.reactor_states(g, ng, "c3" if wl == "c5" else wl, seed=1001)
                rounds = max(1, pairs // ng)
                Xp, Tp = pr.generate_pairs(mf, tf, T0, P0, Y0, rounds=rounds, seed=5)
                t_gen = time.perf_counter() - t0
                t0 = time.perf_counter()
                mlp, xs, ts, hist = pr.train(Xp, Tp, epochs=8 if Xp.shape[0] > 300000 else 12,
                                             batch=4096, lr=1e-3)
                net = (mlp, xs, ts)
                res["learned_predictor"] = {"pairs": int(Xp.shape[0]), "generate_s": t_gen,
                                            "train_s": time.perf_counter() - t0,
                                            "loss_first_last": [hist[0], hist[-1]]}
                print(json.dumps({name: {"learned_predictor": res["learned_predictor"]}}), flush=True)
            dense = len(g.species) + 1 <= 256
            ends, cost = {}, None
            for form, opts, use_net in FORMS[1:] + FORMS[:1]:  # the plain path last
                if (use_net and not learned) or (form == "plain_fp64" and not dense):
                    continue
                if form == "plain_fp64":
                    sample, note = _plain_pick(nr, n_plain, cost)
                    res[form], e, _ = _run_form(mf, tf, T[sample], P[sample], Y[sample], dt, opts,
                                                cost=cost[sample], warm=False)
                    res[form]["sample"] = note
                    ends[form] = (sample, e)
                else:
                    res[form], e, c = _run_form(mf, tf, T, P, Y, dt, opts, net if use_net else None,
                                                warm=warm)
                    if form == "batched_fp64":
                        cost = c
                    ends[form] = (np.arange(nr), e)
                print(json.dumps({name: {form: res[form]}}), flush=True)
            sample = ends["plain_fp64"][0] if "plain_fp64" in ends else np.flatnonzero(cost > 0)
            if "plain_fp64" in res:
                _ratios(res)
            else:
                res["note"] = ("the plain group path needs the dense Newton block (at most 255 "
                               "species); this mechanism runs on the batched sparse path only")
                for form in list(res):
                    if form.startswith("batched_") and form != "batched_fp64":
                        res[form]["over_batched_fp64"] = res[form]["value"] / res["batched_fp64"]["value"]
            # end-state error on a sample against the oracle and its tight run
            pm = zb.Mechanism(mf, tf, device=False)
            ot = _oracle_tables(pm, zo)
            m = min(nr, msamp)
            idx = sample[:m]
            t0 = time.perf_counter()
            To, Po, Yo, so = ot.solve(T[idx], P[idx], Y[idx], dt, nthreads=nth)
            t_oracle = time.perf_counter() - t0
            Tt, Pt, Yt, stt = ot.solve(T[idx], P[idx], Y[idx], dt, nthreads=nth, rtol=1e-12,
                                       atol=1e-24, max_steps=400000, fail_caps=0)
            ok = (so["status"] == 0) & (stt["status"] == 0)
            res["cpu_oracle"] = {"value": m / t_oracle, "unit": "reactors/s", "cores": nth,
                                 "kind": "port", "sample": f"{m} reactors of the plain path's sample",
                                 "failed": int((~ok).sum())}
            eo_T = np.abs(To - Tt)[ok]
            eo_Y = np.max(np.abs(Yo - Yt), axis=1)[ok]
            fT = 10 * np.median(eo_T) if eo_T.size else 0.0
            fY = 10 * np.median(eo_Y) if eo_Y.size else 0.0
            for form, (ix, (Tg, Yg)) in ends.items():
                pos = np.searchsorted(ix, idx)
                eg_T = np.abs(Tg[pos] - Tt)[ok]
                eg_Y = np.max(np.abs(Yg[pos] - Yt), axis=1)[ok]
                bound_T = 50 * np.maximum(eo_T, fT) + 1e-5 * Tt[ok]
                bound_Y = 50 * np.maximum(eo_Y, fY) + 1e-8
                res[form]["max_abs_dT_vs_tight"] = float(eg_T.max()) if eg_T.size else None
                res[form]["max_abs_dY_vs_tight"] = float(eg_Y.max()) if eg_Y.size else None
                res[form]["oracle_max_abs_dT_vs_tight"] = float(eo_T.max()) if eo_T.size else None
                res[form]["within_tolerance"] = bool(np.all(eg_T <= bound_T) and np.all(eg_Y <= bound_Y))
        out[name] = res
        print(json.dumps({name: res}), flush=True)
    return out


def _oracle_tables(pm, zo):
    """CPU oracle tables from the product loader's tables (the loader is pinned
    bit-exact to the reference's own tables by the test suite)."""
    return zo.OracleTables(zo.with_counts(pm.tables()))


def run_reference_arm(a, rank, world):
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as d:
        g, files, T, P, Y = make_workload(d, min(a.states, 1 << 16), seed=7)
        per_step = []
        nthreads = os.cpu_count()
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import zrk_oracle as zo
        kind = "fmath" if zo.ref_available("fmath") else "libc"
        if not zo.ref_available(kind):
            print(json.dumps({"impl": "reference",
                              "unavailable": "oracle/_ref not built (reference sources absent)"}))
            return
        ref = zo.RefMechanism(files[0], files[1], kind=kind)
        ot = zo.OracleTables(ref.tables)
        m = 96 * nthreads  # bounded sample per step
        for i in range(a.warmup + a.steps):
            lo = (i * m) % (len(T) - m)
            t0 = time.perf_counter()
            ref.batch_rates_jac(files, ot, T[lo:lo + m], P[lo:lo + m], Y[lo:lo + m],
                                nthreads=nthreads)
            if i >= a.warmup:
                per_step.append(time.perf_counter() - t0)
        ms = 1e3 * float(np.mean(per_step))
        v = m / (ms / 1e3)
        line = {"metric": METRIC, "value": v, "unit": "states/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
                "config": {"workload": "rates+jacobian, 53 species / 325 reactions, "
                                       f"bounded sample of {m} states per step",
                           "l2": "inputs per step exceed nothing on CPU"},
                "cpu_baseline": {"value": v, "unit": "states/s", "cores": nthreads,
                                 "kind": "reference",
                                 "sample": f"{m} states per step, zerork::mechanism ({kind} exp)"
                                           " + restated SetupJacobianSparse"},
                "e2e": {"value": v, "unit": "states/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        # the reference's own GPU rate path (rates only) on the full state set
        try:
            gT, gP, gY = make_workload(d, a.states, seed=7)[2:]
            line["reference_gpu"] = reference_gpu_rates(files, gT, gP, gY)
        except Exception as ex:  # no GPU on this host: the CPU line stands alone
            line["reference_gpu"] = {"unavailable": str(ex)[:200]}
        print(json.dumps(line))


def main():
    a = args_()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        run_reference_arm(a, rank, world)
        return
    if a.integration_suite:
        res = integration_suite([x for x in a.integration_suite.split(",") if x], a.suite_scale,
                                a.suite_pairs, n_plain=a.plain_sample)
        print(json.dumps({"integration_suite": res}))
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    import zerork_b200 as zb
    dev = torch.device("cuda", local)
    tmp = tempfile.TemporaryDirectory()
    g, files, T, P, Y = make_workload(tmp.name, a.states, seed=7 + rank)
    n = a.states
    pm = zb.Mechanism(*files)
    S, nnz = pm.nsp, pm.nnz
    Td = torch.from_numpy(T).to(dev)
    Pd = torch.from_numpy(P).to(dev)
    Yd = torch.from_numpy(np.ascontiguousarray(Y.T)).to(dev)
    W = torch.empty((S, n), dtype=torch.float64, device=dev)
    J = torch.empty((nnz, n), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def step():
        pm.rates_jac(Td, Pd, Yd, W, J, stream=sptr)

    # project autotuner: time every tile/warp mapping on the first 2^16 states
    if a.launch:
        ts, v, wp, flags = (int(x) for x in a.launch.split(","))
        pm.set_launch(ts, v, wp, bool(flags & 1), 0, stage=bool(flags & 2), two_ctas=bool(flags & 4))
        tuned_ms = None
    else:
        tuned, tuned_ms = pm.autotune(Td, Pd, Yd, W, J, n=min(n, 1 << 16), stream=sptr)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(a.steps)]
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for i in range(a.steps):
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        t_end.record(stream)
        torch.cuda.synchronize()
    total_ms = t_start.elapsed_time(t_end)
    launch_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    if world > 1:
        tt = torch.tensor([total_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
        dist.barrier()
    ms = total_ms / a.steps
    value = world * n / (ms / 1e3)
    # roofline of the (single) kernel per step
    alg_bytes = n * 8 * ((S + 2) + S + nnz)
    launch_avg = float(np.mean(launch_ms))
    achieved = alg_bytes / (launch_avg / 1e3) / 1e9
    peak, peak_kind = peaks()
    tps = traffic_per_state()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": (tps * n if tps else None),
            "peak_source": f"{peak_kind} hbm_gbs",
            "algorithmic_bytes_per_state": 8 * ((S + 2) + S + nnz)}
    # FP64-pipe roofline: transcendental count per state (two rate evaluations:
    # at T and at the forward-difference temperature) at the measured exp rate
    try:
        fma_gflops, exp_gps = zb.measure_fp64()
        fo_type = pm.table("fo_type")
        troe_exps = int(np.sum(fo_type == 1) * 2 + np.sum(fo_type == 2) * 3)
        per_eval = (len(pm.table("arr_step")) + len(pm.table("keq_step")) + len(fo_type) * 3
                    + troe_exps + 2)
        trans = 2 * per_eval
        t_exp = trans * n / (exp_gps * 1e9)
        roof["fp64"] = {"fma_gflops_measured": fma_gflops, "exp_g_per_s_measured": exp_gps,
                        "transcendentals_per_state": trans,
                        "exp_bound_ms": 1e3 * t_exp, "frac": 1e3 * t_exp / launch_avg}
    except Exception as ex:  # diagnostics only
        roof["fp64"] = {"error": str(ex)}
    # end-to-end through the host C-ABI entry (pinned host buffers)
    e2e = None
    if not a.no_e2e:
        Th = torch.from_numpy(T).pin_memory()
        Ph = torch.from_numpy(P).pin_memory()
        Yh = torch.from_numpy(np.ascontiguousarray(Y.T)).pin_memory()
        Wh = torch.empty((S, n), dtype=torch.float64).pin_memory()
        Jh = torch.empty((nnz, n), dtype=torch.float64).pin_memory()
        L = zb.lib()

        def e2e_step():
            zb.check(L.zrk_rates_jac_host(pm.handle, n, zb._ptr(Th), zb._ptr(Ph), zb._ptr(Yh),
                                          zb._ptr(Wh), zb._ptr(Jh)))
        e2e_step()
        e2e_steps = max(2, min(a.steps, 5))
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        dt = (time.perf_counter() - t0) / e2e_steps
        if world > 1:
            tt = torch.tensor([dt], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            dt = float(tt.item())
        e2e = {"value": world * n / dt, "unit": "states/s",
               "h2d_bytes_per_step": int(Th.nbytes + Ph.nbytes + Yh.nbytes),
               "d2h_bytes_per_step": int(Wh.nbytes + Jh.nbytes), "steps": e2e_steps}
    rates_only = rates_only_b200(files, T, P, Y) if rank == 0 else None
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_reference(files, T, P, Y)
    integ = None
    if rank == 0 and world == 1 and a.reactors > 0:
        integ = integration_bench(a.reactors, cpu=not a.no_cpu, dt=a.integ_dt,
                                  learned=not a.no_learned, n_plain=a.plain_sample, warm=a.integ_warm != 0)
        # the small config (64 reactors, 10 species), where the plain group
        # path finishes: every form with its end-state verdict
        integ["c1"] = integration_suite(["c1"], pairs=1 << 16, warm=True)["c1"]
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "states/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded mechanism and states)",
                "config": {"workload": "rates+jacobian: 53 species / 325 reactions / "
                                       f"{pm.nstep} steps, {n} states per GPU, nnz {nnz}",
                           "global_states": world * n, "parallelism": f"shard{world}",
                           "l2": "inputs 445 MB + outputs 15 GB per step exceed L2; no flush",
                           "launch": pm.get_launch(), "autotune_sample_ms": tuned_ms},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "rates_only": rates_only,
                "integration": integ,
                "gpu_launches": a.steps, "clocks": clk.summary()}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
