"""The reference's cfd_plugin tester cases and shipped mechanisms as test inputs.

Reads the committed fixtures of tests/golden (make_plugin_golden.py): the
gzip copies of the reference's mechanism files and plugin_tester.npz, the
tester's initial states and the reactor histories the reference printed
(examples/cfd_plugin_tester/outputs.ref/*_sparse_000.hist).  Nothing here
reads the reference checkout, so the GPU tests run from the fixtures alone.
"""
import gzip
import os
import tempfile

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
_dir = None


def mech_path(name):
    """Path of a decompressed fixture mechanism/thermo file (session temp dir)."""
    global _dir
    if _dir is None:
        _dir = tempfile.mkdtemp(prefix="zrk_golden_mech_")
    out = os.path.join(_dir, name)
    if not os.path.exists(out):
        with gzip.open(os.path.join(GOLDEN, "mech", name + ".gz"), "rb") as f:
            data = f.read()
        with open(out, "wb") as g:
            g.write(data)
    return out


def plugin_tester_case(key):
    """One tester case ("h2", "dme", "nc7h16"): files, initial state, time
    step, the plugin options of inputs/base_plugin.yml, the logged species'
    indexes and the reference history rows (step, time, T, P, logged Y)."""
    d = np.load(os.path.join(GOLDEN, "plugin_tester.npz"))
    mf, tf = (str(x) for x in d[f"{key}_files"])
    species = [str(s) for s in d[f"{key}_species"]]
    logged = [str(s) for s in d[f"{key}_logged"]]
    opts = {str(k): float(v) for k, v in zip(d["plugin_opts_keys"], d["plugin_opts_vals"])}
    opts["max_steps"] = int(opts["max_steps"])
    return dict(mech=mech_path(mf), therm=mech_path(tf), species=species,
                Y0=np.array(d[f"{key}_Y0"]), T0=float(d[f"{key}_TP0"][0]),
                P0=float(d[f"{key}_TP0"][1]), dt=float(d[f"{key}_dt"]),
                logged=[species.index(s) for s in logged], hist=np.array(d[f"{key}_hist"]),
                opts=opts, dT_ign=float(d["dT_ign"]))


def sig6_units(ours, ref):
    """|ours - ref| in units of the 6th significant digit of the printed ref
    (the reference history is printed with 6 significant digits, so an exact
    match of the underlying value gives at most 0.5)."""
    ours, ref = np.asarray(ours, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    mag = np.floor(np.log10(np.maximum(np.abs(ref), 1e-300)))
    unit = 10.0 ** (mag - 5)
    return np.abs(ours - ref) / unit


def compare_history(rows, hist, y_floor=1e-12):
    """Max 6th-digit units over T, P and the logged mass fractions; logged
    mass fractions whose reference value is below y_floor are compared
    absolutely (|diff| <= y_floor counts as 0 units), since at atol 1e-18 a
    trace species far below the major ones is not resolved to 6 digits."""
    rows = np.asarray(rows)
    uT = sig6_units(rows[:, 0], hist[:, 2])
    uP = sig6_units(rows[:, 1], hist[:, 3])
    uY = sig6_units(rows[:, 2:], hist[:, 4:])
    tiny = np.abs(hist[:, 4:]) < y_floor
    uY = np.where(tiny, np.where(np.abs(rows[:, 2:] - hist[:, 4:]) <= y_floor, 0.0, np.inf), uY)
    return float(max(uT.max(), uP.max(), uY.max())), (uT, uP, uY)
