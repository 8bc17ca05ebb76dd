"""The C++ mechanism surface (include/zerork_b200_mechanism.h), the mirror of
zerork::mechanism / zerork::mechanism_cuda (src/zerork/mechanism.h:20-285,
mechanism_cuda.h:9-45), driven by a compiled C++ program
(tests/cpp/mechanism_api.cpp) the way reference callers use the classes.

* CPU: the program compiles and links against lib/libzerork_b200.so; without
  a GPU, creating the mechanism fails loudly (exit code 2, the library's
  "no CUDA device" message).
* GPU: on the reference's H2 mechanism and the states of the committed
  golden fixture (tests/golden/ref_h2.npz, outputs of the reference's own
  zerork::mechanism library), getReactionRatesLimiter (limit 1e22 per step)
  and mechanism_cuda::getReactionRatesLimiter_CUDA_mr_dev match the
  reference's net / create / destroy rates and rates of progress at 1e-12 of
  each entry's rounding scale (create + destroy for species, the step's own
  magnitude for rates of progress); getReactionRates and getNetReactionRates
  (no limiter) match the oracle's calcRatesFromTC restatement; the host
  thermodynamic helpers match the oracle's NASA-7 values.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden, have_gpu, oracle_tables
from plugin_cases import mech_path

TOL = 1e-12


def _build(tmp):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    exe = os.path.join(tmp, "mechanism_api")
    lib = os.path.join(ROOT, "zerork_b200", "lib")
    cuda = "/usr/local/cuda"
    cmd = [gxx, "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "mechanism_api.cpp"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
           "-L", lib, "-lzerork_b200", f"-Wl,-rpath,{lib}", "-L", os.path.join(cuda, "lib64"),
           "-lcudart", f"-Wl,-rpath,{os.path.join(cuda, 'lib64')}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _states_file(tmp, T, P, Y):
    path = os.path.join(tmp, "states.bin")
    with open(path, "wb") as f:
        np.array([len(T)], dtype=np.int32).tofile(f)
        np.column_stack([T, P, Y]).astype(np.float64).tofile(f)
    return path


def test_cpp_surface_builds_and_fails_loudly_without_gpu(tmp_path):
    exe = _build(str(tmp_path))
    if have_gpu():
        pytest.skip("a GPU is visible: the GPU test covers the run")
    gd = golden("h2")
    st = _states_file(str(tmp_path), gd["T"][:2], gd["P"][:2], gd["Y"][:2])
    r = subprocess.run([exe, mech_path("h2_v1b_mech.txt"), mech_path("h2_v1a_therm.txt"), st,
                        str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 2 and "no CUDA device" in r.stderr


@pytest.mark.gpu
def test_cpp_surface_matches_reference_rates(tmp_path):
    if not have_gpu():
        pytest.skip("no CUDA device")
    import zerork_b200 as zb
    exe = _build(str(tmp_path))
    gd = golden("h2")
    T, P, Y = gd["T"], gd["P"], gd["Y"]
    n = len(T)
    mf, tf = mech_path("h2_v1b_mech.txt"), mech_path("h2_v1a_therm.txt")
    st = _states_file(str(tmp_path), T, P, Y)
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, mf, tf, st, out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    pm = zb.Mechanism(mf, tf, device=False)
    ns, nst = pm.nsp, pm.nstep
    raw = np.fromfile(out, dtype=np.float64)
    per = 3 * ns + nst + ns + ns + ns + 1
    host = raw[:n * per].reshape(n, per)
    dev = raw[n * per:]
    assert dev.size == (3 * ns + nst) * n
    net, cre, des = host[:, :ns], host[:, ns:2 * ns], host[:, 2 * ns:3 * ns]
    rop = host[:, 3 * ns:3 * ns + nst]
    o = 3 * ns + nst
    net_nolim, net_rr, u_rt, cvm = host[:, o:o + ns], host[:, o + ns:o + 2 * ns], \
        host[:, o + 2 * ns:o + 3 * ns], host[:, o + 3 * ns]
    sc = np.abs(gd["cre"]) + np.abs(gd["des"])
    for a, b in ((net, gd["net"]), (cre, gd["cre"]), (des, gd["des"])):
        assert np.all(np.abs(a - b) <= TOL * sc + 1e-300), np.max(np.abs(a - b) / (sc + 1e-300))
    assert np.all(np.abs(rop - gd["rop"]) <= TOL * np.abs(gd["rop"]) + 1e-300)
    # multi-reactor device entry, species-major with nReactors leading
    dnet = dev[:ns * n].reshape(ns, n).T
    dcre = dev[ns * n:2 * ns * n].reshape(ns, n).T
    drop = dev[3 * ns * n:].reshape(nst, n).T
    assert np.all(np.abs(dnet - gd["net"]) <= TOL * sc + 1e-300)
    assert np.all(np.abs(dcre - gd["cre"]) <= TOL * sc + 1e-300)
    assert np.all(np.abs(drop - gd["rop"]) <= TOL * np.abs(gd["rop"]) + 1e-300)
    # no limiter: the oracle's calcRatesFromTC restatement; host helpers
    ot = oracle_tables(pm)
    mw = pm.table("mw")
    for i in range(n):
        rho = P[i] * (1.0 / np.sum(Y[i] / mw)) / (8.314462618e3 * T[i])
        C = (1.0 / (1.0 / rho)) * (1.0 / mw) * Y[i]
        on, oc, od, orop = ot.rates(T[i], C, None)
        s = np.abs(oc) + np.abs(od)
        assert np.all(np.abs(net_nolim[i] - on) <= TOL * s + 1e-300)
        assert np.all(np.abs(net_rr[i] - on) <= TOL * s + 1e-300)
        cp, h, g = ot.thermo(T[i])
        np.testing.assert_allclose(u_rt[i], h - 1.0, rtol=1e-14, atol=1e-14)
        cv_ref = np.sum((cp - 1.0) * (8.314462618e3 / mw) * Y[i])
        assert abs(cvm[i] - cv_ref) <= 1e-13 * abs(cv_ref)
