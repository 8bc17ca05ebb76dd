"""Pin the CPU oracle (oracle/zrk_oracle.c) before trusting it.

* against the reference's own zerork::mechanism library compiled from its
  sources (oracle/_ref), on the reference's shipped mechanisms and on the
  synthetic ones;
* against the committed golden fixtures (reference outputs, tests/golden);
* against the closed-form Troe known answers of the reference's
  tests/reactions/troe_gtest.cpp (6e-15 relative there), restated here.
"""
import math
import os

import numpy as np
import pytest

from conftest import REF_DATA, golden, oracle_tables, ref_built, scaled_err

import zrk_oracle as zo

needs_ref = pytest.mark.skipif(not ref_built(), reason="oracle/_ref or reference data missing")


def _conc(tables, T, P, Y):
    mw = tables["mw"]
    rho = P / (8.314462618e3 * T * np.sum(Y * (1.0 / mw)))
    return (1.0 / (1.0 / rho)) * (1.0 / mw) * Y


@needs_ref
@pytest.mark.parametrize("mech,therm", [
    ("hydrogen/h2_v1b_mech.txt", "hydrogen/h2_v1a_therm.txt"),
    ("ideal/troe_test.mech", "ideal/const_specific_heat.therm"),
    ("ideal/sri_reaction.mech", "ideal/const_specific_heat.therm"),
    ("ideal/hydrogen_no_falloff.mech", "ideal/const_specific_heat.therm"),
    ("dme/dme_24_mech.txt", "dme/dme_24_therm.txt"),
    ("n-heptane_reduced/heptanesymp159_mec.txt", "n-heptane_reduced/heptanesymp_therm.txt"),
    ("plog/plog_test.mech", "plog/plog_test.therm"),
    ("ideal/plog_test.mech", "ideal/const_specific_heat.therm"),
])
def test_oracle_matches_reference_library(mech, therm):
    m, t = os.path.join(REF_DATA, mech), os.path.join(REF_DATA, therm)
    if not (os.path.exists(m) and os.path.exists(t)):
        pytest.skip("mechanism not shipped")
    ref = zo.RefMechanism(m, t)
    ot = zo.OracleTables(ref.tables)
    rng = np.random.default_rng(0)
    lim = np.full(ref.nstep, 1e22)
    for _ in range(40):
        T = rng.uniform(300, 3000)
        C = rng.uniform(0, 1, ref.nsp) * 10 ** rng.uniform(-4, 1)
        for a, b in zip(ref.rates(T, C, lim), ot.rates(T, C, lim)):
            np.testing.assert_array_equal(a, b)  # same arithmetic, libc exp
        for a, b in zip(ref.thermo(T), ot.thermo(T)):
            np.testing.assert_array_equal(a, b)


@needs_ref
def test_oracle_batch_jacobian_on_reference_rates(tmp_path):
    """The restated Jacobian assembly gives identical values whether it runs on
    the oracle's rates or on the reference library's rates."""
    from zerork_b200 import mechgen
    g = mechgen.generate(mechgen.SPECS["c1_h2"])
    m, t = g.write(str(tmp_path))
    ref = zo.RefMechanism(m, t)
    ot = zo.OracleTables(ref.tables)
    T, P, Y = mechgen.rate_states(g, 64, seed=5)
    w1, j1 = ref.batch_rates_jac((m, t), ot, T, P, Y, nthreads=2)
    w2, j2, _ = ot.batch_rates_jac(T, P, Y, nthreads=2)
    np.testing.assert_array_equal(w1, w2)
    np.testing.assert_array_equal(j1, j2)


def _src_states(g, n, seed):
    """States, energies and sources for the constant-pressure / source pins."""
    from zerork_b200 import mechgen
    T, P, Y = mechgen.rate_states(g, n, seed=seed)
    rng = np.random.default_rng(seed)
    return T, P, Y, rng


@needs_ref
@pytest.mark.parametrize("mech,therm", [
    ("hydrogen/h2_v1b_mech.txt", "hydrogen/h2_v1a_therm.txt"),
    ("dme/dme_24_mech.txt", "dme/dme_24_therm.txt"),
])
def test_mixture_thermo_matches_reference_library(mech, therm):
    """Density, pressure, mass u / h / c_p and the T(E, Y) / T(H, Y) Newton
    inversions (mechanism.cpp:279-547) equal the reference library's,
    including the extrapolation below 100 K and above 5000 K."""
    m, t = os.path.join(REF_DATA, mech), os.path.join(REF_DATA, therm)
    if not (os.path.exists(m) and os.path.exists(t)):
        pytest.skip("mechanism not shipped")
    ref = zo.RefMechanism(m, t)
    ot = zo.OracleTables(ref.tables)
    rng = np.random.default_rng(3)
    n = 200
    T = rng.uniform(300, 3000, n)
    P = 10 ** rng.uniform(4, 7, n)
    Y = rng.dirichlet(np.full(ref.nsp, 0.5), n)
    # energies of a temperature elsewhere in [20, 7000] K: Newton from T, and
    # both extrapolations
    T2 = np.concatenate([rng.uniform(150, 4900, n - 40), rng.uniform(20, 90, 20),
                         rng.uniform(5100, 7000, 20)])
    E = ot.mix_thermo(T2, P, Y, np.zeros(n), np.zeros(n))[:, 2]
    H = ot.mix_thermo(T2, P, Y, np.zeros(n), np.zeros(n))[:, 3]
    a = ref.mix_thermo(T, P, Y, E, H)
    b = ot.mix_thermo(T, P, Y, E, H)
    np.testing.assert_array_equal(a, b)
    inner = (T2 > 100) & (T2 < 5000)
    assert np.max(np.abs(b[inner, 5] - T2[inner])) < 1e-5
    assert np.max(np.abs(b[inner, 6] - T2[inner])) < 1e-3  # c_v steps: slower, same root


@needs_ref
@pytest.mark.parametrize("cp", [0, 1])
def test_reactor_rhs_sources_on_reference_functions(tmp_path, cp):
    """The restated constant-volume / constant-pressure right-hand side with
    DPDT, E_SRC and Y_SRC gives identical values on the oracle's and on the
    reference library's mechanism functions."""
    from zerork_b200 import mechgen
    g = mechgen.generate(mechgen.SPECS["c1_h2"])
    m, t = g.write(str(tmp_path))
    ref = zo.RefMechanism(m, t)
    ot = zo.OracleTables(ref.tables)
    T, P, Y, rng = _src_states(g, 96, 7)
    n, ns = len(T), ref.nsp
    # sources that move P by ~1e4 Pa and T by ~30 K over tm (<= 1 ms)
    dpdt = np.where(rng.uniform(size=n) < 0.5, rng.normal(0, 1e7, n), 0.0)
    esrc = np.where(rng.uniform(size=n) < 0.5, rng.normal(0, 3e7, n), 0.0)
    ysrc = rng.normal(0, 10.0, (n, ns))
    tm = rng.uniform(0, 1e-3, n)
    # small composition changes: at fixed energy, heats of formation turn a
    # large one into a temperature outside the NASA-7 range
    Yp = Y * rng.uniform(0.999, 1.001, (n, ns))
    Yp /= Yp.sum(axis=1, keepdims=True)
    y = np.concatenate([Yp, (T * rng.uniform(0.95, 1.05, n))[:, None]], axis=1)
    for srcs in ({}, {"dpdt": dpdt}, {"e_src": esrc}, {"dpdt": dpdt, "e_src": esrc},
                 {"dpdt": dpdt, "e_src": esrc, "y_src": ysrc}):
        a = ref.reactor_rhs(ot, cp, T, P, Y, tm, y, **srcs)
        b = ot.reactor_rhs(cp, T, P, Y, tm, y, **srcs)
        np.testing.assert_array_equal(a, b)
        assert np.all(np.isfinite(b))
    # the sources act: without them the temperature derivative differs
    base = ot.reactor_rhs(cp, T, P, Y, tm, y)
    with_e = ot.reactor_rhs(cp, T, P, Y, tm, y, e_src=esrc)
    assert np.all((with_e[:, ns] != base[:, ns]) == (esrc != 0))


@pytest.mark.parametrize("name", ["c1_h2", "c2_53"])
def test_oracle_against_golden(name, mech_dir):
    """Golden fixtures = reference-library outputs; regenerate with tests/golden/make_golden.py."""
    import hashlib
    from conftest import synth
    g, (m, t) = synth(name, mech_dir)
    gd = golden(name)
    assert str(gd["text_hash"]) == hashlib.sha256((g.mech_text + g.therm_text).encode()).hexdigest()
    import zerork_b200 as zb
    pm = zb.Mechanism(m, t, device=False)
    ot = oracle_tables(pm)
    w, j, ws, js = ot.batch_rates_jac_scaled(gd["T"], gd["P"], gd["Y"])
    assert scaled_err(w, gd["wdot"], ws) < 1e-13
    assert scaled_err(j, gd["jac"], js) < 1e-12
    for i in range(len(gd["T"])):
        C = _conc(ot.d, gd["T"][i], gd["P"][i], gd["Y"][i])
        net, cre, des, rop = ot.rates(gd["T"][i], C, np.full(ot.nstep, 1e22))
        np.testing.assert_allclose(rop, gd["rop"][i], rtol=1e-14, atol=0)
        np.testing.assert_allclose(cre, gd["cre"][i], rtol=1e-14, atol=0)


TROE_MECH = """ELEMENTS
H
END
SPECIES
H H2
END
REACTIONS CAL/MOLE
H2(+M) => H + H (+M)   2.0E12 0.0 0.0
  LOW / 2.0E9 0.0 0.0 /
  TROE / 0.68 78.0 1995.0 /
H2(+M) => H + H (+M)   2.0E12 0.0 0.0
  LOW / 2.0E9 0.0 0.0 /
  TROE / 0.68 78.0 1995.0 5590.0 /
END
"""


def _nasa_const_cp(name, comp, a0, a5, a6):
    def e(v):
        return f"{v:15.8E}"
    l1 = f"{name:<16s}{'KA':<8s}{comp:<20s}G{300.0:10.2f}{5000.0:10.2f}{1000.0:8.2f}"
    l1 = f"{l1:<79s}1"
    l2 = e(a0) + e(0) * 4
    l3 = e(a5) + e(a6) + e(a0) + e(0) * 2
    l4 = e(0) * 2 + e(a5) + e(a6)
    return [l1, f"{l2:<79s}2", f"{l3:<79s}3", f"{l4:<79s}4"]


def test_troe_known_answer(tmp_path):
    """Closed-form Troe falloff (3- and 4-parameter) as in the reference's
    tests/reactions/troe_gtest.cpp: Khigh = 2e12 (1/s), Klow = 2e6 (m^3/kmol/s
    after the mol/cm^3 -> kmol/m^3 conversion), alpha = 0.68, T*** = 78,
    T* = 1995, T** = 5590, uniform composition at 1000 K and 1 atm."""
    th = ["THERMO ALL", f"{300.0:10.3f}{1000.0:10.3f}{5000.0:10.3f}"]
    th += _nasa_const_cp("H", "H   1", 2.5, 2.54737667e4, -4.46703359e-1)
    th += _nasa_const_cp("H2", "H   2", 3.5, -1.043525e3, -4.22439182)
    th.append("END")
    (tmp_path / "t.mech").write_text(TROE_MECH)
    (tmp_path / "t.therm").write_text("\n".join(th) + "\n")
    import zerork_b200 as zb
    pm = zb.Mechanism(str(tmp_path / "t.mech"), str(tmp_path / "t.therm"), device=False)
    ot = oracle_tables(pm)
    T, P = 1000.0, 1.01325e5
    C = np.full(2, 0.5 * P / (8.314462618e3 * T))
    K = ot.rate_coefs(T, C)
    Csum = C.sum()
    for rxn, four in ((0, False), (1, True)):
        Pr = 2.0e6 * Csum / 2.0e12
        Fc = (1 - 0.68) * math.exp(-T / 78.0) + 0.68 * math.exp(-T / 1995.0)
        if four:
            Fc += math.exp(-5590.0 / T)
        f = math.log10(Fc)
        n = 0.75 - 1.27 * f
        lp = math.log10(Pr) - (0.4 + 0.67 * f)
        lp = lp / (n - 0.14 * lp)
        F = 10 ** (f / (1 + lp * lp))
        expect = 2.0e12 * F * Pr / (1 + Pr)
        assert abs(K[rxn] - expect) <= 6e-15 * abs(expect)


def test_plog_known_answers():
    """PLOG rate coefficients of data/mechanisms/ideal/plog_test.mech against
    the closed forms of the reference's tests/reactions/plog_gtest.cpp (6e-15
    relative there): single-pressure tables (positive, negative and summed
    duplicate lines) give A T^2 exp(-1000 K / T) at every pressure, and a
    three-pressure table with duplicate lines interpolates log-linearly in
    pressure and stays flat outside its range.  Product loader tables, oracle
    evaluation (committed fixture copy of the mechanism).  Tolerance 2e-14
    relative (the gtest's 6e-15 with room for the closed form's own
    rounding)."""
    import zerork_b200 as zb
    from plugin_cases import mech_path
    pm = zb.Mechanism(mech_path("plog_test_ideal.mech"), mech_path("const_specific_heat.therm"),
                      device=False)
    ot = oracle_tables(pm)
    steps = pm.table("step_rxn")
    fwd = [int(np.nonzero((steps == j) & (pm.table("step_dir") == 1))[0][0]) for j in range(pm.nrxn)]
    ru, patm = 8.314462618e3, 1.01325e5

    def kf(T, p_atm):
        P = p_atm * patm
        c = np.full(pm.nsp, P / (ru * T) / pm.nsp)
        return ot.rate_coefs(T, c)

    def near(a, b):  # the closed form's own rounding (Ta = 1000 K up to 1 ulp) needs 2e-14
        return abs(a - b) <= 2e-14 * max(abs(a), abs(b))

    for T in (300.0, 1000.0, 2500.0):
        base = 1.0e6 * T ** 2 * math.exp(-1000.0 / T)
        for p in (0.1, 1.0, 10.0):
            K = kf(T, p)
            assert near(K[fwd[0]], base) and near(K[fwd[1]], -base)
            assert near(K[fwd[2]], 0.9 * base)
        # duplicates summed per pressure: 6.2 at 1 atm, 1.3 at 2 atm, 10.01 at 4 atm
        # (cgs A / 1000 for a second-order step); flat outside [1, 4] atm
        K = kf(T, 1.5)
        want = 6.2 * 1.5 ** (math.log(1.3 / 6.2) / math.log(2.0))
        assert abs(K[fwd[5]] - want) <= 1e-13 * want
        assert near(kf(T, 0.5)[fwd[5]], 6.2) and near(kf(T, 8.0)[fwd[5]], 10.01)
