"""The product's own CHEMKIN loader against the reference's internal tables.

The reference builds its tables inside zerork::mechanism (info_net, rate_const);
oracle/_ref exposes them.  The product must reproduce every table bit for bit:
species order, step order, expanded reactant/product lists, converted and
merged Arrhenius parameters, Keq lists, third-body and falloff data, and the
fixed Jacobian pattern (reactor_nvector_serial.cpp:122-281).
"""
import os

import numpy as np
import pytest

from conftest import REF_DATA, oracle_tables, ref_built, synth

import zerork_b200 as zb

needs_ref = pytest.mark.skipif(not ref_built(), reason="oracle/_ref or reference data missing")

SHIPPED = [
    ("hydrogen/h2_v1b_mech.txt", "hydrogen/h2_v1a_therm.txt"),
    ("ideal/troe_test.mech", "ideal/const_specific_heat.therm"),
    ("ideal/sri_reaction.mech", "ideal/const_specific_heat.therm"),
    ("ideal/hydrogen_recombination.mech", "ideal/const_specific_heat.therm"),
    ("ideal/hydrogen_recombination_rev_zero.mech", "ideal/const_specific_heat.therm"),
    ("ideal/hydrogen_no_falloff.mech", "ideal/const_specific_heat.therm"),
    ("dme/dme_24_mech.txt", "dme/dme_24_therm.txt"),
    ("n-heptane_reduced/heptanesymp159_mec.txt", "n-heptane_reduced/heptanesymp_therm.txt"),
    ("plog/plog_test.mech", "plog/plog_test.therm"),
    ("ideal/plog_test.mech", "ideal/const_specific_heat.therm"),
]


def _compare(mf, tf):
    import zrk_oracle as zo
    ref = zo.RefMechanism(mf, tf)
    pm = zb.Mechanism(mf, tf, device=False)
    assert pm.species == ref.species
    pt = pm.tables()
    for k in zb.TABLE_NAMES:
        a, b = np.asarray(ref.tables[k]), np.asarray(pt[k])
        assert a.shape == b.shape, k
        assert np.array_equal(a, b), k
    cp, ri = pm.jac_pattern()
    cpo, rio = zo.OracleTables(ref.tables).jac_pattern()
    assert np.array_equal(cp, cpo) and np.array_equal(ri, rio)


@needs_ref
@pytest.mark.parametrize("mech,therm", SHIPPED)
def test_tables_match_reference_shipped(mech, therm):
    mf, tf = os.path.join(REF_DATA, mech), os.path.join(REF_DATA, therm)
    if not (os.path.exists(mf) and os.path.exists(tf)):
        pytest.skip("not shipped")
    _compare(mf, tf)


@needs_ref
@pytest.mark.parametrize("name", ["c1_h2", "c2_53", "c3_160", "c4_650"])
def test_tables_match_reference_synthetic(name, mech_dir):
    g, (mf, tf) = synth(name, mech_dir)
    _compare(mf, tf)


def test_pattern_structure(c2):
    """Diagonal, full temperature row and column, rows ascending per column."""
    pm = zb.Mechanism(*c2[1], device=False)
    cp, ri = pm.jac_pattern()
    n = pm.nsp + 1
    assert cp[0] == 0 and cp[-1] == pm.nnz
    for j in range(n):
        rows = ri[cp[j]:cp[j + 1]]
        assert np.all(np.diff(rows) > 0)
        assert j in rows and (n - 1) in rows
    assert cp[n] - cp[n - 1] == n


def test_parse_errors(tmp_path, c1):
    mf, tf = c1[1]
    with pytest.raises(zb.ZeroRKError) as e:
        zb.Mechanism(str(tmp_path / "missing.mech"), tf, device=False)
    assert e.value.code == 3
    bad = tmp_path / "ford.mech"
    bad.write_text("ELEMENTS\nH\nEND\nSPECIES\nH H2\nEND\nREACTIONS\n"
                   "H2 <=> H + H 1e10 0 0\n FORD / H2 0.5 /\nEND\n")
    with pytest.raises(zb.ZeroRKError, match="FORD"):
        zb.Mechanism(str(bad), tf, device=False)
    # PLOG excludes third-body data and REV (CKParser.cpp:312-350)
    for extra, msg in (("H2 + M <=> H + H + M 1e10 0 0\n PLOG / 1.0 1e10 0 0 /\n", "third-body"),
                       ("H2 <=> H + H 1e10 0 0\n PLOG / 1.0 1e10 0 0 /\n REV / 1e10 0 0 /\n", "REV")):
        bad = tmp_path / "plog_bad.mech"
        bad.write_text("ELEMENTS\nH\nEND\nSPECIES\nH H2\nEND\nREACTIONS\n" + extra + "END\n")
        with pytest.raises(zb.ZeroRKError, match=msg):
            zb.Mechanism(str(bad), tf, device=False)
    und = tmp_path / "und.mech"
    und.write_text("ELEMENTS\nH\nEND\nSPECIES\nH2\nEND\nREACTIONS\nH2 <=> HX + HX 1e10 0 0\nEND\n")
    with pytest.raises(zb.ZeroRKError, match="undeclared"):
        zb.Mechanism(str(und), tf, device=False)


def test_oracle_consumes_product_tables(c1):
    pm = zb.Mechanism(*c1[1], device=False)
    ot = oracle_tables(pm)
    assert ot.jac_pattern()[1].size == pm.nnz
