"""Regenerate the cfd_plugin golden fixtures from the reference checkout.

    python tests/golden/make_plugin_golden.py      (ZERORK_REFERENCE names the checkout)

Writes, next to this script:

* mech/<file>.gz -- gzip copies of the reference's shipped mechanism and
  thermo files that the golden tests load (data inputs of the reference's
  own golden outputs; the GPU box has no reference checkout);
* plugin_tester.npz -- the reference's cfd_plugin tester cases
  (examples/cfd_plugin_tester/run.sh.in: h2, dme, nc7h16-skel) with their
  initial states and the reactor histories the reference printed
  (examples/cfd_plugin_tester/outputs.ref/<case>_sparse_000.hist, 6
  significant digits), plus the plugin options of
  examples/cfd_plugin_tester/inputs/base_plugin.yml.

The initial mass fractions restate the tester's setup
(applications/cfd_plugin/zerork_cfd_plugin_tester.cpp):
getFracsFromCompMap (:480-500) normalises the fuel and oxidizer mole
fractions, setReactorMassFrac (:502-551) mixes phi * fuel with the
stoichiometric oxidizer amount |O_rem(fuel)| / O_rem(oxid), where O_rem is
mechanism::getMolarAtomicOxygenRemainder (src/zerork/mechanism.cpp:731-742,
x * (nO - 2 nC - nH / 2)), renormalises and converts with getYfromX
(mechanism.cpp:299-304).  Molecular weights come from the reference library
built in oracle/_ref; element counts from the thermo file's composition
columns.
"""
import gzip
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import refpath  # noqa: E402
import zrk_oracle as zo  # noqa: E402

MECH_FILES = {
    "h2_v1b_mech.txt": "hydrogen/h2_v1b_mech.txt",
    "h2_v1a_therm.txt": "hydrogen/h2_v1a_therm.txt",
    "dme_24_mech.txt": "dme/dme_24_mech.txt",
    "dme_24_therm.txt": "dme/dme_24_therm.txt",
    "heptanesymp159_mec.txt": "n-heptane_reduced/heptanesymp159_mec.txt",
    "heptanesymp_therm.txt": "n-heptane_reduced/heptanesymp_therm.txt",
    "sri_reaction.mech": "ideal/sri_reaction.mech",
    "troe_test.mech": "ideal/troe_test.mech",
    "hydrogen_no_falloff.mech": "ideal/hydrogen_no_falloff.mech",
    "const_specific_heat.therm": "ideal/const_specific_heat.therm",
    "hydrogen_recombination.mech": "ideal/hydrogen_recombination.mech",
    "plog_test.mech": "plog/plog_test.mech",
    "plog_test.therm": "plog/plog_test.therm",
    "plog_test_ideal.mech": "ideal/plog_test.mech",
    "ford_propane.mech": "real_order/ford_propane.mech",
    "rord_propane.mech": "real_order/rord_propane.mech",
    "non_integer_test.mech": "ideal/non_integer_test.mech",
}

# run.sh.in: name, mechanism, thermo, ignition delay time (simulated twice)
CASES = [
    ("h2", "h2_v1b_mech.txt", "h2_v1a_therm.txt", "8.2565998e-07"),
    ("dme", "dme_24_mech.txt", "dme_24_therm.txt", "1.1e-05"),
    ("nc7h16-skel", "heptanesymp159_mec.txt", "heptanesymp_therm.txt", "1.35e-05"),
]

# inputs/base_tester.yml
T0, P0, PHI, N_STEPS, DT_IGN = 1450.0, 2.02650e6, 1.0, 10, 400.0
# inputs/base_plugin.yml (gpu 0; the sparse run: analytic 1, iterative 1)
PLUGIN_OPTS = {"rel_tol": 1.0e-8, "abs_tol": 1.0e-18, "max_steps": 3000, "eps_lin": 0.1,
               "nonlinear_convergence_coeff": 0.05, "preconditioner_threshold": 3.2e-5}


def element_counts(therm_path, species):
    """{species: {element: count}} from the NASA-7 first lines (columns 25-44)."""
    want = {s.lower() for s in species}
    out = {}
    with open(therm_path) as f:
        for line in f:
            if len(line) < 80 or line[79] != "1":
                continue
            name = line[:18].split()[0].lower() if line[:18].split() else ""
            if name not in want or name in out:
                continue
            comp = {}
            for k in range(4):
                chunk = line[24 + 5 * k: 29 + 5 * k]
                el, cnt = chunk[:2].strip().lower(), chunk[2:].strip()
                if el and el != "0" and cnt:
                    comp[el] = comp.get(el, 0) + int(float(cnt))
            out[name] = comp
    return out


def fracs(name):
    path = os.path.join(refpath.REFERENCE, "examples", "cfd_plugin_tester", "inputs",
                        f"{name}_fracs.log")
    fuel, oxid = {}, {}
    with open(path) as f:
        for line in f:
            if line.startswith("#") or ":" not in line:
                continue
            k, v = line.split(":")
            k = k.strip()
            (oxid if k.lower() in ("o2", "n2") else fuel)[k] = float(v)
    return fuel, oxid


def initial_mass_fractions(species, mw, comp, fuel, oxid):
    idx = {s.lower(): i for i, s in enumerate(species)}
    nsp = len(species)

    def vec(m):
        x = np.zeros(nsp)
        for k, v in m.items():
            x[idx[k.lower()]] = v
        return x / x.sum() if x.sum() != 0.0 else x

    def o_rem(x):
        r = 0.0
        for j in range(nsp):
            if x[j] == 0.0:
                continue
            c = comp[species[j].lower()]
            r += x[j] * (c.get("o", 0) - 2.0 * c.get("c", 0) - 0.5 * c.get("h", 0))
        return r

    xf, xo = vec(fuel), vec(oxid)
    stoic = abs(o_rem(xf)) / o_rem(xo)
    fr = PHI * xf + stoic * xo
    fr = fr / fr.sum()
    inv_mix = 1.0 / np.sum(fr * mw)
    return inv_mix * fr * mw


def read_hist(path):
    with open(path) as f:
        head = f.readline().lstrip("#").split()
        rows = [[float(v) for v in line.split()] for line in f if line.strip()]
    return head, np.array(rows)


def main():
    os.makedirs(os.path.join(HERE, "mech"), exist_ok=True)
    for dst, src in MECH_FILES.items():
        with open(os.path.join(refpath.REF_DATA, src), "rb") as f:
            data = f.read()
        with gzip.GzipFile(os.path.join(HERE, "mech", dst + ".gz"), "wb", mtime=0) as g:
            g.write(data)
    out = {}
    for name, mf, tf, idt in CASES:
        m = os.path.join(refpath.REF_DATA, MECH_FILES[mf])
        t = os.path.join(refpath.REF_DATA, MECH_FILES[tf])
        ref = zo.RefMechanism(m, t)
        mw = np.asarray(ref.tables["mw"])
        fuel, oxid = fracs(name)
        comp = element_counts(t, list(fuel) + list(oxid))
        Y0 = initial_mass_fractions(ref.species, mw, comp, fuel, oxid)
        head, rows = read_hist(os.path.join(refpath.REFERENCE, "examples", "cfd_plugin_tester",
                                            "outputs.ref", f"{name}_sparse_000.hist"))
        logged = head[4:]
        key = name.split("-")[0]
        out[f"{key}_files"] = np.array([mf, tf])
        out[f"{key}_species"] = np.array(ref.species)
        out[f"{key}_Y0"] = Y0
        out[f"{key}_TP0"] = np.array([T0, P0])
        out[f"{key}_dt"] = np.array(2.0 * float(idt) / N_STEPS)
        out[f"{key}_logged"] = np.array(logged)
        out[f"{key}_hist"] = rows  # step, time, T, P, logged mass fractions
        ref.close()
    out["plugin_opts_keys"] = np.array(list(PLUGIN_OPTS))
    out["plugin_opts_vals"] = np.array(list(PLUGIN_OPTS.values()), dtype=np.float64)
    out["dT_ign"] = np.array(DT_IGN)
    np.savez_compressed(os.path.join(HERE, "plugin_tester.npz"), **out)
    print("wrote plugin_tester.npz and", len(MECH_FILES), "mechanism files")


if __name__ == "__main__":
    main()
