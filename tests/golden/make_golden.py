"""Regenerate the golden fixtures in this directory from the reference itself.

Run in a checkout where oracle/_ref was built from the reference sources
(`make -C oracle ref`):  python tests/golden/make_golden.py

Each fixture holds seeded states and the outputs of the reference's own
zerork::mechanism library (ZERORK_EXP_LIBC build) for them:
  * rate coefficients Kfwd/Krev (getKrxnFromTC, mechanism.h:111)
  * net/create/destroy rates and ROP (getReactionRatesLimiter, mechanism.h:143)
  * reactor wdot and Jacobian values: reference rates + the restated
    SetupJacobianSparse assembly (reactor_nvector_serial.cpp:610-771)
for the H2 mechanism shipped with the reference, the Troe known-answer
mechanism, and the two smallest synthetic mechanisms (whose text hash is
stored so a generator change is detected).
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

from zerork_b200 import mechgen  # noqa: E402
import zrk_oracle as zo  # noqa: E402

from refpath import REF_DATA as REF  # noqa: E402
N_STATES = 12


def states(nsp, n, seed):
    rng = np.random.default_rng(seed)
    T = rng.uniform(300.0, 3000.0, n)
    P = 101325.0 * 10 ** rng.uniform(0.0, 2.0, n)
    Y = rng.dirichlet(np.full(nsp, 0.5), size=n)
    return T, P, Y


def make(name, mech, therm, seed, text_hash=""):
    ref = zo.RefMechanism(mech, therm)
    ot = zo.OracleTables(ref.tables)
    T, P, Y = states(ref.nsp, N_STATES, seed)
    Kf, Kr, net, cre, des, rop = [], [], [], [], [], []
    lim = np.full(ref.nstep, 1e22)
    for i in range(N_STATES):
        rho = P[i] / (zo_ru() * T[i] * np.sum(Y[i] / ref.tables["mw"]))
        Cc = rho * Y[i] / ref.tables["mw"]
        a, b = ref.krxn(T[i], Cc)
        Kf.append(a)
        Kr.append(b)
        n_, c_, d_, r_ = ref.rates(T[i], Cc, lim)
        net.append(n_); cre.append(c_); des.append(d_); rop.append(r_)
    wdot, jac = ref.batch_rates_jac((mech, therm), ot, T, P, Y)
    out = os.path.join(HERE, f"ref_{name}.npz")
    np.savez_compressed(out, T=T, P=P, Y=Y, Kf=np.array(Kf), Kr=np.array(Kr), net=np.array(net),
                        cre=np.array(cre), des=np.array(des), rop=np.array(rop), wdot=wdot,
                        jac=jac, text_hash=np.array(text_hash))
    print("wrote", out)


def zo_ru():
    return 8.314462618e3


def main():
    make("h2", f"{REF}/hydrogen/h2_v1b_mech.txt", f"{REF}/hydrogen/h2_v1a_therm.txt", 1)
    make("troe", f"{REF}/ideal/troe_test.mech", f"{REF}/ideal/const_specific_heat.therm", 2)
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        for nm, seed in (("c1_h2", 3), ("c2_53", 4)):
            g = mechgen.generate(mechgen.SPECS[nm])
            m, t = g.write(d)
            h = hashlib.sha256((g.mech_text + g.therm_text).encode()).hexdigest()
            make(nm, m, t, seed, h)


if __name__ == "__main__":
    main()
