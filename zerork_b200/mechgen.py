"""Seeded synthetic CHEMKIN mechanisms and reactor states.

Writes element-balanced CHEMKIN-II mechanism text plus NASA-7 two-range
thermodynamic fits, in the same file formats that Zero-RK's CHEMKIN reader
consumes (src/CKconverter/CKParser.cpp:860-1050 for the fixed-column NASA
entries, :1060-1700 for the REACTIONS section).  Nothing here depends on a
public benchmark suite: every species, reaction and state is drawn from
numpy's PCG64 generator with a recorded seed.

Parameter distributions (per workload):
  * Arrhenius high-pressure/elementary rates: pre-exponential factor
    log-uniform on [1e8, 1e16] (cm-mol-s units) referenced to 1000 K, i.e.
    the file's A is A' / 1000**n so that A T**n equals A' at 1000 K; n uniform
    on [-2, 3], Ea uniform on [0, 50] kcal/mol.  (Unreferenced, A = 1e16 with
    n = 3 gives bimolecular rate constants ~1e26 cm^3/mol/s and net rates that
    are pure rounding noise at rtol 1e-8.)
  * Falloff low-pressure limit: A_low' = A' * 10**U(3, 8) referenced the same
    way, same n/Ea laws;
    Troe alpha U(0.1, 0.9), T*** U(10, 500) K, T* U(500, 5000) K and, for
    half of them, T** U(1000, 10000) K.
  * Third-body efficiencies: 0-3 collision partners with efficiency U(0.5, 6).
  * NASA-7 fits: least-squares fits of a smooth model cp(T) on [300, 1000] K
    and [1000, 5000] K with cp, h and s continuous at Tmid = 1000 K.
"""
from __future__ import annotations

import itertools
import math
import os
from dataclasses import dataclass, field

import numpy as np

RU_KJ = 8.314462618e-3  # kJ/(mol K)
ATOM_HF = {"C": 716.7, "H": 218.0, "O": 249.2, "N": 472.7}  # kJ/mol, gas-phase atoms
VALENCE = {"C": 4, "H": 1, "O": 2, "N": 3}


@dataclass
class SynthSpec:
    """Size and reaction mix of a synthetic mechanism."""
    name: str
    n_species: int
    n_reactions: int
    elements: tuple
    n_third_body: int
    n_falloff: int
    n_irreversible: int
    n_troe: int | None = None  # falloff reactions that carry TROE (rest Lindemann)
    seed: int = 1234


# The four mechanism sizes of the benchmark workloads.
SPECS = {
    "c1_h2": SynthSpec("c1_h2", 10, 27, ("H", "O", "N"), 5, 2, 0, n_troe=2, seed=101),
    "c2_53": SynthSpec("c2_53", 53, 325, ("C", "H", "O", "N", "AR"), 49, 33, 65, seed=202),
    "c3_160": SynthSpec("c3_160", 160, 900, ("C", "H", "O", "N", "AR"), 135, 90, 180, seed=303),
    "c4_650": SynthSpec("c4_650", 650, 2800, ("C", "H", "O", "N", "AR"), 420, 280, 560, seed=404),
}

_C1_SPECIES = [
    ("H", {"H": 1}), ("H2", {"H": 2}), ("O", {"O": 1}), ("O2", {"O": 2}),
    ("OH", {"O": 1, "H": 1}), ("H2O", {"H": 2, "O": 1}), ("HO2", {"H": 1, "O": 2}),
    ("H2O2", {"H": 2, "O": 2}), ("N2", {"N": 2}), ("N2O", {"N": 2, "O": 1}),
]
_CORE = [
    ("AR", {"AR": 1}), ("N2", {"N": 2}), ("O2", {"O": 2}), ("H2", {"H": 2}), ("H", {"H": 1}),
    ("O", {"O": 1}), ("OH", {"O": 1, "H": 1}), ("H2O", {"H": 2, "O": 1}),
    ("HO2", {"H": 1, "O": 2}), ("H2O2", {"H": 2, "O": 2}), ("CO", {"C": 1, "O": 1}),
    ("CO2", {"C": 1, "O": 2}),
]


def _formula(comp):
    s = ""
    for e in ("C", "H", "O", "N"):
        n = comp.get(e, 0)
        if n:
            s += e + (str(n) if n > 1 else "")
    return s or "X"


def _lattice(n_needed, rng):
    """CxHyOzNw compositions ordered by heavy-atom count, then isomers."""
    out = []
    for heavy in range(1, 40):
        level = []
        for c in range(0, heavy + 1):
            for o in range(0, min(heavy - c, 4) + 1):
                n = heavy - c - o
                if n > 2:
                    continue
                hmax = 2 * c + 2 + n
                for h in range(0, hmax + 1):
                    comp = {k: v for k, v in (("C", c), ("H", h), ("O", o), ("N", n)) if v}
                    level.append(comp)
        rng.shuffle(level)
        out.extend(level)
        if len(out) >= 4 * n_needed:
            break
    return out


def _species(spec: SynthSpec, rng):
    if spec.name == "c1_h2":
        return [(n, dict(c)) for n, c in _C1_SPECIES]
    sp = [(n, dict(c)) for n, c in _CORE]
    seen = {tuple(sorted(c.items())) for _, c in sp}
    names = {n for n, _ in sp}
    lat = _lattice(spec.n_species, rng)
    # prefer small molecules: take the lattice in order (heavy-atom count)
    i = 0
    while len(sp) < spec.n_species and i < len(lat):
        comp = lat[i]
        i += 1
        key = tuple(sorted(comp.items()))
        if key in seen:
            continue
        seen.add(key)
        nm = _formula(comp)
        base, k = nm, 1
        while nm in names:
            k += 1
            nm = f"{base}-{k}"
        names.add(nm)
        sp.append((nm, comp))
    # isomers if the lattice ran short (large mechanisms)
    j = 0
    while len(sp) < spec.n_species:
        nm0, comp = sp[12 + (j % (len(sp) - 12))]
        j += 1
        base, k = _formula(comp), 2
        nm = f"{base}-{k}"
        while nm in names:
            k += 1
            nm = f"{base}-{k}"
        names.add(nm)
        sp.append((nm, dict(comp)))
    return sp[: spec.n_species]


def _cp_model(comp, rng):
    """Smooth cp/R(T): translation + rotation + Einstein-like vibrations."""
    natoms = sum(v for k, v in comp.items())
    if natoms == 1:
        return lambda T: 2.5 + 0.0 * T
    rot = 1.0 if natoms == 2 else 1.5
    nvib = 3 * natoms - (5 if natoms == 2 else 6)
    thetas = rng.uniform(500.0, 4000.0, size=nvib)

    def cp(T):
        T = np.asarray(T, dtype=np.float64)
        x = thetas[None, :] / T[:, None]
        ex = np.exp(-x)
        vib = (x * x * ex / (1.0 - ex) ** 2).sum(axis=1)
        return 2.5 + rot + vib
    return cp


def _fit_nasa(cp, hf_R, s_R, tmid=1000.0):
    """NASA-7 low/high coefficients, cp/h/s continuous at tmid."""
    tl = np.linspace(300.0, tmid, 60)
    th = np.linspace(tmid, 5000.0, 120)
    # unknowns: 5 low + 5 high cp coefficients; equality cp_lo(tmid)=cp_hi(tmid)
    A = np.zeros((tl.size + th.size, 10))
    b = np.concatenate([cp(tl), cp(th)])
    for k in range(5):
        A[: tl.size, k] = tl ** k
        A[tl.size:, 5 + k] = th ** k
    Ceq = np.zeros((1, 10))
    for k in range(5):
        Ceq[0, k] = tmid ** k
        Ceq[0, 5 + k] = -(tmid ** k)
    # scale columns for conditioning
    sc = np.concatenate([tmid ** -np.arange(5.0), tmid ** -np.arange(5.0)])
    As, Cs = A * sc, Ceq * sc
    K = np.block([[As.T @ As, Cs.T], [Cs, np.zeros((1, 1))]])
    rhs = np.concatenate([As.T @ b, [0.0]])
    sol = np.linalg.solve(K, rhs)[:10] * sc
    lo, hi = list(sol[:5]), list(sol[5:])

    def h_int(a, T):  # h/R without a6
        return a[0] * T + a[1] * T**2 / 2 + a[2] * T**3 / 3 + a[3] * T**4 / 4 + a[4] * T**5 / 5

    def s_int(a, T):  # s/R without a7
        return a[0] * math.log(T) + a[1] * T + a[2] * T**2 / 2 + a[3] * T**3 / 3 + a[4] * T**4 / 4

    T0 = 298.15
    a6l = hf_R - h_int(lo, T0)
    a7l = s_R - s_int(lo, T0)
    a6h = (h_int(lo, tmid) + a6l) - h_int(hi, tmid)
    a7h = (s_int(lo, tmid) + a7l) - s_int(hi, tmid)
    return lo + [a6l, a7l], hi + [a6h, a7h]


def _thermo_entry(name, comp, lo, hi, tmid=1000.0):
    elems = ""
    for e in ("C", "H", "O", "N", "AR"):
        n = comp.get(e, 0)
        if n:
            elems += f"{e:<2s}{n:3d}"
    elems = f"{elems:<20s}"[:20]
    l1 = f"{name:<16s}{'SYN':<8s}{elems}G{300.0:10.2f}{5000.0:10.2f}{tmid:8.2f}"
    l1 = f"{l1:<79s}1"
    f = lambda v: f"{v:15.8E}"
    l2 = "".join(f(v) for v in hi[0:5])
    l3 = "".join(f(v) for v in hi[5:7]) + "".join(f(v) for v in lo[0:3])
    l4 = "".join(f(v) for v in lo[3:7])
    return [l1, f"{l2:<79s}2", f"{l3:<79s}3", f"{l4:<79s}4"]


def _hf_kJ(comp, rng):
    if comp.get("AR"):
        return 0.0
    atoms = sum(ATOM_HF[e] * n for e, n in comp.items())
    vsum = sum(VALENCE[e] * n for e, n in comp.items())
    nat = sum(comp.values())
    bonds = min(vsum // 2, 3 * nat)
    if nat == 1:
        return atoms
    return atoms - 360.0 * bonds + rng.normal(0.0, 35.0)


@dataclass
class SynthMechanism:
    spec: SynthSpec
    species: list = field(default_factory=list)  # (name, comp)
    mech_text: str = ""
    therm_text: str = ""

    def write(self, directory):
        os.makedirs(directory, exist_ok=True)
        m = os.path.join(directory, f"{self.spec.name}.mech")
        t = os.path.join(directory, f"{self.spec.name}.therm")
        with open(m, "w") as f:
            f.write(self.mech_text)
        with open(t, "w") as f:
            f.write(self.therm_text)
        return m, t

    def index(self, name):
        return [n for n, _ in self.species].index(name)


def _key(comp, elems):
    return tuple(comp.get(e, 0) for e in elems)


def generate(spec: SynthSpec) -> SynthMechanism:
    rng = np.random.default_rng(spec.seed)
    species = _species(spec, rng)
    S = len(species)
    names = [n for n, _ in species]
    elems = ("C", "H", "O", "N")
    comps = [_key(c, elems) for _, c in species]
    reactive = [i for i, (n, c) in enumerate(species) if not c.get("AR")]

    # -- candidate reactions (index tuples), balanced by construction
    single = {}
    for i in reactive:
        single.setdefault(comps[i], []).append(i)
    pair = {}
    for a, i in enumerate(reactive):
        for j in reactive[a:]:
            k = tuple(x + y for x, y in zip(comps[i], comps[j]))
            pair.setdefault(k, []).append((i, j))
    decomp = []  # (A,), (B, C)
    for k, lst in pair.items():
        for a in single.get(k, []):
            for (i, j) in lst:
                if a not in (i, j):
                    decomp.append(((a,), (i, j)))
    exch = []
    for k, lst in pair.items():
        if len(lst) < 2:
            continue
        for p, q in itertools.combinations(lst, 2):
            if set(p) & set(q):
                continue
            exch.append((p, q))
    if spec.name == "c1_h2" or len(exch) < spec.n_reactions:
        # 2 -> 3 rearrangements for very small species sets
        trip = {}
        for a, i in enumerate(reactive):
            for b, j in enumerate(reactive[a:], a):
                for l in reactive[b:]:
                    k = tuple(x + y + z for x, y, z in zip(comps[i], comps[j], comps[l]))
                    trip.setdefault(k, []).append((i, j, l))
        for k, lst in pair.items():
            for p in lst:
                for q in trip.get(k, []):
                    if not set(p) & set(q):
                        exch.append((p, q))
    rng.shuffle(decomp)
    rng.shuffle(exch)

    used = set()

    def canon(r, p):
        a, b = tuple(sorted(r)), tuple(sorted(p))
        return (a, b) if a <= b else (b, a)

    chosen = []  # (reactants, products, kind)
    n_pm = spec.n_third_body + spec.n_falloff
    for (a, bc) in decomp:
        if len([c for c in chosen if c[2] != "x"]) >= n_pm:
            break
        key = canon(a, bc)
        if key in used:
            continue
        used.add(key)
        kind = "tb" if len([c for c in chosen if c[2] == "tb"]) < spec.n_third_body else "fo"
        # write recombination direction half of the time
        if rng.random() < 0.5:
            chosen.append((bc, a, kind))
        else:
            chosen.append((a, bc, kind))
    n_ex = spec.n_reactions - len(chosen)
    for (p, q) in exch:
        if n_ex <= 0:
            break
        key = canon(p, q)
        if key in used:
            continue
        used.add(key)
        chosen.append((p, q, "x"))
        n_ex -= 1
    if len(chosen) < spec.n_reactions:
        raise RuntimeError(f"{spec.name}: only {len(chosen)} balanced reactions found")
    order = rng.permutation(len(chosen))
    chosen = [chosen[i] for i in order]
    irrev = set(rng.choice(len(chosen), size=spec.n_irreversible, replace=False).tolist()) \
        if spec.n_irreversible else set()
    fo_ids = [i for i, c in enumerate(chosen) if c[2] == "fo"]
    n_troe = spec.n_troe if spec.n_troe is not None else int(round(0.75 * len(fo_ids)))
    troe = set(fo_ids[:n_troe])

    # -- text
    lines = ["! synthetic mechanism " + spec.name + f" (seed {spec.seed})",
             "ELEMENTS", " ".join(spec.elements), "END", "SPECIES"]
    for k in range(0, S, 8):
        lines.append(" ".join(names[k:k + 8]))
    lines += ["END", "REACTIONS CAL/MOLE MOLES"]
    colliders = [i for i in range(S)]
    for idx, (r, p, kind) in enumerate(chosen):
        Aref = 10 ** rng.uniform(8.0, 16.0)
        n = rng.uniform(-2.0, 3.0)
        Ea = rng.uniform(0.0, 50000.0)
        A = Aref / 1000.0 ** n
        lhs = " + ".join(names[i] for i in r)
        rhs = " + ".join(names[i] for i in p)
        arrow = " => " if idx in irrev else " <=> "
        if kind == "tb":
            eq = f"{lhs} + M{arrow}{rhs} + M"
        elif kind == "fo":
            eq = f"{lhs} (+M){arrow}{rhs} (+M)"
        else:
            eq = f"{lhs}{arrow}{rhs}"
        lines.append(f"{eq:<48s} {A:12.5E} {n:8.4f} {Ea:12.3f}")
        if kind == "fo":
            nl = rng.uniform(-2.0, 3.0)
            Al = Aref * 10 ** rng.uniform(3.0, 8.0) / 1000.0 ** nl
            El = rng.uniform(0.0, 50000.0)
            lines.append(f"   LOW / {Al:12.5E} {nl:8.4f} {El:12.3f} /")
            if idx in troe:
                al = rng.uniform(0.1, 0.9)
                t3 = rng.uniform(10.0, 500.0)
                t1 = rng.uniform(500.0, 5000.0)
                if rng.random() < 0.5:
                    t2 = rng.uniform(1000.0, 10000.0)
                    lines.append(f"   TROE / {al:8.4f} {t3:10.2f} {t1:10.2f} {t2:10.2f} /")
                else:
                    lines.append(f"   TROE / {al:8.4f} {t3:10.2f} {t1:10.2f} /")
        if kind in ("tb", "fo"):
            ne = int(rng.integers(0, 4))
            eff = sorted(rng.choice(colliders, size=ne, replace=False).tolist())
            if eff:
                lines.append("   " + " ".join(f"{names[i]}/{rng.uniform(0.5, 6.0):.3f}/" for i in eff))
    lines.append("END")
    mech_text = "\n".join(lines) + "\n"

    tl = ["THERMO ALL", f"{300.0:10.3f}{1000.0:10.3f}{5000.0:10.3f}"]
    for nm, comp in species:
        cp = _cp_model(comp, rng)
        hf_R = _hf_kJ(comp, rng) / RU_KJ
        nat = sum(comp.values())
        s_R = 12.0 + 3.5 * nat + rng.normal(0.0, 1.5)
        lo, hi = _fit_nasa(cp, hf_R, s_R)
        tl += _thermo_entry(nm, comp, lo, hi)
    tl.append("END")
    therm_text = "\n".join(tl) + "\n"
    return SynthMechanism(spec, species, mech_text, therm_text)


def write_mechanism(name: str, directory: str):
    """Generate the named synthetic mechanism and write (mech, therm) files."""
    return generate(SPECS[name]).write(directory)


# ----------------------------------------------------------------- states
P_ATM = 101325.0


def _mw(comp):
    w = {"C": 12.0107, "H": 1.00794, "O": 15.9994, "N": 14.0067, "AR": 39.948}
    return sum(w[e] * n for e, n in comp.items())


def rate_states(mech: SynthMechanism, n, seed=7):
    """Independent rate-evaluation states: T U[300,3000] K, log10 P U[0,2] atm,
    mass fractions Dirichlet(0.5) over all species."""
    rng = np.random.default_rng(seed)
    S = len(mech.species)
    T = rng.uniform(300.0, 3000.0, n)
    P = P_ATM * 10 ** rng.uniform(0.0, 2.0, n)
    Y = rng.dirichlet(np.full(S, 0.5), size=n)
    return T, P, Y


def reactor_states(mech: SynthMechanism, n, workload, seed=11):
    """Initial reactor states for the integration workloads.

    c1: T U[900,1500] K, P U[1,50] atm; Y = f*Dirichlet(1) over H2, O2, H2O, OH
        with f ~ U(0.2, 0.6) and N2 the balance.
    c3/c4/c5: 1-4 fuel-like C/H species at 0-5 % total mole fraction in air
        (O2:N2 = 21:79 by moles); T, P ranges per workload.
    """
    rng = np.random.default_rng(seed)
    S = len(mech.species)
    mw = np.array([_mw(c) for _, c in mech.species])
    Y = np.zeros((n, S))
    if workload == "c1":
        T = rng.uniform(900.0, 1500.0, n)
        P = P_ATM * rng.uniform(1.0, 50.0, n)
        ids = [mech.index(s) for s in ("H2", "O2", "H2O", "OH")]
        f = rng.uniform(0.2, 0.6, n)
        Y[:, ids] = f[:, None] * rng.dirichlet(np.ones(4), size=n)
        Y[:, mech.index("N2")] = 1.0 - f
        return T, P, Y
    if workload in ("c3", "c5"):
        T = rng.uniform(700.0, 2500.0, n)
        P = P_ATM * rng.uniform(1.0, 100.0, n)
    elif workload == "c4":
        T = rng.uniform(800.0, 1800.0, n)
        P = P_ATM * rng.uniform(10.0, 80.0, n)
    else:
        raise ValueError(workload)
    fuels = [i for i, (nm, c) in enumerate(mech.species)
             if c.get("C", 0) >= 1 and c.get("H", 0) >= 2 and c.get("O", 0) == 0
             and c.get("N", 0) == 0]
    iO2, iN2 = mech.index("O2"), mech.index("N2")
    for r in range(n):
        k = int(rng.integers(1, 5))
        pick = rng.choice(fuels, size=k, replace=False)
        xf = rng.uniform(0.0, 0.05) * rng.dirichlet(np.ones(k))
        X = np.zeros(S)
        X[pick] = xf
        rest = 1.0 - xf.sum()
        X[iO2] = 0.21 * rest
        X[iN2] = 0.79 * rest
        y = X * mw
        Y[r] = y / y.sum()
    return T, P, Y
