// mech.cpp -- CHEMKIN-II loader and mechanism tables (see mech.h).
//
// Supported: ELEMENTS, SPECIES, THERMO (in the mechanism or thermo file),
// REACTIONS with CAL/MOLE, KCAL/MOLE, JOULES/MOLE, KJOULES/MOLE, KELVINS and
// MOLES units; elementary, +M third-body and (+M)/(+species) falloff
// reactions with LOW, TROE (3/4 parameters), SRI (3/5 parameters), REV, DUP,
// PLOG and collision efficiencies.  FORD/RORD, HIGH and Landau-Teller
// reactions, and non-integer stoichiometry, are rejected with a ParseError.
#include "mech.h"

#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace zrk {
namespace {

// Universal gas constant [J/kmol/K] and energy conversions, as defined in
// src/zerork/constants.h:10-24.
const double kRu = 8.314462618e3;
const double kCalPerMolTact = 4184.0 / kRu;
const double kKcalPerMolTact = 4184.0 / kRu * 1000.0;
const double kKjoulesPerMolTact = 238.846 * kCalPerMolTact;
const double kJoulesPerMolTact = 238.846 * kCalPerMolTact / 1000.0;
const double kConvertC = 1000.0;  // mol/cm^3 -> kmol/m^3
const double kPatm = 1.01325e5;   // src/zerork/constants.h:12
const double kArrheniusRtol = 1.0e-6;

// IUPAC 2007 standard atomic weights [kg/kmol] (the table Zero-RK uses,
// src/zerork/atomicMassDB.h), for the elements combustion mechanisms carry.
struct ElemW {
  const char *sym;
  double w;
};
const ElemW kElemW[] = {
    {"H", 1.00794},      {"HE", 4.002602},  {"LI", 6.941},      {"BE", 9.012182},
    {"B", 10.811},       {"C", 12.0107},    {"N", 14.0067},     {"O", 15.9994},
    {"F", 18.9984032},   {"NE", 20.1797},   {"NA", 22.98976928}, {"MG", 24.3050},
    {"AL", 26.9815386},  {"SI", 28.0855},   {"P", 30.973762},   {"S", 32.065},
    {"CL", 35.453},      {"AR", 39.948},    {"K", 39.0983},     {"CA", 40.078},
    {"FE", 55.845},      {"CU", 63.546},    {"BR", 79.904},     {"KR", 83.798},
    {"I", 126.90447},    {"XE", 131.293},
};

std::string upper(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}
std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}
std::string strip_ws(const std::string &s) {
  std::string o;
  for (char c : s)
    if (!std::isspace((unsigned char)c)) o += c;
  return o;
}
std::vector<std::string> tokens(const std::string &s) {
  std::vector<std::string> t;
  std::istringstream is(s);
  std::string w;
  while (is >> w) t.push_back(w);
  return t;
}
// Fortran-style number: accepts D/d exponents.
bool to_num(std::string s, double *v) {
  for (auto &c : s)
    if (c == 'D' || c == 'd') c = 'E';
  s = trim(s);
  if (s.empty()) return false;
  char *end = nullptr;
  *v = std::strtod(s.c_str(), &end);
  return end && *end == '\0';
}
double num_or_throw(const std::string &s, const std::string &what) {
  double v;
  if (!to_num(s, &v)) throw ParseError("bad number '" + s + "' in " + what);
  return v;
}

double elem_weight(const std::string &sym) {
  std::string u = upper(trim(sym));
  for (const auto &e : kElemW)
    if (u == e.sym) return e.w;
  throw ParseError("unknown element '" + sym + "'");
}

struct Line {
  std::string text;
  int no;
};
std::vector<Line> read_lines(const std::string &file, bool strip_comments) {
  std::ifstream in(file);
  if (!in) throw ParseError("cannot open " + file);
  std::vector<Line> out;
  std::string s;
  int no = 0;
  while (std::getline(in, s)) {
    ++no;
    if (!s.empty() && s.back() == '\r') s.pop_back();
    if (strip_comments) {
      size_t c = s.find('!');
      if (c != std::string::npos) s = s.substr(0, c);
    }
    out.push_back({s, no});
  }
  return out;
}

bool kw(const std::string &line, const char *key4) {
  std::string t = upper(trim(line));
  return t.compare(0, std::strlen(key4), key4) == 0;
}

struct Species {
  std::string name;
  std::vector<std::pair<std::string, int>> elements;  // in file order
  double tmid = 0;
  double lo[7], hi[7];
  bool have = false;
};

// One NASA-7 entry (fixed columns; CKParser.cpp:860-1050 reads the same layout).
void parse_thermo_block(const std::vector<Line> &L, size_t begin, size_t end, double tmid_default,
                        std::map<std::string, Species *> &byname,
                        std::map<std::string, Species *> &byupper) {
  for (size_t i = begin; i < end; ++i) {
    const std::string &s = L[i].text;
    if (s.size() < 80 || s[79] != '1') continue;
    if (i + 3 >= L.size()) throw ParseError("truncated thermo entry");
    std::vector<std::string> nt = tokens(s.substr(0, 16));
    if (nt.empty()) continue;
    std::string nm = nt[0];
    Species *sp = nullptr;
    auto it = byname.find(nm);
    if (it != byname.end()) sp = it->second;
    else {
      auto iu = byupper.find(upper(nm));
      if (iu != byupper.end()) sp = iu->second;
    }
    if (!sp || sp->have) {  // not in the mechanism, or a later duplicate
      i += 3;
      continue;
    }
    if (s.size() >= 81 && s[80] == '&')
      throw ParseError("free-form thermo composition is not supported (" + nm + ")");
    sp->elements.clear();
    auto add = [&](const std::string &sym, const std::string &cnt) {
      std::string e = trim(sym);
      double a = 0.0;
      to_num(cnt, &a);
      if (e.empty() || a == 0.0) return;
      sp->elements.push_back({e, (int)a});
    };
    for (int k = 0; k < 4; ++k) {
      int loc = 24 + 5 * k;
      std::string sym;
      if (s[loc] != ' ') sym = (s[loc + 1] != ' ') ? s.substr(loc, 2) : s.substr(loc, 1);
      else if (s[loc + 1] != ' ') sym = s.substr(loc + 1, 1);
      add(sym, s.substr(loc + 2, 3));
    }
    double tm = 0.0;
    if (!to_num(s.substr(65, 8), &tm) || tm == 0.0) tm = tmid_default;
    if (s.size() >= 78) {
      std::string sym;
      if (s[73] != ' ') sym += s[73];
      if (s[74] != ' ') sym += s[74];
      add(sym, s.substr(75, 3));
    }
    sp->tmid = tm;
    double c[15];
    int nc = 0;
    for (int ln = 1; ln <= 3; ++ln) {
      const std::string &t = L[i + ln].text;
      if (t.size() < 80 || t[79] != (char)('1' + ln))
        throw ParseError("thermo entry for " + nm + ": bad line " + std::to_string(L[i + ln].no));
      int nf = (ln == 3) ? 4 : 5;
      for (int f = 0; f < nf; ++f) c[nc++] = num_or_throw(t.substr(15 * f, 15), "thermo of " + nm);
    }
    for (int k = 0; k < 7; ++k) {
      sp->hi[k] = c[k];
      sp->lo[k] = c[7 + k];
    }
    sp->have = true;
    i += 3;
  }
}

struct RCoef {
  double A = -1.0e300, n = 0.0, E = 0.0;
};
struct Reaction {
  std::vector<std::pair<std::string, double>> reac, prod;
  bool reversible = true, third_body = false, falloff = false;
  std::string third = "<none>";
  RCoef kf, krev, klow;
  bool have_low = false;
  int ftype = kLindemann;
  std::vector<double> fpar;
  std::map<std::string, double> e3b;  // std::map: efficiency order by name
  std::vector<std::array<double, 4>> plog;  // PLOG lines: p [atm], A, n, E
  int line = 0;
};

// Split one side of an equation at '+' separators (after whitespace removal),
// with an optional leading numeric stoichiometric coefficient.
void side_species(const std::string &s0, std::vector<std::pair<std::string, double>> &out,
                  int line) {
  std::string s = strip_ws(s0);
  std::vector<std::string> parts;
  std::string cur;
  for (size_t i = 0; i < s.size(); ++i) {
    if (s[i] == '+' && !cur.empty() && i + 1 < s.size() && s[i + 1] != '+') {
      parts.push_back(cur);
      cur.clear();
    } else {
      cur += s[i];
    }
  }
  if (!cur.empty()) parts.push_back(cur);
  for (auto &p : parts) {
    size_t k = 0;
    while (k < p.size() && (std::isdigit((unsigned char)p[k]) || p[k] == '.')) ++k;
    double nu = 1.0;
    if (k > 0) nu = std::atof(p.substr(0, k).c_str());
    out.push_back({p.substr(k), nu});
  }
  if (out.empty()) throw ParseError("empty reaction side at line " + std::to_string(line));
}

}  // namespace

MechTables load_chemkin(const std::string &mech_file, const std::string &therm_file) {
  std::vector<Line> L = read_lines(mech_file, true);
  MechTables t;
  std::vector<Species> sp;
  std::vector<Reaction> rx;
  double convertE = kCalPerMolTact;
  size_t i = 0;
  int thermo_begin = -1, thermo_end = -1;
  while (i < L.size()) {
    std::string s = trim(L[i].text);
    if (s.empty()) { ++i; continue; }
    if (kw(s, "ELEM")) {
      std::vector<std::string> tk = tokens(s);
      tk.erase(tk.begin());
      ++i;
      bool done = false;
      for (;;) {
        for (auto &w : tk) {
          if (upper(w) == "END") { done = true; break; }
          if (w.find('/') != std::string::npos) throw ParseError("element masses not supported");
          t.elements.push_back(w);
        }
        if (done || i >= L.size()) break;
        tk = tokens(L[i].text);
        ++i;
      }
      continue;
    }
    if (kw(s, "SPEC")) {
      std::vector<std::string> tk = tokens(s);
      tk.erase(tk.begin());
      ++i;
      bool done = false;
      for (;;) {
        for (auto &w : tk) {
          if (upper(w) == "END") { done = true; break; }
          bool dup = false;
          for (auto &q : sp) dup |= (q.name == w);
          if (!dup) {
            Species x;
            x.name = w;
            sp.push_back(x);
          }
        }
        if (done || i >= L.size()) break;
        tk = tokens(L[i].text);
        ++i;
      }
      continue;
    }
    if (kw(s, "THER")) {
      thermo_begin = (int)i;
      ++i;
      while (i < L.size() && !kw(L[i].text, "END")) ++i;
      thermo_end = (int)i;
      ++i;
      continue;
    }
    if (kw(s, "REAC")) {
      for (auto &w : tokens(s)) {
        std::string u = upper(w);
        if (u == "CAL/MOLE") convertE = kCalPerMolTact;
        else if (u == "KCAL/MOLE") convertE = kKcalPerMolTact;
        else if (u == "JOULES/MOLE") convertE = kJoulesPerMolTact;
        else if (u == "KJOULES/MOLE") convertE = kKjoulesPerMolTact;
        else if (u == "KELVINS") convertE = 1.0;
        else if (u == "EVOLTS" || u == "MOLECULES")
          throw ParseError(u + " units not supported");
      }
      ++i;
      for (; i < L.size(); ++i) {
        std::string r = L[i].text;
        if (trim(r).empty()) continue;
        if (kw(r, "END")) { ++i; break; }
        if (r.find('=') != std::string::npos) {
          Reaction R;
          R.line = L[i].no;
          std::string left, right;
          size_t e;
          if ((e = r.find("<=>")) != std::string::npos) {
            left = r.substr(0, e); right = r.substr(e + 3);
          } else if ((e = r.find("=>")) != std::string::npos) {
            R.reversible = false; left = r.substr(0, e); right = r.substr(e + 2);
          } else {
            e = r.find('='); left = r.substr(0, e); right = r.substr(e + 1);
          }
          left = strip_ws(left);
          size_t m = left.find("(+");
          if (m != std::string::npos) {
            size_t c = left.find(')', m);
            if (c == std::string::npos) throw ParseError("missing ) at line " + std::to_string(R.line));
            std::string ms = left.substr(m + 2, c - m - 2);
            R.falloff = true;
            R.third = (ms == "M" || ms == "m") ? "M" : ms;
            left = left.substr(0, m);
          } else if (left.size() >= 2 && (left.compare(left.size() - 2, 2, "+M") == 0 ||
                                          left.compare(left.size() - 2, 2, "+m") == 0)) {
            R.third_body = true;
            R.third = "M";
            left = left.substr(0, left.size() - 2);
          }
          side_species(left, R.reac, R.line);
          std::vector<std::string> tk = tokens(right);
          if (tk.size() < 3) throw ParseError("expected 3 Arrhenius parameters at line " + std::to_string(R.line));
          R.kf.A = num_or_throw(tk[tk.size() - 3], "A");
          R.kf.n = num_or_throw(tk[tk.size() - 2], "n");
          R.kf.E = num_or_throw(tk[tk.size() - 1], "E");
          // a negative A is kept: only a PLOG reaction may carry one (its
          // lines replace the rate), checked when the reaction is complete
          std::string rs;
          for (size_t k = 0; k + 3 < tk.size(); ++k) rs += tk[k];
          m = rs.find("(+");
          if (m != std::string::npos) {
            if (R.third_body) throw ParseError("mismatched +M or (+M)");
            size_t c = rs.find(')', m);
            if (c == std::string::npos) throw ParseError("missing )");
            std::string ms = rs.substr(m + 2, c - m - 2);
            R.falloff = true;
            std::string third = (ms == "M" || ms == "m") ? "M" : ms;
            if (R.third != "<none>" && R.third != third) throw ParseError("mismatched third body");
            R.third = third;
            rs = rs.substr(0, m);
          } else if (rs.size() >= 2 && (rs.compare(rs.size() - 2, 2, "+M") == 0 ||
                                        rs.compare(rs.size() - 2, 2, "+m") == 0)) {
            if (R.falloff) throw ParseError("mismatched +M or (+M)");
            R.third_body = true;
            R.third = "M";
            rs = rs.substr(0, rs.size() - 2);
          }
          side_species(rs, R.prod, R.line);
          rx.push_back(R);
          continue;
        }
        // auxiliary data line: NAME / data / pairs, or bare keywords
        if (rx.empty()) throw ParseError("auxiliary data before first reaction");
        Reaction &R = rx.back();
        std::string rest = r;
        for (;;) {
          rest = trim(rest);
          if (rest.empty()) break;
          size_t a = rest.find('/');
          std::string name, data;
          bool has = false;
          if (a == std::string::npos) {
            name = trim(rest);
            rest.clear();
          } else {
            name = trim(rest.substr(0, a));
            size_t b = rest.find('/', a + 1);
            if (b == std::string::npos) throw ParseError("unterminated / at line " + std::to_string(L[i].no));
            data = rest.substr(a + 1, b - a - 1);
            rest = rest.substr(b + 1);
            has = true;
          }
          // a bare keyword may be followed by more pairs on the same line
          std::vector<std::string> nt = tokens(name);
          while (nt.size() > 1) {
            std::string u = upper(nt.front());
            if (u.compare(0, 3, "DUP") == 0) { nt.erase(nt.begin()); continue; }
            throw ParseError("cannot parse auxiliary line " + std::to_string(L[i].no));
          }
          name = nt.empty() ? "" : nt[0];
          std::string u = upper(name);
          std::vector<std::string> dt = tokens(data);
          if (u == "LOW") {
            if (dt.size() != 3) throw ParseError("expected 3 LOW parameters");
            R.klow.A = num_or_throw(dt[0], "LOW");
            R.klow.n = num_or_throw(dt[1], "LOW");
            R.klow.E = num_or_throw(dt[2], "LOW");
            R.have_low = true;
          } else if (u == "TROE") {
            R.ftype = kTroe3;
            for (auto &x : dt) R.fpar.push_back(num_or_throw(x, "TROE"));
            if (R.fpar.size() == 4) R.ftype = kTroe4;
            else if (R.fpar.size() != 3) throw ParseError("TROE needs 3 or 4 parameters");
          } else if (u == "SRI") {
            R.ftype = kSRI;
            for (auto &x : dt) R.fpar.push_back(num_or_throw(x, "SRI"));
            if (R.fpar.size() != 3 && R.fpar.size() != 5) throw ParseError("SRI needs 3 or 5 parameters");
          } else if (u == "REV") {
            if (!R.reversible) throw ParseError("REV on an irreversible reaction");
            if (dt.size() != 3) throw ParseError("expected 3 REV parameters");
            R.krev.A = num_or_throw(dt[0], "REV");
            R.krev.n = num_or_throw(dt[1], "REV");
            R.krev.E = num_or_throw(dt[2], "REV");
          } else if (u.compare(0, 3, "DUP") == 0) {
            // duplicate marker: no effect on the tables
          } else if (u == "PLOG") {  // CKParser.cpp:1642-1660: p [atm], A, n, E
            if (dt.size() != 4) throw ParseError("expected 4 PLOG parameters at line " + std::to_string(L[i].no));
            std::array<double, 4> v;
            for (int q = 0; q < 4; ++q) v[q] = num_or_throw(dt[q], "PLOG");
            R.plog.push_back(v);
          } else if (u == "FORD" || u == "RORD" || u == "HIGH" || u == "LT" || u == "RLT") {
            throw ParseError(u + " reactions are not supported by this build");
          } else if (!name.empty()) {
            bool is_sp = false;
            for (auto &q : sp) is_sp |= (q.name == name);
            // CKParser.cpp:1686-1700 keeps unknown keyword data without using it
            if (!is_sp) continue;
            if (!has) throw ParseError("missing efficiency for " + name);
            if (R.third == name || R.third == "M") R.e3b[name] = num_or_throw(data, "efficiency");
            else throw ParseError("third-body efficiency error at line " + std::to_string(L[i].no));
          }
        }
      }
      continue;
    }
    ++i;
  }
  if (sp.empty()) throw ParseError("no species");

  // thermo: the thermo file first, then a THERMO section of the mechanism file
  std::map<std::string, Species *> byname, byupper;
  for (auto &q : sp) {
    byname[q.name] = &q;
    byupper[upper(q.name)] = &q;
  }
  auto load_thermo = [&](const std::vector<Line> &T, size_t b, size_t e) {
    double tmid = 1000.0;
    for (size_t k = b; k < e && k < b + 3; ++k) {
      const std::string &s = T[k].text;
      if (s.size() >= 80 && s[79] == '1') break;
      std::vector<std::string> tk = tokens(s);
      double a, m, c;
      if (tk.size() >= 3 && to_num(tk[0], &a) && to_num(tk[1], &m) && to_num(tk[2], &c)) {
        tmid = m;
        break;
      }
    }
    parse_thermo_block(T, b, e, tmid, byname, byupper);
  };
  if (!therm_file.empty()) {
    std::vector<Line> T = read_lines(therm_file, false);
    size_t b = 0, e = T.size();
    for (size_t k = 0; k < T.size(); ++k)
      if (kw(T[k].text, "THER")) { b = k + 1; break; }
    for (size_t k = b; k < T.size(); ++k)
      if (kw(T[k].text, "END") && (T[k].text.size() < 80)) { e = k; break; }
    load_thermo(T, b, e);
  }
  if (thermo_begin >= 0) {
    std::vector<Line> M = read_lines(mech_file, false);
    load_thermo(M, (size_t)thermo_begin + 1, (size_t)thermo_end);
  }
  for (auto &q : sp)
    if (!q.have) throw ParseError("no thermo data for species " + q.name);

  // PLOG reactions exclude falloff, third-body and REV data (CKParser.cpp:
  // 312-350); other reactions need a non-negative prefactor
  for (auto &R : rx) {
    if (R.plog.empty()) {
      if (R.kf.A < 0.0) throw ParseError("negative prefactor at line " + std::to_string(R.line));
      continue;
    }
    if (R.falloff || R.have_low) throw ParseError("PLOG and falloff are exclusive at line " + std::to_string(R.line));
    if (R.third_body) throw ParseError("PLOG and third-body are exclusive at line " + std::to_string(R.line));
    if (R.krev.A > -1.0e299) throw ParseError("PLOG does not take REV at line " + std::to_string(R.line));
  }

  // ---- species tables
  t.nsp = (int)sp.size();
  std::map<std::string, int> idx;
  for (int k = 0; k < t.nsp; ++k) {
    idx[sp[k].name] = k;
    t.species.push_back(sp[k].name);
    double w = 0.0;  // species.cpp:44: sum over the entry's elements in order
    for (auto &e : sp[k].elements) w += e.second * elem_weight(e.first);
    t.mw.push_back(w);
    t.thermo.push_back(sp[k].tmid);
    for (int c = 0; c < 7; ++c) t.thermo.push_back(sp[k].lo[c]);
    for (int c = 0; c < 7; ++c) t.thermo.push_back(sp[k].hi[c]);
    t.thermo.push_back(0.0);
  }

  // ---- steps
  t.nrxn = (int)rx.size();
  std::vector<int> fwd_of(t.nrxn), rev_of(t.nrxn, -1);
  auto expand = [&](const std::vector<std::pair<std::string, double>> &side, std::vector<int> &out,
                    int line) {
    for (auto &p : side) {
      auto it = idx.find(p.first);
      if (it == idx.end()) throw ParseError("undeclared species " + p.first + " at line " + std::to_string(line));
      int n = (int)(p.second + 0.5);
      if (std::fabs(p.second - n) >= 1.0e-14)
        throw ParseError("non-integer stoichiometry is not supported (line " + std::to_string(line) + ")");
      for (int m = 0; m < n; ++m) out.push_back(it->second);
    }
  };
  t.reac_ptr.push_back(0);
  t.prod_ptr.push_back(0);
  for (int j = 0; j < t.nrxn; ++j) {
    const Reaction &R = rx[j];
    bool rev = R.reversible && R.krev.A != 0.0;
    t.rxn_reversible.push_back(rev ? 1 : 0);
    t.rxn_third_body.push_back(R.third_body ? 1 : 0);
    t.rxn_falloff.push_back(R.falloff ? 1 : 0);
    t.rxn_plog.push_back(R.plog.empty() ? 0 : 1);
    fwd_of[j] = (int)t.step_rxn.size();
    t.step_rxn.push_back(j);
    t.step_dir.push_back(1);
    expand(R.reac, t.reac_spc, R.line);
    expand(R.prod, t.prod_spc, R.line);
    t.reac_ptr.push_back((int)t.reac_spc.size());
    t.prod_ptr.push_back((int)t.prod_spc.size());
    if (rev) {
      rev_of[j] = (int)t.step_rxn.size();
      t.step_rxn.push_back(j);
      t.step_dir.push_back(-1);
      expand(R.prod, t.reac_spc, R.line);
      expand(R.reac, t.prod_spc, R.line);
      t.reac_ptr.push_back((int)t.reac_spc.size());
      t.prod_ptr.push_back((int)t.prod_spc.size());
    }
  }
  t.nstep = (int)t.step_rxn.size();
  auto order = [&](int s) { return (double)(t.reac_ptr[s + 1] - t.reac_ptr[s]); };

  // ---- Arrhenius steps with the distinct-parameter merge
  struct AE {
    int step;
    double A, n, Ta;
  };
  std::vector<AE> ae;
  for (int s = 0; s < t.nstep; ++s) {
    const Reaction &R = rx[t.step_rxn[s]];
    const RCoef *k = nullptr;
    if (t.step_dir[s] == 1) {
      if (R.plog.empty()) k = &R.kf;  // PLOG steps have their own list
    } else if (R.krev.A > 0.0) {
      k = &R.krev;
    }
    if (!k) continue;
    AE e;
    e.step = s;
    e.A = k->A * std::pow(kConvertC, (1.0 - order(s)));
    e.n = k->n;
    e.Ta = k->E * convertE;
    if (R.third_body) e.A /= kConvertC;
    ae.push_back(e);
  }
  auto less_arr = [](const AE &x, const AE &y) {
    if (x.A != y.A) return x.A < y.A;
    if (x.Ta != y.Ta) return x.Ta > y.Ta;
    if (x.n != y.n) return x.n < y.n;
    return x.step < y.step;
  };
  auto same = [](const AE &x, const AE &y) {
    auto diff = [](double a, double b) { return std::fabs(a - b) > kArrheniusRtol * std::fabs(0.5 * (a + b)) && std::fabs(a - b) > 0.0; };
    return !(diff(x.A, y.A) || diff(x.n, y.n) || diff(x.Ta, y.Ta));
  };
  std::vector<AE> sorted = ae;
  std::sort(sorted.begin(), sorted.end(), less_arr);
  std::vector<std::pair<int, AE>> per_step;  // step -> distinct params
  if (!sorted.empty()) {
    AE last = sorted[0];
    AE lead = sorted[0];
    lead.A = std::log(sorted[0].A);
    for (size_t k = 0; k < sorted.size(); ++k) {
      if (k > 0 && !same(last, sorted[k])) {
        last = sorted[k];
        lead = sorted[k];
        lead.A = std::log(sorted[k].A);
      }
      per_step.push_back({sorted[k].step, lead});
    }
  }
  std::sort(per_step.begin(), per_step.end(), [](const std::pair<int, AE> &a, const std::pair<int, AE> &b) { return a.first < b.first; });
  for (auto &p : per_step) {
    t.arr_step.push_back(p.first);
    t.arr_lnA.push_back(p.second.A);
    t.arr_n.push_back(p.second.n);
    t.arr_Ta.push_back(p.second.Ta);
  }

  // ---- reverse steps from equilibrium constants
  for (int j = 0; j < t.nrxn; ++j) {
    const Reaction &R = rx[j];
    if (R.reversible && R.krev.A < 0.0) {
      int f = fwd_of[j];
      t.keq_step.push_back(rev_of[j]);
      t.keq_fwd.push_back(f);
      t.keq_dn.push_back((double)((t.prod_ptr[f + 1] - t.prod_ptr[f]) - (t.reac_ptr[f + 1] - t.reac_ptr[f])));
    }
  }

  // ---- PLOG reactions (rate_const.cpp:1146-1185, plog_reaction.cpp:8-132):
  // pressure [atm] -> Pa, E -> K, A * convertC^(1 - order); lines sorted by
  // pressure (selection sort: the first strict minimum of the rest swaps in),
  // then grouped into distinct pressures at relative tolerance 1e-8
  t.plog_pt_ptr.push_back(0);
  t.plog_ln_ptr.push_back(0);
  for (int j = 0; j < t.nrxn; ++j) {
    const Reaction &R = rx[j];
    if (R.plog.empty()) continue;
    const int f = fwd_of[j];
    t.plog_step.push_back(f);
    std::vector<std::array<double, 5>> ln;  // p, ln|A|, sign, n, Ta
    for (auto &v : R.plog) {
      const double A = v[1] * std::pow(kConvertC, (1.0 - order(f)));
      ln.push_back({v[0] * kPatm, std::log(std::fabs(A)), (A < 0.0) ? -1.0 : 1.0, v[2], v[3] * convertE});
    }
    for (size_t a = 0; a + 1 < ln.size(); ++a) {
      size_t mi = a;
      for (size_t b = a + 1; b < ln.size(); ++b)
        if (ln[b][0] < ln[mi][0]) mi = b;
      if (mi != a) std::swap(ln[a], ln[mi]);
    }
    double last = ln[0][0];
    t.plog_p.push_back(last);
    for (size_t a = 0; a < ln.size(); ++a) {
      if (a > 0 && std::fabs(ln[a][0] - last) > std::fabs(last * 1.0e-8)) {
        t.plog_ln_ptr.push_back((int)t.plog_lnA.size());
        last = ln[a][0];
        t.plog_p.push_back(last);
      }
      t.plog_lnA.push_back(ln[a][1]);
      t.plog_sgn.push_back(ln[a][2]);
      t.plog_n.push_back(ln[a][3]);
      t.plog_Ta.push_back(ln[a][4]);
    }
    t.plog_ln_ptr.push_back((int)t.plog_lnA.size());
    t.plog_pt_ptr.push_back((int)t.plog_p.size());
  }
  for (double p : t.plog_p) t.plog_lnp.push_back(std::log(p));

  // ---- third-body and falloff lists
  t.tb_ptr.push_back(0);
  t.fo_ptr.push_back(0);
  for (int j = 0; j < t.nrxn; ++j) {
    const Reaction &R = rx[j];
    if (R.third_body) {
      t.tb_fwd.push_back(fwd_of[j]);
      t.tb_rev.push_back(rev_of[j]);
      for (auto &e : R.e3b) {
        auto it = idx.find(e.first);
        if (it == idx.end()) continue;
        t.tb_spc.push_back(it->second);
        t.tb_alpha.push_back(e.second - 1.0);
      }
      t.tb_ptr.push_back((int)t.tb_spc.size());
    }
    if (R.falloff) {
      if (!R.have_low) throw ParseError("falloff reaction without LOW at line " + std::to_string(R.line));
      t.fo_fwd.push_back(fwd_of[j]);
      t.fo_rev.push_back(rev_of[j]);
      int fs = -1;
      if (R.third != "M") {
        auto it = idx.find(R.third);
        if (it == idx.end()) throw ParseError("unknown falloff species " + R.third);
        fs = it->second;
      }
      t.fo_spc.push_back(fs);
      if (fs < 0) {
        for (auto &e : R.e3b) {
          auto it = idx.find(e.first);
          if (it == idx.end()) continue;
          t.fo_eff_spc.push_back(it->second);
          t.fo_alpha.push_back(e.second - 1.0);
        }
      }
      t.fo_ptr.push_back((int)t.fo_eff_spc.size());
      double p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      double Alow = R.klow.A * std::pow(kConvertC, -order(fwd_of[j]));
      p[0] = std::log(Alow);
      p[1] = R.klow.n;
      p[2] = R.klow.E * convertE;
      t.fo_type.push_back(R.ftype);
      if (R.ftype == kTroe3 || R.ftype == kTroe4) {
        p[3] = R.fpar[0];
        p[4] = R.fpar[1];
        p[5] = R.fpar[2];
        if (R.ftype == kTroe4) p[6] = R.fpar[3];
      } else if (R.ftype == kSRI) {
        p[3] = R.fpar[0];
        p[4] = R.fpar[1];
        p[5] = (R.fpar[2] > 0) ? 1.0 / R.fpar[2] : -1.0;
        p[6] = (R.fpar.size() >= 4) ? R.fpar[3] : 1.0;
        p[7] = (R.fpar.size() >= 5) ? R.fpar[4] : 0.0;
      }
      for (int k = 0; k < 8; ++k) t.fo_par.push_back(p[k]);
    }
  }
  return t;
}

JacPattern build_jac_pattern(const MechTables &t) {
  const int ns = t.nsp, nv = ns + 1;
  std::vector<int> mark((size_t)nv * nv, 0);  // [col*nv + row]
  for (int j = 0; j < ns; ++j) {
    mark[(size_t)j * nv + j] = 1;
    mark[(size_t)j * nv + ns] = 1;
  }
  for (int k = 0; k < nv; ++k) mark[(size_t)ns * nv + k] = 1;
  JacPattern p;
  p.n = nv;
  for (int s = 0; s < t.nstep; ++s) {
    for (int a = t.reac_ptr[s]; a < t.reac_ptr[s + 1]; ++a) {
      int col = t.reac_spc[a];
      for (int b = t.reac_ptr[s]; b < t.reac_ptr[s + 1]; ++b) {
        int row = t.reac_spc[b];
        mark[(size_t)col * nv + row] = 1;
        p.des_conc.push_back(col); p.des_step.push_back(s); p.des_nz.push_back(row);
      }
      for (int b = t.prod_ptr[s]; b < t.prod_ptr[s + 1]; ++b) {
        int row = t.prod_spc[b];
        mark[(size_t)col * nv + row] = 1;
        p.cre_conc.push_back(col); p.cre_step.push_back(s); p.cre_nz.push_back(row);
      }
    }
  }
  std::vector<int> addr((size_t)nv * nv, -1);
  p.col_ptr.assign(nv + 1, 0);
  int cnt = 0;
  for (int j = 0; j < nv; ++j) {
    for (int k = 0; k < nv; ++k)
      if (mark[(size_t)j * nv + k]) {
        addr[(size_t)j * nv + k] = cnt++;
        p.row_idx.push_back(k);
      }
    p.col_ptr[j + 1] = cnt;
  }
  p.nnz = cnt;
  p.last_row.resize(nv);
  for (int j = 0; j < nv; ++j) p.last_row[j] = addr[(size_t)j * nv + ns];
  for (size_t q = 0; q < p.des_nz.size(); ++q) p.des_nz[q] = addr[(size_t)p.des_conc[q] * nv + p.des_nz[q]];
  for (size_t q = 0; q < p.cre_nz.size(); ++q) p.cre_nz[q] = addr[(size_t)p.cre_conc[q] * nv + p.cre_nz[q]];
  return p;
}

}  // namespace zrk
