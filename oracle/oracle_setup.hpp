// Oracle (test infrastructure only): restatement of the reference's setup
// (L4) in REAL*4, so that the per-step restatement and the product can be fed
// identical tables, maps and topology.  Every routine cites the reference
// file:line it follows.  Arrays keep Fortran's 1-based indices: a 1-D array
// has an unused slot 0; a 2-D array (I,A) is column-major, element
// (I,A) at [(A-1)*ld + (I-1)].
#pragma once
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>
#include "oracle_io.hpp"

namespace orc {

struct Tab {  // one tabulated family: X(NT,0:W-1) and POT/FORCE, type-fastest
  int nt = 0, w = 0;
  std::vector<float> x, pot, force, bin;  // x/pot/force: [t-1 + nt*k]
  std::vector<int> ndat;                  // 1-based
  void alloc(int n, int width) {
    nt = n; w = width;
    x.assign((size_t)n * width, 0.f); pot.assign((size_t)n * width, 0.f); force.assign((size_t)n * width, 0.f);
    bin.assign(n + 1, 0.f); ndat.assign(n + 1, 0);
  }
  float& X(int t, int k) { return x[(size_t)(t - 1) + (size_t)nt * k]; }
  float& P(int t, int k) { return pot[(size_t)(t - 1) + (size_t)nt * k]; }
  float& F(int t, int k) { return force[(size_t)(t - 1) + (size_t)nt * k]; }
};

struct Setup {
  std::string err;
  // UNIT.f90
  float KB, NA, PI, MMOLY, MASSSCALE, RSCALE, ESCALE, TEMPSCALE, PSCALE, TIMESCALE,
      FSCALE, DSCALE, VSCALE, CONV, R2D, D2R;
  // RDCONTROL.f90
  int ENSEMBLE = 10, RESTART = 10, NATOMS = 0, NSTEP = 0, NVIRTA = 0, NITEMS = 0, IBRDESCR = 10,
      NONBEXC_ATOM = 4, NONBEXC_BEAD = 4, NUPDATE = 1, NTRJ = 1, HALT_DRIFT = 1, NMTS = 0;
  float TEMP0 = 0, TEMP = 0, TEMP_IN = 0, PRESSURE0 = 0, PRESSURE = 0, DT0 = 0, DT = 0, TAUT0 = 0,
        TAUT = 0, TAUP0 = 0, TAUP = 0, BETA0 = 0, BETA = 0, RCUT_ATOM = 0, RCUTSQ_ATOM = 0,
        RLIST_ATOM = 0, RCUT_BEAD = 0, RCUTSQ_BEAD = 0, RLIST_BEAD = 0;
  // ALLOCATEVAR.f90
  float FAC = 0, PFAC = 0, MKTEMP = 0, MKTEMP_ATOM = 0, MKTEMP_BEAD = 0;
  // RDINTERACT.f90
  int NTYPE = 0;
  std::vector<float> MASS0, MASS, INVMASS;  // 1-based
  std::vector<char> NAME_LABEL;             // first character of the A/B label
  Tab bond, bend, tors, nb, oop;            // nb is stored index-fastest in the reference; the
                                            // values are the same, only the layout differs
  std::vector<int> IBONDT, INBONDT, IANGT, ITORT, IOOPT;  // dense 0-based [t1-1 + NTYPE*(t2-1)+...]
  std::vector<int> BOND_TYPE_LABEL, ANGLE_TYPE_LABEL, TORSION_TYPE_LABEL, OOP_TYPE_LABEL;  // 1-based
  // RDCOOR.f90
  float BOX[3] = {0, 0, 0}, BOXINV[3], BOX2[3];
  float INITIME = 0;
  int NMOL = 0;
  std::vector<int> NATM;
  std::vector<int> ITYPE, TYPE_LABEL, NBONDS, MOL;  // 1-based, NITEMS
  std::vector<int> JBOND;                           // (NITEMS,4)
  std::vector<float> SXYZ, VXYZ;                    // (3,NITEMS) / (3,NATOMS) at [3*(i-1)+c]
  // RDVIRTUAL.f90
  std::vector<int> VITYPE, VIRT_CENTER, VIRT_NUMATOMS, VIRT_ATM_IND;  // VIRT_ATM_IND(NVIRTA,MAXV)
  int VIRT_MAXATOMS = 0;
  std::vector<float> VIRT_MASS, VIRT_INVMASS, VIRT_MASSCOEFF;  // coeff (NTYPE,NTYPE) 0-based dense
  // MAKE_LISTS.f90
  int NUMATOMS = 0, NUMBEADS = 0, NCOARSE = 0;
  std::vector<int> ATOM, BEAD;  // 1-based
  // SETLIS.f90 (ld NITEMS for angles, NATOMS for torsion/OOP)
  std::vector<int> NIJK, JANGLEIJK, KANGLEIJK, NOANGLEIJK, NOJANGLEIJK, NOKANGLEIJK;
  std::vector<int> NIJKL, JTORIJKL, KTORIJKL, LTORIJKL, FNIJKL, FJTORIJKL, FKTORIJKL, FLTORIJKL;
  std::vector<int> NOOPIJKL, JOOPIJKL, KOOPIJKL, LOOPIJKL;
  // BUILD_CONNECTIVITY.f90 / RDVIRTBONDS.f90
  static const int MAXCONNECTIONS = 20;
  std::vector<int> CONNECTIONS, CONNECTED_TO;  // CONNECTED_TO(NITEMS,20)
  int connectivity_overflow = 0;               // rows that would overrun 20 entries
  // ALLOCATEVAR2.f90
  int NCELLX_ATOM = 0, NCELLY_ATOM = 0, NCELLZ_ATOM = 0, NCELLX_BEAD = 0, NCELLY_BEAD = 0, NCELLZ_BEAD = 0;
  // sizes of the per-atom bonded slots
  static const int MAXBONDS = 4, MAXANG = 10, MAXTOR = 10, MAXOOP = 20;

  int& jbond(int i, int a) { return JBOND[(size_t)(a - 1) * NITEMS + (i - 1)]; }
  int& jang(int i, int a) { return JANGLEIJK[(size_t)(a - 1) * NITEMS + (i - 1)]; }
  int& kang(int i, int a) { return KANGLEIJK[(size_t)(a - 1) * NITEMS + (i - 1)]; }
  int& nojang(int i, int a) { return NOJANGLEIJK[(size_t)(a - 1) * NITEMS + (i - 1)]; }
  int& nokang(int i, int a) { return NOKANGLEIJK[(size_t)(a - 1) * NITEMS + (i - 1)]; }
  int& jtor(int i, int a) { return JTORIJKL[(size_t)(a - 1) * NATOMS + (i - 1)]; }
  int& ktor(int i, int a) { return KTORIJKL[(size_t)(a - 1) * NATOMS + (i - 1)]; }
  int& ltor(int i, int a) { return LTORIJKL[(size_t)(a - 1) * NATOMS + (i - 1)]; }
  int& fjtor(int i, int a) { return FJTORIJKL[(size_t)(a - 1) * NATOMS + (i - 1)]; }
  int& fktor(int i, int a) { return FKTORIJKL[(size_t)(a - 1) * NATOMS + (i - 1)]; }
  int& fltor(int i, int a) { return FLTORIJKL[(size_t)(a - 1) * NATOMS + (i - 1)]; }
  int& joop(int i, int a) { return JOOPIJKL[(size_t)(a - 1) * NATOMS + (i - 1)]; }
  int& koop(int i, int a) { return KOOPIJKL[(size_t)(a - 1) * NATOMS + (i - 1)]; }
  int& loop(int i, int a) { return LOOPIJKL[(size_t)(a - 1) * NATOMS + (i - 1)]; }
  int& conn(int i, int c) { return CONNECTED_TO[(size_t)(c - 1) * NITEMS + (i - 1)]; }
  int& vatm(int v, int a) { return VIRT_ATM_IND[(size_t)(a - 1) * NVIRTA + (v - 1)]; }
  int t2(int a, int b) const { return (a - 1) + NTYPE * (b - 1); }
  int t3(int a, int b, int c) const { return (a - 1) + NTYPE * ((b - 1) + NTYPE * (c - 1)); }
  int t4(int a, int b, int c, int d) const {
    return (a - 1) + NTYPE * ((b - 1) + NTYPE * ((c - 1) + NTYPE * (d - 1)));
  }
  float& coeff(int tv, int ta) { return VIRT_MASSCOEFF[(size_t)(tv - 1) + (size_t)NTYPE * (ta - 1)]; }
};

// ---------------------------------------------------------------- UNIT.f90:9-23
inline void unit_constants(Setup& s) {
  s.KB = (float)1.380658e-23;
  s.NA = (float)6.0221367e+23;
  s.PI = 3.14159265358f;
  s.MMOLY = (float)0.012;
  s.MASSSCALE = s.MMOLY / s.NA;
  s.RSCALE = (float)1.0e-9;
  s.ESCALE = s.KB * 300.0f;
  s.TEMPSCALE = s.ESCALE / s.KB;
  s.PSCALE = (float)((double)(s.ESCALE / powf(s.RSCALE, 3.0f)) / 1000.0);
  s.TIMESCALE = s.RSCALE * sqrtf(s.MASSSCALE / s.ESCALE);
  s.FSCALE = s.ESCALE / s.RSCALE;
  s.DSCALE = s.MASSSCALE / powf(s.RSCALE, 3.0f);
  s.VSCALE = s.RSCALE / s.TIMESCALE;
  s.CONV = (float)((double)(s.NA * s.ESCALE) / 1000.0);
  s.R2D = 180.0f / s.PI;
  s.D2R = s.PI / 180.0f;
}

// ------------------------------------------------------------ RDCONTROL.f90
// Each keyword is found by rewinding and scanning (RDCONTROL.f90:59-517).
inline bool find_key(Unit& u, const char* key, std::vector<std::string>* words) {
  u.rewind();
  std::string line;
  while (u.read_a80(&line)) {
    auto w = parse_line(line);
    if (!w.empty() && w[0] == key) { *words = w; return true; }
  }
  return false;
}

inline bool rdcontrol(Setup& s, const std::string& dir) {
  Unit u;
  if (!u.open(dir + "/control")) { s.err = "File control does not exist"; return false; }
  std::vector<std::string> w;
  auto fval = [&](const char* k, float* out) -> bool {
    if (!find_key(u, k, &w) || w.size() < 2) return false;
    return parse_float(w[1], out);
  };
  auto ival = [&](const char* k, int* out) -> bool {
    if (!find_key(u, k, &w) || w.size() < 2) return false;
    return parse_int(w[1], out);
  };
  if (find_key(u, "ensemble", &w) && w.size() >= 2) {  // :59-80
    if (w[1] == "NVE" || w[1] == "nve") s.ENSEMBLE = 0;
    if (w[1] == "NVT" || w[1] == "nvt") s.ENSEMBLE = 1;
    if (w[1] == "NPT" || w[1] == "npt") s.ENSEMBLE = 2;
  }
  if (s.ENSEMBLE == 10) { s.err = "invalid ensemble"; return false; }
  if (!fval("temperature", &s.TEMP0)) { s.err = "temperature"; return false; }  // :86-92
  s.TEMP = s.TEMP0 / s.TEMPSCALE;
  s.TEMP_IN = s.TEMP;
  if (!fval("pressure", &s.PRESSURE0)) { s.err = "pressure"; return false; }  // :106-110
  s.PRESSURE = s.PRESSURE0 / s.PSCALE;
  if (!ival("atoms", &s.NATOMS)) { s.err = "atoms"; return false; }
  if (!ival("num_of_time_steps", &s.NSTEP)) { s.err = "num_of_time_steps"; return false; }
  if (!fval("time_step", &s.DT0)) { s.err = "time_step"; return false; }  // :160-165
  s.DT = (float)((double)s.DT0 * 1.0e-12 / (double)s.TIMESCALE);
  if (!ival("virtual_sites", &s.NVIRTA)) { s.err = "virtual_sites"; return false; }  // :180-191
  s.NITEMS = s.NATOMS + s.NVIRTA;
  s.IBRDESCR = s.NVIRTA > 0 ? 0 : 1;
  bool ok = fval("bead_cutoff", &s.RCUT_BEAD);  // :203-215
  if (ok) s.RCUTSQ_BEAD = s.RCUT_BEAD * s.RCUT_BEAD;
  if (!ok && s.IBRDESCR != 1) { s.err = "bead_cutoff"; return false; }
  ok = fval("bead_neighbour_list_cutoff", &s.RLIST_BEAD);  // :222-240
  if (ok && s.RLIST_BEAD < s.RCUT_BEAD) { s.err = "bead list cutoff below cutoff"; return false; }
  if (!ok && s.IBRDESCR != 1) { s.err = "bead_neighbour_list_cutoff"; return false; }
  if (s.IBRDESCR == 0) {  // :242-273
    if (!ival("non_bonded_bead", &s.NONBEXC_BEAD)) { s.err = "non_bonded_bead"; return false; }
    if (s.NONBEXC_BEAD != 4 && s.NONBEXC_BEAD != 5) { s.err = "invalid non_bonded_bead"; return false; }
  }
  if (!ival("update_neighbour_list", &s.NUPDATE)) { s.err = "update_neighbour_list"; return false; }
  ok = fval("temperature_coupling_time", &s.TAUT0);  // :298-310
  if (ok) s.TAUT = (float)((double)s.TAUT0 * 1.0e-12 / (double)s.TIMESCALE);
  if (!ok && (s.ENSEMBLE == 1 || s.ENSEMBLE == 2)) { s.err = "temperature_coupling_time"; return false; }
  ok = fval("pressure_coupling_time", &s.TAUP0);  // :316-328
  if (ok) s.TAUP = (float)((double)s.TAUP0 * 1.0e-12 / (double)s.TIMESCALE);
  if (!ok && s.ENSEMBLE == 2) { s.err = "pressure_coupling_time"; return false; }
  ok = fval("isothermal_compressibility", &s.BETA0);  // :335-347
  if (ok) s.BETA = s.BETA0 * s.PSCALE;
  if (!ok && s.ENSEMBLE == 2) { s.err = "isothermal_compressibility"; return false; }
  if (!fval("cutoff", &s.RCUT_ATOM)) { s.err = "cutoff"; return false; }  // :353-365
  s.RCUTSQ_ATOM = s.RCUT_ATOM * s.RCUT_ATOM;
  if (!fval("neighbour_list_cutoff", &s.RLIST_ATOM)) { s.err = "neighbour_list_cutoff"; return false; }
  if (s.RLIST_ATOM < s.RCUT_ATOM) { s.err = "list cutoff below cutoff"; return false; }
  if (!ival("trajectory", &s.NTRJ)) { s.err = "trajectory"; return false; }
  if (!ival("halt_drift", &s.HALT_DRIFT)) { s.err = "halt_drift"; return false; }
  if (!ival("non_bonded", &s.NONBEXC_ATOM)) { s.err = "non_bonded"; return false; }
  if (s.NONBEXC_ATOM != 4 && s.NONBEXC_ATOM != 5) { s.err = "invalid non_bonded"; return false; }
  if (find_key(u, "initialize_velocities", &w) && w.size() >= 2) {  // :462-481
    char c = w[1][0];
    if (c == 'Y' || c == 'y') s.RESTART = 1;
    if (c == 'N' || c == 'n') s.RESTART = 0;
  }
  if (s.RESTART == 10) { s.err = "initialize_velocities"; return false; }
  // :485-497: the last 'mts' line wins (the scan does not stop at the first match)
  {
    u.rewind();
    std::string line;
    bool found = false;
    while (u.read_a80(&line)) {
      auto ww = parse_line(line);
      if (!ww.empty() && ww[0] == "mts" && ww.size() >= 2) found = parse_int(ww[1], &s.NMTS);
    }
    if (!found) { s.err = "mts"; return false; }
  }
  {  // :502-517
    u.rewind();
    std::string line;
    bool found = false;
    while (u.read_a80(&line)) {
      auto ww = parse_line(line);
      if (!ww.empty() && (ww[0] == "END" || ww[0] == "end" || ww[0] == "End")) { found = true; break; }
    }
    if (!found) { s.err = "end"; return false; }
  }
  // ALLOCATEVAR.f90:42-46
  s.FAC = s.DT / s.TAUT;
  s.PFAC = s.BETA * s.DT * (float)10 / s.TAUP;
  s.MKTEMP = (float)(2.0 / (double)(float)(3.0 * (double)(s.NATOMS - 1)));
  return true;
}

// ----------------------------------------------------------- RDINTERACT.f90
inline float to_reduced(const Setup& s, float v) { return v * 1000.0f / s.NA / s.ESCALE; }

struct RawTable { std::vector<float> x, p; };

inline bool read_pairs(const std::string& path, RawTable* t, bool stop_on_error_before_convert) {
  (void)stop_on_error_before_convert;
  Unit u;
  if (!u.open(path)) return false;
  std::vector<std::string> it;
  t->x.clear(); t->p.clear();
  while (u.read_items(2, &it)) {
    float a, b;
    if (!parse_float(it[0], &a) || !parse_float(it[1], &b)) break;
    t->x.push_back(a); t->p.push_back(b);
  }
  return true;
}

inline int what_type(char c) {  // RDINTERACT.f90:754-771
  if (c == 'A' || c == 'a') return 1;
  if (c == 'B' || c == 'b') return 2;
  return 100;
}

inline bool rdinteract(Setup& s, const std::string& dir) {
  Unit u;
  if (!u.open(dir + "/interaction")) { s.err = "File interaction does not exist"; return false; }
  std::string line;
  std::vector<std::string> w;
  auto next_words = [&]() -> bool {
    if (!u.read_a80(&line)) return false;
    w = parse_line(line);
    return true;
  };
  // atom types :88-130
  if (!next_words() || w.size() < 2 || w[0] != "atom_types" || !parse_int(w[1], &s.NTYPE)) {
    s.err = "atom_types"; return false;
  }
  int NT = s.NTYPE;
  s.MASS0.assign(NT + 1, 0.f); s.MASS.assign(NT + 1, 0.f); s.INVMASS.assign(NT + 1, 0.f);
  s.NAME_LABEL.assign(NT + 1, ' ');
  u.skip();
  for (int i = 1; i <= NT; ++i) {
    if (!next_words() || w.size() < 4) { s.err = "atom type line"; return false; }
    if (w[0] == "bond_types") { s.err = "Number of atom_types different"; return false; }
    int ti;
    if (!parse_int(w[0], &ti) || ti < 1 || ti > NT) { s.err = "type index"; return false; }
    parse_float(w[2], &s.MASS0[ti]);
    s.NAME_LABEL[ti] = w[3][0];
    if (what_type(w[3][0]) == 100 || w[3].size() != 1) { s.err = "label must be A or B"; return false; }
    // :128-129  MASS(I) uses the loop index, not TYPEI
    s.MASS[i] = s.MASS0[i] / s.NA / s.MASSSCALE;
    s.INVMASS[i] = (float)(1.0 / (double)s.MASS[i]);
  }
  s.IBONDT.assign((size_t)NT * NT, 0);
  s.INBONDT.assign((size_t)NT * NT, 0);
  s.IANGT.assign((size_t)NT * NT * NT, 0);
  s.ITORT.assign((size_t)NT * NT * NT * NT, 0);
  s.IOOPT.assign((size_t)NT * NT * NT * NT, 0);
  std::vector<int> bi, bj, ai, aj, ak, ti_, tj_, tk_, tl_, oi, oj, ok_, ol;

  // bonds :144-223  (no row-0 insertion; BONDS.inc offsets by RBOND(TIJ,0))
  int nbt;
  if (!next_words() || w.size() < 2 || w[0] != "bond_types" || !parse_int(w[1], &nbt)) { s.err = "bond_types"; return false; }
  u.skip();
  std::vector<RawTable> braw(nbt);
  std::vector<std::string> bfiles(nbt);
  for (int i = 0; i < nbt; ++i) {
    if (!next_words() || w.size() < 3) { s.err = "bond line"; return false; }
    if (w[0] == "angle_types") { s.err = "Number of bond_types different"; return false; }
    int ib, jb; parse_int(w[0], &ib); parse_int(w[1], &jb);
    bi.push_back(ib); bj.push_back(jb);
    if (s.IBONDT[s.t2(ib, jb)] != 0) { s.err = "Duplicate bond"; return false; }
    s.IBONDT[s.t2(ib, jb)] = i + 1; s.IBONDT[s.t2(jb, ib)] = i + 1;
    if (!read_pairs(dir + "/" + w[2], &braw[i], false)) { s.err = "missing file " + w[2]; return false; }
  }
  {
    int maxn = 0;
    for (auto& r : braw) maxn = std::max<int>(maxn, (int)r.x.size());
    s.bond.alloc(nbt, maxn + 2);
    for (int i = 1; i <= nbt; ++i) {
      auto& r = braw[i - 1];
      int K = (int)r.x.size();
      for (int k = 0; k < K; ++k) { s.bond.X(i, k) = r.x[k]; s.bond.P(i, k) = r.p[k]; }
      s.bond.ndat[i] = K - 1;
      for (int j = 0; j <= s.bond.ndat[i]; ++j) s.bond.P(i, j) = to_reduced(s, s.bond.P(i, j));
      s.bond.bin[i] = s.bond.X(i, 1) - s.bond.X(i, 0);
    }
  }

  // angles :229-332 / torsions :337-442 / OOP :543-666 share the row-0 insertion rule
  auto read_angular = [&](Tab& T, int ntab, const std::vector<std::string>& files, bool oop_bin) -> bool {
    std::vector<RawTable> raw(ntab);
    int maxn = 0;
    for (int i = 0; i < ntab; ++i) {
      if (!read_pairs(dir + "/" + files[i], &raw[i], false)) { s.err = "missing file " + files[i]; return false; }
      maxn = std::max<int>(maxn, (int)raw[i].x.size());
    }
    T.alloc(ntab, maxn + 3);
    for (int i = 1; i <= ntab; ++i) {
      auto& r = raw[i - 1];
      if (r.x.size() < 2) { s.err = "table too short"; return false; }
      T.X(i, 0) = r.x[0]; T.P(i, 0) = to_reduced(s, r.p[0]);
      T.X(i, 1) = r.x[1]; T.P(i, 1) = to_reduced(s, r.p[1]);
      if (oop_bin && T.X(i, 1) < T.X(i, 0)) T.bin[i] = T.X(i, 0) - T.X(i, 1);
      else T.bin[i] = T.X(i, 1) - T.X(i, 0);
      int K;
      if (T.X(i, 0) != 0.0f) {
        T.X(i, 0) = 0.0f;
        T.X(i, 2) = T.X(i, 1); T.P(i, 2) = T.P(i, 1);
        T.X(i, 1) = T.bin[i]; T.P(i, 1) = T.P(i, 0);
        K = 3;
      } else {
        K = 2;
      }
      for (size_t k = 2; k < r.x.size(); ++k) {
        T.X(i, K) = r.x[k]; T.P(i, K) = to_reduced(s, r.p[k]);
        ++K;
      }
      T.ndat[i] = K - 1;
    }
    return true;
  };

  int nat;
  if (!next_words() || w.size() < 2 || w[0] != "angle_types" || !parse_int(w[1], &nat)) { s.err = "angle_types"; return false; }
  u.skip();
  std::vector<std::string> afiles;
  for (int i = 0; i < nat; ++i) {
    if (!next_words() || w.size() < 4) { s.err = "angle line"; return false; }
    if (w[0] == "torsion_types") { s.err = "Number of angle_types different"; return false; }
    int ia, ja, ka; parse_int(w[0], &ia); parse_int(w[1], &ja); parse_int(w[2], &ka);
    ai.push_back(ia); aj.push_back(ja); ak.push_back(ka);
    if (s.IANGT[s.t3(ia, ja, ka)] != 0) { s.err = "Duplicate angle"; return false; }
    s.IANGT[s.t3(ia, ja, ka)] = i + 1; s.IANGT[s.t3(ka, ja, ia)] = i + 1;
    afiles.push_back(w[3]);
  }
  if (!read_angular(s.bend, nat, afiles, false)) return false;

  int ntt;
  if (!next_words() || w.size() < 2 || w[0] != "torsion_types" || !parse_int(w[1], &ntt)) { s.err = "torsion_types"; return false; }
  u.skip();
  std::vector<std::string> tfiles;
  for (int i = 0; i < ntt; ++i) {
    if (!next_words() || w.size() < 5) { s.err = "torsion line"; return false; }
    if (w[0] == "non_bonded_interaction_types") { s.err = "Number of torsion_types different"; return false; }
    int a, b, c, d; parse_int(w[0], &a); parse_int(w[1], &b); parse_int(w[2], &c); parse_int(w[3], &d);
    ti_.push_back(a); tj_.push_back(b); tk_.push_back(c); tl_.push_back(d);
    if (s.ITORT[s.t4(a, b, c, d)] != 0) { s.err = "Duplicate torsion"; return false; }
    s.ITORT[s.t4(a, b, c, d)] = i + 1; s.ITORT[s.t4(d, c, b, a)] = i + 1;
    tfiles.push_back(w[4]);
  }
  if (!read_angular(s.tors, ntt, tfiles, false)) return false;

  // nonbonded :448-537
  int nnb;
  if (!next_words() || w.size() < 2 || w[0] != "non_bonded_interaction_types" || !parse_int(w[1], &nnb)) {
    s.err = "non_bonded_interaction_types"; return false;
  }
  u.skip();
  {
    std::vector<RawTable> raw(nnb);
    int maxn = 0;
    for (int i = 0; i < nnb; ++i) {
      if (!next_words() || w.size() < 3) { s.err = "nonbonded line"; return false; }
      if (w[0] == "Out_of_Planes") { s.err = "Number of non_bonded_interaction_types different"; return false; }
      int a, b; parse_int(w[0], &a); parse_int(w[1], &b);
      if (s.INBONDT[s.t2(a, b)] != 0) { s.err = "Duplicate nonbonded"; return false; }
      s.INBONDT[s.t2(a, b)] = i + 1; s.INBONDT[s.t2(b, a)] = i + 1;
      if (!read_pairs(dir + "/" + w[2], &raw[i], false)) { s.err = "missing file " + w[2]; return false; }
      maxn = std::max<int>(maxn, (int)raw[i].x.size());
    }
    s.nb.alloc(nnb, maxn + 3);
    for (int i = 1; i <= nnb; ++i) {
      auto& r = raw[i - 1];
      if (r.x.size() < 2) { s.err = "table too short"; return false; }
      s.nb.X(i, 0) = r.x[0]; s.nb.P(i, 0) = to_reduced(s, r.p[0]);
      s.nb.X(i, 1) = r.x[1]; s.nb.P(i, 1) = to_reduced(s, r.p[1]);
      s.nb.bin[i] = s.nb.X(i, 1) - s.nb.X(i, 0);
      int K;
      if (s.nb.X(i, 0) != 0.0f) {
        s.nb.X(i, 0) = 0.0f;
        s.nb.X(i, 2) = s.nb.X(i, 1); s.nb.P(i, 2) = s.nb.P(i, 1);
        s.nb.X(i, 1) = s.nb.bin[i]; s.nb.P(i, 1) = s.nb.P(i, 0);
        K = 3;
      } else {
        K = 2;
      }
      for (size_t k = 2; k < r.x.size(); ++k) {
        s.nb.X(i, K) = r.x[k]; s.nb.P(i, K) = to_reduced(s, r.p[k]);
        ++K;
      }
      s.nb.ndat[i] = K - 1;
    }
  }

  // out of planes :543-666
  int notype;
  if (!next_words() || w.size() < 2 || w[0] != "Out_of_Planes" || !parse_int(w[1], &notype)) { s.err = "Out_of_Planes"; return false; }
  u.skip();
  std::vector<std::string> ofiles;
  for (int i = 0; i < notype; ++i) {
    if (!next_words() || w.size() < 5) { s.err = "Number of Out_of_Planes different"; return false; }
    int a, b, c, d; parse_int(w[0], &a); parse_int(w[1], &b); parse_int(w[2], &c); parse_int(w[3], &d);
    oi.push_back(a); oj.push_back(b); ok_.push_back(c); ol.push_back(d);
    if (s.IOOPT[s.t4(a, b, c, d)] != 0) { s.err = "Duplicate out of plane"; return false; }
    s.IOOPT[s.t4(a, b, c, d)] = i + 1;
    ofiles.push_back(w[4]);
  }
  if (notype > 0) {
    std::string l2;
    if (u.read_a80(&l2)) { s.err = "Number of Out_of_Planes different"; return false; }  // :596-606
  }
  if (!read_angular(s.oop, notype, ofiles, true)) return false;

  // class labels :676-749
  auto lab = [&](int t) { return what_type(s.NAME_LABEL[t]); };
  s.BOND_TYPE_LABEL.assign(nbt + 1, 0);
  for (int i = 1; i <= nbt; ++i) {
    int h = lab(bi[i - 1]) + lab(bj[i - 1]);
    s.BOND_TYPE_LABEL[i] = h == 2 ? 1 : (h == 4 ? 2 : 3);
  }
  s.ANGLE_TYPE_LABEL.assign(nat + 1, 0);
  for (int i = 1; i <= nat; ++i) {
    int h = lab(ai[i - 1]) + lab(aj[i - 1]) + lab(ak[i - 1]);
    s.ANGLE_TYPE_LABEL[i] = h == 3 ? 1 : (h == 6 ? 2 : 3);
  }
  s.TORSION_TYPE_LABEL.assign(ntt + 1, 0);
  for (int i = 1; i <= ntt; ++i) {
    int h = lab(ti_[i - 1]) + lab(tj_[i - 1]) + lab(tk_[i - 1]) + lab(tl_[i - 1]);
    s.TORSION_TYPE_LABEL[i] = h == 4 ? 1 : (h == 8 ? 2 : 3);
  }
  s.OOP_TYPE_LABEL.assign(notype + 1, 0);
  for (int i = 1; i <= notype; ++i) {
    int h = lab(oi[i - 1]) + lab(oj[i - 1]) + lab(ok_[i - 1]) + lab(ol[i - 1]);
    s.OOP_TYPE_LABEL[i] = h == 4 ? 1 : (h == 8 ? 2 : 3);
  }
  return true;
}

// ---------------------------------------------------------------- RDCOOR.f90
inline bool rdcoor(Setup& s, const std::string& dir) {
  Unit u;
  if (!u.open(dir + "/coordinate")) { s.err = "File coordinate does not exist"; return false; }
  std::string line;
  std::vector<std::string> it;
  if (!u.read_a80(&line)) { s.err = "coordinate header"; return false; }  // :55-58 (TITLE)
  if (!u.read_a80(&line)) { s.err = "coordinate header"; return false; }  // :60-65
  {
    auto w = parse_line(line);
    if (w.size() >= 2 && w[0] == "Time") parse_float(w[1], &s.INITIME);
  }
  u.skip();
  if (!u.read_items(3, &it)) { s.err = "box"; return false; }  // :67
  for (int c = 0; c < 3; ++c) parse_float(it[c], &s.BOX[c]);
  for (int c = 0; c < 3; ++c) { s.BOXINV[c] = 1.0f / s.BOX[c]; s.BOX2[c] = s.BOX[c] / 2.0f; }
  for (int k = 0; k < 5; ++k) u.skip();
  if (!u.read_items(2, &it) || !parse_int(it[1], &s.NMOL)) { s.err = "num_of_molecules"; return false; }
  const int N = s.NITEMS, NA_ = s.NATOMS;
  s.NATM.assign(s.NMOL + 1, 0);
  s.ITYPE.assign(N + 1, 0); s.TYPE_LABEL.assign(N + 1, 1); s.NBONDS.assign(N + 1, 0); s.MOL.assign(NA_ + 1, 0);
  s.JBOND.assign((size_t)N * Setup::MAXBONDS, 0);
  s.SXYZ.assign((size_t)3 * N, 0.f); s.VXYZ.assign((size_t)3 * NA_, 0.f);
  int L = 0;
  for (int i = 1; i <= s.NMOL; ++i) {
    if (!u.read_items(4, &it) || !parse_int(it[0], &s.NATM[i])) { s.err = "molecule name missing"; return false; }
    for (int j = 1; j <= s.NATM[i]; ++j) {
      ++L;
      if (L > NA_) { s.err = "No. Atoms in coordinate does not equal NATOMS"; return false; }
      if (!u.read_items(6, &it)) { s.err = "RDCOOR"; return false; }  // :103
      int ll;
      parse_int(it[0], &ll); parse_int(it[1], &s.ITYPE[L]); parse_int(it[2], &s.NBONDS[L]);
      for (int c = 0; c < 3; ++c) parse_float(it[3 + c], &s.SXYZ[3 * (L - 1) + c]);
      int nb = s.NBONDS[L];
      if (nb < 0 || nb > Setup::MAXBONDS) { s.err = "too many bonds"; return false; }
      if (!u.read_items(3 + nb, &it)) { s.err = "RDCOOR"; return false; }  // :104
      for (int c = 0; c < 3; ++c) parse_float(it[c], &s.VXYZ[3 * (L - 1) + c]);
      for (int k = 1; k <= nb; ++k) parse_int(it[3 + k - 1], &s.jbond(L, k));
      s.MOL[L] = i;
      if (s.IBRDESCR == 0) {  // :110-123
        char c = s.NAME_LABEL[s.ITYPE[L]];
        if (c == 'A' || c == 'a') s.TYPE_LABEL[L] = 1;
        else if (c == 'B' || c == 'b') s.TYPE_LABEL[L] = 2;
        else { s.err = "label must be A or B"; return false; }
      }
      for (int c = 0; c < 3; ++c) {  // :125
        float& v = s.VXYZ[3 * (L - 1) + c];
        v = v * 1.e3f / s.VSCALE;
      }
    }
  }
  if (L != NA_) { s.err = "No. Atoms in coordinate does not equal NATOMS"; return false; }
  return true;
}

// ------------------------------------------------------------ RDVIRTUAL.f90
inline bool rdvirtual(Setup& s, const std::string& dir) {
  Unit u;
  if (!u.open(dir + "/virtual")) { s.err = "File virtual site does not exist"; return false; }
  std::vector<std::string> it;
  u.skip(); u.skip();
  int nv;
  if (!u.read_items(1, &it) || !parse_int(it[0], &nv)) { s.err = "virtual header"; return false; }
  s.NVIRTA = nv;  // :210 (the file's count wins)
  u.skip(); u.skip();
  const int NT = s.NTYPE, MAXA = 15;
  s.VIRT_NUMATOMS.assign(NT + 1, 0);
  s.VIRT_MASS.assign(NT + 1, 0.f); s.VIRT_INVMASS.assign(NT + 1, 0.f);
  s.VIRT_MASSCOEFF.assign((size_t)NT * NT, 0.f);
  s.VITYPE.assign(nv + 1, 0); s.VIRT_CENTER.assign(nv + 1, 0);
  std::vector<int> indx((size_t)nv * MAXA, 0);
  for (int i = 1; i <= nv; ++i) {  // :236-263
    if (!u.read_items(4, &it)) { s.err = "ERROR READING VIRTUAL, TOO SHORT"; return false; }
    int k = 0, numatom = 0;
    parse_int(it[0], &k); parse_int(it[1], &s.VITYPE[i]); parse_int(it[2], &numatom); parse_int(it[3], &s.VIRT_CENTER[i]);
    s.ITYPE[s.NATOMS + i] = s.VITYPE[i];
    if (numatom > MAXA) { s.err = "Number of atoms in VS exceeds maximum"; return false; }
    if (!u.read_items(numatom, &it)) { s.err = "ERROR READING VIRTUAL, TOO SHORT"; return false; }
    for (int j = 0; j < numatom; ++j) parse_int(it[j], &indx[(size_t)(i - 1) * MAXA + j]);
    int& vn = s.VIRT_NUMATOMS[s.VITYPE[i]];
    if (vn == 0) vn = numatom;
    else if (vn != numatom) { s.err = "Disagreement in number of atoms in a VS type"; return false; }
  }
  int amax = 0;
  for (int t = 1; t <= NT; ++t) amax = std::max(amax, s.VIRT_NUMATOMS[t]);
  s.VIRT_MAXATOMS = amax;
  s.VIRT_ATM_IND.assign((size_t)nv * std::max(amax, 1), 0);
  for (int i = 1; i <= nv; ++i)
    for (int j = 1; j <= s.VIRT_NUMATOMS[s.VITYPE[i]]; ++j) s.vatm(i, j) = indx[(size_t)(i - 1) * MAXA + (j - 1)];
  for (int i = 1; i <= nv; ++i) {  // :287-309
    int ti = s.VITYPE[i];
    double sum = 0.0;
    for (int j = 1; j <= s.VIRT_NUMATOMS[ti]; ++j) sum += (double)s.MASS[s.ITYPE[s.vatm(i, j)]];
    if (s.VIRT_MASS[ti] == 0.0f) {
      s.VIRT_MASS[ti] = (float)sum;
      s.VIRT_INVMASS[ti] = (float)(1.0 / sum);
    } else if (std::fabs((double)s.VIRT_MASS[ti] - sum) > (double)0.0001f) {
      s.err = "Disagreement in VS mass"; return false;
    }
    for (int j = 1; j <= s.VIRT_NUMATOMS[ti]; ++j) {
      int tj = s.ITYPE[s.vatm(i, j)];
      s.coeff(ti, tj) = s.MASS[tj] * s.VIRT_INVMASS[ti];
    }
  }
  return true;
}

// ------------------------------------------------------------ MAKE_LISTS.f90
inline bool make_lists(Setup& s) {
  if (s.IBRDESCR != 0) {  // main.F90:139-146
    s.NUMATOMS = s.NATOMS; s.NUMBEADS = 0; s.NCOARSE = 0;
    s.ATOM.assign(s.NUMATOMS + 1, 0);
    for (int i = 1; i <= s.NATOMS; ++i) s.ATOM[i] = i;
    s.BEAD.assign(1, 0);
    return true;
  }
  s.NUMATOMS = 0; s.NUMBEADS = 0;  // MAKE_LISTS.f90:24-60
  for (int i = 1; i <= s.NATOMS; ++i) {
    if (s.TYPE_LABEL[i] == 1) ++s.NUMATOMS;
    else if (s.TYPE_LABEL[i] == 2) ++s.NUMBEADS;
    else { s.err = "invalid type label"; return false; }
  }
  s.NCOARSE = s.NUMBEADS + s.NVIRTA;
  s.ATOM.assign(s.NUMATOMS + 1, 0); s.BEAD.assign(s.NCOARSE + 1, 0);
  int na = 0, nb = 0;
  for (int i = 1; i <= s.NATOMS; ++i) {
    if (s.TYPE_LABEL[i] == 1) s.ATOM[++na] = i;
    else s.BEAD[++nb] = i;
  }
  for (int i = 1; i <= s.NVIRTA; ++i) s.BEAD[++nb] = s.NATOMS + i;
  return true;
}

// ---------------------------------------------------------------- FTABLE.f90
inline void ftable(Setup& s) {
  Tab& b = s.bond;  // :26-32, including the vector-subscript store at :31
  for (int i = 1; i <= b.nt; ++i) {
    for (int j = 1; j <= b.ndat[i] - 1; ++j) {
      float t = -(b.P(i, j + 1) - b.P(i, j - 1)) / b.bin[i] / b.X(i, j);
      b.F(i, j) = (float)((double)t / 2.0);
    }
    b.F(i, 0) = b.F(i, 1);
    float last = b.F(i, b.ndat[i] - 1);
    for (int k = 1; k <= b.nt; ++k) b.F(i, b.ndat[k]) = last;
  }
  auto angular = [&](Tab& T, bool tail_from_zero) {  // :35-43, :47-55, :78-86
    for (int i = 1; i <= T.nt; ++i) {
      for (int j = 1; j <= T.ndat[i] - 1; ++j) {
        float t = -(T.P(i, j + 1) - T.P(i, j - 1)) / T.bin[i] / s.D2R;
        T.F(i, j) = (float)((double)t / 2.0);
      }
      T.F(i, 0) = T.F(i, 1);
      T.F(i, T.ndat[i]) = tail_from_zero ? T.F(i, 0) : T.F(i, T.ndat[i] - 1);
    }
  };
  angular(s.bend, false);
  angular(s.tors, true);
  angular(s.oop, true);
  Tab& n = s.nb;  // :59-75 (runs to NDATNB, using the zero POT row NDATNB+1)
  for (int i = 1; i <= n.nt; ++i) {
    for (int j = 1; j <= n.ndat[i]; ++j) {
      float t = -(n.P(i, j + 1) - n.P(i, j - 1)) / n.bin[i] / n.X(i, j);
      n.F(i, j) = (float)((double)t / 2.0);
    }
    n.F(i, 0) = n.F(i, 1);
  }
}

// ---------------------------------------------------------------- SCALEV.f90
// SCALEV.f90:13-26, called at main.F90:168-171 when initialize_velocities is
// Y.  The reference calls COMVEL (COMVEL.f90:17-79) first, which draws new
// velocities from gfortran's RANDOM_NUMBER; that draw is not reproducible, so
// the coordinate file's velocities stand in for it.  EK and FACTOR are REAL*8,
// each term MASS*(vx**2+vy**2+vz**2) REAL*4; the scaled velocity is rounded
// back to REAL*4.
inline void scalev(Setup& s) {
  double ek = 0.0;
  for (int i = 1; i <= s.NATOMS; ++i) {
    const float* v = &s.VXYZ[3 * (size_t)(i - 1)];
    const float sq = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
    ek = ek + (double)(s.MASS[s.ITYPE[i]] * sq);
  }
  ek = 0.5 * ek;
  const double t = ek * (double)s.MKTEMP;
  const double factor = (double)s.TEMP_IN / t;
  for (size_t k = 0; k < 3 * (size_t)s.NATOMS; ++k) s.VXYZ[k] = (float)(std::sqrt(factor) * (double)s.VXYZ[k]);
}

// ---------------------------------------------------------------- SETLIS.f90
inline bool setlis(Setup& s) {
  const int NI = s.NITEMS, NA_ = s.NATOMS, NT = s.NTYPE;
  s.NIJK.assign(NI + 1, 0); s.NOANGLEIJK.assign(NI + 1, 0);
  s.NIJKL.assign(NI + 1, 0); s.FNIJKL.assign(NI + 1, 0); s.NOOPIJKL.assign(NI + 1, 0);
  s.JANGLEIJK.assign((size_t)NI * Setup::MAXANG, 0); s.KANGLEIJK.assign((size_t)NI * Setup::MAXANG, 0);
  s.NOJANGLEIJK.assign((size_t)NI * Setup::MAXANG, 0); s.NOKANGLEIJK.assign((size_t)NI * Setup::MAXANG, 0);
  s.JTORIJKL.assign((size_t)NA_ * Setup::MAXTOR, 0); s.KTORIJKL.assign((size_t)NA_ * Setup::MAXTOR, 0);
  s.LTORIJKL.assign((size_t)NA_ * Setup::MAXTOR, 0);
  s.FJTORIJKL.assign((size_t)NA_ * Setup::MAXTOR, 0); s.FKTORIJKL.assign((size_t)NA_ * Setup::MAXTOR, 0);
  s.FLTORIJKL.assign((size_t)NA_ * Setup::MAXTOR, 0);
  s.JOOPIJKL.assign((size_t)NA_ * Setup::MAXOOP, 0); s.KOOPIJKL.assign((size_t)NA_ * Setup::MAXOOP, 0);
  s.LOOPIJKL.assign((size_t)NA_ * Setup::MAXOOP, 0);
  const int NBT = s.bond.nt, NAT = s.bend.nt, NTT = s.tors.nt, NOT = s.oop.nt;
  if (NBT <= 0) return true;  // :17
  auto full = [&](int n, int cap) -> bool {
    if (n > cap) { s.err = "per-atom bonded slot capacity exceeded"; return false; }
    return true;
  };
  int I = 0;
  for (int n = 1; n <= s.NMOL; ++n) {
    for (int m = 1; m <= s.NATM[n]; ++m) {
      ++I;
      int IT = s.ITYPE[I];
      if (NOT > 0 && s.NBONDS[I] == 3) {  // :33-97
        static const int perm[6][3] = {{1, 2, 3}, {3, 1, 2}, {2, 1, 3}, {1, 3, 2}, {2, 3, 1}, {3, 2, 1}};
        for (int ll = 0; ll < 6; ++ll) {
          int Z = s.jbond(I, perm[ll][0]), P = s.jbond(I, perm[ll][1]), O = s.jbond(I, perm[ll][2]);
          int ZT = s.ITYPE[Z], PT = s.ITYPE[P], OT = s.ITYPE[O];
          if (s.IOOPT[s.t4(IT, ZT, PT, OT)] != 0 && s.NOOPIJKL[I] == 0) {
            int c = ++s.NOOPIJKL[I];
            if (!full(c, Setup::MAXOOP)) return false;
            s.joop(I, c) = Z; s.koop(I, c) = P; s.loop(I, c) = O;
          }
        }
      }
      for (int j1 = 1; j1 <= s.NBONDS[I]; ++j1) {  // :99-415
        int J = s.jbond(I, j1), JT = s.ITYPE[J];
        if (s.IBONDT[s.t2(IT, JT)] == 0) { s.err = "No parameters found for a bond"; return false; }
        if (NAT > 0) {
          for (int k1 = 1; k1 <= s.NBONDS[J]; ++k1) {
            int K = s.jbond(J, k1), KT = s.ITYPE[K];
            if (K == I) continue;  // :153
            if (K > I) {           // :155-240
              if (s.IANGT[s.t3(IT, JT, KT)] == 0) {
                int c = ++s.NOANGLEIJK[I];
                if (!full(c, Setup::MAXANG)) return false;
                s.nojang(I, c) = J; s.nokang(I, c) = K;
              } else {
                int c = ++s.NIJK[I];
                if (!full(c, Setup::MAXANG)) return false;
                s.jang(I, c) = J; s.kang(I, c) = K;
              }
            }
            if (NTT > 0) {  // :243-410, searched for every K != I
              for (int l1 = 1; l1 <= s.NBONDS[K]; ++l1) {
                int L = s.jbond(K, l1), LT = s.ITYPE[L];
                if (L == J) continue;
                if (L > I) {
                  if (s.ITORT[s.t4(IT, JT, KT, LT)] == 0) {
                    if (NOT > 0 && s.IOOPT[s.t4(IT, JT, KT, LT)] != 0) {
                      int c = ++s.NOOPIJKL[I];
                      if (!full(c, Setup::MAXOOP)) return false;
                      s.joop(I, c) = J; s.koop(I, c) = K; s.loop(I, c) = L;
                    } else {
                      int c = ++s.FNIJKL[I];
                      if (!full(c, Setup::MAXTOR)) return false;
                      s.fjtor(I, c) = J; s.fktor(I, c) = K; s.fltor(I, c) = L;
                    }
                  } else {
                    int c = ++s.NIJKL[I];
                    if (!full(c, Setup::MAXTOR)) return false;
                    s.jtor(I, c) = J; s.ktor(I, c) = K; s.ltor(I, c) = L;
                  }
                }
              }
            }
          }
        }
      }
    }
  }
  (void)NT;
  return true;
}

// ---------------------------------------------------------- RDVIRTANGLES.f90
inline bool rdvirtangles(Setup& s, const std::string& dir) {
  Unit u;
  if (!u.open(dir + "/virtangles")) return true;  // optional file
  std::vector<std::string> it;
  while (u.read_items(4, &it)) {
    int i, j, k, t;
    if (!parse_int(it[0], &i) || !parse_int(it[1], &j) || !parse_int(it[2], &k) || !parse_int(it[3], &t)) break;
    int c = ++s.NIJK[i];
    if (c > Setup::MAXANG) { s.err = "per-atom angle capacity exceeded"; return false; }
    s.jang(i, c) = j; s.kang(i, c) = k;
  }
  return true;
}

// ---------------------------------------------------- BUILD_CONNECTIVITY.f90
// Restated from the dense IS_CONNECTED(NITEMS,NITEMS) marking (:27-93) and
// row compaction over J=1..NATOMS in ascending order (:95-110), using one
// sorted set per row instead of the N^2 array.  Rows of VS indices are never
// compacted (:99-101).
inline void build_connectivity(Setup& s, const std::vector<int>& index_list, int n, int exclusion) {
  const int NI = s.NITEMS, NA_ = s.NATOMS;
  std::vector<std::vector<int>> adj(NI + 1);
  auto mark = [&](int a, int b) { adj[a].push_back(b); adj[b].push_back(a); };
  for (int I = 1; I <= NA_; ++I) {
    for (int b = 1; b <= s.NBONDS[I]; ++b) mark(I, s.jbond(I, b));
    for (int b = 1; b <= s.NIJK[I]; ++b) { mark(I, s.jang(I, b)); mark(I, s.kang(I, b)); }
    for (int b = 1; b <= s.NOANGLEIJK[I]; ++b) { mark(I, s.nojang(I, b)); mark(I, s.nokang(I, b)); }
    if (exclusion == 5) {
      for (int b = 1; b <= s.NIJKL[I]; ++b) { mark(I, s.jtor(I, b)); mark(I, s.ktor(I, b)); mark(I, s.ltor(I, b)); }
      for (int b = 1; b <= s.FNIJKL[I]; ++b) { mark(I, s.fjtor(I, b)); mark(I, s.fktor(I, b)); mark(I, s.fltor(I, b)); }
      for (int b = 1; b <= s.NOOPIJKL[I]; ++b) { mark(I, s.joop(I, b)); mark(I, s.koop(I, b)); mark(I, s.loop(I, b)); }
    }
  }
  for (int a = 1; a <= n; ++a) {
    int I = index_list[a];
    if (I > NA_) return;
    auto& row = adj[I];
    std::sort(row.begin(), row.end());
    row.erase(std::unique(row.begin(), row.end()), row.end());
    int counter = 0;
    for (int J : row) {
      if (J < 1 || J > NA_) continue;
      ++counter;
      if (counter > Setup::MAXCONNECTIONS) { ++s.connectivity_overflow; continue; }
      s.conn(I, counter) = J;
    }
    s.CONNECTIONS[I] = std::min(counter, (int)Setup::MAXCONNECTIONS);
  }
}

// ----------------------------------------------------------- RDVIRTBONDS.f90
inline bool rdvirtbonds(Setup& s, const std::string& dir) {
  Unit u;
  if (!u.open(dir + "/virtbonds")) return true;  // optional file
  std::vector<std::string> it;
  while (u.read_items(2, &it)) {
    int i, j;
    if (!parse_int(it[0], &i) || !parse_int(it[1], &j)) break;
    if (++s.CONNECTIONS[i] > Setup::MAXCONNECTIONS) { s.err = "Max number of connections exceeded"; return false; }
    s.conn(i, s.CONNECTIONS[i]) = j;
    if (++s.CONNECTIONS[j] > Setup::MAXCONNECTIONS) { s.err = "Max number of connections exceeded"; return false; }
    s.conn(j, s.CONNECTIONS[j]) = i;
  }
  return true;
}

// main.F90:107-218 in order (the I/O-free part of L4)
inline bool setup_from_dir(Setup& s, const std::string& dir) {
  unit_constants(s);
  if (!rdcontrol(s, dir)) return false;
  if (!rdinteract(s, dir)) return false;
  if (!rdcoor(s, dir)) return false;
  // ALLOCATEVAR2.f90:19-42
  s.NCELLX_ATOM = (int)(s.BOX[0] / s.RLIST_ATOM);
  s.NCELLY_ATOM = (int)(s.BOX[1] / s.RLIST_ATOM);
  s.NCELLZ_ATOM = (int)(s.BOX[2] / s.RLIST_ATOM);
  if (s.IBRDESCR == 0) {
    s.NCELLX_BEAD = (int)(s.BOX[0] / s.RLIST_BEAD);
    s.NCELLY_BEAD = (int)(s.BOX[1] / s.RLIST_BEAD);
    s.NCELLZ_BEAD = (int)(s.BOX[2] / s.RLIST_BEAD);
    if (!rdvirtual(s, dir)) return false;
  }
  if (!make_lists(s)) return false;
  ftable(s);
  if (s.RESTART == 1) scalev(s);  // main.F90:168-171
  // main.F90:177-178
  s.MKTEMP_ATOM = 2.0f / (3.0f * (float)(s.NUMATOMS - 1));
  s.MKTEMP_BEAD = 2.0f / (3.0f * (float)(s.NUMBEADS - 1));
  if (!setlis(s)) return false;
  if (s.IBRDESCR == 0 && !rdvirtangles(s, dir)) return false;
  s.CONNECTIONS.assign(s.NITEMS + 1, 0);
  s.CONNECTED_TO.assign((size_t)s.NITEMS * Setup::MAXCONNECTIONS, 0);
  build_connectivity(s, s.ATOM, s.NUMATOMS, s.NONBEXC_ATOM);
  if (s.IBRDESCR == 0) {
    build_connectivity(s, s.BEAD, s.NCOARSE, s.NONBEXC_BEAD);
    if (!rdvirtbonds(s, dir)) return false;
  }
  if (s.connectivity_overflow) { s.err = "more than 20 exclusions for one particle"; return false; }
  return true;
}

}  // namespace orc
