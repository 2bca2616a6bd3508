// Host-side setup of one Hybrid IBIsCO system from its reference input files.
//
// This is the part of the reference's program that runs before the MD loop
// (main.F90:107-218): unit constants (UNIT.f90), the control keywords
// (RDCONTROL.f90), tables and type maps (RDINTERACT.f90), coordinates
// (RDCOOR.f90), virtual sites (RDVIRTUAL.f90), the atom/bead index lists
// (MAKE_LISTS.f90), force tables (FTABLE.f90), angles/torsions/out-of-planes
// (SETLIS.f90, RDVIRTANGLES.f90) and nonbonded exclusions
// (BUILD_CONNECTIVITY.f90, RDVIRTBONDS.f90).  Its output is an ibg_desc with
// the same values, in REAL*4, that the Fortran host holds in MODULE VAR, so that
// a host without the Fortran program can drive the device step.
//
// Differences of method (not of result):
//  * exclusions are built from sorted per-particle adjacency vectors instead
//    of the dense NITEMS x NITEMS LOGICAL matrix (BUILD_CONNECTIVITY.f90:23),
//    so a 2-million-particle system sets up in seconds;
//  * tables are kept with a leading dimension of (longest table + 3) rather
//    than MAXINPUT+1.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/ibisco_gpu.h"

namespace {

// ------------------------------------------------------------ text records
// Input files of the reader chain held in memory (ibg_setup_read_mem): file
// name -> contents.  While set on the calling thread, every file the readers
// open is looked up here by its name instead of on disk.
thread_local const std::map<std::string, std::string>* t_files = nullptr;

struct Records {
  std::vector<std::string> line;
  size_t at = 0;
  bool load(const std::string& path) {
    std::string all;
    if (t_files) {
      const size_t k = path.find_last_of('/');
      auto it = t_files->find(k == std::string::npos ? path : path.substr(k + 1));
      if (it == t_files->end()) return false;
      all = it->second;
    } else {
      std::ifstream f(path, std::ios::binary);
      if (!f) return false;
      std::stringstream ss;
      ss << f.rdbuf();
      all = ss.str();
    }
    line.clear();
    size_t b = 0;
    for (size_t i = 0; i <= all.size(); ++i) {
      if (i == all.size() || all[i] == '\n') {
        if (i > b || i < all.size()) line.emplace_back(all, b, i - b);
        b = i + 1;
      }
    }
    at = 0;
    return true;
  }
  bool more() const { return at < line.size(); }
};

// Words of a keyword/section line: the reference reads 80 columns, blanks the
// 80th, splits on blanks and tabs and drops '#'-delimited comments
// (PARSE.f90:78-149).
std::vector<std::string> words80(const std::string& raw) {
  std::string l = raw.substr(0, std::min<size_t>(raw.size(), 80));
  if (l.size() == 80) l[79] = ' ';
  std::vector<std::string> out;
  std::string cur;
  bool in_comment = false;
  for (char c : l) {
    if (in_comment) {
      if (c == '#') in_comment = false;
      continue;
    }
    if (c == '#') {
      if (!cur.empty()) { out.push_back(cur); cur.clear(); }
      in_comment = true;
      continue;
    }
    if (c == ' ' || c == '\t' || c == '\r') {
      if (!cur.empty()) { out.push_back(cur); cur.clear(); }
    } else {
      cur.push_back(c);
    }
  }
  if (!cur.empty() && !in_comment) out.push_back(cur);
  return out;
}

// List-directed input: a READ takes its values from the next record(s) and
// discards the rest of the last record it touched.
void split_ld(const std::string& l, std::vector<std::string>* t) {
  size_t i = 0, n = l.size();
  while (i < n) {
    char c = l[i];
    if (c == ' ' || c == '\t' || c == ',' || c == '\r') { ++i; continue; }
    if (c == '/') return;
    size_t b = i;
    while (i < n && l[i] != ' ' && l[i] != '\t' && l[i] != ',' && l[i] != '\r') ++i;
    t->emplace_back(l, b, i - b);
  }
}
bool read_ld(Records& r, size_t n, std::vector<std::string>* v) {
  v->clear();
  if (!r.more()) return false;
  while (v->size() < n) {
    if (!r.more()) return false;
    std::vector<std::string> t;
    split_ld(r.line[r.at++], &t);
    for (auto& s : t)
      if (v->size() < n) v->push_back(std::move(s));
  }
  return true;
}

bool to_f32(const std::string& s, float* out) {  // REAL*4, 'D' exponents allowed
  char buf[64];
  if (s.size() >= sizeof(buf)) return false;
  for (size_t i = 0; i < s.size(); ++i) buf[i] = (s[i] == 'd' || s[i] == 'D') ? 'E' : s[i];
  buf[s.size()] = 0;
  char* e = nullptr;
  float v = std::strtof(buf, &e);
  if (e == buf || *e) return false;
  *out = v;
  return true;
}
bool to_i32(const std::string& s, int* out) {
  char* e = nullptr;
  long v = std::strtol(s.c_str(), &e, 10);
  if (e == s.c_str() || *e) return false;
  *out = (int)v;
  return true;
}

struct Table {  // one tabulated family
  int n = 0, ld = 0;
  bool index_fastest = false;  // nonbonded layout (0:ld-1, NNBTYPE)
  std::vector<float> x, pot, frc, bin;
  std::vector<int> ndat;
  size_t at(int t, int k) const {  // t 1-based, k 0-based
    return index_fastest ? (size_t)k + (size_t)ld * (t - 1) : (size_t)(t - 1) + (size_t)n * k;
  }
  float& X(int t, int k) { return x[at(t, k)]; }
  float& P(int t, int k) { return pot[at(t, k)]; }
  float& F(int t, int k) { return frc[at(t, k)]; }
  void init(int ntab, int width, bool idxfast) {
    n = ntab; ld = width; index_fastest = idxfast;
    size_t sz = (size_t)std::max(ntab, 1) * width;
    x.assign(sz, 0.f); pot.assign(sz, 0.f); frc.assign(sz, 0.f);
    bin.assign(std::max(ntab, 1), 0.f); ndat.assign(std::max(ntab, 1), 0);
  }
};

}  // namespace

struct ibg_setup {
  ibg_desc d;
  std::string err;
  // UNIT.f90 constants (REAL*4)
  float NA = 0, MASSSCALE = 0, ESCALE = 0, TEMPSCALE = 0, PSCALE = 0, TIMESCALE = 0, VSCALE = 0, R2D = 0, D2R = 0,
        CONV = 0;
  // coordinate file header (RDCOOR.f90:55-65) and molecule names, for the output files
  std::string title;
  float initime = 0;
  std::vector<std::string> molname;
  // control values not in the descriptor
  int nstep = 0, ntrj = 0, restart = 0, nonbexc_atom = 4, nonbexc_bead = 4;
  float taut = 0, taup = 0, beta = 0;
  // particles
  float box[3] = {0, 0, 0};
  int nmol = 0;
  std::vector<int> natm;
  std::vector<float> mass, invmass;
  std::vector<char> label;
  std::vector<int> itype, type_label, atom, bead, nbonds, jbond;
  std::vector<float> sxyz, vxyz;
  // topology, (ld, slots) column-major, 0 = empty
  std::vector<int> nijk, jang, kang, noang, nojang, nokang;
  std::vector<int> nijkl, jtor, ktor, ltor, fnijkl, fjtor, fktor, fltor;
  std::vector<int> noop, joop, koop, loop;
  std::vector<int> connections, connected_to;
  // type maps
  std::vector<int> ibondt, inbondt, iangt, itort, ioopt;
  std::vector<int> lab_b, lab_a, lab_t, lab_o;
  Table tb, ta, tt, tn, to;
  // virtual sites
  std::vector<int> vitype, vcenter, vnum, vatm;
  std::vector<float> vmass, vinvmass, vcoeff;
  int vmax = 0;
};

namespace {

bool fail(ibg_setup* s, const std::string& m) {
  s->err = m;
  return false;
}

void units(ibg_setup* s) {  // UNIT.f90:9-23, all REAL*4
  const float KB = (float)1.380658e-23;
  s->NA = (float)6.0221367e+23;
  const float PI = 3.14159265358f;
  const float MMOLY = (float)0.012;
  s->MASSSCALE = MMOLY / s->NA;
  const float RSCALE = (float)1.0e-9;
  s->ESCALE = KB * 300.0f;
  s->TEMPSCALE = s->ESCALE / KB;
  s->PSCALE = (float)((double)(s->ESCALE / powf(RSCALE, 3.0f)) / 1000.0);
  s->TIMESCALE = RSCALE * sqrtf(s->MASSSCALE / s->ESCALE);
  s->VSCALE = RSCALE / s->TIMESCALE;
  s->R2D = 180.0f / PI;
  s->D2R = PI / 180.0f;
  s->CONV = (float)((double)(s->NA * s->ESCALE) / 1000.0);
}

// ---------------------------------------------------------- RDCONTROL.f90
bool control(ibg_setup* s, const std::string& dir) {
  Records r;
  if (!r.load(dir + "/control")) return fail(s, "File control does not exist");
  // first line that starts with each keyword; 'mts' is scanned to the end
  // (RDCONTROL.f90:485-493) so its last occurrence counts
  std::map<std::string, std::string> first;
  std::string mts;
  bool have_mts = false, have_end = false;
  for (auto& l : r.line) {
    auto w = words80(l);
    if (w.empty()) continue;
    if (w[0] == "mts" && w.size() > 1) { mts = w[1]; have_mts = true; }
    if (w[0] == "END" || w[0] == "end" || w[0] == "End") have_end = true;
    if (w.size() > 1 && !first.count(w[0])) first[w[0]] = w[1];
  }
  auto F = [&](const char* k, float* v) { auto it = first.find(k); return it != first.end() && to_f32(it->second, v); };
  auto I = [&](const char* k, int* v) { auto it = first.find(k); return it != first.end() && to_i32(it->second, v); };
  ibg_desc& d = s->d;
  auto it = first.find("ensemble");
  int ens = 10;
  if (it != first.end()) {
    if (it->second == "NVE" || it->second == "nve") ens = 0;
    if (it->second == "NVT" || it->second == "nvt") ens = 1;
    if (it->second == "NPT" || it->second == "npt") ens = 2;
  }
  if (ens == 10) return fail(s, "control: no valid ensemble (NVE/NVT/NPT)");
  d.ensemble = ens;
  float temp0, p0, dt0, rc, rl;
  if (!F("temperature", &temp0)) return fail(s, "control: keyword temperature missing");
  d.temp_in = temp0 / s->TEMPSCALE;
  if (!F("pressure", &p0)) return fail(s, "control: keyword pressure missing");
  d.pressure = p0 / s->PSCALE;
  if (!I("atoms", &d.natoms)) return fail(s, "control: keyword atoms missing");
  if (!I("num_of_time_steps", &s->nstep)) return fail(s, "control: keyword num_of_time_steps missing");
  if (!F("time_step", &dt0)) return fail(s, "control: keyword time_step missing");
  d.dt = (float)((double)dt0 * 1.0e-12 / (double)s->TIMESCALE);
  if (!I("virtual_sites", &d.nvirta)) return fail(s, "control: keyword virtual_sites missing");
  d.nitems = d.natoms + d.nvirta;
  d.ibrdescr = d.nvirta > 0 ? 0 : 1;
  bool ok = F("bead_cutoff", &rc);
  if (ok) { d.rcut_bead = rc; d.rcutsq_bead = rc * rc; }
  if (!ok && d.ibrdescr != 1) return fail(s, "control: keyword bead_cutoff missing");
  ok = F("bead_neighbour_list_cutoff", &rl);
  if (ok) {
    d.rlist_bead = rl;
    if (rl < d.rcut_bead) return fail(s, "control: neighbour list cutoff must be larger than the cutoff");
  }
  if (!ok && d.ibrdescr != 1) return fail(s, "control: keyword bead_neighbour_list_cutoff missing");
  if (d.ibrdescr == 0) {
    if (!I("non_bonded_bead", &s->nonbexc_bead)) return fail(s, "control: keyword non_bonded_bead missing");
    if (s->nonbexc_bead != 4 && s->nonbexc_bead != 5) return fail(s, "control: invalid non_bonded_bead");
  }
  if (!I("update_neighbour_list", &d.nupdate)) return fail(s, "control: keyword update_neighbour_list missing");
  float t0;
  if (F("temperature_coupling_time", &t0)) s->taut = (float)((double)t0 * 1.0e-12 / (double)s->TIMESCALE);
  else if (ens == 1 || ens == 2) return fail(s, "control: keyword temperature_coupling_time missing");
  if (F("pressure_coupling_time", &t0)) s->taup = (float)((double)t0 * 1.0e-12 / (double)s->TIMESCALE);
  else if (ens == 2) return fail(s, "control: keyword pressure_coupling_time missing");
  if (F("isothermal_compressibility", &t0)) s->beta = t0 * s->PSCALE;
  else if (ens == 2) return fail(s, "control: keyword isothermal_compressibility missing");
  if (!F("cutoff", &rc)) return fail(s, "control: keyword cutoff missing");
  d.rcut_atom = rc; d.rcutsq_atom = rc * rc;
  if (!F("neighbour_list_cutoff", &rl)) return fail(s, "control: keyword neighbour_list_cutoff missing");
  d.rlist_atom = rl;
  if (rl < rc) return fail(s, "control: neighbour list cutoff must be larger than the cutoff");
  if (!I("trajectory", &s->ntrj)) return fail(s, "control: keyword trajectory missing");
  if (!I("halt_drift", &d.halt_drift)) return fail(s, "control: keyword halt_drift missing");
  if (!I("non_bonded", &s->nonbexc_atom)) return fail(s, "control: keyword non_bonded missing");
  if (s->nonbexc_atom != 4 && s->nonbexc_atom != 5) return fail(s, "control: invalid non_bonded");
  it = first.find("initialize_velocities");
  int rs = 10;
  if (it != first.end()) {
    char c = it->second[0];
    if (c == 'Y' || c == 'y') rs = 1;
    if (c == 'N' || c == 'n') rs = 0;
  }
  if (rs == 10) return fail(s, "control: keyword initialize_velocities missing");
  s->restart = rs;
  if (!have_mts || !to_i32(mts, &d.nmts)) return fail(s, "control: keyword mts missing");
  if (!have_end) return fail(s, "control: keyword end missing");
  // ALLOCATEVAR.f90:42-46
  d.fac = d.dt / s->taut;
  d.pfac = s->beta * d.dt * 10.0f / s->taup;
  d.mktemp = (float)(2.0 / (double)(float)(3.0 * (double)(d.natoms - 1)));
  d.maxnab = 1000;  // main.F90:156,159
  return true;
}

// --------------------------------------------------------- RDINTERACT.f90
struct XY { std::vector<float> x, y; };
bool table_file(const std::string& path, XY* t) {
  Records r;
  if (!r.load(path)) return false;
  std::vector<std::string> v;
  while (read_ld(r, 2, &v)) {
    float a, b;
    if (!to_f32(v[0], &a) || !to_f32(v[1], &b)) break;
    t->x.push_back(a); t->y.push_back(b);
  }
  return true;
}

// One nonbonded table into column i of s->tn (RDINTERACT.f90:504-533): the
// potential converted from kJ/mol to reduced units, and a row at r = 0
// inserted (row 1 then holds r = bin with row 0's potential) when the file's
// first r is not 0.  The column must be zero and at least rows + 4 long.
bool nb_table(ibg_setup* s, int i, const XY& t) {
  auto energy = [&](float v) { return v * 1000.0f / s->NA / s->ESCALE; };  // RDINTERACT.f90:506-507,526
  if (t.x.size() < 2) return false;
  const float x0 = t.x[0], x1 = t.x[1], bin = x1 - x0;
  s->tn.bin[i - 1] = bin;
  int K;
  if (x0 != 0.0f) {
    s->tn.X(i, 0) = 0.0f; s->tn.P(i, 0) = energy(t.y[0]);
    s->tn.X(i, 1) = bin;  s->tn.P(i, 1) = energy(t.y[0]);
    s->tn.X(i, 2) = x1;   s->tn.P(i, 2) = energy(t.y[1]);
    K = 3;
  } else {
    s->tn.X(i, 0) = x0; s->tn.P(i, 0) = energy(t.y[0]);
    s->tn.X(i, 1) = x1; s->tn.P(i, 1) = energy(t.y[1]);
    K = 2;
  }
  for (size_t k = 2; k < t.x.size(); ++k, ++K) { s->tn.X(i, K) = t.x[k]; s->tn.P(i, K) = energy(t.y[k]); }
  s->tn.ndat[i - 1] = K - 1;
  return true;
}

bool interaction(ibg_setup* s, const std::string& dir) {
  Records r;
  if (!r.load(dir + "/interaction")) return fail(s, "File interaction does not exist");
  auto next = [&]() -> std::vector<std::string> {
    if (!r.more()) return {};
    return words80(r.line[r.at++]);
  };
  auto energy = [&](float v) { return v * 1000.0f / s->NA / s->ESCALE; };  // RDINTERACT.f90:217
  ibg_desc& d = s->d;
  auto w = next();
  if (w.size() < 2 || w[0] != "atom_types" || !to_i32(w[1], &d.ntype)) return fail(s, "interaction: atom_types");
  const int NT = d.ntype;
  if (NT < 1) return fail(s, "interaction: atom_types");
  s->mass.assign(NT, 0.f); s->invmass.assign(NT, 0.f); s->label.assign(NT, ' ');
  std::vector<float> mass0(NT, 0.f);
  if (r.more()) ++r.at;
  for (int i = 0; i < NT; ++i) {  // :101-130
    w = next();
    if (w.size() < 4 || w[0] == "bond_types") return fail(s, "interaction: number of atom_types different from number of atoms");
    int ti;
    if (!to_i32(w[0], &ti) || ti < 1 || ti > NT) return fail(s, "interaction: bad atom type index");
    to_f32(w[2], &mass0[ti - 1]);
    char c = w[3][0];
    if (w[3].size() != 1 || !(c == 'A' || c == 'a' || c == 'B' || c == 'b')) return fail(s, "interaction: label must be A or B");
    s->label[ti - 1] = c;
    // MASS is filled by line order (RDINTERACT.f90:128)
    s->mass[i] = mass0[i] / s->NA / s->MASSSCALE;
    s->invmass[i] = (float)(1.0 / (double)s->mass[i]);
  }
  auto cls = [&](int t) { char c = s->label[t - 1]; return (c == 'A' || c == 'a') ? 1 : 2; };
  s->ibondt.assign((size_t)NT * NT, 0);
  s->inbondt.assign((size_t)NT * NT, 0);
  s->iangt.assign((size_t)NT * NT * NT, 0);
  s->itort.assign((size_t)NT * NT * NT * NT, 0);
  s->ioopt.assign((size_t)NT * NT * NT * NT, 0);
  auto T2 = [&](int a, int b) { return (size_t)(a - 1) + (size_t)NT * (b - 1); };
  auto T3 = [&](int a, int b, int c) { return (size_t)(a - 1) + (size_t)NT * ((b - 1) + (size_t)NT * (c - 1)); };
  auto T4 = [&](int a, int b, int c, int e) {
    return (size_t)(a - 1) + (size_t)NT * ((b - 1) + (size_t)NT * ((c - 1) + (size_t)NT * (e - 1)));
  };
  auto section = [&](const char* key, int* count) -> bool {
    auto ww = next();
    if (ww.size() < 2 || ww[0] != key || !to_i32(ww[1], count)) return false;
    if (r.more()) ++r.at;
    return true;
  };
  auto ints = [&](const std::vector<std::string>& ww, int n, int* o) {
    for (int k = 0; k < n; ++k)
      if (!to_i32(ww[k], &o[k]) || o[k] < 1 || o[k] > NT) return false;
    return true;
  };

  // bonds (:144-223): read as is, offset lookup in BONDS.inc
  int nb;
  if (!section("bond_types", &nb)) return fail(s, "interaction: bond_types");
  std::vector<XY> bx(nb);
  s->lab_b.assign(std::max(nb, 1), 0);
  for (int i = 0; i < nb; ++i) {
    w = next();
    if (w.size() < 3 || w[0] == "angle_types") return fail(s, "interaction: number of bond_types different from number of bonds");
    int t[2];
    if (!ints(w, 2, t)) return fail(s, "interaction: bad bond types");
    if (s->ibondt[T2(t[0], t[1])]) return fail(s, "interaction: duplicate bond entry");
    s->ibondt[T2(t[0], t[1])] = s->ibondt[T2(t[1], t[0])] = i + 1;
    int h = cls(t[0]) + cls(t[1]);
    s->lab_b[i] = h == 2 ? 1 : (h == 4 ? 2 : 3);
    if (!table_file(dir + "/" + w[2], &bx[i])) return fail(s, "interaction: table file " + w[2] + " does not exist");
  }
  {
    size_t maxn = 2;
    for (auto& t : bx) maxn = std::max(maxn, t.x.size());
    s->tb.init(nb, (int)maxn + 3, false);
    for (int i = 1; i <= nb; ++i) {
      auto& t = bx[i - 1];
      int K = (int)t.x.size();
      if (K < 2) return fail(s, "interaction: bond table too short");
      for (int k = 0; k < K; ++k) { s->tb.X(i, k) = t.x[k]; s->tb.P(i, k) = energy(t.y[k]); }
      s->tb.ndat[i - 1] = K - 1;
      s->tb.bin[i - 1] = s->tb.X(i, 1) - s->tb.X(i, 0);
    }
  }
  // angle, torsion and out-of-plane tables start at 0: a table that does not
  // gets a row 0 copied from its first row (:312-321, :420-429, :644-653)
  auto angular = [&](Table& T, std::vector<XY>& raw, bool oop) -> bool {
    size_t maxn = 2;
    for (auto& t : raw) maxn = std::max(maxn, t.x.size());
    T.init((int)raw.size(), (int)maxn + 4, false);
    for (int i = 1; i <= (int)raw.size(); ++i) {
      auto& t = raw[i - 1];
      if (t.x.size() < 2) return false;
      float x0 = t.x[0], x1 = t.x[1];
      float bin = (oop && x1 < x0) ? x0 - x1 : x1 - x0;
      T.bin[i - 1] = bin;
      int K = 0;
      if (x0 != 0.0f) {
        T.X(i, 0) = 0.0f; T.P(i, 0) = energy(t.y[0]);
        T.X(i, 1) = bin;  T.P(i, 1) = energy(t.y[0]);
        T.X(i, 2) = x1;   T.P(i, 2) = energy(t.y[1]);
        K = 3;
      } else {
        T.X(i, 0) = x0; T.P(i, 0) = energy(t.y[0]);
        T.X(i, 1) = x1; T.P(i, 1) = energy(t.y[1]);
        K = 2;
      }
      for (size_t k = 2; k < t.x.size(); ++k, ++K) { T.X(i, K) = t.x[k]; T.P(i, K) = energy(t.y[k]); }
      T.ndat[i - 1] = K - 1;
    }
    return true;
  };
  int na;
  if (!section("angle_types", &na)) return fail(s, "interaction: angle_types");
  std::vector<XY> ax(na);
  s->lab_a.assign(std::max(na, 1), 0);
  for (int i = 0; i < na; ++i) {
    w = next();
    if (w.size() < 4 || w[0] == "torsion_types") return fail(s, "interaction: number of angle_types different from number of angles");
    int t[3];
    if (!ints(w, 3, t)) return fail(s, "interaction: bad angle types");
    if (s->iangt[T3(t[0], t[1], t[2])]) return fail(s, "interaction: duplicate angle entry");
    s->iangt[T3(t[0], t[1], t[2])] = s->iangt[T3(t[2], t[1], t[0])] = i + 1;
    int h = cls(t[0]) + cls(t[1]) + cls(t[2]);
    s->lab_a[i] = h == 3 ? 1 : (h == 6 ? 2 : 3);
    if (!table_file(dir + "/" + w[3], &ax[i])) return fail(s, "interaction: table file " + w[3] + " does not exist");
  }
  if (!angular(s->ta, ax, false)) return fail(s, "interaction: angle table too short");
  int nt;
  if (!section("torsion_types", &nt)) return fail(s, "interaction: torsion_types");
  std::vector<XY> tx(nt);
  s->lab_t.assign(std::max(nt, 1), 0);
  for (int i = 0; i < nt; ++i) {
    w = next();
    if (w.size() < 5 || w[0] == "non_bonded_interaction_types") return fail(s, "interaction: number of torsion_types different from number of torsions");
    int t[4];
    if (!ints(w, 4, t)) return fail(s, "interaction: bad torsion types");
    if (s->itort[T4(t[0], t[1], t[2], t[3])]) return fail(s, "interaction: duplicate torsion entry");
    s->itort[T4(t[0], t[1], t[2], t[3])] = s->itort[T4(t[3], t[2], t[1], t[0])] = i + 1;
    int h = cls(t[0]) + cls(t[1]) + cls(t[2]) + cls(t[3]);
    s->lab_t[i] = h == 4 ? 1 : (h == 8 ? 2 : 3);
    if (!table_file(dir + "/" + w[4], &tx[i])) return fail(s, "interaction: table file " + w[4] + " does not exist");
  }
  if (!angular(s->tt, tx, false)) return fail(s, "interaction: torsion table too short");
  // nonbonded (:448-537), index-fastest, row 0 inserted when missing
  int nn;
  if (!section("non_bonded_interaction_types", &nn)) return fail(s, "interaction: non_bonded_interaction_types");
  std::vector<XY> nx(nn);
  for (int i = 0; i < nn; ++i) {
    w = next();
    if (w.size() < 3 || w[0] == "Out_of_Planes") return fail(s, "interaction: number of non_bonded_interaction_types different");
    int t[2];
    if (!ints(w, 2, t)) return fail(s, "interaction: bad nonbonded types");
    if (s->inbondt[T2(t[0], t[1])]) return fail(s, "interaction: duplicate nonbonded entry");
    s->inbondt[T2(t[0], t[1])] = s->inbondt[T2(t[1], t[0])] = i + 1;
    if (!table_file(dir + "/" + w[2], &nx[i])) return fail(s, "interaction: table file " + w[2] + " does not exist");
  }
  {
    size_t maxn = 2;
    for (auto& t : nx) maxn = std::max(maxn, t.x.size());
    s->tn.init(nn, (int)maxn + 4, true);
    for (int i = 1; i <= nn; ++i)
      if (!nb_table(s, i, nx[i - 1])) return fail(s, "interaction: nonbonded table too short");
  }
  // out of planes (:543-666); the map is not symmetrised (:608-616)
  int no;
  if (!section("Out_of_Planes", &no)) return fail(s, "interaction: Out_of_Planes");
  std::vector<XY> ox(no);
  s->lab_o.assign(std::max(no, 1), 0);
  for (int i = 0; i < no; ++i) {
    w = next();
    if (w.size() < 5) return fail(s, "interaction: number of Out_of_Planes different");
    int t[4];
    if (!ints(w, 4, t)) return fail(s, "interaction: bad out-of-plane types");
    if (s->ioopt[T4(t[0], t[1], t[2], t[3])]) return fail(s, "interaction: duplicate out-of-plane entry");
    s->ioopt[T4(t[0], t[1], t[2], t[3])] = i + 1;
    int h = cls(t[0]) + cls(t[1]) + cls(t[2]) + cls(t[3]);
    s->lab_o[i] = h == 4 ? 1 : (h == 8 ? 2 : 3);
    if (!table_file(dir + "/" + w[4], &ox[i])) return fail(s, "interaction: table file " + w[4] + " does not exist");
  }
  if (no > 0 && r.more()) return fail(s, "interaction: number of Out_of_Planes different");
  if (!angular(s->to, ox, true)) return fail(s, "interaction: out-of-plane table too short");
  return true;
}

// ---------------------------------------------------------------- FTABLE.f90
// Nonbonded table i (FTABLE.f90:59-75); the last row uses the zero potential
// past the table.
void ftable_nb(ibg_setup* s, int i) {
  Table& n = s->tn;
  int nd = n.ndat[i - 1];
  for (int j = 1; j <= nd; ++j)
    n.F(i, j) = (float)((double)(-(n.P(i, j + 1) - n.P(i, j - 1)) / n.bin[i - 1] / n.X(i, j)) / 2.0);
  n.F(i, 0) = n.F(i, 1);
}

void ftable(ibg_setup* s) {
  const float D2R = s->D2R;
  Table& b = s->tb;  // bonds :26-32, F/r; the end store at :31 indexes with the
  for (int i = 1; i <= b.n; ++i) {  // whole NDATB array, i.e. one store per bond type
    int nd = b.ndat[i - 1];
    for (int j = 1; j <= nd - 1; ++j)
      b.F(i, j) = (float)((double)(-(b.P(i, j + 1) - b.P(i, j - 1)) / b.bin[i - 1] / b.X(i, j)) / 2.0);
    b.F(i, 0) = b.F(i, 1);
    float last = b.F(i, nd - 1);
    for (int k = 0; k < b.n; ++k) b.F(i, b.ndat[k]) = last;
  }
  auto ang = [&](Table& T, bool end_from_first) {
    for (int i = 1; i <= T.n; ++i) {
      int nd = T.ndat[i - 1];
      for (int j = 1; j <= nd - 1; ++j)
        T.F(i, j) = (float)((double)(-(T.P(i, j + 1) - T.P(i, j - 1)) / T.bin[i - 1] / D2R) / 2.0);
      T.F(i, 0) = T.F(i, 1);
      T.F(i, nd) = end_from_first ? T.F(i, 0) : T.F(i, nd - 1);
    }
  };
  ang(s->ta, false);  // :35-43
  ang(s->tt, true);   // :47-55
  ang(s->to, true);   // :78-86
  for (int i = 1; i <= s->tn.n; ++i) ftable_nb(s, i);
}

// ---------------------------------------------------------------- SCALEV.f90
// Initial velocity rescale to TEMP_IN (SCALEV.f90:13-26), run at
// main.F90:168-171 when initialize_velocities is Y.  The reference first
// calls COMVEL (COMVEL.f90:17-79), whose draw from gfortran's RANDOM_NUMBER
// cannot be reproduced; the coordinate file's velocities take its place.
// Kinetic energy and factor in double over REAL*4 terms, velocities rounded
// back to REAL*4, as the reference does.
void scalev(ibg_setup* s) {
  const ibg_desc& d = s->d;
  double ek = 0.0;
  for (int i = 0; i < d.natoms; ++i) {
    const float* v = &s->vxyz[3 * (size_t)i];
    const float sq = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
    ek = ek + (double)(s->mass[s->itype[i] - 1] * sq);
  }
  ek = 0.5 * ek;
  const double t = ek * (double)d.mktemp;
  const double factor = (double)d.temp_in / t;
  for (size_t k = 0; k < 3 * (size_t)d.natoms; ++k) s->vxyz[k] = (float)(std::sqrt(factor) * (double)s->vxyz[k]);
}

// ----------------------------------------------------------------- RDCOOR.f90
bool coordinate(ibg_setup* s, const std::string& dir) {
  Records r;
  if (!r.load(dir + "/coordinate")) return fail(s, "File coordinate does not exist");
  ibg_desc& d = s->d;
  if (r.line.size() < 11) return fail(s, "coordinate: header too short");
  {  // RDCOOR.f90:55-65: TITLE is the first word of line 1; INITIME follows 'Time' on line 2
    auto w0 = words80(r.line[0]);
    s->title = w0.empty() ? "" : w0[0].substr(0, 72);
    auto w1 = words80(r.line[1]);
    s->initime = 0.0f;
    if (w1.size() >= 2 && w1[0] == "Time") to_f32(w1[1], &s->initime);
  }
  r.at = 3;
  std::vector<std::string> v;
  if (!read_ld(r, 3, &v)) return fail(s, "coordinate: box");
  for (int c = 0; c < 3; ++c)
    if (!to_f32(v[c], &s->box[c])) return fail(s, "coordinate: box");
  r.at += 5;
  if (!read_ld(r, 2, &v) || !to_i32(v[1], &s->nmol)) return fail(s, "coordinate: num_of_molecules");
  const int N = d.nitems, NA = d.natoms;
  s->natm.assign(s->nmol, 0);
  s->molname.assign(s->nmol, "");
  s->itype.assign(N, 0); s->type_label.assign(N, 1); s->nbonds.assign(N, 0);
  s->jbond.assign((size_t)N * 4, 0);
  s->sxyz.assign((size_t)3 * NA, 0.f); s->vxyz.assign((size_t)3 * NA, 0.f);
  int L = 0;
  for (int m = 0; m < s->nmol; ++m) {
    if (!read_ld(r, 4, &v) || !to_i32(v[0], &s->natm[m])) return fail(s, "coordinate: molecule name missing");
    s->molname[m] = v[3];
    for (int k = 0; k < s->natm[m]; ++k) {
      if (L >= NA) return fail(s, "coordinate: number of atoms differs from NATOMS");
      if (!read_ld(r, 6, &v)) return fail(s, "coordinate: record");
      int ll, t, nbd;
      if (!to_i32(v[0], &ll) || !to_i32(v[1], &t) || !to_i32(v[2], &nbd)) return fail(s, "coordinate: record");
      if (t < 1 || t > d.ntype || nbd < 0 || nbd > 4) return fail(s, "coordinate: bad type or bond count");
      s->itype[L] = t; s->nbonds[L] = nbd;
      for (int c = 0; c < 3; ++c)
        if (!to_f32(v[3 + c], &s->sxyz[3 * (size_t)L + c])) return fail(s, "coordinate: position");
      if (!read_ld(r, 3 + nbd, &v)) return fail(s, "coordinate: record");
      for (int c = 0; c < 3; ++c) {
        float x;
        if (!to_f32(v[c], &x)) return fail(s, "coordinate: velocity");
        s->vxyz[3 * (size_t)L + c] = x * 1.e3f / s->VSCALE;  // RDCOOR.f90:125
      }
      for (int b = 0; b < nbd; ++b) {
        int j;
        if (!to_i32(v[3 + b], &j) || j < 1 || j > NA) return fail(s, "coordinate: bonded index");
        s->jbond[(size_t)b * N + L] = j;
      }
      if (d.ibrdescr == 0) {
        char c = s->label[t - 1];
        s->type_label[L] = (c == 'A' || c == 'a') ? 1 : 2;
      }
      ++L;
    }
  }
  if (L != NA) return fail(s, "coordinate: number of atoms differs from NATOMS");
  return true;
}

// -------------------------------------------------------------- RDVIRTUAL.f90
bool virtual_sites(ibg_setup* s, const std::string& dir) {
  Records r;
  if (!r.load(dir + "/virtual")) return fail(s, "File virtual does not exist");
  ibg_desc& d = s->d;
  const int NT = d.ntype;
  r.at = 2;
  std::vector<std::string> v;
  int nv;
  if (!read_ld(r, 1, &v) || !to_i32(v[0], &nv)) return fail(s, "virtual: header");
  if (nv != d.nvirta) return fail(s, "virtual: number of virtual sites differs from control");
  r.at += 2;
  s->vnum.assign(NT, 0);
  s->vitype.assign(nv, 0); s->vcenter.assign(nv, 0);
  std::vector<std::vector<int>> members(nv);
  for (int i = 0; i < nv; ++i) {
    int k, n;
    if (!read_ld(r, 4, &v) || !to_i32(v[0], &k) || !to_i32(v[1], &s->vitype[i]) || !to_i32(v[2], &n) ||
        !to_i32(v[3], &s->vcenter[i]))
      return fail(s, "virtual: record too short");
    int t = s->vitype[i];
    if (t < 1 || t > NT) return fail(s, "virtual: bad type");
    if (n > 15) return fail(s, "virtual: number of atoms in a virtual site exceeds 15");
    if (!read_ld(r, n, &v)) return fail(s, "virtual: record too short");
    for (auto& x : v) {
      int a;
      if (!to_i32(x, &a) || a < 1 || a > d.natoms) return fail(s, "virtual: bad member index");
      members[i].push_back(a);
    }
    s->itype[d.natoms + i] = t;
    if (s->vnum[t - 1] == 0) s->vnum[t - 1] = n;
    else if (s->vnum[t - 1] != n) return fail(s, "virtual: disagreement in number of atoms of a site type");
  }
  s->vmax = 0;
  for (int t = 0; t < NT; ++t) s->vmax = std::max(s->vmax, s->vnum[t]);
  s->vatm.assign((size_t)nv * std::max(s->vmax, 1), 0);
  for (int i = 0; i < nv; ++i)
    for (int j = 0; j < s->vnum[s->vitype[i] - 1]; ++j) s->vatm[(size_t)j * nv + i] = members[i][j];
  s->vmass.assign(NT, 0.f); s->vinvmass.assign(NT, 0.f); s->vcoeff.assign((size_t)NT * NT, 0.f);
  for (int i = 0; i < nv; ++i) {  // :287-309
    int t = s->vitype[i];
    double m = 0.0;
    for (int a : members[i]) m += (double)s->mass[s->itype[a - 1] - 1];
    if (s->vmass[t - 1] == 0.0f) {
      s->vmass[t - 1] = (float)m;
      s->vinvmass[t - 1] = (float)(1.0 / m);
    } else if (std::fabs((double)s->vmass[t - 1] - m) > (double)0.0001f) {
      return fail(s, "virtual: disagreement in site mass");
    }
    for (int a : members[i]) {
      int ta = s->itype[a - 1];
      s->vcoeff[(size_t)(t - 1) + (size_t)NT * (ta - 1)] = s->mass[ta - 1] * s->vinvmass[t - 1];
    }
  }
  return true;
}

// ------------------------------------------------------ SETLIS.f90 et al.
bool topology(ibg_setup* s, const std::string& dir) {
  ibg_desc& d = s->d;
  const int N = d.nitems, NA = d.natoms, NT = d.ntype;
  s->nijk.assign(N, 0); s->noang.assign(N, 0); s->nijkl.assign(N, 0); s->fnijkl.assign(N, 0); s->noop.assign(N, 0);
  s->jang.assign((size_t)N * 10, 0); s->kang.assign((size_t)N * 10, 0);
  s->nojang.assign((size_t)N * 10, 0); s->nokang.assign((size_t)N * 10, 0);
  s->jtor.assign((size_t)NA * 10, 0); s->ktor.assign((size_t)NA * 10, 0); s->ltor.assign((size_t)NA * 10, 0);
  s->fjtor.assign((size_t)NA * 10, 0); s->fktor.assign((size_t)NA * 10, 0); s->fltor.assign((size_t)NA * 10, 0);
  s->joop.assign((size_t)NA * 20, 0); s->koop.assign((size_t)NA * 20, 0); s->loop.assign((size_t)NA * 20, 0);
  auto B = [&](int i, int k) { return s->jbond[(size_t)(k - 1) * N + (i - 1)]; };  // JBOND(i,k)
  auto TY = [&](int i) { return s->itype[i - 1]; };
  auto m4 = [&](const std::vector<int>& m, int a, int b, int c, int e) {
    return m[(size_t)(a - 1) + (size_t)NT * ((b - 1) + (size_t)NT * ((c - 1) + (size_t)NT * (e - 1)))];
  };
  auto push = [&](std::vector<int>& cnt, int i, int cap, int ld, std::initializer_list<std::vector<int>*> dst,
                  std::initializer_list<int> val) -> bool {
    int c = ++cnt[i - 1];
    if (c > cap) return false;
    auto vit = val.begin();
    for (auto* v : dst) (*v)[(size_t)(c - 1) * ld + (i - 1)] = *vit++;
    return true;
  };
  const bool have_oop = s->to.n > 0, have_ang = s->ta.n > 0, have_tor = s->tt.n > 0;
  if (s->tb.n > 0) {
    for (int I = 1; I <= NA; ++I) {  // molecules are contiguous, so this is SETLIS's order
      int IT = TY(I);
      if (have_oop && s->nbonds[I - 1] == 3) {  // :33-97, first matching permutation only
        static const int P[6][3] = {{1, 2, 3}, {3, 1, 2}, {2, 1, 3}, {1, 3, 2}, {2, 3, 1}, {3, 2, 1}};
        for (auto& p : P) {
          int Z = B(I, p[0]), Pp = B(I, p[1]), O = B(I, p[2]);
          if (m4(s->ioopt, IT, TY(Z), TY(Pp), TY(O)) && s->noop[I - 1] == 0)
            if (!push(s->noop, I, 20, NA, {&s->joop, &s->koop, &s->loop}, {Z, Pp, O})) return fail(s, "SETLIS: more than 20 out-of-planes on one atom");
        }
      }
      for (int b1 = 1; b1 <= s->nbonds[I - 1]; ++b1) {
        int J = B(I, b1), JT = TY(J);
        if (!s->ibondt[(size_t)(IT - 1) + (size_t)NT * (JT - 1)])
          return fail(s, "SETLIS: no parameters found for the bond between atoms " + std::to_string(I) + " and " + std::to_string(J));
        if (!have_ang) continue;
        for (int b2 = 1; b2 <= s->nbonds[J - 1]; ++b2) {
          int K = B(J, b2), KT = TY(K);
          if (K == I) continue;
          if (K > I) {
            bool known = s->iangt[(size_t)(IT - 1) + (size_t)NT * ((JT - 1) + (size_t)NT * (KT - 1))] != 0;
            bool ok = known ? push(s->nijk, I, 10, N, {&s->jang, &s->kang}, {J, K})
                            : push(s->noang, I, 10, N, {&s->nojang, &s->nokang}, {J, K});
            if (!ok) return fail(s, "SETLIS: more than 10 angles on one atom");
          }
          if (!have_tor) continue;
          for (int b3 = 1; b3 <= s->nbonds[K - 1]; ++b3) {
            int L = B(K, b3), LT = TY(L);
            if (L == J || L <= I) continue;
            bool ok;
            if (m4(s->itort, IT, JT, KT, LT)) ok = push(s->nijkl, I, 10, NA, {&s->jtor, &s->ktor, &s->ltor}, {J, K, L});
            else if (have_oop && m4(s->ioopt, IT, JT, KT, LT)) ok = push(s->noop, I, 20, NA, {&s->joop, &s->koop, &s->loop}, {J, K, L});
            else ok = push(s->fnijkl, I, 10, NA, {&s->fjtor, &s->fktor, &s->fltor}, {J, K, L});
            if (!ok) return fail(s, "SETLIS: more than 10 torsions (20 out-of-planes) on one atom");
          }
        }
      }
    }
  }
  if (d.ibrdescr == 0) {  // RDVIRTANGLES.f90:35-50 (optional file)
    Records r;
    if (r.load(dir + "/virtangles")) {
      std::vector<std::string> v;
      while (read_ld(r, 4, &v)) {
        int i, j, k, t;
        if (!to_i32(v[0], &i) || !to_i32(v[1], &j) || !to_i32(v[2], &k) || !to_i32(v[3], &t)) break;
        if (i < 1 || i > N || j < 1 || j > N || k < 1 || k > N) return fail(s, "virtangles: bad index");
        if (!push(s->nijk, i, 10, N, {&s->jang, &s->kang}, {j, k})) return fail(s, "virtangles: more than 10 angles on one particle");
      }
    }
  }
  return true;
}

// Nonbonded exclusions.  For every atom I the reference marks the particles
// it shares a bond, angle (with or without parameters) and, for
// non_bonded 5, a torsion or out-of-plane with, symmetrically; each row of a
// list's particles then holds the marked atoms (ids <= NATOMS) ascending.
bool exclusions(ibg_setup* s, const std::string& dir) {
  ibg_desc& d = s->d;
  const int N = d.nitems, NA = d.natoms;
  s->connections.assign(N, 0);
  s->connected_to.assign((size_t)N * 20, 0);
  auto build = [&](const std::vector<int>& list, int excl) -> bool {
    std::vector<std::vector<int>> adj(N + 1);
    auto link = [&](int a, int b) { adj[a].push_back(b); adj[b].push_back(a); };
    for (int I = 1; I <= NA; ++I) {
      for (int k = 0; k < s->nbonds[I - 1]; ++k) link(I, s->jbond[(size_t)k * N + I - 1]);
      for (int k = 0; k < s->nijk[I - 1]; ++k) { link(I, s->jang[(size_t)k * N + I - 1]); link(I, s->kang[(size_t)k * N + I - 1]); }
      for (int k = 0; k < s->noang[I - 1]; ++k) { link(I, s->nojang[(size_t)k * N + I - 1]); link(I, s->nokang[(size_t)k * N + I - 1]); }
      if (excl == 5) {
        for (int k = 0; k < s->nijkl[I - 1]; ++k)
          for (auto* m : {&s->jtor, &s->ktor, &s->ltor}) link(I, (*m)[(size_t)k * NA + I - 1]);
        for (int k = 0; k < s->fnijkl[I - 1]; ++k)
          for (auto* m : {&s->fjtor, &s->fktor, &s->fltor}) link(I, (*m)[(size_t)k * NA + I - 1]);
        for (int k = 0; k < s->noop[I - 1]; ++k)
          for (auto* m : {&s->joop, &s->koop, &s->loop}) link(I, (*m)[(size_t)k * NA + I - 1]);
      }
    }
    for (int I : list) {
      if (I > NA) break;  // virtual sites follow the beads (BUILD_CONNECTIVITY.f90:99-101)
      auto& a = adj[I];
      std::sort(a.begin(), a.end());
      a.erase(std::unique(a.begin(), a.end()), a.end());
      int c = 0;
      for (int j : a) {
        if (j > NA) continue;
        if (c == 20) return fail(s, "exclusions: more than 20 excluded partners for particle " + std::to_string(I));
        s->connected_to[(size_t)c * N + I - 1] = j;
        ++c;
      }
      s->connections[I - 1] = c;
    }
    return true;
  };
  if (!build(s->atom, s->nonbexc_atom)) return false;
  if (d.ibrdescr == 0) {
    if (!build(s->bead, s->nonbexc_bead)) return false;
    Records r;  // RDVIRTBONDS.f90 (optional file): appended, unsorted
    if (r.load(dir + "/virtbonds")) {
      std::vector<std::string> v;
      while (read_ld(r, 2, &v)) {
        int i, j;
        if (!to_i32(v[0], &i) || !to_i32(v[1], &j)) break;
        if (i < 1 || i > N || j < 1 || j > N) return fail(s, "virtbonds: bad index");
        for (int q : {i, j}) {
          int other = q == i ? j : i;
          if (s->connections[q - 1] == 20) return fail(s, "virtbonds: max number of connections exceeded");
          s->connected_to[(size_t)s->connections[q - 1] * N + q - 1] = other;
          ++s->connections[q - 1];
        }
      }
    }
  }
  return true;
}

void fill_desc(ibg_setup* s) {
  ibg_desc& d = s->d;
  const int N = d.nitems;
  d.mass = s->mass.data(); d.invmass = s->invmass.data();
  d.itype = s->itype.data(); d.type_label = s->type_label.data();
  d.atom = s->atom.data(); d.bead = s->bead.data();
  d.nbonds = s->nbonds.data(); d.jbond = s->jbond.data(); d.ld_bond = N;
  d.nijk = s->nijk.data(); d.jangleijk = s->jang.data(); d.kangleijk = s->kang.data(); d.ld_angle = N;
  d.nijkl = s->nijkl.data(); d.jtorijkl = s->jtor.data(); d.ktorijkl = s->ktor.data(); d.ltorijkl = s->ltor.data();
  d.ld_torsion = d.natoms;
  d.noopijkl = s->noop.data(); d.joopijkl = s->joop.data(); d.koopijkl = s->koop.data(); d.loopijkl = s->loop.data();
  d.ld_oop = d.natoms;
  d.connections = s->connections.data(); d.connected_to = s->connected_to.data(); d.ld_conn = N;
  d.ibondt = s->ibondt.data(); d.inbondt = s->inbondt.data(); d.iangt = s->iangt.data();
  d.itort = s->itort.data(); d.ioopt = s->ioopt.data();
  d.bond_type_label = s->lab_b.data(); d.angle_type_label = s->lab_a.data();
  d.torsion_type_label = s->lab_t.data(); d.oop_type_label = s->lab_o.data();
  d.nbtype = s->tb.n; d.natype = s->ta.n; d.nttype = s->tt.n; d.nnbtype = s->tn.n; d.notype = s->to.n;
  d.ld_b = s->tb.ld; d.ld_a = s->ta.ld; d.ld_t = s->tt.ld; d.ld_nb = s->tn.ld; d.ld_o = s->to.ld;
  d.ndatb = s->tb.ndat.data(); d.binb = s->tb.bin.data(); d.rbond = s->tb.x.data(); d.bond_pot = s->tb.pot.data(); d.bond_force = s->tb.frc.data();
  d.ndatan = s->ta.ndat.data(); d.bina = s->ta.bin.data(); d.angle = s->ta.x.data(); d.bend_pot = s->ta.pot.data(); d.bend_force = s->ta.frc.data();
  d.ndatt = s->tt.ndat.data(); d.bint = s->tt.bin.data(); d.angle_tor = s->tt.x.data(); d.tor_pot = s->tt.pot.data(); d.tor_force = s->tt.frc.data();
  d.ndatnb = s->tn.ndat.data(); d.binnb = s->tn.bin.data(); d.rnbond = s->tn.x.data(); d.nbond_pot = s->tn.pot.data(); d.nbond_force = s->tn.frc.data();
  d.ndato = s->to.ndat.data(); d.bino = s->to.bin.data(); d.angle_oop = s->to.x.data(); d.oop_pot = s->to.pot.data(); d.oop_force = s->to.frc.data();
  d.ld_vs = d.nvirta; d.vs_maxatoms = s->vmax;
  d.vitype = s->vitype.data(); d.virt_center = s->vcenter.data(); d.virt_numatoms = s->vnum.data();
  d.virt_atm_ind = s->vatm.data(); d.virt_invmass = s->vinvmass.data(); d.virt_masscoeff = s->vcoeff.data();
}

bool read_all(ibg_setup* s, const std::string& dir) {
  std::memset(&s->d, 0, sizeof(s->d));
  units(s);
  if (!control(s, dir)) return false;
  if (!interaction(s, dir)) return false;
  if (!coordinate(s, dir)) return false;
  ibg_desc& d = s->d;
  if (d.ibrdescr == 0) {
    if (!virtual_sites(s, dir)) return false;
    for (int i = 1; i <= d.natoms; ++i)  // MAKE_LISTS.f90:46-60
      (s->type_label[i - 1] == 1 ? s->atom : s->bead).push_back(i);
    d.numatoms = (int)s->atom.size();
    d.numbeads = (int)s->bead.size();
    for (int i = 1; i <= d.nvirta; ++i) s->bead.push_back(d.natoms + i);
    d.ncoarse = (int)s->bead.size();
  } else {
    for (int i = 1; i <= d.natoms; ++i) s->atom.push_back(i);
    d.numatoms = d.natoms; d.numbeads = 0; d.ncoarse = 0;
  }
  ftable(s);
  if (s->restart == 1) scalev(s);  // main.F90:168-171
  d.mktemp_atom = 2.0f / (3.0f * (float)(d.numatoms - 1));  // main.F90:177-178
  d.mktemp_bead = 2.0f / (3.0f * (float)(d.numbeads - 1));
  if (!topology(s, dir)) return false;
  if (!exclusions(s, dir)) return false;
  fill_desc(s);
  return true;
}

}  // namespace

extern "C" {

int ibg_setup_read(const char* dir, ibg_setup** out, char* err, int errlen) {
  if (!dir || !out) return IBG_E_INVALID;
  auto* s = new ibg_setup();
  if (!read_all(s, dir)) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", s->err.c_str());
    delete s;
    *out = nullptr;
    return IBG_E_IO;
  }
  *out = s;
  return IBG_OK;
}

int ibg_setup_read_mem(int nfiles, const char* const* names, const char* const* data, const long* sizes,
                       ibg_setup** out, char* err, int errlen) {
  if (!out || nfiles < 0 || (nfiles > 0 && (!names || !data || !sizes))) return IBG_E_INVALID;
  *out = nullptr;
  std::map<std::string, std::string> files;
  for (int k = 0; k < nfiles; ++k) {
    if (!names[k] || sizes[k] < 0 || (sizes[k] > 0 && !data[k])) return IBG_E_INVALID;
    files[names[k]] = std::string(data[k] ? data[k] : "", (size_t)sizes[k]);
  }
  auto* s = new ibg_setup();
  t_files = &files;
  const bool ok = read_all(s, "");
  t_files = nullptr;
  if (!ok) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", s->err.c_str());
    delete s;
    return IBG_E_IO;
  }
  *out = s;
  return IBG_OK;
}

int ibg_setup_set_nb_table(ibg_setup* s, int table, int nrows, const float* r, const float* v) {
  if (!s || !r || !v || nrows < 2 || table < 1 || table > s->tn.n) return IBG_E_INVALID;
  Table& n = s->tn;
  const int need = nrows + 4;  // a possible inserted row 0, rows up to NDATNB+1 and the zero row past it
  if (need > n.ld) {           // a longer table: widen every column
    Table w;
    w.init(n.n, need, true);
    for (int i = 1; i <= n.n; ++i) {
      for (int k = 0; k < n.ld; ++k) { w.X(i, k) = n.X(i, k); w.P(i, k) = n.P(i, k); w.F(i, k) = n.F(i, k); }
      w.bin[i - 1] = n.bin[i - 1];
      w.ndat[i - 1] = n.ndat[i - 1];
    }
    n = std::move(w);
  }
  for (int k = 0; k < n.ld; ++k) n.X(table, k) = n.P(table, k) = n.F(table, k) = 0.0f;
  XY t;
  t.x.assign(r, r + nrows);
  t.y.assign(v, v + nrows);
  nb_table(s, table, t);
  ftable_nb(s, table);
  fill_desc(s);
  return IBG_OK;
}

const ibg_desc* ibg_setup_desc(const ibg_setup* s) { return s ? &s->d : nullptr; }

int ibg_setup_initial_state(const ibg_setup* s, float* sxyz, float* vxyz, float* box) {
  if (!s) return IBG_E_INVALID;
  if (sxyz) std::memcpy(sxyz, s->sxyz.data(), sizeof(float) * s->sxyz.size());
  if (vxyz) std::memcpy(vxyz, s->vxyz.data(), sizeof(float) * s->vxyz.size());
  if (box) std::memcpy(box, s->box, sizeof(float) * 3);
  return IBG_OK;
}

int ibg_setup_control(const ibg_setup* s, int* iv, int n) {
  if (!s || !iv) return IBG_E_INVALID;
  int v[] = {s->nstep, s->ntrj, s->restart, s->nonbexc_atom, s->nonbexc_bead, s->nmol};
  for (int i = 0; i < n && i < (int)(sizeof(v) / sizeof(v[0])); ++i) iv[i] = v[i];
  return IBG_OK;
}

long ibg_setup_array_i(const ibg_setup* s, const char* name, int* out, long n) {
  if (!s || !name) return -1;
  const std::map<std::string, const std::vector<int>*> m = {
      {"ITYPE", &s->itype}, {"TYPE_LABEL", &s->type_label}, {"ATOM", &s->atom}, {"BEAD", &s->bead},
      {"NBONDS", &s->nbonds}, {"JBOND", &s->jbond},
      {"NIJK", &s->nijk}, {"JANGLEIJK", &s->jang}, {"KANGLEIJK", &s->kang},
      {"NOANGLEIJK", &s->noang}, {"NOJANGLEIJK", &s->nojang}, {"NOKANGLEIJK", &s->nokang},
      {"NIJKL", &s->nijkl}, {"JTORIJKL", &s->jtor}, {"KTORIJKL", &s->ktor}, {"LTORIJKL", &s->ltor},
      {"FNIJKL", &s->fnijkl}, {"FJTORIJKL", &s->fjtor}, {"FKTORIJKL", &s->fktor}, {"FLTORIJKL", &s->fltor},
      {"NOOPIJKL", &s->noop}, {"JOOPIJKL", &s->joop}, {"KOOPIJKL", &s->koop}, {"LOOPIJKL", &s->loop},
      {"CONNECTIONS", &s->connections}, {"CONNECTED_TO", &s->connected_to},
      {"IBONDT", &s->ibondt}, {"INBONDT", &s->inbondt}, {"IANGT", &s->iangt}, {"ITORT", &s->itort}, {"IOOPT", &s->ioopt},
      {"VITYPE", &s->vitype}, {"VIRT_CENTER", &s->vcenter}, {"VIRT_NUMATOMS", &s->vnum}, {"VIRT_ATM_IND", &s->vatm},
      {"NDATB", &s->tb.ndat}, {"NDATAN", &s->ta.ndat}, {"NDATT", &s->tt.ndat}, {"NDATNB", &s->tn.ndat}, {"NDATO", &s->to.ndat},
      {"BOND_TYPE_LABEL", &s->lab_b}, {"ANGLE_TYPE_LABEL", &s->lab_a}, {"TORSION_TYPE_LABEL", &s->lab_t}, {"OOP_TYPE_LABEL", &s->lab_o}};
  auto it = m.find(name);
  if (it == m.end()) return -1;
  long sz = (long)it->second->size();
  if (out) {
    if (n < sz) return -1;
    std::memcpy(out, it->second->data(), sizeof(int) * sz);
  }
  return sz;
}

long ibg_setup_array_f(const ibg_setup* s, const char* name, float* out, long n) {
  if (!s || !name) return -1;
  const std::map<std::string, const std::vector<float>*> m = {
      {"MASS", &s->mass}, {"INVMASS", &s->invmass}, {"SXYZ", &s->sxyz}, {"VXYZ", &s->vxyz},
      {"VIRT_MASS", &s->vmass}, {"VIRT_INVMASS", &s->vinvmass}, {"VIRT_MASSCOEFF", &s->vcoeff},
      {"RBOND", &s->tb.x}, {"BOND_POT", &s->tb.pot}, {"BOND_FORCE", &s->tb.frc}, {"BINB", &s->tb.bin},
      {"ANGLE", &s->ta.x}, {"BEND_POT", &s->ta.pot}, {"BEND_FORCE", &s->ta.frc}, {"BINA", &s->ta.bin},
      {"ANGLE_TOR", &s->tt.x}, {"TOR_POT", &s->tt.pot}, {"TOR_FORCE", &s->tt.frc}, {"BINT", &s->tt.bin},
      {"RNBOND", &s->tn.x}, {"NBOND_POT", &s->tn.pot}, {"NBOND_FORCE", &s->tn.frc}, {"BINNB", &s->tn.bin},
      {"ANGLE_OOP", &s->to.x}, {"OOP_POT", &s->to.pot}, {"OOP_FORCE", &s->to.frc}, {"BINO", &s->to.bin}};
  auto it = m.find(name);
  if (it == m.end()) return -1;
  long sz = (long)it->second->size();
  if (out) {
    if (n < sz) return -1;
    std::memcpy(out, it->second->data(), sizeof(float) * sz);
  }
  return sz;
}

void ibg_setup_free(ibg_setup* s) { delete s; }

}  // extern "C"

// ------------------------------------------------------------ WRITETRJ.F90
namespace {

// One Fortran unformatted sequential record as gfortran writes it: the
// payload between two 4-byte length markers.
bool record(std::FILE* f, const void* p, size_t n) {
  const unsigned m = (unsigned)n;
  return std::fwrite(&m, 4, 1, f) == 1 && (n == 0 || std::fwrite(p, 1, n, f) == n) && std::fwrite(&m, 4, 1, f) == 1;
}

// Fortran Gw.d output editing: F(w-4).(d-k) and four blanks when the value
// rounded to d digits has decimal exponent k in 0..d (0.1 <= |x| < 10^d),
// Ew.d (0.ddd...E+ee) otherwise; zero as F(w-4).(d-1).
std::string fortran_g(double x, int w, int d) {
  char buf[96];
  const double a = std::fabs(x);
  if (a == 0.0) {
    std::snprintf(buf, sizeof buf, "%*.*f    ", w - 4, d - 1, 0.0);
    return buf;
  }
  std::snprintf(buf, sizeof buf, "%.*e", d - 1, a);  // m.mmm...e+XX, d digits
  const char* e = std::strchr(buf, 'e');
  const int k = std::atoi(e + 1) + 1;  // 10^(k-1) <= |x| < 10^k after rounding
  if (k >= 0 && k <= d) {
    char out[96];
    std::snprintf(out, sizeof out, "%*.*f    ", w - 4, d - k, x);
    return out;
  }
  std::string digits;
  for (const char* c = buf; c < e; ++c)
    if (*c >= '0' && *c <= '9') digits.push_back(*c);
  char tail[16];
  std::snprintf(tail, sizeof tail, "E%c%02d", k < 0 ? '-' : '+', std::abs(k));
  std::string v = std::string(x < 0 ? "-" : "") + "0." + digits + tail;
  return std::string(v.size() < (size_t)w ? w - v.size() : 0, ' ') + v;
}

}  // namespace

struct ibg_trz {
  const ibg_setup* s;
  std::FILE* f;
  int nframe;
};

extern "C" {

int ibg_trz_open(const ibg_setup* s, const char* path, ibg_trz** out) {
  if (!s || !path || !out) return IBG_E_INVALID;
  std::FILE* f = std::fopen(path, "wb");
  if (!f) return IBG_E_IO;
  *out = new ibg_trz{s, f, 0};
  return IBG_OK;
}

int ibg_trz_write(ibg_trz* t, int step, const ibg_obs* obs, const float* sxyz, const float* vxyz) {
  if (!t || !obs || !sxyz || !vxyz) return IBG_E_INVALID;
  const ibg_setup* s = t->s;
  const ibg_desc& d = s->d;
  const int NA = d.natoms;
  const double small = 1.0 / 1.0e12 / (double)s->TIMESCALE;  // WRITETRJ.F90:31
  std::vector<float> col((size_t)NA);
  bool ok = true;
  t->nframe += 1;
  if (t->nframe == 1) {  // :51-55, header with the first frame
    char title[80];
    std::memset(title, ' ', sizeof title);
    std::memcpy(title, s->title.data(), std::min<size_t>(s->title.size(), 72));
    const int nrec = 10;
    ok = ok && record(t->f, title, 80) && record(t->f, &nrec, 4);
  }
  // :56-58: frame number, its step index, NATOMS and the time in ps
  const double treal = (double)((float)step * d.dt * s->TIMESCALE) * 1.0e12 + (double)s->initime;
  unsigned char hdr[20];
  const int hi[3] = {t->nframe, s->ntrj * t->nframe, NA};
  std::memcpy(hdr, hi, 12);
  std::memcpy(hdr + 12, &treal, 8);
  ok = ok && record(t->f, hdr, 20);
  const double boxr[9] = {(double)(float)obs->box[0], 0.0, 0.0, 0.0, (double)(float)obs->box[1], 0.0,
                          0.0, 0.0, (double)(float)obs->box[2]};  // :60-66
  ok = ok && record(t->f, boxr, sizeof boxr);
  // :68-79, the pressure tensor of the step in REAL*4 as the host holds it
  float pt[6];
  for (int k = 0; k < 6; ++k) pt[k] = (float)obs->pt[k];  // PT11, PT22, PT33, PT12, PT13, PT23
  const double pr[7] = {(double)(((pt[0] + pt[1]) + pt[2]) * s->PSCALE) / 3.0, (double)(pt[0] * s->PSCALE),
                        (double)(pt[3] * s->PSCALE), (double)(pt[1] * s->PSCALE), (double)(pt[4] * s->PSCALE),
                        (double)(pt[5] * s->PSCALE), (double)(pt[2] * s->PSCALE)};
  ok = ok && record(t->f, pr, sizeof pr);
  // :81-85, energies
  auto sum3 = [](const double* v) { return (v[0] + v[1]) + v[2]; };
  const double ptot = (((sum3(obs->v_bond) + sum3(obs->v_angle)) + sum3(obs->v_torsion)) + sum3(obs->v_oop)) +
                      sum3(obs->v_nb);
  const double ek = obs->ek[0] + obs->ek[1];
  const double etot = ptot + ek;
  const double temp = ek * (double)d.mktemp;
  unsigned char en[52];
  const int six = 6;
  const double ev[6] = {etot * (double)s->CONV, ptot * (double)s->CONV, ek * (double)s->CONV, temp, 0.0, 0.0};
  std::memcpy(en, &six, 4);
  std::memcpy(en + 4, ev, 48);
  ok = ok && record(t->f, en, 52);
  for (int c = 0; c < 3 && ok; ++c) {  // :87-90
    for (int j = 0; j < NA; ++j) col[j] = sxyz[3 * (size_t)j + c];
    ok = record(t->f, col.data(), sizeof(float) * NA);
  }
  for (int c = 0; c < 3 && ok; ++c) {  // :39-47, :92-95
    for (int j = 0; j < NA; ++j) col[j] = (float)((double)vxyz[3 * (size_t)j + c] * small);
    ok = record(t->f, col.data(), sizeof(float) * NA);
  }
  ok = ok && std::fflush(t->f) == 0;
  return ok ? IBG_OK : IBG_E_IO;
}

void ibg_trz_close(ibg_trz* t) {
  if (!t) return;
  if (t->f) std::fclose(t->f);
  delete t;
}

int ibg_write_restart(const ibg_setup* s, const char* path, int step, const float* box, const float* sxyz,
                      const float* vxyz) {
  if (!s || !path || !box || !sxyz || !vxyz) return IBG_E_INVALID;
  const ibg_desc& d = s->d;
  std::FILE* f = std::fopen(path, "w");
  if (!f) return IBG_E_IO;
  // WRITETRJ.F90:129-143: title, time, box, a five-line header, molecule count
  const float treal = (float)((double)((float)step * d.dt * s->TIMESCALE) * 1.0e12 + (double)s->initime);
  std::fprintf(f, " %s\n Time\t%.9g\t(ps)\n *** box lengths X, Y, Z in nm ***\n %.9g %.9g %.9g\n", s->title.c_str(),
               (double)treal, (double)box[0], (double)box[1], (double)box[2]);
  std::fprintf(f, "%s\n", std::string(70, '*').c_str());
  std::fprintf(f, "*** per atom: index, type, number of bonds, x y z (nm)\n");
  std::fprintf(f, "*** then vx vy vz (nm/ps) and the bonded atoms\n");
  std::fprintf(f, "*** written as WRITE_RESTART writes them\n");
  std::fprintf(f, "%s\n", std::string(70, '*').c_str());
  std::fprintf(f, " num_of_molecules  %d\n", s->nmol);
  const int N = d.nitems;
  int L = 0;
  for (int m = 0; m < s->nmol; ++m) {  // :144-173
    std::fprintf(f, " %d  Atoms_in_Molecule_No. %d %s\n", s->natm[m], m + 1, s->molname[m].c_str());
    for (int j = 0; j < s->natm[m]; ++j, ++L) {
      const int nb = s->nbonds[L];
      std::string line = " ";
      char buf[64];
      std::snprintf(buf, sizeof buf, "%6d %2d %1d ", L + 1, s->itype[L], nb);
      line += buf;
      for (int c = 0; c < 3; ++c) line += fortran_g((double)sxyz[3 * (size_t)L + c], 21, 14) + " ";
      std::fprintf(f, "%s\n", line.c_str());
      line.clear();
      const char* sep = nb == 2 ? "  " : " ";  // FORMAT 9060 spaces its velocities by two
      for (int c = 0; c < 3; ++c) {
        const double v = (double)(vxyz[3 * (size_t)L + c] * s->VSCALE) * 1.0e-3;
        std::snprintf(buf, sizeof buf, "%16.10f%s", v, sep);
        line += buf;
      }
      for (int b = 0; b < nb; ++b) {
        std::snprintf(buf, sizeof buf, nb == 1 ? "%5d" : "%5d  ", s->jbond[(size_t)b * N + L]);
        line += buf;
      }
      std::fprintf(f, "%s\n", line.c_str());
    }
  }
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  return ok ? IBG_OK : IBG_E_IO;
}

}  // extern "C"
