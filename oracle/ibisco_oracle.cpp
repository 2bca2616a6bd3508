// Oracle for the Hybrid IBIsCO force-and-integrate path.
//
// TEST INFRASTRUCTURE ONLY.  This is a CPU restatement of the reference
// (richardjgowers/ibisco, Fortran 90 + OpenMP) used to check the CUDA path and
// as the timed CPU baseline.  Nothing in the product links or calls it; only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm
// load it.
//
// Pinning: Engine<float> is checked against the reference's own golden
// trajectories (testsuite/tests.py:10-68) by tests/test_oracle_golden.py.
//
// C interface (ctypes):  handles own one Setup (REAL*4, read from a directory
// of reference-format input files) and two engines: precision 0 = REAL*4
// restatement, precision 1 = the same algorithm in double.
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include "oracle_engine.hpp"
#include "oracle_setup.hpp"

using namespace orc;

struct OrcHandle {
  Setup s;
  Engine<float> ef;
  Engine<double> ed;
  std::string err;
  std::map<std::string, std::pair<const int*, long>> ints;
  std::map<std::string, std::pair<const float*, long>> floats;
};

static void register_arrays(OrcHandle* h) {
  Setup& s = h->s;
  auto I = [&](const char* n, const std::vector<int>& v) { h->ints[n] = {v.data(), (long)v.size()}; };
  auto Fv = [&](const char* n, const std::vector<float>& v) { h->floats[n] = {v.data(), (long)v.size()}; };
  I("ITYPE", s.ITYPE); I("TYPE_LABEL", s.TYPE_LABEL); I("NBONDS", s.NBONDS); I("JBOND", s.JBOND);
  I("ATOM", s.ATOM); I("BEAD", s.BEAD);
  I("NIJK", s.NIJK); I("JANGLEIJK", s.JANGLEIJK); I("KANGLEIJK", s.KANGLEIJK);
  I("NOANGLEIJK", s.NOANGLEIJK); I("NOJANGLEIJK", s.NOJANGLEIJK); I("NOKANGLEIJK", s.NOKANGLEIJK);
  I("NIJKL", s.NIJKL); I("JTORIJKL", s.JTORIJKL); I("KTORIJKL", s.KTORIJKL); I("LTORIJKL", s.LTORIJKL);
  I("FNIJKL", s.FNIJKL); I("FJTORIJKL", s.FJTORIJKL); I("FKTORIJKL", s.FKTORIJKL); I("FLTORIJKL", s.FLTORIJKL);
  I("NOOPIJKL", s.NOOPIJKL); I("JOOPIJKL", s.JOOPIJKL); I("KOOPIJKL", s.KOOPIJKL); I("LOOPIJKL", s.LOOPIJKL);
  I("CONNECTIONS", s.CONNECTIONS); I("CONNECTED_TO", s.CONNECTED_TO);
  I("IBONDT", s.IBONDT); I("INBONDT", s.INBONDT); I("IANGT", s.IANGT); I("ITORT", s.ITORT); I("IOOPT", s.IOOPT);
  I("BOND_TYPE_LABEL", s.BOND_TYPE_LABEL); I("ANGLE_TYPE_LABEL", s.ANGLE_TYPE_LABEL);
  I("TORSION_TYPE_LABEL", s.TORSION_TYPE_LABEL); I("OOP_TYPE_LABEL", s.OOP_TYPE_LABEL);
  I("VITYPE", s.VITYPE); I("VIRT_CENTER", s.VIRT_CENTER); I("VIRT_NUMATOMS", s.VIRT_NUMATOMS);
  I("VIRT_ATM_IND", s.VIRT_ATM_IND);
  I("NDATB", s.bond.ndat); I("NDATAN", s.bend.ndat); I("NDATT", s.tors.ndat); I("NDATNB", s.nb.ndat); I("NDATO", s.oop.ndat);
  Fv("MASS", s.MASS); Fv("INVMASS", s.INVMASS); Fv("SXYZ", s.SXYZ); Fv("VXYZ", s.VXYZ);
  Fv("VIRT_MASS", s.VIRT_MASS); Fv("VIRT_INVMASS", s.VIRT_INVMASS); Fv("VIRT_MASSCOEFF", s.VIRT_MASSCOEFF);
  Fv("RBOND", s.bond.x); Fv("BOND_POT", s.bond.pot); Fv("BOND_FORCE", s.bond.force); Fv("BINB", s.bond.bin);
  Fv("ANGLE", s.bend.x); Fv("BEND_POT", s.bend.pot); Fv("BEND_FORCE", s.bend.force); Fv("BINA", s.bend.bin);
  Fv("ANGLE_TOR", s.tors.x); Fv("TOR_POT", s.tors.pot); Fv("TOR_FORCE", s.tors.force); Fv("BINT", s.tors.bin);
  Fv("RNBOND", s.nb.x); Fv("NBOND_POT", s.nb.pot); Fv("NBOND_FORCE", s.nb.force); Fv("BINNB", s.nb.bin);
  Fv("ANGLE_OOP", s.oop.x); Fv("OOP_POT", s.oop.pot); Fv("OOP_FORCE", s.oop.force); Fv("BINO", s.oop.bin);
}

template <typename E>
static int nonbonded_list(E& e, const orc::Setup& st, int which, double* fxyz, double* sums) {
  using R = decltype(e.PT11);
  e.zero_force_stage();
  if (which == 0) e.nonbonded_force(st.ATOM, st.NUMATOMS, e.la, (R)st.RCUTSQ_ATOM);
  else e.nonbonded_force(st.BEAD, st.NCOARSE, e.lb, (R)st.RCUTSQ_BEAD);
  for (size_t k = 0; k < e.F.size(); ++k) fxyz[k] = (double)e.F[k];
  const double v[9] = {e.V_NB[0], e.V_NB[1], e.V_NB[2], (double)e.PT11, (double)e.PT22, (double)e.PT33,
                       (double)e.PT12, (double)e.PT13, (double)e.PT23};
  for (int k = 0; k < 9; ++k) sums[k] = v[k];
  return e.err;
}

extern "C" {

void* orc_open(const char* dir, int nthreads, char* errbuf, int errlen) {
  auto* h = new OrcHandle();
  if (!setup_from_dir(h->s, dir)) {
    if (errbuf && errlen > 0) std::snprintf(errbuf, errlen, "%s", h->s.err.c_str());
    delete h;
    return nullptr;
  }
  h->ef.attach(&h->s, nthreads);
  h->ed.attach(&h->s, nthreads);
  register_arrays(h);
  return h;
}

void orc_close(void* p) { delete static_cast<OrcHandle*>(p); }

void orc_set_threads(void* p, int n) {
  auto* h = static_cast<OrcHandle*>(p);
  h->ef.nthreads = h->ed.nthreads = std::max(1, n);
  h->ef.fpriv.assign(h->ef.nthreads, std::vector<float>((size_t)3 * h->s.NITEMS, 0.f));
  h->ed.fpriv.assign(h->ed.nthreads, std::vector<double>((size_t)3 * h->s.NITEMS, 0.0));
}

void orc_set_com_fix(void* p, int on) {
  auto* h = static_cast<OrcHandle*>(p);
  h->ef.com_fix = h->ed.com_fix = on != 0;
}

// Integer scalars of the setup, in this order.
int orc_info_int(void* p, int* out, int n) {
  auto& s = static_cast<OrcHandle*>(p)->s;
  int v[] = {s.NATOMS, s.NVIRTA, s.NITEMS, s.NTYPE, s.NUMATOMS, s.NUMBEADS, s.NCOARSE, s.ENSEMBLE,
             s.NSTEP, s.NUPDATE, s.HALT_DRIFT, s.NTRJ, s.NMTS, s.IBRDESCR, s.NONBEXC_ATOM, s.NONBEXC_BEAD,
             s.bond.nt, s.bend.nt, s.tors.nt, s.nb.nt, s.oop.nt, s.bond.w, s.bend.w, s.tors.w, s.nb.w, s.oop.w,
             s.VIRT_MAXATOMS, s.RESTART, s.NMOL};
  int m = (int)(sizeof(v) / sizeof(v[0]));
  for (int i = 0; i < n && i < m; ++i) out[i] = v[i];
  return m;
}
// Float scalars of the setup, in this order.
int orc_info_float(void* p, float* out, int n) {
  auto& s = static_cast<OrcHandle*>(p)->s;
  float v[] = {s.DT, s.FAC, s.PFAC, s.TEMP_IN, s.PRESSURE, s.MKTEMP, s.MKTEMP_ATOM, s.MKTEMP_BEAD,
               s.RCUT_ATOM, s.RCUTSQ_ATOM, s.RLIST_ATOM, s.RCUT_BEAD, s.RCUTSQ_BEAD, s.RLIST_BEAD,
               s.BOX[0], s.BOX[1], s.BOX[2], s.R2D, s.D2R, s.TIMESCALE, s.VSCALE, s.CONV, s.PSCALE,
               s.TEMPSCALE, s.ESCALE, s.NA, s.MASSSCALE};
  int m = (int)(sizeof(v) / sizeof(v[0]));
  for (int i = 0; i < n && i < m; ++i) out[i] = v[i];
  return m;
}

long orc_array_size(void* p, const char* name) {
  auto* h = static_cast<OrcHandle*>(p);
  auto it = h->ints.find(name);
  if (it != h->ints.end()) return it->second.second;
  auto jt = h->floats.find(name);
  if (jt != h->floats.end()) return jt->second.second;
  return -1;
}
int orc_get_int_array(void* p, const char* name, int* out, long n) {
  auto* h = static_cast<OrcHandle*>(p);
  auto it = h->ints.find(name);
  if (it == h->ints.end() || n < it->second.second) return -1;
  std::memcpy(out, it->second.first, sizeof(int) * it->second.second);
  return 0;
}
int orc_get_float_array(void* p, const char* name, float* out, long n) {
  auto* h = static_cast<OrcHandle*>(p);
  auto it = h->floats.find(name);
  if (it == h->floats.end() || n < it->second.second) return -1;
  std::memcpy(out, it->second.first, sizeof(float) * it->second.second);
  return 0;
}

#define ENG(h, prec, body)        \
  do {                            \
    if (prec == 0) {              \
      auto& e = h->ef;            \
      body;                       \
    } else {                      \
      auto& e = h->ed;            \
      body;                       \
    }                             \
  } while (0)

// Set positions (3,NATOMS), velocities (3,NATOMS) and box, then run the
// reference's pre-loop initialisation (VS define, SHIFT, initial kinetic
// energy and temperatures, cell maps and the first Verlet list).
int orc_set_state(void* p, int prec, const float* sxyz, const float* vxyz, const float* box) {
  auto* h = static_cast<OrcHandle*>(p);
  ENG(h, prec, { e.set_state(sxyz, vxyz, box); return e.err; });
}
// The state read from the coordinate file.
int orc_init(void* p, int prec) {
  auto* h = static_cast<OrcHandle*>(p);
  return orc_set_state(p, prec, h->s.SXYZ.data(), h->s.VXYZ.data(), h->s.BOX);
}
int orc_step(void* p, int prec, int step) {
  auto* h = static_cast<OrcHandle*>(p);
  ENG(h, prec, { return e.step(step); });
}
int orc_run(void* p, int prec, int first, int nsteps) {
  auto* h = static_cast<OrcHandle*>(p);
  for (int k = 0; k < nsteps; ++k) {
    int rc = orc_step(p, prec, first + k);
    if (rc) return rc;
  }
  (void)h;
  return 0;
}
// SHIFT, VIRTUAL_DEF, the list rebuild when due and the force stage of one
// step, without MOVE.
int orc_forces(void* p, int prec, int step) {
  auto* h = static_cast<OrcHandle*>(p);
  ENG(h, prec, { e.force_stage(step); return e.err; });
}
// NONBONDED_FORCE.F90 on one list alone (which: 0 atom list, 1 bead list) at
// the current positions: forces (3,NITEMS) and sums[9] = V_NB(1..3), PT11,
// PT22, PT33, PT12, PT13, PT23 (not divided by the volume).  It replaces the
// engine's force arrays; call orc_forces or orc_step to rebuild them.
int orc_nonbonded_list(void* p, int prec, int which, double* fxyz, double* sums) {
  auto* h = static_cast<OrcHandle*>(p);
  return prec == 0 ? nonbonded_list(h->ef, h->s, which, fxyz, sums) : nonbonded_list(h->ed, h->s, which, fxyz, sums);
}
const char* orc_error(void* p, int prec) {
  auto* h = static_cast<OrcHandle*>(p);
  return prec == 0 ? h->ef.errmsg.c_str() : h->ed.errmsg.c_str();
}

// Arrays are (3,N) in Fortran order, returned as double.
int orc_get_state(void* p, int prec, double* sxyz, double* rxyz, double* vxyz, double* fxyz) {
  auto* h = static_cast<OrcHandle*>(p);
  ENG(h, prec, {
    for (size_t k = 0; k < e.S.size(); ++k) {
      if (sxyz) sxyz[k] = (double)e.S[k];
      if (rxyz) rxyz[k] = (double)e.RW[k];
      if (fxyz) fxyz[k] = (double)e.F[k];
    }
    if (vxyz) for (size_t k = 0; k < e.V.size(); ++k) vxyz[k] = (double)e.V[k];
    return 0;
  });
}

// obs: EK[2], TEMP, TEMP_ATOM, TEMP_BEAD, V_NB[3], V_BOND[3], V_ANGLE[3],
// V_TORSION[3], V_OOP[3], PT11, PT22, PT33, PT12, PT13, PT23, BOX[3],
// bond over-extensions, cell clamps   (32 doubles)
int orc_get_obs(void* p, int prec, double* o) {
  auto* h = static_cast<OrcHandle*>(p);
  ENG(h, prec, {
    int k = 0;
    o[k++] = e.EK[0]; o[k++] = e.EK[1];
    o[k++] = e.TEMP; o[k++] = e.TEMP_ATOM; o[k++] = e.TEMP_BEAD;
    for (int c = 0; c < 3; ++c) o[k++] = e.V_NB[c];
    for (int c = 0; c < 3; ++c) o[k++] = e.V_BOND[c];
    for (int c = 0; c < 3; ++c) o[k++] = e.V_ANGLE[c];
    for (int c = 0; c < 3; ++c) o[k++] = e.V_TORSION[c];
    for (int c = 0; c < 3; ++c) o[k++] = e.V_OOP[c];
    o[k++] = e.PT11; o[k++] = e.PT22; o[k++] = e.PT33; o[k++] = e.PT12; o[k++] = e.PT13; o[k++] = e.PT23;
    for (int c = 0; c < 3; ++c) o[k++] = e.BOX[c];
    o[k++] = e.bond_overext; o[k++] = e.cell_clamps;
    return k;
  });
}

// Verlet list `which` (0 atom list, 1 bead list) as LIST(maxnab,N): column A
// holds the neighbours of INDEX_LIST(A) as 1-based global ids, 0-terminated.
// nnebs receives NNEBS(INDEX_LIST(A)).  Returns N, or -1 if maxnab is too small.
int orc_get_list(void* p, int prec, int which, int* list, int maxnab, int* nnebs) {
  auto* h = static_cast<OrcHandle*>(p);
  ENG(h, prec, {
    auto& L = which == 0 ? e.la : e.lb;
    int n = which == 0 ? h->s.NUMATOMS : h->s.NCOARSE;
    for (int a = 1; a <= n; ++a) {
      auto& l = L.list[a];
      if ((int)l.size() >= maxnab) return -1;
      if (nnebs) nnebs[a - 1] = (int)l.size();
      if (list) {
        int* col = list + (size_t)(a - 1) * maxnab;
        for (int k = 0; k < maxnab; ++k) col[k] = k < (int)l.size() ? l[k] : 0;
      }
    }
    return n;
  });
}

}  // extern "C"
