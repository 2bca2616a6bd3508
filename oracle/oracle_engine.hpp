// Oracle (test infrastructure only): restatement of the reference's per-step
// force-and-integrate path.  Engine<float> follows the REAL*4 semantics of the
// Fortran source (mixed-mode FP64 promotions where the source writes 1.0D0 /
// 2.0D0, ANINT = round half away from zero, INT = truncation, no FMA,
// OpenMP REDUCTION semantics: private copies that start at zero and are added
// to the shared value at the end).  Engine<double> is the same algorithm with
// every REAL*4 quantity of the step held in double; it is the FP64 reference
// for the force/energy tolerance checks.
#pragma once
#include <omp.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>
#include "oracle_setup.hpp"

namespace orc {

enum OrcErr {
  ORC_OK = 0,
  ORC_E_LIST_OVERFLOW = -2,   // NEW_NEIGHBOUR_WITHLIST.f90:72,113
  ORC_E_TORSION_TABLE = -3,   // TORSIONS.inc:105-109
  ORC_E_OOP_RANGE = -4,       // OUTOFPLANES.inc:62-100
  ORC_E_CELL_GRID = -6,       // MAPS.f90 needs >= 3 cells per dimension
  ORC_E_TABLE_RANGE = -9,     // nonbonded lookup beyond the table
  ORC_E_MISSING_TABLE = -10,  // a listed pair has no nonbonded table
};

template <typename R>
inline R anint(R x) { return std::round(x); }
template <typename R>
inline int fint(R x) {  // Fortran INT (truncation); saturates instead of UB
  if (!(x == x)) return std::numeric_limits<int>::min();
  if (x >= (R)2147483647) return 2147483647;
  if (x <= (R)-2147483647) return -2147483647;
  return (int)x;
}

template <typename R>
struct Engine {
  using D = double;
  Setup* s = nullptr;
  int nthreads = 1;
  bool com_fix = true;  // VIRTUAL_DEF.f90:31 zeroes only the x sum; see com_bug below
  int err = 0;
  std::string errmsg;
  int NI_ = 0, NA_ = 0;
  // state (1-based particle index i lives at [3*(i-1)+c])
  std::vector<R> S, RW, V, VT, F, FNB;
  R BOX[3], BOXINV[3], BOX2[3];
  R PT11 = 0, PT22 = 0, PT33 = 0, PT12 = 0, PT13 = 0, PT23 = 0;
  double V_NB[3], V_BOND[3], V_ANGLE[3], V_TORSION[3], V_OOP[3], EK[2];
  R TEMP = 0, TEMP_ATOM = 0, TEMP_BEAD = 0;
  std::vector<int> TYPE_LABEL;
  // tables in R
  struct TabR {
    int nt = 0, w = 0;
    std::vector<R> x, p, f, bin;
    std::vector<int> ndat;
    R X(int t, int k) const { return x[(size_t)(t - 1) + (size_t)nt * k]; }
    R P(int t, int k) const { return p[(size_t)(t - 1) + (size_t)nt * k]; }
    R Fo(int t, int k) const { return f[(size_t)(t - 1) + (size_t)nt * k]; }
  } bond, bend, tors, nb, oop;
  // cell lists and Verlet lists
  struct NList {
    int ncx = 0, ncy = 0, ncz = 0;
    std::vector<int> map, head, lclist, cell;
    std::vector<std::vector<int>> list;  // list[A] = neighbour global ids in reference order
  } la, lb;
  std::vector<int> NNEBS;
  int cell_clamps = 0;
  int bond_overext = 0;
  // MTS (module_MTS.f90)
  std::vector<R> MTS_FXYZ;  // (3,3,NCOARSE)
  R MTS_V_NB[3][3];         // (m, label)
  R MTS_PT[6][3];           // PT11,PT22,PT33,PT12,PT13,PT23 for m=1..3; PT23 is never saved
  // SCALEBP
  int IAVP = 0;
  R SP[10];
  // thread-private buffers
  std::vector<std::vector<R>> fpriv;

  static void promote(const Tab& t, TabR& o) {
    o.nt = t.nt; o.w = t.w;
    o.x.assign(t.x.begin(), t.x.end()); o.p.assign(t.pot.begin(), t.pot.end());
    o.f.assign(t.force.begin(), t.force.end()); o.bin.assign(t.bin.begin(), t.bin.end());
    o.ndat = t.ndat;
  }

  void attach(Setup* setup, int threads) {
    s = setup; nthreads = std::max(1, threads);
    NI_ = s->NITEMS; NA_ = s->NATOMS;
    promote(s->bond, bond); promote(s->bend, bend); promote(s->tors, tors); promote(s->nb, nb); promote(s->oop, oop);
    S.assign((size_t)3 * NI_, 0); RW.assign((size_t)3 * NI_, 0);
    V.assign((size_t)3 * NA_, 0); VT.assign((size_t)3 * NA_, 0);
    F.assign((size_t)3 * NI_, 0); FNB.assign((size_t)3 * NA_, 0);
    NNEBS.assign(NI_ + 1, 0);
    MTS_FXYZ.assign((size_t)9 * std::max(1, s->NCOARSE), 0);
    for (auto& a : MTS_V_NB) for (auto& b : a) b = 0;
    for (auto& a : MTS_PT) for (auto& b : a) b = 0;
    for (auto& x : SP) x = 0;
    fpriv.assign(nthreads, std::vector<R>((size_t)3 * NI_, 0));
  }

  void fail(int code, const std::string& m) {
    if (err == 0) { err = code; errmsg = m; }
  }

  R& sx(int i, int c) { return S[3 * (size_t)(i - 1) + c]; }
  R& rx(int i, int c) { return RW[3 * (size_t)(i - 1) + c]; }
  R& vx(int i, int c) { return V[3 * (size_t)(i - 1) + c]; }
  R& fx(int i, int c) { return F[3 * (size_t)(i - 1) + c]; }

  // ------------------------------------------------------------- SHIFT.f90:36-44
  void fold(R* r, const R* src) {  // the three-component fold used by SHIFT and VIRTUAL_DEF
    R sp[3];
    for (int c = 0; c < 3; ++c) r[c] = src[c] / BOX2[c];
    for (int c = 0; c < 3; ++c) sp[c] = r[c] - (R)2.0 * (R)fint(r[c] / (R)2.0);
    for (int c = 0; c < 3; ++c) r[c] = (sp[c] - (R)2.0 * (R)fint(sp[c])) * BOX2[c];
  }
  static bool outside(const R* p, const R* b2) {
    for (int c = 0; c < 3; ++c) if (p[c] > b2[c] || p[c] < -b2[c]) return true;
    return false;
  }
  void shift() {
    for (int i = 1; i <= NA_; ++i) {
      R* si = &S[3 * (size_t)(i - 1)];
      R* ri = &RW[3 * (size_t)(i - 1)];
      if (outside(si, BOX2)) fold(ri, si);
      else for (int c = 0; c < 3; ++c) ri[c] = si[c];
    }
  }

  // -------------------------------------------------------- VIRTUAL_DEF.f90:19-47
  void virtual_def() {
    R sum[3] = {0, 0, 0};  // with com_fix off the y/z sums carry from site to site (:31)
    for (int i = 1; i <= s->NVIRTA; ++i) {
      int pos = i + NA_;
      TYPE_LABEL[pos] = 3;
      if (s->VIRT_CENTER[i] != 0) {
        int j = s->VIRT_CENTER[i];
        for (int c = 0; c < 3; ++c) { rx(pos, c) = sx(j, c); sx(pos, c) = sx(j, c); }
      } else {
        int ti = s->VITYPE[i];
        sum[0] = 0;
        if (com_fix) { sum[1] = 0; sum[2] = 0; }
        for (int j = 1; j <= s->VIRT_NUMATOMS[ti]; ++j) {
          int k = s->vatm(i, j);
          R m = (R)s->MASS[s->ITYPE[k]];
          for (int c = 0; c < 3; ++c) sum[c] = sum[c] + m * sx(k, c);
        }
        R inv = (R)s->VIRT_INVMASS[ti];
        for (int c = 0; c < 3; ++c) { rx(pos, c) = sum[c] * inv; sx(pos, c) = rx(pos, c); }
      }
      R* sp = &S[3 * (size_t)(pos - 1)];
      if (outside(sp, BOX2)) {
        R tmp[3] = {rx(pos, 0), rx(pos, 1), rx(pos, 2)};
        fold(&RW[3 * (size_t)(pos - 1)], tmp);
      }
    }
  }

  // -------------------------------------------------------------- MAPS.f90:20-77
  static int icell(int ix, int iy, int iz, int nx, int ny, int nz) {
    return 1 + ((iz - 1 + nz) % nz) + ((iy - 1 + ny) % ny) * nz + ((ix - 1 + nx) % nx) * nz * ny;
  }
  void maps(NList& L) {
    int nx = L.ncx, ny = L.ncy, nz = L.ncz;
    L.map.assign((size_t)13 * nx * ny * nz + 1, 0);
    for (int ix = 1; ix <= nx; ++ix)
      for (int iy = 1; iy <= ny; ++iy)
        for (int iz = 1; iz <= nz; ++iz) {
          int im = (icell(ix, iy, iz, nx, ny, nz) - 1) * 13;
          int* m = &L.map[im + 1];
          m[0] = icell(ix + 1, iy, iz, nx, ny, nz);
          m[1] = icell(ix + 1, iy + 1, iz, nx, ny, nz);
          m[2] = icell(ix, iy + 1, iz, nx, ny, nz);
          m[3] = icell(ix - 1, iy + 1, iz, nx, ny, nz);
          m[4] = icell(ix + 1, iy, iz - 1, nx, ny, nz);
          m[5] = icell(ix + 1, iy + 1, iz - 1, nx, ny, nz);
          m[6] = icell(ix, iy + 1, iz - 1, nx, ny, nz);
          m[7] = icell(ix - 1, iy + 1, iz - 1, nx, ny, nz);
          m[8] = icell(ix + 1, iy, iz + 1, nx, ny, nz);
          m[9] = icell(ix + 1, iy + 1, iz + 1, nx, ny, nz);
          m[10] = icell(ix, iy + 1, iz + 1, nx, ny, nz);
          m[11] = icell(ix - 1, iy + 1, iz + 1, nx, ny, nz);
          m[12] = icell(ix, iy, iz + 1, nx, ny, nz);
        }
  }

  // ------------------------------------------------------------- LINKS.f90:13-23
  // A component equal to NCELL (a coordinate at +L/2 after rounding) would index
  // past the grid in the reference; it is clamped to NCELL-1 and counted.
  int cell_component(R x, R binv, int nc) {
    int k = fint((x * binv + (R)0.5) * (R)nc);
    if (k >= nc) { k = nc - 1; ++cell_clamps; }
    if (k < 0) { k = 0; ++cell_clamps; }
    return k;
  }
  void links(NList& L, const std::vector<int>& idx, int n) {
    L.head.assign((size_t)L.ncx * L.ncy * L.ncz + 1, 0);
    L.lclist.assign(n + 1, 0);
    L.cell.assign(n + 1, 0);
    for (int a = 1; a <= n; ++a) {
      int i = idx[a];
      int jc = 1 + cell_component(rx(i, 0), BOXINV[0], L.ncx) * L.ncz * L.ncy +
               cell_component(rx(i, 1), BOXINV[1], L.ncy) * L.ncz +
               cell_component(rx(i, 2), BOXINV[2], L.ncz);
      L.lclist[a] = L.head[jc];
      L.head[jc] = a;
      L.cell[a] = jc;
    }
  }

  // ------------------------------------------- NEW_NEIGHBOUR_WITHLIST.f90:26-123
  void new_neighbour(NList& L, const std::vector<int>& idx, int n, R rlist, int maxnab) {
    R rlistsq = rlist * rlist;
    L.list.assign(n + 1, std::vector<int>());
    bool hybrid = s->IBRDESCR == 0;
    int overflow = 0;
#pragma omp parallel for num_threads(nthreads) schedule(static, 1) reduction(+ : overflow)
    for (int a = 1; a <= n; ++a) {
      int i = idx[a];
      auto& lst = L.list[a];
      R ri[3] = {rx(i, 0), rx(i, 1), rx(i, 2)};
      auto consider = [&](int b) {
        int j = idx[b];
        bool nonbond = true;
        int nc = s->CONNECTIONS[i];
        for (int c = 1; c <= nc; ++c)
          if (s->conn(i, c) == j) { nonbond = false; break; }
        if (hybrid && i > NA_ && j > NA_) nonbond = false;
        if (!nonbond) return;
        R d[3];
        for (int c = 0; c < 3; ++c) d[c] = ri[c] - rx(j, c);
        for (int c = 0; c < 3; ++c) d[c] = d[c] - anint(d[c] * BOXINV[c]) * BOX[c];
        R r2 = d[0] * d[0];
        r2 = r2 + d[1] * d[1];
        r2 = r2 + d[2] * d[2];
        if (r2 < rlistsq) {
          lst.push_back(j);
          if ((int)lst.size() == maxnab) ++overflow;
        }
      };
      for (int b = L.lclist[a]; b != 0; b = L.lclist[b]) consider(b);
      int jc0 = 13 * (L.cell[a] - 1);
      for (int nab = 1; nab <= 13; ++nab) {
        int jc = L.map[jc0 + nab];
        for (int b = L.head[jc]; b != 0; b = L.lclist[b]) consider(b);
      }
      NNEBS[i] = (int)lst.size();
    }
    if (overflow) fail(ORC_E_LIST_OVERFLOW, "LIST TOO SMALL");
  }

  bool grid_ok(const NList& L) {
    if (L.ncx < 3 || L.ncy < 3 || L.ncz < 3) {
      fail(ORC_E_CELL_GRID, "fewer than 3 cells in a dimension");
      return false;
    }
    return true;
  }

  // ----------------------------------------------- UPDATE_NEIGHBOURLIST.F90:14-85
  void update_neighbourlist(bool force_regrid = false) {
    if (s->ENSEMBLE == 2 || force_regrid) {
      la.ncx = fint(BOX[0] / (R)s->RLIST_ATOM); la.ncy = fint(BOX[1] / (R)s->RLIST_ATOM); la.ncz = fint(BOX[2] / (R)s->RLIST_ATOM);
      if (!grid_ok(la)) return;
      maps(la);
      if (s->IBRDESCR == 0) {
        lb.ncx = fint(BOX[0] / (R)s->RLIST_BEAD); lb.ncy = fint(BOX[1] / (R)s->RLIST_BEAD); lb.ncz = fint(BOX[2] / (R)s->RLIST_BEAD);
        if (!grid_ok(lb)) return;
        maps(lb);
      }
    }
    links(la, s->ATOM, s->NUMATOMS);
    new_neighbour(la, s->ATOM, s->NUMATOMS, (R)s->RLIST_ATOM, 1000);
    if (s->IBRDESCR == 0) {
      links(lb, s->BEAD, s->NCOARSE);
      new_neighbour(lb, s->BEAD, s->NCOARSE, (R)s->RLIST_BEAD, 1000);
    }
  }

  // ------------------------------------------------ NONBONDED_FORCE.F90:45-104
  void nonbonded_force(const std::vector<int>& idx, int n, NList& L, R rcutsq) {
    const int T = nthreads;
    std::vector<double> vnb((size_t)3 * T, 0.0);
    std::vector<R> pt((size_t)6 * T, (R)0);
    int bad_range = 0, missing = 0;
#pragma omp parallel num_threads(T) reduction(+ : bad_range, missing)
    {
      int t = omp_get_thread_num();
      std::vector<R>& fp = fpriv[t];
      std::fill(fp.begin(), fp.end(), (R)0);
      double* vn = &vnb[(size_t)3 * t];
      R* p = &pt[(size_t)6 * t];
      for (int a = 1 + t; a <= n; a += T) {
        int i = idx[a];
        R ri[3] = {rx(i, 0), rx(i, 1), rx(i, 2)};
        R fi[3] = {0, 0, 0};
        int ti = s->ITYPE[i];
        const auto& lst = L.list[a];
        int cnt = NNEBS[i];
        for (int jn = 0; jn < cnt; ++jn) {
          int j = lst[jn];
          int tj = s->ITYPE[j];
          int tij = s->INBONDT[s->t2(ti, tj)];
          R d[3];
          for (int c = 0; c < 3; ++c) d[c] = ri[c] - rx(j, c);
          for (int c = 0; c < 3; ++c) d[c] = d[c] - anint(d[c] * BOXINV[c]) * BOX[c];
          R r2 = d[0] * d[0];
          r2 = r2 + d[1] * d[1];
          r2 = r2 + d[2] * d[2];
          if (r2 < rcutsq) {
            if (tij == 0) { ++missing; continue; }
            R r = std::sqrt(r2);
            R bin = nb.bin[tij];
            int k = fint(r / bin);
            if (k < 0 || k + 1 >= nb.w || k > nb.ndat[tij]) { ++bad_range; continue; }
            R alpha = (r - nb.X(tij, k)) / bin;
            R fij = nb.Fo(tij, k) * ((R)1.0 - alpha) + nb.Fo(tij, k + 1) * alpha;
            R vij = nb.P(tij, k) * ((R)1.0 - alpha) + nb.P(tij, k + 1) * alpha;
            int li = TYPE_LABEL[i];
            if (li == 1) vn[0] += (double)vij;
            else if (li == 2) {
              int lj = TYPE_LABEL[j];
              if (lj == 2) vn[1] += (double)vij;
              else if (lj == 3) vn[2] += (double)vij;
            } else if (li == 3) vn[2] += (double)vij;
            for (int c = 0; c < 3; ++c) fi[c] = fi[c] + fij * d[c];
            for (int c = 0; c < 3; ++c) fp[3 * (size_t)(j - 1) + c] = fp[3 * (size_t)(j - 1) + c] - fij * d[c];
            p[0] = p[0] + fij * d[0] * d[0];
            p[1] = p[1] + fij * d[1] * d[1];
            p[2] = p[2] + fij * d[2] * d[2];
            p[3] = p[3] + fij * d[1] * d[0];
            p[4] = p[4] + fij * d[2] * d[0];
            p[5] = p[5] + fij * d[2] * d[1];
          }
        }
        for (int c = 0; c < 3; ++c) fp[3 * (size_t)(i - 1) + c] = fp[3 * (size_t)(i - 1) + c] + fi[c];
      }
    }
    for (int t = 0; t < T; ++t) {
      const std::vector<R>& fp = fpriv[t];
      for (size_t k = 0; k < F.size(); ++k) F[k] = F[k] + fp[k];
      for (int c = 0; c < 3; ++c) V_NB[c] += vnb[(size_t)3 * t + c];
      const R* p = &pt[(size_t)6 * t];
      PT11 = PT11 + p[0]; PT22 = PT22 + p[1]; PT33 = PT33 + p[2];
      PT12 = PT12 + p[3]; PT13 = PT13 + p[4]; PT23 = PT23 + p[5];
    }
    if (missing) fail(ORC_E_MISSING_TABLE, "pair without a nonbonded table");
    if (bad_range) fail(ORC_E_TABLE_RANGE, "nonbonded distance beyond its table");
  }

  // ------------------------------------------------- BONDED_FORCE.F90:38-99
  void bonded_force() {
    const int T = nthreads;
    std::vector<double> vb((size_t)12 * T, 0.0);
    int tor_err = 0, oop_err = 0, overext = 0;
    const R eps = (R)(float)1.0e-7;  // REAL*4 :: eps = 1.0D-7
#pragma omp parallel num_threads(T) reduction(+ : tor_err, oop_err, overext)
    {
      int t = omp_get_thread_num();
      std::vector<R>& FL = fpriv[t];
      std::fill(FL.begin(), FL.end(), (R)0);
      double* vbond = &vb[(size_t)12 * t];
      double* vang = vbond + 3;
      double* vtor = vbond + 6;
      double* voop = vbond + 9;
      auto fl = [&](int i, int c) -> R& { return FL[3 * (size_t)(i - 1) + c]; };
      for (int I = 1 + t; I <= NI_; I += T) {
        R ri[3] = {sx(I, 0), sx(I, 1), sx(I, 2)};
        R fi[3] = {0, 0, 0};
        int TI = s->ITYPE[I];
        // BONDS.inc:3-57
        for (int A = 1; A <= s->NBONDS[I]; ++A) {
          int J = s->jbond(I, A);
          if (J > I) {
            int TIJ = s->IBONDT[s->t2(TI, s->ITYPE[J])];
            R d[3];
            for (int c = 0; c < 3; ++c) d[c] = ri[c] - sx(J, c);
            R rijsq = d[0] * d[0] + d[1] * d[1];
            rijsq = rijsq + d[2] * d[2];
            R rij = std::sqrt(rijsq);
            int k = fint((rij - bond.X(TIJ, 0)) / bond.bin[TIJ]);
            if (k > bond.ndat[TIJ]) { ++overext; k = bond.ndat[TIJ]; }
            else if (k < 0) k = 0;
            R alpha = (rij - bond.X(TIJ, k)) / bond.bin[TIJ];
            R fij = (R)((D)bond.Fo(TIJ, k) * (1.0 - (D)alpha) + (D)(alpha * bond.Fo(TIJ, k + 1)));
            R vij = (R)((D)bond.P(TIJ, k) * (1.0 - (D)alpha) + (D)(alpha * bond.P(TIJ, k + 1)));
            vbond[s->BOND_TYPE_LABEL[TIJ] - 1] += (double)vij;
            R fij3[3];
            for (int c = 0; c < 3; ++c) fij3[c] = fij * d[c];
            for (int c = 0; c < 3; ++c) fi[c] = fi[c] + fij3[c];
            for (int c = 0; c < 3; ++c) fl(J, c) = fl(J, c) - fij3[c];
          }
        }
        // ANGLES.inc:2-75
        for (int A = 1; A <= s->NIJK[I]; ++A) {
          int J = s->jang(I, A), K = s->kang(I, A);
          int TIJK = s->IANGT[s->t3(TI, s->ITYPE[J], s->ITYPE[K])];
          R ij[3], kj[3];
          for (int c = 0; c < 3; ++c) ij[c] = ri[c] - sx(J, c);
          for (int c = 0; c < 3; ++c) kj[c] = sx(K, c) - sx(J, c);
          R rij = std::sqrt((ij[0] * ij[0] + ij[1] * ij[1]) + ij[2] * ij[2]);
          R rkj = std::sqrt((kj[0] * kj[0] + kj[1] * kj[1]) + kj[2] * kj[2]);
          R ct = ((ij[0] * kj[0] + ij[1] * kj[1]) + ij[2] * kj[2]) / rij / rkj;
          // ANGLES.inc:20-21 takes ACOS(CT) unclamped; rounding can put |CT| of a
          // straight angle just above 1, where the reference's result is NaN.  The
          // restatement clamps there, as TORSIONS.inc:93-96 does for its cosine.
          if (ct > (R)1) ct = (R)1;
          if (ct < (R)-1) ct = (R)-1;
          R theta = std::acos(ct) * (R)s->R2D;
          R m[3];
          m[0] = -(ij[1] * kj[2] - ij[2] * kj[1]);
          m[1] = -(-ij[0] * kj[2] + ij[2] * kj[0]);
          m[2] = -(ij[0] * kj[1] - ij[1] * kj[0]);
          R rm = std::sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
          for (int c = 0; c < 3; ++c) m[c] = m[c] / rm;
          R nn[3], ss[3];
          nn[0] = (m[1] * ij[2] - m[2] * ij[1]) / rij;
          nn[1] = (-m[0] * ij[2] + m[2] * ij[0]) / rij;
          nn[2] = (m[0] * ij[1] - m[1] * ij[0]) / rij;
          ss[0] = -(m[1] * kj[2] - m[2] * kj[1]) / rkj;
          ss[1] = -(-m[0] * kj[2] + m[2] * kj[0]) / rkj;
          ss[2] = -(m[0] * kj[1] - m[1] * kj[0]) / rkj;
          int k = fint(theta / bend.bin[TIJK]);
          // NaN or beyond the table (ANGLES.inc:43-49 reads row NI alone at 180 deg)
          if (k < 0 || k >= bend.w || (k + 1 >= bend.w && theta != (R)180.0)) { ++tor_err; continue; }
          R fijk, vijk;
          if (theta == (R)180.0) {
            fijk = bend.Fo(TIJK, k); vijk = bend.P(TIJK, k);
          } else {
            R alpha = (theta - bend.X(TIJK, k)) / bend.bin[TIJK];
            fijk = (R)((D)bend.Fo(TIJK, k) * (1.0 - (D)alpha) + (D)(alpha * bend.Fo(TIJK, k + 1)));
            vijk = (R)((D)bend.P(TIJK, k) * (1.0 - (D)alpha) + (D)(alpha * bend.P(TIJK, k + 1)));
          }
          vang[s->ANGLE_TYPE_LABEL[TIJK] - 1] += (double)vijk;
          R fijk3[3];
          for (int c = 0; c < 3; ++c) fijk3[c] = fijk * nn[c] / rij;
          for (int c = 0; c < 3; ++c) fi[c] = fi[c] + fijk3[c];
          for (int c = 0; c < 3; ++c) fl(K, c) = fl(K, c) + fijk * ss[c] / rkj;
          for (int c = 0; c < 3; ++c) fl(J, c) = fl(J, c) - fijk * ss[c] / rkj - fijk3[c];
        }
        // TORSIONS.inc:1-152
        R cosm = 0, sinm = 0, cotanm = 0, cosn = 0, sinn = 0, cotann = 0;
        for (int A = 1; A <= s->NIJKL[I]; ++A) {
          int J = s->jtor(I, A), K = s->ktor(I, A), L = s->ltor(I, A);
          int TIJKL = s->ITORT[s->t4(TI, s->ITYPE[J], s->ITYPE[K], s->ITYPE[L])];
          R ij[3], jk[3], kl[3];
          for (int c = 0; c < 3; ++c) ij[c] = ri[c] - sx(J, c);
          for (int c = 0; c < 3; ++c) jk[c] = sx(J, c) - sx(K, c);
          for (int c = 0; c < 3; ++c) kl[c] = sx(K, c) - sx(L, c);
          R rij = std::sqrt((ij[0] * ij[0] + ij[1] * ij[1]) + ij[2] * ij[2]);
          R rjk = std::sqrt((jk[0] * jk[0] + jk[1] * jk[1]) + jk[2] * jk[2]);
          R rkl = std::sqrt((kl[0] * kl[0] + kl[1] * kl[1]) + kl[2] * kl[2]);
          R m[3], nn[3];
          auto cross_m = [&]() {
            m[0] = ij[1] * jk[2] - ij[2] * jk[1];
            m[1] = -ij[0] * jk[2] + ij[2] * jk[0];
            m[2] = ij[0] * jk[1] - ij[1] * jk[0];
          };
          auto cross_n = [&]() {
            nn[0] = jk[1] * kl[2] - jk[2] * kl[1];
            nn[1] = -jk[0] * kl[2] + jk[2] * kl[0];
            nn[2] = jk[0] * kl[1] - jk[1] * kl[0];
          };
          cross_m();
          R rm = std::sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
          if (rm > (R)0) {
            for (int c = 0; c < 3; ++c) m[c] = m[c] / rm;
            cosm = ((ij[0] * jk[0] + ij[1] * jk[1]) + ij[2] * jk[2]) / rij / rjk;
            sinm = std::sqrt((R)1 - cosm * cosm);
            cotanm = cosm / sinm;
          } else if (rm == (R)0) {
            ij[0] = ri[0] * (R)0.99f - sx(J, 0);
            rij = std::sqrt((ij[0] * ij[0] + ij[1] * ij[1]) + ij[2] * ij[2]);
            cross_m();
            rm = std::sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
            for (int c = 0; c < 3; ++c) m[c] = m[c] / rm;
            cosm = ((ij[0] * jk[0] + ij[1] * jk[1]) + ij[2] * jk[2]) / rij / rjk;
            sinm = std::sqrt((R)1 - cosm * cosm);
            cotanm = cosm / sinm;
          }
          cross_n();
          R rn = std::sqrt((nn[0] * nn[0] + nn[1] * nn[1]) + nn[2] * nn[2]);
          if (rn > (R)0) {
            for (int c = 0; c < 3; ++c) nn[c] = nn[c] / rn;
            cosn = ((jk[0] * kl[0] + jk[1] * kl[1]) + jk[2] * kl[2]) / rjk / rkl;
            sinn = std::sqrt((R)1 - cosn * cosn);
            cotann = cosn / sinn;
          } else if (rn == (R)0) {
            kl[0] = sx(K, 0) - sx(L, 0) * (R)0.99f;
            rkl = std::sqrt((kl[0] * kl[0] + kl[1] * kl[1]) + kl[2] * kl[2]);
            cross_n();
            rn = std::sqrt((nn[0] * nn[0] + nn[1] * nn[1]) + nn[2] * nn[2]);
            for (int c = 0; c < 3; ++c) nn[c] = nn[c] / rn;
            cosn = ((jk[0] * kl[0] + jk[1] * kl[1]) + jk[2] * kl[2]) / rjk / rkl;
            sinn = std::sqrt((R)1 - cosn * cosn);
            cotann = cosn / sinn;
          }
          R cost = (m[0] * nn[0] + m[1] * nn[1]) + m[2] * nn[2];
          R signt = -((m[0] * kl[0] + m[1] * kl[1]) + m[2] * kl[2]);
          if (cost > (R)1.0) cost = 1.0;
          else if (cost < (R)-1.0) cost = -1.0;
          R phi = std::acos(cost) * (R)s->R2D;
          if (signt < (R)0) phi = (R)360.0 - phi;
          int k = fint(phi / tors.bin[TIJKL]);
          if (k > tors.ndat[TIJKL] || k < 0) { ++tor_err; continue; }
          R fijkl, vijkl;
          if (phi == (R)360.0) {
            fijkl = tors.Fo(TIJKL, k); vijkl = tors.P(TIJKL, k);
          } else {
            R alpha = (phi - tors.X(TIJKL, k)) / tors.bin[TIJKL];
            fijkl = tors.Fo(TIJKL, k) * ((R)1.0 - alpha) + alpha * tors.Fo(TIJKL, k + 1);
            vijkl = tors.P(TIJKL, k) * ((R)1.0 - alpha) + alpha * tors.P(TIJKL, k + 1);
          }
          vtor[s->TORSION_TYPE_LABEL[TIJKL] - 1] += (double)vijkl;
          R f1[3], f4[3], f12[3];
          for (int c = 0; c < 3; ++c) f1[c] = -(fijkl * m[c] / sinm / rij);
          for (int c = 0; c < 3; ++c) fi[c] = fi[c] + f1[c];
          for (int c = 0; c < 3; ++c) f4[c] = fijkl * nn[c] / sinn / rkl;
          for (int c = 0; c < 3; ++c) fl(L, c) = fl(L, c) + f4[c];
          for (int c = 0; c < 3; ++c) f12[c] = fijkl * (cotanm * m[c] + cotann * nn[c]) / rjk;
          for (int c = 0; c < 3; ++c) fl(J, c) = fl(J, c) - f1[c] + f12[c];
          for (int c = 0; c < 3; ++c) fl(K, c) = fl(K, c) - f4[c] - f12[c];
        }
        // OUTOFPLANES.inc:1-141
        for (int A = 1; A <= s->NOOPIJKL[I]; ++A) {
          int J = s->joop(I, A), K = s->koop(I, A), L = s->loop(I, A);
          int TO = s->IOOPT[s->t4(TI, s->ITYPE[J], s->ITYPE[K], s->ITYPE[L])];
          R ij[3], jk[3], kl[3];
          for (int c = 0; c < 3; ++c) ij[c] = ri[c] - sx(J, c);
          for (int c = 0; c < 3; ++c) jk[c] = sx(K, c) - sx(J, c);
          for (int c = 0; c < 3; ++c) kl[c] = sx(K, c) - sx(L, c);
          R rij = std::sqrt((ij[0] * ij[0] + ij[1] * ij[1]) + ij[2] * ij[2]);
          R rjk = std::sqrt((jk[0] * jk[0] + jk[1] * jk[1]) + jk[2] * jk[2]);
          R rkl = std::sqrt((kl[0] * kl[0] + kl[1] * kl[1]) + kl[2] * kl[2]);
          R m[3], nn[3], mn[3];
          m[0] = ij[1] * jk[2] - ij[2] * jk[1];
          m[1] = -ij[0] * jk[2] + ij[2] * jk[0];
          m[2] = ij[0] * jk[1] - ij[1] * jk[0];
          R rm = std::sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
          for (int c = 0; c < 3; ++c) m[c] = m[c] / rm;
          R cm = ((ij[0] * jk[0] + ij[1] * jk[1]) + ij[2] * jk[2]) / rij / rjk;
          R sm = std::sqrt((R)1 - cm * cm);
          R ctm = cm / sm;
          nn[0] = jk[1] * kl[2] - jk[2] * kl[1];
          nn[1] = -jk[0] * kl[2] + jk[2] * kl[0];
          nn[2] = jk[0] * kl[1] - jk[1] * kl[0];
          R rn = std::sqrt((nn[0] * nn[0] + nn[1] * nn[1]) + nn[2] * nn[2]);
          for (int c = 0; c < 3; ++c) nn[c] = nn[c] / rn;
          R cn = ((jk[0] * kl[0] + jk[1] * kl[1]) + jk[2] * kl[2]) / rjk / rkl;
          R sn = std::sqrt((R)1 - cn * cn);
          R ctn = cn / sn;
          R cost = (m[0] * nn[0] + m[1] * nn[1]) + m[2] * nn[2];
          mn[0] = m[1] * nn[2] - m[2] * nn[1];
          mn[1] = -m[0] * nn[2] + m[2] * nn[0];
          mn[2] = m[0] * nn[1] - m[1] * nn[0];
          R sgn = std::copysign((R)1.0, (mn[0] * jk[0] + mn[1] * jk[1]) + mn[2] * jk[2]);
          if (cost > (R)1.0 + eps || cost < -((R)1.0 + eps)) { ++oop_err; continue; }
          if (cost > (R)1.0) cost = 1.0;
          else if (cost < (R)-1.0) cost = -1.0;
          R phi = std::acos(cost);
          phi = sgn * phi;
          phi = phi * (R)s->R2D;
          R phit = (R)180.0 + phi;
          int k = fint(anint(phit / oop.bin[TO]));
          if (k < 0 || k > oop.ndat[TO]) { ++oop_err; continue; }
          R alpha = std::fabs(std::fabs(phi) - std::fabs(oop.X(TO, k))) / oop.bin[TO];
          if (alpha > (R)1.0) {
            k = k + 1;
            alpha = std::fabs(std::fabs(phi) - std::fabs(oop.X(TO, k))) / oop.bin[TO];
          }
          R fijkl = oop.Fo(TO, k) * ((R)1.0 - alpha) + alpha * oop.Fo(TO, k + 1);
          R vijkl = oop.P(TO, k) * ((R)1.0 - alpha) + alpha * oop.P(TO, k + 1);
          voop[s->OOP_TYPE_LABEL[TO] - 1] += (double)vijkl;
          R f1[3], f4[3], f12[3];
          for (int c = 0; c < 3; ++c) f1[c] = fijkl * m[c] / sm / rij;
          for (int c = 0; c < 3; ++c) fi[c] = fi[c] + f1[c];
          for (int c = 0; c < 3; ++c) f4[c] = -(fijkl * nn[c] / sn / rkl);
          for (int c = 0; c < 3; ++c) fl(L, c) = fl(L, c) + f4[c];
          for (int c = 0; c < 3; ++c) f12[c] = fijkl * (ctm * m[c] + ctn * nn[c]) / rjk;
          for (int c = 0; c < 3; ++c) fl(J, c) = fl(J, c) - f1[c] + f12[c];
          for (int c = 0; c < 3; ++c) fl(K, c) = fl(K, c) - f4[c] - f12[c];
        }
        for (int c = 0; c < 3; ++c) fl(I, c) = fl(I, c) + fi[c];
      }
    }
    for (int t = 0; t < T; ++t) {
      const std::vector<R>& FL = fpriv[t];
      for (size_t k = 0; k < F.size(); ++k) F[k] = F[k] + ((R)0 + FL[k]);
      for (int c = 0; c < 3; ++c) {
        V_BOND[c] += vb[(size_t)12 * t + c];
        V_ANGLE[c] += vb[(size_t)12 * t + 3 + c];
        V_TORSION[c] += vb[(size_t)12 * t + 6 + c];
        V_OOP[c] += vb[(size_t)12 * t + 9 + c];
      }
    }
    bond_overext += overext;
    if (tor_err) fail(ORC_E_TORSION_TABLE, "Entry in torsion table does not exist");
    if (oop_err) fail(ORC_E_OOP_RANGE, "out of plane angle outside its table");
  }

  // ------------------------------------------------ DISTRIBUTE_VSFORCE.f90:27-37
  void distribute_vsforce() {
    for (int i = 1; i <= s->NVIRTA; ++i) {
      int ti = s->VITYPE[i], vs = NA_ + i;
      for (int a = 1; a <= s->VIRT_NUMATOMS[ti]; ++a) {
        int j = s->vatm(i, a);
        R cf = (R)s->coeff(ti, s->ITYPE[j]);
        for (int c = 0; c < 3; ++c) fx(j, c) = fx(j, c) + fx(vs, c) * cf;
      }
      for (int c = 0; c < 3; ++c) fx(vs, c) = 0;
    }
  }

  void zero_force_stage() {
    std::fill(F.begin(), F.end(), (R)0);
    std::fill(FNB.begin(), FNB.end(), (R)0);
    PT11 = PT22 = PT33 = PT12 = PT13 = PT23 = 0;
    for (int c = 0; c < 3; ++c) V_NB[c] = V_BOND[c] = V_ANGLE[c] = V_TORSION[c] = V_OOP[c] = 0.0;
  }
  void bonded_virial() {  // NEW_FORCE.F90:73-80 / MTS_LOOP.f90:126-133
    for (int i = 1; i <= NA_; ++i) {
      R d0 = fx(i, 0) - FNB[3 * (size_t)(i - 1) + 0];
      R d1 = fx(i, 1) - FNB[3 * (size_t)(i - 1) + 1];
      R d2 = fx(i, 2) - FNB[3 * (size_t)(i - 1) + 2];
      PT11 = PT11 + d0 * sx(i, 0);
      PT22 = PT22 + d1 * sx(i, 1);
      PT33 = PT33 + d2 * sx(i, 2);
      PT12 = PT12 + d1 * sx(i, 0);
      PT13 = PT13 + d2 * sx(i, 0);
      PT23 = PT23 + d2 * sx(i, 1);
    }
  }
  void copy_fnb() {
    for (size_t k = 0; k < (size_t)3 * NA_; ++k) FNB[k] = F[k];
  }

  // ------------------------------------------------------ NEW_FORCE.F90:17-80
  void new_force() {
    zero_force_stage();
    nonbonded_force(s->ATOM, s->NUMATOMS, la, (R)s->RCUTSQ_ATOM);
    if (s->IBRDESCR == 0) {
      nonbonded_force(s->BEAD, s->NCOARSE, lb, (R)s->RCUTSQ_BEAD);
      distribute_vsforce();
    }
    copy_fnb();
    bonded_force();
    distribute_vsforce();
    bonded_virial();
  }

  // ------------------------------------------------------ MTS_LOOP.f90:71-224
  R& mts_f(int c, int m, int a) { return MTS_FXYZ[(size_t)c + 3 * ((size_t)(m - 1) + 3 * (size_t)(a - 1))]; }
  void mts_force(int step) {
    zero_force_stage();
    int m = step % (3 + s->NMTS);
    if (m >= 1 && m <= 3) {
      nonbonded_force(s->BEAD, s->NCOARSE, lb, (R)s->RCUTSQ_BEAD);
      for (int a = 1; a <= s->NCOARSE; ++a)
        for (int c = 0; c < 3; ++c) mts_f(c, m, a) = fx(s->BEAD[a], c);
      for (int c = 0; c < 3; ++c) MTS_V_NB[m - 1][c] = (R)V_NB[c];
      MTS_PT[0][m - 1] = PT11; MTS_PT[1][m - 1] = PT22; MTS_PT[2][m - 1] = PT33;
      MTS_PT[3][m - 1] = PT12; MTS_PT[4][m - 1] = PT13;  // PT23 is not saved (:193-199)
    } else {
      R coef = (R)(m - 3) * (R)0.5;
      for (int a = 1; a <= s->NCOARSE; ++a)
        for (int c = 0; c < 3; ++c) {
          R f3 = mts_f(c, 3, a), f1 = mts_f(c, 1, a);
          fx(s->BEAD[a], c) = f3 + coef * (f3 - f1);
        }
      for (int c = 0; c < 3; ++c) {
        R v3 = MTS_V_NB[2][c], v1 = MTS_V_NB[0][c];
        V_NB[c] = (double)(v3 + coef * (v3 - v1));
      }
      R* pts[6] = {&PT11, &PT22, &PT33, &PT12, &PT13, &PT23};
      for (int q = 0; q < 6; ++q) *pts[q] = MTS_PT[q][2] + coef * (MTS_PT[q][2] - MTS_PT[q][0]);
    }
    distribute_vsforce();
    nonbonded_force(s->ATOM, s->NUMATOMS, la, (R)s->RCUTSQ_ATOM);
    copy_fnb();
    bonded_force();
    distribute_vsforce();
    bonded_virial();
  }

  // ------------------------------------------------------------ MOVE.F90:9-118
  void move() {
    R k11[2] = {0, 0}, k22[2] = {0, 0}, k33[2] = {0, 0}, k12[2] = {0, 0}, k23[2] = {0, 0}, k13[2] = {0, 0};
    R lam[2];
    if (s->ENSEMBLE == 1 || s->ENSEMBLE == 2) {
      R tin = (R)s->TEMP_IN, fac = (R)s->FAC;
      lam[0] = std::sqrt((R)1.0 + fac * ((tin / TEMP_ATOM) - (R)1.0));
      lam[1] = std::sqrt((R)1.0 + fac * ((tin / TEMP_BEAD) - (R)1.0));
    } else {
      lam[0] = lam[1] = 1.0;
    }
    R dt = (R)s->DT;
    auto one = [&](int i, int cls) {
      int ti = s->ITYPE[i];
      R m = (R)s->MASS[ti], invm = (R)s->INVMASS[ti];
      R vo[3] = {vx(i, 0), vx(i, 1), vx(i, 2)};
      for (int c = 0; c < 3; ++c) vx(i, c) = (vo[c] + dt * fx(i, c) * invm) * lam[cls];
      for (int c = 0; c < 3; ++c) sx(i, c) = sx(i, c) + dt * vx(i, c);
      R vt[3];
      for (int c = 0; c < 3; ++c) { vt[c] = (R)0.5 * (vx(i, c) + vo[c]); VT[3 * (size_t)(i - 1) + c] = vt[c]; }
      k11[cls] = k11[cls] + m * vt[0] * vt[0];
      k22[cls] = k22[cls] + m * vt[1] * vt[1];
      k33[cls] = k33[cls] + m * vt[2] * vt[2];
      k12[cls] = k12[cls] + m * vt[0] * vt[1];
      k13[cls] = k13[cls] + m * vt[0] * vt[2];
      k23[cls] = k23[cls] + m * vt[1] * vt[2];
    };
    for (int a = 1; a <= s->NUMATOMS; ++a) one(s->ATOM[a], 0);
    for (int a = 1; a <= s->NUMBEADS; ++a) one(s->BEAD[a], 1);
    PT11 = PT11 + (k11[0] + k11[1]);
    PT22 = PT22 + (k22[0] + k22[1]);
    PT33 = PT33 + (k33[0] + k33[1]);
    PT12 = PT12 + (k12[0] + k12[1]);
    PT13 = PT13 + (k13[0] + k13[1]);
    PT23 = PT23 + (k23[0] + k23[1]);
    EK[0] = (double)((R)0.5 * (k11[0] + k22[0] + k33[0]));
    EK[1] = (double)((R)0.5 * (k11[1] + k22[1] + k33[1]));
    TEMP = (R)((EK[0] + EK[1]) * (double)(R)s->MKTEMP);
    TEMP_ATOM = (R)(EK[0] * (double)(R)s->MKTEMP_ATOM);
    TEMP_BEAD = (R)(EK[1] * (double)(R)s->MKTEMP_BEAD);
    R vol = BOX[0] * BOX[1] * BOX[2];
    R inv = (R)1.0 / vol;
    PT11 = PT11 * inv; PT22 = PT22 * inv; PT33 = PT33 * inv;
    PT12 = PT12 * inv; PT13 = PT13 * inv; PT23 = PT23 * inv;
  }

  // -------------------------------------------------------- MOMENTUM.f90:14-29
  void momentum() {
    R sum[3] = {0, 0, 0};
    for (int i = 1; i <= NA_; ++i) {
      R m = (R)s->MASS[s->ITYPE[i]];
      for (int c = 0; c < 3; ++c) sum[c] = sum[c] + vx(i, c) * m;
    }
    for (int c = 0; c < 3; ++c) sum[c] = sum[c] / (R)NA_;
    for (int i = 1; i <= NA_; ++i) {
      R invm = (R)s->INVMASS[s->ITYPE[i]];
      for (int c = 0; c < 3; ++c) vx(i, c) = vx(i, c) - sum[c] * invm;
    }
  }

  // --------------------------------------------------------- SCALEBP.f90:18-41
  void scalebp(int tm) {
    IAVP = IAVP + 1;
    if (IAVP > 10) IAVP -= 10;
    SP[IAVP - 1] = (R)((double)(PT11 + PT22 + PT33) / 3.0);
    if (tm % 10 == 0) {
      R avp = 0;
      for (int i = 0; i < 10; ++i) avp = avp + SP[i];
      R p = avp / (R)10;
      R base = (R)1.0 + (p - (R)s->PRESSURE) * (R)s->PFAC;
      R miu = std::pow(base, (R)1.0 / (R)3.0);
      for (int c = 0; c < 3; ++c) {
        BOX[c] = BOX[c] * miu;
        BOXINV[c] = (R)1.0 / BOX[c];
        BOX2[c] = BOX[c] / (R)2.0;
      }
      for (int i = 1; i <= NA_; ++i)
        for (int c = 0; c < 3; ++c) sx(i, c) = sx(i, c) * miu;
    }
  }

  // ---------------------------------------------------- main.F90:148-234 (init)
  void set_state(const float* sxyz, const float* vxyz, const float* box) {
    err = 0; errmsg.clear();
    for (size_t k = 0; k < (size_t)3 * NA_; ++k) { S[k] = (R)sxyz[k]; V[k] = (R)vxyz[k]; }
    for (int c = 0; c < 3; ++c) {
      BOX[c] = (R)box[c];
      BOXINV[c] = (R)1.0 / BOX[c];
      BOX2[c] = BOX[c] / (R)2.0;
    }
    TYPE_LABEL = s->TYPE_LABEL;
    IAVP = 0;
    cell_clamps = 0; bond_overext = 0;
    la.ncx = fint(BOX[0] / (R)s->RLIST_ATOM); la.ncy = fint(BOX[1] / (R)s->RLIST_ATOM); la.ncz = fint(BOX[2] / (R)s->RLIST_ATOM);
    if (s->IBRDESCR == 0) {
      lb.ncx = fint(BOX[0] / (R)s->RLIST_BEAD); lb.ncy = fint(BOX[1] / (R)s->RLIST_BEAD); lb.ncz = fint(BOX[2] / (R)s->RLIST_BEAD);
    }
    if (s->IBRDESCR == 0) virtual_def();
    shift();
    // main.F90:174-195
    EK[0] = EK[1] = 0.0;
    for (int a = 1; a <= s->NUMATOMS; ++a) {
      int i = s->ATOM[a];
      R m = (R)s->MASS[s->ITYPE[i]];
      EK[0] += (double)(m * ((vx(i, 0) * vx(i, 0) + vx(i, 1) * vx(i, 1)) + vx(i, 2) * vx(i, 2)));
    }
    for (int a = 1; a <= s->NUMBEADS; ++a) {
      int i = s->BEAD[a];
      R m = (R)s->MASS[s->ITYPE[i]];
      EK[1] += (double)(m * ((vx(i, 0) * vx(i, 0) + vx(i, 1) * vx(i, 1)) + vx(i, 2) * vx(i, 2)));
    }
    EK[0] = 0.5 * EK[0];
    EK[1] = 0.5 * EK[1];
    TEMP = (R)((EK[0] + EK[1]) * (double)(R)s->MKTEMP);
    TEMP_ATOM = (R)(EK[0] * (double)(R)s->MKTEMP_ATOM);
    TEMP_BEAD = (R)(EK[1] * (double)(R)s->MKTEMP_BEAD);
    if (!grid_ok(la)) return;
    maps(la);
    if (s->IBRDESCR == 0) {
      if (!grid_ok(lb)) return;
      maps(lb);
    }
    update_neighbourlist();
  }

  // one body of NEW_LOOP.F90:66-124 / MTS_LOOP.f90:24-44 without I/O
  void force_stage(int step) {
    shift();
    if (s->IBRDESCR == 0 || s->NMTS > 0) virtual_def();
    if (step % s->NUPDATE == 0) update_neighbourlist();
    if (err) return;
    if (s->NMTS == 0) new_force();
    else mts_force(step);
  }
  int step(int st) {
    force_stage(st);
    if (err) return err;
    move();
    if (st % s->HALT_DRIFT == 0) momentum();
    if (s->ENSEMBLE == 2) scalebp(st);
    return err;
  }
};

}  // namespace orc
