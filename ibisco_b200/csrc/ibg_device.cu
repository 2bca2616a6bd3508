// Device context of one Hybrid IBIsCO system and the C ABI of ibisco_gpu.h.
//
// Layout in HBM (per system):
//   S, V            FP64 (3,NATOMS[+NVIRTA]) unwrapped positions / velocities
//   su              unwrapped positions in the step precision (bonded terms)
//   fnb, fb         nonbonded / bonded forces, global order, 64-bit fixed
//                   point (FP32 path) or double (FP64 path)
//   per list (atom list, bead list):
//     pos4          wrapped positions in cell order, type|label in .w
//     fsort         nonbonded forces per slot (cell order), in blocks of 32 slots: x, y, z sums (fs_at)
//     cells         counting-sorted cell index (LINKS.f90 grid)
//     entries       Verlet list as slot indices, sliced-ELL: slice g of 32
//                   slots stores entry k of slot s at off[g] + 32 k + (s & 31)
//     tables        the nonbonded tables of the list's type pairs
//   bonded terms    flat (i,j[,k[,l]],table,label) arrays + float4 tables
//   Scalars         box, thermostat, MTS/barostat history, error bits
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "../../include/ibisco_gpu.h"
#include "ibg_common.cuh"
#include "ibg_kernels.cuh"

using namespace ibg;

namespace {

// Particles per SM from which a list is built with a thread per particle:
// 64 resident warps of 32 particles each, twice over.  Measured: the
// 2,000,000-bead melt builds in 1.97 ms a thread per particle against 3.0 ms a
// warp per particle; the 40,000-bead melt takes 225 us against 140 us.
constexpr long long kThreadBuildMin = 2LL * 64 * 32;

struct CudaError {
  cudaError_t e;
};

#define CK(x)                                 \
  do {                                        \
    cudaError_t e_ = (x);                     \
    if (e_ != cudaSuccess) throw CudaError{e_}; \
  } while (0)

// Device allocations of a context or batch, with their sizes (the device
// footprint that admission control accounts for).
struct Owned {
  std::vector<std::pair<void*, size_t>> a;
  size_t bytes = 0;
  void add(void* p, size_t n) { a.emplace_back(p, n); bytes += n; }
  void release(void* p) {
    for (size_t k = 0; k < a.size(); ++k)
      if (a[k].first == p) {
        bytes -= a[k].second;
        a.erase(a.begin() + (long)k);
        cudaFree(p);
        return;
      }
  }
  void free_all() {
    for (auto& x : a) cudaFree(x.first);
    a.clear();
    bytes = 0;
  }
};

template <typename T>
T* dalloc(size_t n, Owned& owned) {
  void* p = nullptr;
  if (n == 0) n = 1;
  CK(cudaMalloc(&p, n * sizeof(T)));
  CK(cudaMemset(p, 0, n * sizeof(T)));
  owned.add(p, n * sizeof(T));
  return (T*)p;
}
template <typename T>
T* dupload(const std::vector<T>& h, Owned& owned) {
  T* p = dalloc<T>(h.size(), owned);
  if (!h.empty()) CK(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return p;
}

enum Variant : unsigned {
  V_REBUILD = 1u,
  V_MOMENTUM = 2u,
  V_SCALE = 4u,
  V_FORCE_ONLY = 8u,
  V_MTS_APPROX = 16u,
};

struct DevList {
  int n = 0, which = 0, present = 0;
  int T = 1;  // lanes per particle in the list build and the nonbonded kernel (1, 2, 4 or 8)
  // list form: 0 = a list per particle, T lanes per particle (k_list_build_*,
  // k_nonbonded_f32 / k_nonbonded); 1 = a list per slice of four slots, each
  // neighbour once with a mask of its pairs (k_list_build_slices,
  // k_nonbonded_slices; FP32 path only)
  int form = 0;
  int cell_cap = 0, nslices = 0;
  int w_cap = 0;  // rows of 32 list entries per slice
  int *idx = nullptr, *cell_of = nullptr, *cell_count = nullptr, *cell_start = nullptr, *cell_fill = nullptr;
  int *sorted = nullptr, *sorted_new = nullptr, *slot_of = nullptr, *slot_of_new = nullptr;
  int *counts = nullptr, *slice_w = nullptr, *entries = nullptr;
  void *pos4 = nullptr, *pos4_new = nullptr, *fsort = nullptr, *mtsf = nullptr;
  int4 *posq = nullptr, *posq_new = nullptr;  // FP32 path: positions as box fractions
  int4* near = nullptr;                       // FP32 path: pairs at the cutoff (k_nb_near)
  int near_cap = 0;
  size_t pos_bytes = 0;
  // tables of this list
  int *ltab = nullptr, *toff = nullptr, *tndat = nullptr;
  int4* ptab = nullptr;  // per type pair: first row, NDAT, 1/bin bits, table present
  void *tbin = nullptr, *tinv = nullptr, *tfp = nullptr, *tx = nullptr;
  float4* tcoef = nullptr;  // FP32 path: per row {F - dF e, P - dP e, dF, dP} (NBArgs::tcoef)
  int ntab = 0, nrows = 0;
  size_t smem = 0;
  bool use_smem = false;
  float rlist = 0, rlistsq = 0, rcutsq = 0;
  float rgroupsq = 0;  // FP32 path: outer group of the stored lists (ListArgs::rgroupsq); 0: reference order
  bool mixed = true;   // the list holds particles of more than one label (k_nonbonded_f32's MIXED)
  int grid_nb = 0;
};

// Argument blocks of every kernel of one system.  The host copy is passed by
// value to single-system launches; a device copy serves batched launches,
// which read it through a table of per-system pointers.
template <typename R>
struct SysArgs {
  PosArgs pos;
  ListArgs list[2];
  NBArgs<R> nb[2];
  CollectArgs<R> col[2];
  DistArgs<R> dist;
  BondedArgs<R> bond;
  MoveArgs<R> move;
  MomArgs mom;
  FinalArgs fin;
};

}  // namespace

struct ibg_ctx {
  int prec = 0;
  int dev = 0, nsm = 148;
  cudaStream_t st = nullptr, st2 = nullptr;  // st2: bonded branch of a step
  cudaEvent_t fork_ev[2] = {nullptr, nullptr};
  Owned owned;
  std::string err;
  // descriptor scalars
  int natoms = 0, nvirta = 0, nitems = 0, ntype = 0, numatoms = 0, numbeads = 0, ncoarse = 0;
  int ensemble = 0, nupdate = 1, halt_drift = 1, nmts = 0, ibrdescr = 1, maxnab = 1000;
  float dt = 0, fac = 0, pfac = 0, temp_in = 0, pressure = 0, mktemp = 0, mktemp_atom = 0, mktemp_bead = 0;
  float r2d = 0;
  // device arrays
  double *S = nullptr, *V = nullptr, *mass = nullptr, *invmass = nullptr;
  float* xfer = nullptr;  // device staging of REAL*4 state for ibg_set_state / ibg_get_state (12 x NITEMS)
  void *su = nullptr, *fnb = nullptr, *fb = nullptr;
  int *tbits = nullptr, *gslot = nullptr, *excl_n = nullptr, *excl = nullptr;
  int *vcenter = nullptr, *vnum = nullptr, *vmem = nullptr;
  float *vmass = nullptr, *vinv = nullptr, *vcoef = nullptr;
  // bonded
  int nb = 0, na = 0, nt = 0, no = 0;
  int4 *bonds = nullptr, *angles = nullptr, *tors = nullptr, *oops = nullptr;
  int2 *tors_t = nullptr, *oops_t = nullptr;
  float4 *tb = nullptr, *ta = nullptr, *tt = nullptr, *to = nullptr;
  int *tb_off = nullptr, *ta_off = nullptr, *tt_off = nullptr, *to_off = nullptr;
  int *tb_nd = nullptr, *ta_nd = nullptr, *tt_nd = nullptr, *to_nd = nullptr;
  float *tb_bin = nullptr, *ta_bin = nullptr, *tt_bin = nullptr, *to_bin = nullptr;
  DevList L[2];
  Scalars* sc = nullptr;
  Scalars* hsc = nullptr;    // pinned host copy of *sc, read back once per run
  SysArgs<float> af;
  SysArgs<double> ad;
  void* dargs = nullptr;  // device copy of af or ad
  int g_list[2] = {1, 1}, g_regrid[2] = {1, 1}, g_build[2] = {1, 1}, g_dist = 1;
  int nb_blocks_per_sm = 0;  // tuning: resident nonbonded blocks per SM (0: all that fit)
  int nb_chunk = 0;          // tuning (FP32): 256ths of the units taken dynamically after the block ranges (0: all, per warp)
  int nb_rows = 16;          // tuning: list rows per nonbonded work unit (8 or 16)
  int nb_window = 0;         // tuning (FP32, nb_chunk > 0): units per run dealt to the blocks in turn (0: one range per block)
  int vs_com_form = IBG_VS_COM_FIXED;  // centre-of-mass virtual sites: fixed or the reference's form
  int list_form = IBG_LIST_AUTO;       // FP32 path: list form of new lists (DevList::form, list_form_of)
  void* vchain = nullptr;              // the reference form's per-site terms (k_vsite_chain)
  ObsD* ring = nullptr;
  int ring_cap = 0;
  double *p_b = nullptr, *p_mv = nullptr, *p_mom = nullptr;
  int g_b = 0, g_mv = 0, g_pos = 0;
  bool fb_dirty = false;
  bool state_set = false;
  int step_now = 0;  // last completed step (host mirror of the device counter)
  bool in_batch = false;
  std::map<unsigned, cudaGraphExec_t> graphs;
  std::vector<cudaGraph_t> graph_defs;
  long long launches_per_variant[32] = {0};
  // timing: stage events (timing mode, direct launches) and whole-run events
  bool timing = false;
  // programmatic dependent launches in the step (off while the autotuner
  // times single launches between memsets and events)
  bool pdl = true;
  double stage_ms[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  std::vector<std::pair<cudaEvent_t, int>> marks;  // event, stage that starts there
  cudaEvent_t run_ev[2] = {nullptr, nullptr};
  long long launches = 0;
  long long list_growths = 0;
  // L2 flush between timed steps
  size_t flush_bytes = 0;
  void* flush_buf = nullptr;
  std::vector<cudaEvent_t> step_ev;
};

namespace {

int fail(ibg_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}

int status_from_bits(unsigned b) {
  if (!b) return IBG_OK;
  if (b & EB_CELL_GRID) return IBG_E_CELL_GRID;  // a bad grid also overflows the lists
  if (b & EB_LIST_OVERFLOW) return IBG_E_LIST_OVERFLOW;
  if (b & EB_TORSION) return IBG_E_TORSION_TABLE;
  if (b & EB_OOP) return IBG_E_OOP_RANGE;
  if (b & EB_FIXED) return IBG_E_FIXED_OVERFLOW;
  if (b & EB_CELL_GRID) return IBG_E_CELL_GRID;
  if (b & EB_TABLE_RANGE) return IBG_E_TABLE_RANGE;
  if (b & EB_MISSING_TABLE) return IBG_E_MISSING_TABLE;
  if (b & EB_CAPACITY) return IBG_E_CAPACITY;
  return IBG_E_INVALID;
}
const char* bits_message(unsigned b) {
  if (b & EB_CELL_GRID) return "fewer than 3 cells per dimension for the neighbour list";
  if (b & EB_LIST_OVERFLOW) return "LIST TOO SMALL: a particle reached MAXNAB neighbours";
  if (b & EB_TORSION) return "FATAL ERROR: Entry in torsion table does not exist";
  if (b & EB_OOP) return "out of plane angle outside its table";
  if (b & EB_FIXED) return "force outside the 64-bit fixed-point range";
  if (b & EB_CELL_GRID) return "fewer than 3 cells per dimension for the neighbour list";
  if (b & EB_TABLE_RANGE) return "distance or angle outside its table";
  if (b & EB_MISSING_TABLE) return "listed pair without a nonbonded table";
  if (b & EB_CAPACITY) return "device neighbour-list or cell storage exhausted";
  return "unknown device error";
}

size_t rsize(const ibg_ctx* c) { return c->prec == IBG_PREC_FP32_FIXED ? sizeof(float) : sizeof(double); }
size_t accsize(const ibg_ctx* c) { return c->prec == IBG_PREC_FP32_FIXED ? sizeof(unsigned long long) : sizeof(double); }
size_t possize(const ibg_ctx* c) { return c->prec == IBG_PREC_FP32_FIXED ? sizeof(float4) : sizeof(double4); }

// ----------------------------------------------------------- list setup
// The list form of a list of n particles.  Automatic choice on the FP32 path:
// slice lists where the per-particle form would use its thread build (lists
// filling the GPU at a thread per particle), per-particle lists below, where
// the warp build serves them.  Measured on the 2,000,000-bead melt, lists
// rebuilt every 10 steps: 1.656 ms a step with slice lists against 1.669 ms.
int list_form_of(const ibg_ctx* c, int n) {
  if (c->prec != IBG_PREC_FP32_FIXED || n >= (1 << 28)) return IBG_LIST_PER_PARTICLE;
  if (c->list_form == IBG_LIST_AUTO) return n >= kThreadBuildMin * c->nsm ? IBG_LIST_PER_SLICE : IBG_LIST_PER_PARTICLE;
  return c->list_form;
}

void build_list(ibg_ctx* c, const ibg_desc* d, int which) {
  DevList& L = c->L[which];
  L.which = which;
  std::vector<int> idx;
  if (which == 0) for (int a = 0; a < d->numatoms; ++a) idx.push_back(d->atom[a] - 1);
  else for (int a = 0; a < d->ncoarse; ++a) idx.push_back(d->bead[a] - 1);
  L.n = (int)idx.size();
  L.present = L.n > 0;
  if (!L.present) return;
  L.rlist = which == 0 ? d->rlist_atom : d->rlist_bead;
  L.rlistsq = L.rlist * L.rlist;  // RLISTSQ = RLIST*RLIST (NEW_NEIGHBOUR_WITHLIST.f90:26)
  L.rcutsq = which == 0 ? d->rcutsq_atom : d->rcutsq_bead;
  // FP32 path: pairs beyond rc + skin/4 at the rebuild are stored after the
  // rest of each list (the nonbonded kernel then skips most of their rows);
  // ibg_get_neighbour_list restores the reference's order
  if (c->prec == IBG_PREC_FP32_FIXED && L.rcutsq > 0.f && L.rlist * L.rlist > L.rcutsq) {
    const double rc = std::sqrt((double)L.rcutsq);
    const double rg = rc + 0.25 * ((double)L.rlist - rc);
    L.rgroupsq = (float)(rg * rg);
  }
  // lanes per particle: 8 (the list-build and nonbonded launches assume it).  The eight lanes of a particle take eight
  // consecutive entries of its list, whose neighbours lie close together in
  // slot order, so a warp's position gathers and force atomics touch fewer
  // L1 sectors than with one lane per particle, where the 32 lanes of a row
  // belong to 32 particles (the kernel is bound by L1 throughput).  Measured
  // per nonbonded launch on the 2,000,000-bead melt: 1,779 us with 1 lane,
  // 1,635 with 2, 1,505 with 4, 1,472 with 8, 1,465 with 16, 1,788 with 32;
  // on the 40,000-bead melt 72, 61, 59, 59, 62 and 59 us.
  L.T = 8;
  L.nslices = (L.n + 32 / L.T - 1) / (32 / L.T);
  L.form = list_form_of(c, L.n);
  // one label throughout (an atom list, or a CG list without virtual sites):
  // every pair adds to that label's energy term
  {
    auto lab = [&](int i) { return i < d->natoms ? d->type_label[i] : 3; };
    L.mixed = false;
    for (int i : idx) L.mixed = L.mixed || lab(i) != lab(idx[0]);
  }
  auto& o = c->owned;
  L.idx = dupload(idx, o);
  L.cell_of = dalloc<int>(L.n, o);
  L.sorted = dalloc<int>(L.n, o);
  L.sorted_new = dalloc<int>(L.n, o);
  std::vector<int> ident(L.n);
  for (int a = 0; a < L.n; ++a) ident[a] = a;
  L.slot_of = dupload(ident, o);
  CK(cudaMemcpy(L.sorted, ident.data(), sizeof(int) * L.n, cudaMemcpyHostToDevice));
  L.slot_of_new = dalloc<int>(L.n, o);
  L.counts = dalloc<int>(L.n, o);
  L.slice_w = dalloc<int>(L.nslices, o);
  L.pos_bytes = possize(c) * L.n;
  L.pos4 = dalloc<unsigned char>(L.pos_bytes, o);
  L.pos4_new = dalloc<unsigned char>(L.pos_bytes, o);
  if (c->prec == IBG_PREC_FP32_FIXED) {
    L.posq = dalloc<int4>(L.n, o);
    L.posq_new = dalloc<int4>(L.n, o);
    // about 16 pairs a step sit this close to the cutoff on 40,000 beads
    L.near_cap = std::max(4096, L.n / 32);
    L.near = dalloc<int4>(L.near_cap, o);
  }
  L.fsort = dalloc<unsigned char>(accsize(c) * fs_len(L.n), o);
  if (which == 1 && c->nmts > 0) L.mtsf = dalloc<unsigned char>(accsize(c) * 9 * L.n, o);
  L.cell_cap = 0;  // sized in ibg_set_state once the box is known
  // nonbonded tables of the type pairs present in this list
  std::set<int> types;
  for (int a = 0; a < L.n; ++a) types.insert(d->itype[idx[a]] - 1);
  const int NT = d->ntype;
  std::vector<int> ltab((size_t)NT * NT, -1);
  std::map<int, int> local;
  std::vector<int> order;
  for (int ti : types)
    for (int tj : types) {
      int g = d->inbondt[(size_t)ti + (size_t)NT * tj];
      if (g <= 0) continue;
      if (!local.count(g)) { local[g] = (int)order.size(); order.push_back(g); }
      ltab[(size_t)ti * NT + tj] = local[g];
    }
  L.ntab = (int)order.size();
  std::vector<int> toff(L.ntab + 1, 0), tnd(L.ntab, 0);
  std::vector<double> fp, xx, bin(L.ntab);
  for (int t = 0; t < L.ntab; ++t) {
    int g = order[t];  // 1-based table
    int nd = d->ndatnb[g - 1];
    tnd[t] = nd;
    bin[t] = d->binnb[g - 1];
    toff[t] = (int)xx.size();
    int rows = std::min(nd + 2, d->ld_nb);
    for (int k = 0; k < rows; ++k) {
      size_t at = (size_t)k + (size_t)d->ld_nb * (g - 1);
      fp.push_back(d->nbond_force[at]);
      fp.push_back(d->nbond_pot[at]);
      xx.push_back(d->rnbond[at]);
    }
    for (int k = rows; k < nd + 2; ++k) { fp.push_back(0); fp.push_back(0); xx.push_back(0); }
  }
  toff[L.ntab] = (int)xx.size();
  // at least two rows: the FP32 kernel reads a row pair even for a type pair
  // without a table (it then stops the step with an error)
  while (xx.size() < 2) { fp.push_back(0); fp.push_back(0); xx.push_back(0); }
  L.nrows = (int)xx.size();
  L.ltab = dupload(ltab, o);
  L.toff = dupload(toff, o);
  L.tndat = dupload(tnd, o);
  if (c->prec == IBG_PREC_FP32_FIXED) {
    std::vector<float> f1(fp.begin(), fp.end()), x1(xx.begin(), xx.end()), b1(bin.begin(), bin.end()), i1(bin.size());
    for (size_t k = 0; k < bin.size(); ++k) i1[k] = (float)(1.0 / (double)(float)bin[k]);
    L.tfp = dupload(f1, o); L.tx = dupload(x1, o); L.tbin = dupload(b1, o); L.tinv = dupload(i1, o);
    // interpolation coefficients of every row k of table t (local index n =
    // k - toff[t]): with u = r/bin - n, the kernel's alpha = (r - X_k)/bin
    // is u - e_k, e_k = X_k/bin - n, so F = F_k + (F_k+1 - F_k) alpha is
    // (F_k - dF e_k) + dF u, and the same for P; computed in FP64 from the
    // FP32 rows the kernel would otherwise read
    std::vector<float4> co(L.nrows, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int t = 0; t < L.ntab; ++t)
      for (int k = toff[t]; k < toff[t + 1]; ++k) {
        const bool last = k + 1 >= toff[t + 1];
        const double fk = f1[2 * (size_t)k], pk = f1[2 * (size_t)k + 1];
        const double df = last ? 0.0 : (double)f1[2 * (size_t)k + 2] - fk;
        const double dp = last ? 0.0 : (double)f1[2 * (size_t)k + 3] - pk;
        const double e = (double)x1[k] * (double)i1[t] - (double)(k - toff[t]);
        co[k] = make_float4((float)(fk - df * e), (float)(pk - dp * e), (float)df, (float)dp);
      }
    L.tcoef = dupload(co, o);
    std::vector<int4> pt((size_t)NT * NT);
    for (size_t k = 0; k < pt.size(); ++k) {
      const int t = ltab[k];
      float inv = t >= 0 ? i1[t] : 0.f;
      int ib;
      std::memcpy(&ib, &inv, sizeof(int));
      pt[k] = t >= 0 ? make_int4(toff[t], tnd[t], ib, 1) : make_int4(0, 0, 0, 0);
    }
    L.ptab = dupload(pt, o);
  } else {
    L.tfp = dupload(fp, o); L.tx = dupload(xx, o); L.tbin = dupload(bin, o);
  }
  const size_t rs = rsize(c);
  L.smem = c->prec == IBG_PREC_FP32_FIXED
               ? kNbAccBytes + sizeof(int4) * (size_t)NT * NT + sizeof(float4) * (size_t)L.nrows + 64
               : 9 * 256 * sizeof(double) + rs * 3 * (size_t)L.nrows + 2 * rs * L.ntab +
                     sizeof(int) * ((size_t)NT * NT + 2 * L.ntab + 1) + 64;
  // launch defaults (ibg_set_tuning / ibg_autotune change them): the FP32
  // kernel reads its tables through L1, the FP64 kernel stages them
  L.use_smem = c->prec != IBG_PREC_FP32_FIXED && L.smem <= 200 * 1024;
}

void alloc_cells(ibg_ctx* c, DevList& L, const float* box) {
  if (!L.present) return;
  long long ncap = 1;
  for (int k = 0; k < 3; ++k) ncap *= std::max(3, (int)std::ceil(box[k] * 1.25f / L.rlist) + 1);
  if (ncap <= L.cell_cap) return;
  auto& o = c->owned;
  L.cell_cap = (int)ncap;
  L.cell_count = dalloc<int>(ncap, o);
  L.cell_start = dalloc<int>(ncap + 1, o);
  L.cell_fill = dalloc<int>(ncap, o);
}

int grid_for(ibg_ctx* c, long long work, int per_sm = 8) {
  long long g = (work + 255) / 256;
  return (int)std::max<long long>(1, std::min<long long>(g, (long long)c->nsm * per_sm));
}

// ------------------------------------------------------------ step stages
// Stage marks (timing mode only): 0 list build, 1 nonbonded, 2 bonded,
// 3 integrate and reductions, 4 other; 7 ends a step.
void mark(ibg_ctx* c, int stage) {
  if (!c->timing) return;
  cudaEvent_t e;
  CK(cudaEventCreate(&e));
  CK(cudaEventRecord(e, c->st));
  c->marks.emplace_back(e, stage);
}

void collect_marks(ibg_ctx* c) {
  if (c->marks.empty()) return;
  CK(cudaStreamSynchronize(c->st));
  for (size_t k = 0; k + 1 < c->marks.size(); ++k) {
    int stg = c->marks[k].second;
    if (stg == 7) continue;
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->marks[k].first, c->marks[k + 1].first));
    c->stage_ms[stg] += ms;
  }
  for (auto& m : c->marks) cudaEventDestroy(m.first);
  c->marks.clear();
}

template <typename R>
SysArgs<R>& args(ibg_ctx* c);
template <>
SysArgs<float>& args<float>(ibg_ctx* c) { return c->af; }
template <>
SysArgs<double>& args<double>(ibg_ctx* c) { return c->ad; }

// Fill the argument blocks from the context's current arrays and sizes.
template <typename R>
void make_args(ibg_ctx* c) {
  using acc_t = typename Prec<R>::acc_t;
  SysArgs<R>& A = args<R>(c);
  std::memset(&A, 0, sizeof(A));
  Scalars* sc = c->sc;
  PosArgs& p = A.pos;
  p.sc = sc; p.natoms = c->natoms; p.nvirta = c->nvirta; p.nupdate = c->nupdate; p.nmts = c->nmts;
  p.S = c->S; p.Svs = c->S + 3 * (size_t)c->natoms; p.tbits = c->tbits; p.gslot = c->gslot;
  p.pos4[0] = c->L[0].pos4; p.pos4[1] = c->L[1].pos4;
  p.posq[0] = c->L[0].posq; p.posq[1] = c->L[1].posq;
  p.vcenter = c->vcenter; p.vnum = c->vnum; p.vmem = c->vmem; p.vmass = c->vmass; p.vinv = c->vinv;
  p.com_carry = c->vs_com_form == IBG_VS_COM_REFERENCE;
  p.chain = c->vchain;
  for (int w = 0; w < 2; ++w) {
    DevList& L = c->L[w];
    ListArgs& a = A.list[w];
    a.sc = sc;
    a.n = L.n; a.which = w; a.natoms = c->natoms; a.hybrid = c->ibrdescr == 0; a.maxnab = c->maxnab;
    a.cell_cap = L.cell_cap;
    a.nslices = L.nslices;
    a.rlist = L.rlist; a.rlistsq = L.rlistsq; a.rlistd = (double)L.rlist; a.rlistsqd = (double)L.rlist * (double)L.rlist;
    a.idx = L.idx; a.cell_of = L.cell_of; a.cell_count = L.cell_count; a.cell_start = L.cell_start;
    a.cell_fill = L.cell_fill;
    a.sorted = L.sorted; a.sorted_new = L.sorted_new; a.slot_of = L.slot_of; a.slot_of_new = L.slot_of_new;
    a.gslot = c->gslot; a.pos4 = L.pos4; a.pos4_new = L.pos4_new;
    a.posq = L.posq; a.posq_new = L.posq_new;
    a.counts = L.counts; a.slice_w = L.slice_w; a.entries = L.entries; a.w_cap = L.w_cap;
    a.rgroupsq = L.rgroupsq;
    a.excl_n = c->excl_n; a.excl = c->excl;
    NBArgs<R>& n = A.nb[w];
    n.sc = sc; n.mts = (w == 1 && c->nmts > 0);
    n.n = L.n; n.nslices = L.nslices; n.ntype = c->ntype;
    n.pos4 = L.pos4; n.posq = L.posq; n.counts = L.counts; n.slice_w = L.slice_w; n.entries = L.entries;
    n.w_cap = L.w_cap; n.work = w;
    n.fsort = (acc_t*)L.fsort;
    n.ltab = L.ltab; n.toff = L.toff; n.tndat = L.tndat; n.tbin = (const R*)L.tbin; n.tinv = (const R*)L.tinv;
    n.tfp = (const R*)L.tfp; n.tx = (const R*)L.tx; n.ptab = L.ptab; n.chunk = c->nb_chunk;
    n.tcoef = L.tcoef;
    n.rows = c->nb_rows;
    n.window = c->nb_window;
    n.ntab = L.ntab; n.nrows = L.nrows; n.rcutsq = (R)L.rcutsq;
    n.rcut_lo = L.rcutsq * (1.0f - 1e-6f);
    n.rcut_hi = L.rcutsq * (1.0f + 1e-6f);
    n.near = L.near; n.near_cap = L.near_cap;
    n.sorted = L.sorted; n.idx = L.idx; n.S = c->S; n.natoms = c->natoms;
    CollectArgs<R>& k = A.col[w];
    k.sc = sc; k.n = L.n; k.mts = (w == 1 && c->nmts > 0); k.sorted = L.sorted; k.idx = L.idx;
    k.fsort = (acc_t*)L.fsort; k.fnb = (acc_t*)c->fnb; k.mtsf = (acc_t*)L.mtsf;
  }
  DistArgs<R>& d = A.dist;
  d.sc = sc; d.F[0] = (acc_t*)c->fnb; d.F[1] = (acc_t*)c->fb; d.natoms = c->natoms; d.nvirta = c->nvirta;
  d.vnum = c->vnum; d.vmem = c->vmem; d.vcoef = c->vcoef;
  BondedArgs<R>& B = A.bond;
  B.sc = sc; B.su = c->S; B.fb = (acc_t*)c->fb;
  B.nb = c->nb; B.na = c->na; B.nt = c->nt; B.no = c->no;
  B.bonds = c->bonds; B.angles = c->angles; B.tors = c->tors; B.tors_t = c->tors_t; B.oops = c->oops; B.oops_t = c->oops_t;
  B.tb = c->tb; B.tb_off = c->tb_off; B.tb_ndat = c->tb_nd; B.tb_bin = c->tb_bin;
  B.ta = c->ta; B.ta_off = c->ta_off; B.ta_ndat = c->ta_nd; B.ta_bin = c->ta_bin;
  B.tt = c->tt; B.tt_off = c->tt_off; B.tt_ndat = c->tt_nd; B.tt_bin = c->tt_bin;
  B.to = c->to; B.to_off = c->to_off; B.to_ndat = c->to_nd; B.to_bin = c->to_bin;
  B.r2d = c->r2d; B.part = c->p_b; B.part_stride = c->g_b;
  MoveArgs<R>& M = A.move;
  M.sc = sc; M.natoms = c->natoms; M.S = c->S; M.V = c->V;
  M.fnb = (acc_t*)c->fnb; M.fb = (acc_t*)c->fb;
  M.tbits = c->tbits; M.mass = c->mass; M.invmass = c->invmass; M.dt = (double)c->dt; M.update = 1;
  M.part = c->p_mv; M.part_stride = c->g_mv;
  MomArgs& m = A.mom;
  m.sc = sc; m.natoms = c->natoms; m.halt_drift = c->halt_drift; m.V = c->V; m.mass = c->mass; m.invmass = c->invmass;
  m.part = c->p_mom; m.nblocks = c->g_mv;
  FinalArgs& F = A.fin;
  F.sc = sc; F.fixed = c->prec == IBG_PREC_FP32_FIXED;
  F.p_b = c->p_b; F.g_b = c->g_b; F.p_mv = c->p_mv; F.g_mv = c->g_mv;
  F.mts = c->nmts > 0; F.move = 1; F.ensemble = c->ensemble;
  F.temp_in = c->temp_in; F.fac = c->fac; F.pfac = c->pfac; F.pressure = c->pressure;
  F.mktemp = c->mktemp; F.mktemp_atom = c->mktemp_atom; F.mktemp_bead = c->mktemp_bead;
  F.ring = c->ring; F.ring_cap = c->ring_cap;
}

// Rebuild the argument blocks and their device copy (after any change of the
// context's arrays: creation, cell storage, list storage, observable ring).
void refresh_args(ibg_ctx* c) {
  size_t bytes;
  const void* src;
  if (c->prec == IBG_PREC_FP32_FIXED) { make_args<float>(c); bytes = sizeof(c->af); src = &c->af; }
  else { make_args<double>(c); bytes = sizeof(c->ad); src = &c->ad; }
  if (!c->dargs) c->dargs = dalloc<unsigned char>(bytes, c->owned);
  CK(cudaMemcpy(c->dargs, src, bytes, cudaMemcpyHostToDevice));
}

const BlockMap kOne{nullptr, nullptr};

// A launch on stream st, with programmatic stream serialization when pdl is
// set: the kernel may start while the kernel before it in the stream still
// runs, and waits for it in pdl_wait(), so that its launch overlaps the
// other's tail.  Kernels launched this way call pdl_wait() before anything
// else.
template <typename... KArgs, typename... Args>
void launch_on(cudaStream_t st, bool pdl, void (*k)(KArgs...), int grid, int block, size_t smem, const Args&... a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl ? 1 : 0;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, k, a...));
}

// The same on the context's stream.  Timing mode, which separates the stages
// with events, and the autotuner's trial launches are ordinary launches.
template <typename... KArgs, typename... Args>
void launch_pdl(ibg_ctx* c, void (*k)(KArgs...), int grid, int block, size_t smem, const Args&... a) {
  launch_on(c->st, c->pdl && !c->timing, k, grid, block, smem, a...);
  ++c->launches;
}

template <typename R>
void enq_positions(ibg_ctx* c, int begin = 0) {
  const PosArgs& a = args<R>(c).pos;
  k_positions<R, false><<<c->g_pos, 256, 0, c->st>>>(a, nullptr, kOne, begin);
  if (a.com_carry && c->nvirta > 0) {  // the reference's centre-of-mass sums
    k_vsite_chain<R, false><<<1, 256, 0, c->st>>>(a, nullptr, kOne);
    ++c->launches;
  }
  ++c->launches;
}

// always: rebuild whatever the step's flag says (ibg_set_state, growth).
template <typename R>
void enq_rebuild(ibg_ctx* c, DevList& L, int always) {
  if (!L.present) return;
  const ListArgs& a = args<R>(c).list[L.which];
  const int w = L.which, gn = c->g_list[w];
  // the first launch may follow a memset (ibg_set_state): an ordinary one;
  // the rest follow a kernel of the chain
  using LA = const ListArgs* const*;
  k_regrid<R, false><<<c->g_regrid[w], 256, 0, c->st>>>(a, nullptr, kOne, always);
  ++c->launches;
  launch_pdl(c, k_cell_assign<R, false>, gn, 256, 0, a, (LA)nullptr, kOne, always);
  launch_pdl(c, k_scan_cells<false>, 1, 1024, 0, a, (LA)nullptr, kOne, always);
  launch_pdl(c, k_cell_fill<false>, gn, 256, 0, a, (LA)nullptr, kOne, always);
  launch_pdl(c, k_cell_rank<false>, gn, 256, 0, a, (LA)nullptr, kOne, always);
  launch_pdl(c, k_reslot<R, false>, gn, 256, 0, a, (LA)nullptr, kOne, always);
  launch_pdl(c, k_slot_of<R, false>, gn, 256, 0, a, (LA)nullptr, kOne, always);
  const int gl = c->g_build[w];
  // a thread per particle once the list has enough particles to fill the GPU
  // that way (twice the resident warps), a warp per particle below that;
  // both give the same lists
  if (L.form == 1)
    launch_pdl(c, k_list_build_slices<false>, gl, 256, 0, a, (LA)nullptr, kOne, always);
  else if (L.n >= kThreadBuildMin * c->nsm)
    launch_pdl(c, k_list_build_thread<R, 8, false>, gl, 256, 0, a, (LA)nullptr, kOne, always);
  else
    launch_pdl(c, k_list_build_warp<R, 8, false>, gl, 256, 0, a, (LA)nullptr, kOne, always);
}

template <typename R, bool B>
using NBKernel = void (*)(const NBArgs<R>, const NBArgs<R>* const*, const BlockMap);

// The nonbonded kernel of a list: tables staged in shared memory or read
// through L1 (smem), on the FP32 path whether the list mixes labels, and the
// list form (DevList::form).  Per-particle lists are built for eight lanes
// per particle.
template <typename R, bool B>
NBKernel<R, B> nb_kernel(bool smem, bool mixed, int form);

template <bool B>
NBKernel<float, B> nb_kernel_f(bool smem, bool mixed, int form) {
  if (form == 1) {
    if (smem) return mixed ? k_nonbonded_slices<true, true, B> : k_nonbonded_slices<true, false, B>;
    return mixed ? k_nonbonded_slices<false, true, B> : k_nonbonded_slices<false, false, B>;
  }
  if (smem) return mixed ? k_nonbonded_f32<true, true, B> : k_nonbonded_f32<true, false, B>;
  return mixed ? k_nonbonded_f32<false, true, B> : k_nonbonded_f32<false, false, B>;
}
template <>
NBKernel<float, false> nb_kernel<float, false>(bool smem, bool mixed, int form) {
  return nb_kernel_f<false>(smem, mixed, form);
}
template <>
NBKernel<float, true> nb_kernel<float, true>(bool smem, bool mixed, int form) {
  return nb_kernel_f<true>(smem, mixed, form);
}
template <>
NBKernel<double, false> nb_kernel<double, false>(bool smem, bool, int) {
  return smem ? k_nonbonded<double, true, 8, false> : k_nonbonded<double, false, 8, false>;
}
template <>
NBKernel<double, true> nb_kernel<double, true>(bool smem, bool, int) {
  return smem ? k_nonbonded<double, true, 8, true> : k_nonbonded<double, false, 8, true>;
}

// Dynamic shared memory of a nonbonded launch over list L.
size_t nb_smem(const ibg_ctx* c, const DevList& L) {
  const size_t base = c->prec == IBG_PREC_FP32_FIXED ? (size_t)kNbAccBytes : 9 * 8 * sizeof(double);
  return L.use_smem ? L.smem : base;
}

// Blocks per SM the nonbonded kernel of list L reaches (after raising its
// dynamic shared-memory limit when needed).
template <typename R, bool B>
int nb_occupancy(const ibg_ctx* c, const DevList& L, size_t sm) {
  NBKernel<R, B> k = nb_kernel<R, B>(L.use_smem, L.mixed, L.form);
  if (sm > 48 * 1024) CK(cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int per = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k, 256, sm));
  per = std::max(1, per);
  // L1 and shared memory share each SM's 256 KB: ask for the smallest
  // shared-memory carveout that holds `per` blocks and leave the rest to L1,
  // which caches the position gathers and the table rows (the driver rounds
  // the request up to a configuration the SM supports)
  cudaFuncAttributes fa;
  CK(cudaFuncGetAttributes(&fa, (const void*)k));
  int dev = 0, maxsm = 0, resv = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  CK(cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
  const size_t need = (size_t)per * (sm + fa.sharedSizeBytes + (size_t)resv);
  const int pct = maxsm > 0 ? (int)std::min<size_t>(100, (need * 100 + (size_t)maxsm - 1) / (size_t)maxsm) : 100;
  CK(cudaFuncSetAttribute((const void*)k, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
  return per;
}

template <typename R>
void nb_configure(ibg_ctx* c, DevList& L) {
  int per = nb_occupancy<R, false>(c, L, nb_smem(c, L));
  nb_occupancy<R, true>(c, L, nb_smem(c, L));
  if (c->nb_blocks_per_sm > 0) per = std::min(per, c->nb_blocks_per_sm);
  const long long units = (long long)L.nslices * 4;
  L.grid_nb = (int)std::max<long long>(1, std::min<long long>((long long)c->nsm * per, (units + 7) / 8));
}

template <typename R>
void enq_nonbonded(ibg_ctx* c, DevList& L) {
  launch_pdl(c, nb_kernel<R, false>(L.use_smem, L.mixed, L.form), L.grid_nb, 256, nb_smem(c, L), args<R>(c).nb[L.which],
             (const NBArgs<R>* const*)nullptr, kOne);
  if (c->prec == IBG_PREC_FP32_FIXED)
    launch_pdl(c, k_nb_near<false>, 1, 256, 0, args<float>(c).nb[L.which], (const NBArgs<float>* const*)nullptr, kOne);
}

template <typename R>
void enq_collect(ibg_ctx* c, DevList& L) {
  launch_pdl(c, k_nb_collect<R, false>, c->g_list[L.which], 256, 0, args<R>(c).col[L.which],
             (const CollectArgs<R>* const*)nullptr, kOne);
}

template <typename R>
void enq_distribute(ibg_ctx* c, int which) {
  if (c->nvirta == 0) return;
  launch_pdl(c, k_distribute<R, false>, c->g_dist, 256, 0, args<R>(c).dist, (const DistArgs<R>* const*)nullptr, kOne,
             which);
}

template <typename R>
void enq_bonded(ibg_ctx* c) {
  k_bonded<R, false><<<c->g_b, 256, 0, c->st>>>(args<R>(c).bond, nullptr, kOne);
  ++c->launches;
}

template <typename R>
void enq_move(ibg_ctx* c, int update) {
  MoveArgs<R> M = args<R>(c).move;
  M.update = update;
  // an ordinary launch: it follows the join with the bonded branch
  k_move<R, false><<<c->g_mv, 256, 0, c->st>>>(M, nullptr, kOne);
  ++c->launches;
}

template <typename R>
void enq_finalize(ibg_ctx* c, int move) {
  FinalArgs F = args<R>(c).fin;
  F.move = move;
  launch_pdl(c, k_finalize<false>, 1, 1024, 0, F, (const FinalArgs* const*)nullptr, kOne);
}

// One loop body.  In graph mode the bonded branch (bonded terms and their VS
// distribution) runs concurrently with the list build and the nonbonded
// branch; both join before MOVE.  Timing mode keeps one stream so that the
// stage times add up.
template <typename R>
void enqueue_step(ibg_ctx* c, unsigned v) {
  const bool fork = !c->timing;
  const int always = 0;  // rebuild kernels follow the step's own flag
  mark(c, 4);
  enq_positions<R>(c, 1);
  auto bonded_branch = [&]() {
    mark(c, 2);
    enq_bonded<R>(c);
    mark(c, 4);
    enq_distribute<R>(c, 1);
  };
  cudaStream_t main_st = c->st;
  if (fork) {
    CK(cudaEventRecord(c->fork_ev[0], main_st));
    CK(cudaStreamWaitEvent(c->st2, c->fork_ev[0], 0));
    c->st = c->st2;
    bonded_branch();
    CK(cudaEventRecord(c->fork_ev[1], c->st2));
    c->st = main_st;
  }
  if (v & V_REBUILD) {
    mark(c, 0);
    enq_rebuild<R>(c, c->L[0], always);
    enq_rebuild<R>(c, c->L[1], always);
  }
  // nonbonded: MTS runs the bead list first (MTS_LOOP.f90:100-116); sums are
  // order independent, so one sequence serves both loops
  mark(c, 1);
  if (c->L[1].present && !(v & V_MTS_APPROX)) {
    enq_nonbonded<R>(c, c->L[1]);
    c->stage_ms[6] += c->timing;
    c->stage_ms[8] += c->timing;
  }
  if (c->L[0].present) { enq_nonbonded<R>(c, c->L[0]); c->stage_ms[6] += c->timing; }
  mark(c, 4);
  if (c->L[1].present) enq_collect<R>(c, c->L[1]);
  if (c->L[0].present) enq_collect<R>(c, c->L[0]);
  enq_distribute<R>(c, 0);
  if (fork) CK(cudaStreamWaitEvent(main_st, c->fork_ev[1], 0));
  else bonded_branch();
  mark(c, 3);
  if (v & V_FORCE_ONLY) {
    enq_move<R>(c, 0);
    enq_finalize<R>(c, 0);
    mark(c, 7);
    return;
  }
  enq_move<R>(c, 1);
  if (v & V_MOMENTUM) {
    k_mom_sum<false><<<c->g_mv, 256, 0, c->st>>>(args<R>(c).mom, nullptr, kOne);
    k_mom_apply<false><<<c->g_mv, 256, 0, c->st>>>(args<R>(c).mom, nullptr, kOne);
    c->launches += 2;
  }
  enq_finalize<R>(c, 1);
  if (v & V_SCALE) {
    k_scale_positions<R, false><<<c->g_mv, 256, 0, c->st>>>(args<R>(c).move, nullptr, kOne);
    ++c->launches;
  }
  mark(c, 7);
}

unsigned variant_of(const ibg_ctx* c, int step, bool force_only) {
  unsigned v = 0;
  if (step % c->nupdate == 0) v |= V_REBUILD;
  if (c->nmts > 0) {
    int m = step % (3 + c->nmts);
    if (!(m >= 1 && m <= 3)) v |= V_MTS_APPROX;
  }
  if (force_only) return v | V_FORCE_ONLY;
  if (step % c->halt_drift == 0) v |= V_MOMENTUM;
  if (c->ensemble == 2 && step % 10 == 0) v |= V_SCALE;
  return v;
}

void enqueue(ibg_ctx* c, unsigned v) {
  if (c->prec == IBG_PREC_FP32_FIXED) enqueue_step<float>(c, v);
  else enqueue_step<double>(c, v);
}

// The system runs steps step_before+1 .. last; observables of step k go to
// ring slot k - base.
// Step counter, ring base and step limit for the next run, in stream order
// on the context's stream (sync: also wait for it, for launches on another
// stream).
void set_step_counter(ibg_ctx* c, int step_before, int base, int last, bool sync) {
  k_set_counter<<<1, 1, 0, c->st>>>(c->sc, step_before, base, last);
  CK(cudaGetLastError());
  ++c->launches;
  if (sync) CK(cudaStreamSynchronize(c->st));
}

int check_bits(ibg_ctx* c, unsigned bits);

int check_device(ibg_ctx* c) {
  unsigned bits = 0;
  CK(cudaMemcpyAsync(&bits, &c->sc->err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return check_bits(c, bits);
}

// Error bits read from the device: clear them there and report.
int check_bits(ibg_ctx* c, unsigned bits) {
  if (bits) {
    unsigned zero = 0;
    CK(cudaMemcpy(&c->sc->err, &zero, sizeof(unsigned), cudaMemcpyHostToDevice));
    return fail(c, status_from_bits(bits), bits_message(bits));
  }
  return IBG_OK;
}

void obs_to_c(const ObsD& o, ibg_obs* out) {
  std::memcpy(out->ek, o.ek, sizeof(double) * 2);
  out->temp = o.temp; out->temp_atom = o.temp_atom; out->temp_bead = o.temp_bead;
  std::memcpy(out->v_nb, o.v_nb, sizeof(double) * 3);
  std::memcpy(out->v_bond, o.v_bond, sizeof(double) * 3);
  std::memcpy(out->v_angle, o.v_angle, sizeof(double) * 3);
  std::memcpy(out->v_torsion, o.v_torsion, sizeof(double) * 3);
  std::memcpy(out->v_oop, o.v_oop, sizeof(double) * 3);
  std::memcpy(out->pt, o.pt, sizeof(double) * 6);
  std::memcpy(out->box, o.box, sizeof(double) * 3);
  out->bond_overext = o.bond_overext;
  out->cell_clamps = o.cell_clamps;
  out->step = o.step;
  out->status = o.status;
}

int read_obs(ibg_ctx* c, ibg_obs* out) {
  if (!out) return IBG_OK;
  ObsD o;
  CK(cudaMemcpyAsync(&o, &c->sc->obs, sizeof(ObsD), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  obs_to_c(o, out);
  return IBG_OK;
}

// A list build that outgrew its slices raised the abort flag (the remaining
// kernels of the run did nothing).  Enlarge the slices to the recorded need
// plus 25 %, clear the flag and return 1 so the caller repeats from the step
// that aborted.
int grow_lists(ibg_ctx* c) {
  int abort_flag = 0;
  int need[2] = {0, 0};
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(&abort_flag, &c->sc->abort, sizeof(int), cudaMemcpyDeviceToHost));
  if (!abort_flag) return 0;
  int need_near[2] = {0, 0};
  CK(cudaMemcpy(need, c->sc->need_rows, sizeof(need), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(need_near, c->sc->need_near, sizeof(need_near), cudaMemcpyDeviceToHost));
  for (int w = 0; w < 2; ++w) {
    DevList& L = c->L[w];
    if (!L.present) continue;
    if (need[w] > L.w_cap) {
      const int cap = need[w] + need[w] / 4 + 2;
      if (L.entries) c->owned.release(L.entries);
      L.entries = dalloc<int>((size_t)L.nslices * 32 * cap, c->owned);
      L.w_cap = cap;
      ++c->list_growths;
    }
    if (need_near[w] > L.near_cap) {  // pairs at the cutoff (FP32 path)
      const int cap = need_near[w] + need_near[w] / 4 + 64;
      if (L.near) c->owned.release(L.near);
      L.near = dalloc<int4>(cap, c->owned);
      L.near_cap = cap;
    }
  }
  const int zero[3] = {0, 0, 0};
  CK(cudaMemcpy(&c->sc->abort, zero, sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(&c->sc->skip, zero, sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->sc->need_rows, zero, 2 * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->sc->need_near, zero, 2 * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->sc->near_n, zero, 2 * sizeof(unsigned), cudaMemcpyHostToDevice));
  // the bonded branch of the aborted step may have run (it overlaps the list
  // build), and so may its nonbonded kernels (a step aborted for the pairs at
  // the cutoff): their sums are recomputed when the step is repeated
  CK(cudaMemset(c->fb, 0, accsize(c) * 3 * (size_t)c->nitems));
  for (auto& L : c->L)
    if (L.present) CK(cudaMemset(L.fsort, 0, accsize(c) * fs_len(L.n)));
  CK(cudaMemset(c->sc->nbacc, 0, sizeof(c->sc->nbacc)));
  refresh_args(c);
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);  // they bake the old pointers
  c->graphs.clear();
  return 1;
}

template <typename R>
void rebuild_now(ibg_ctx* c) {
  CK(cudaMemsetAsync(c->sc->work, 0, sizeof(c->sc->work), c->st));
  for (auto& L : c->L) {
    if (!L.present) continue;
    enq_rebuild<R>(c, L, 1);
  }
}

}  // namespace

// ======================================================================= C ABI
extern "C" {

const char* ibg_version(void) { return "ibisco_b200 0.1 (sm_100a)"; }

int ibg_set_device(int device) { return cudaSetDevice(device) == cudaSuccess ? IBG_OK : IBG_E_CUDA; }

int ibg_set_list_rows(ibg_ctx* c, int rows) {
  if (!c || rows < 1) return IBG_E_INVALID;
  try {
    CK(cudaStreamSynchronize(c->st));
    for (auto& L : c->L) {
      if (!L.present) continue;
      if (L.entries) c->owned.release(L.entries);
      L.entries = dalloc<int>((size_t)L.nslices * 32 * rows, c->owned);
      L.w_cap = rows;
    }
    refresh_args(c);
    for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
    c->graphs.clear();
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return IBG_OK;
}

int ibg_set_vsite_com(ibg_ctx* c, int form) {
  if (!c || (form != IBG_VS_COM_FIXED && form != IBG_VS_COM_REFERENCE)) return IBG_E_INVALID;
  if (c->in_batch) return fail(c, IBG_E_INVALID, "the context is in a batch");
  try {
    CK(cudaStreamSynchronize(c->st));
    c->vs_com_form = form;
    if (form == IBG_VS_COM_REFERENCE && c->nvirta > 0 && !c->vchain) {
      const size_t nb = c->prec == IBG_PREC_FP32_FIXED ? chain_bytes<float>(c->nvirta) : chain_bytes<double>(c->nvirta);
      c->vchain = dalloc<unsigned char>(nb, c->owned);
    }
    refresh_args(c);
    for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
    c->graphs.clear();
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return IBG_OK;
}

int ibg_get_tuning(const ibg_ctx* c, ibg_tuning* t) {
  if (!c || !t) return IBG_E_INVALID;
  const DevList& L = c->L[c->L[0].present ? 0 : 1];
  t->nb_tables_smem = L.use_smem ? 1 : 0;
  t->nb_blocks_per_sm = c->nb_blocks_per_sm;
  t->nb_chunk = c->nb_chunk;
  t->nb_rows = c->nb_rows;
  t->nb_window = c->nb_window;
  return IBG_OK;
}

int ibg_set_tuning(ibg_ctx* c, const ibg_tuning* t) {
  if (!c || !t || t->nb_blocks_per_sm < 0 || t->nb_chunk < 0 || t->nb_window < 0) return IBG_E_INVALID;
  if (t->nb_rows != 0 && t->nb_rows != 8 && t->nb_rows != 16) return IBG_E_INVALID;
  if (c->in_batch) return fail(c, IBG_E_INVALID, "the context is in a batch");
  try {
    c->nb_blocks_per_sm = t->nb_blocks_per_sm;
    c->nb_chunk = c->prec == IBG_PREC_FP32_FIXED ? t->nb_chunk : 0;
    c->nb_rows = t->nb_rows ? t->nb_rows : 16;
    c->nb_window = c->prec == IBG_PREC_FP32_FIXED ? t->nb_window : 0;
    for (auto& L : c->L) {
      if (!L.present) continue;
      L.use_smem = t->nb_tables_smem != 0 && L.smem <= 200 * 1024;
      if (c->prec == IBG_PREC_FP32_FIXED) nb_configure<float>(c, L);
      else nb_configure<double>(c, L);
    }
    refresh_args(c);
    for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
    c->graphs.clear();
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return IBG_OK;
}

int ibg_set_list_form(ibg_ctx* c, int form) {
  if (!c || form < IBG_LIST_AUTO || form > IBG_LIST_PER_SLICE) return IBG_E_INVALID;
  if (form == 1 && c->prec != IBG_PREC_FP32_FIXED) return fail(c, IBG_E_INVALID, "slice lists are an FP32-path form");
  if (c->in_batch) return fail(c, IBG_E_INVALID, "the context is in a batch");
  try {
    CK(cudaStreamSynchronize(c->st));
    c->list_form = form;
    bool changed = false;
    for (auto& L : c->L) {
      if (!L.present) continue;
      const int f = list_form_of(c, L.n);
      if (f == L.form) continue;
      if (L.entries) c->owned.release(L.entries);
      L.entries = nullptr;
      L.w_cap = 0;  // sized by the next build
      L.form = f;
      if (c->prec == IBG_PREC_FP32_FIXED) nb_configure<float>(c, L);
      else nb_configure<double>(c, L);
      changed = true;
    }
    if (changed) {
      refresh_args(c);
      for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
      c->graphs.clear();
      c->state_set = false;  // the lists are rebuilt by the next ibg_set_state
    }
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return IBG_OK;
}

int ibg_get_list_form(const ibg_ctx* c) {
  if (!c) return IBG_E_INVALID;
  for (const auto& L : c->L)
    if (L.present) return L.form;
  // no list: the form a list would get if it were explicitly chosen, else
  // per particle (never IBG_LIST_AUTO, which equals IBG_E_INVALID)
  return c->prec == IBG_PREC_FP32_FIXED && c->list_form == IBG_LIST_PER_SLICE ? IBG_LIST_PER_SLICE
                                                                              : IBG_LIST_PER_PARTICLE;
}

int ibg_autotune(ibg_ctx* c, int reps, ibg_tuning* best, ibg_tuning* cand_out, double* us, int ncand) {
  if (!c || reps <= 0) return IBG_E_INVALID;
  if (!c->state_set) return fail(c, IBG_E_INVALID, "ibg_set_state has not been called");
  if (c->in_batch) return fail(c, IBG_E_INVALID, "the context is in a batch");
  std::vector<ibg_tuning> cand;
  if (c->prec == IBG_PREC_FP32_FIXED) {
    for (int rows : {8, 16})
      for (int chunk : {0, 12, 24, 48, 96})
        for (int window : {0, 64})
          for (int smem : {0, 1})
            for (int per : {0, 4, 3})
              if (chunk > 0 || window == 0) cand.push_back(ibg_tuning{smem, per, chunk, rows, window});
  } else {
    for (int rows : {8, 16})
      for (int smem : {0, 1})
        for (int per : {0, 3, 2}) cand.push_back(ibg_tuning{smem, per, 0, rows, 0});
  }
  ibg_tuning keep;
  ibg_get_tuning(c, &keep);
  int win = -1;
  double win_us = 0.0;
  std::vector<cudaEvent_t> ev(2 * (size_t)reps, nullptr);
  // the trial launches run in the ordinary way, each on its own between the
  // memsets and events; programmatic launches are restored on every return
  struct PdlOff {
    ibg_ctx* c;
    ~PdlOff() { c->pdl = true; }
  } pdl_off{c};
  c->pdl = false;
  auto drop_events = [&] {
    for (auto& e : ev)
      if (e) {
        cudaEventDestroy(e);
        e = nullptr;
      }
  };
  try {
    for (auto& e : ev) CK(cudaEventCreate(&e));
    // with an L2 flush set, every timed launch starts from a flushed L2 as the
    // nonbonded launch of a timed step does; only the launches are timed
    const bool flush = c->flush_bytes > 0;
    if (flush && !c->flush_buf) CK(cudaMalloc(&c->flush_buf, c->flush_bytes));
    for (size_t k = 0; k < cand.size(); ++k) {
      int rc = ibg_set_tuning(c, &cand[k]);
      if (rc) {
        drop_events();
        return rc;
      }
      for (int r = 0; r <= reps; ++r) {  // the first launch warms up
        CK(cudaMemsetAsync(c->sc->work, 0, sizeof(c->sc->work), c->st));
        if (flush) CK(cudaMemsetAsync(c->flush_buf, r & 0xff, c->flush_bytes, c->st));
        if (r > 0) CK(cudaEventRecord(ev[2 * (r - 1)], c->st));
        for (auto& L : c->L) {
          if (!L.present) continue;
          if (c->prec == IBG_PREC_FP32_FIXED) enq_nonbonded<float>(c, L);
          else enq_nonbonded<double>(c, L);
        }
        if (r > 0) CK(cudaEventRecord(ev[2 * (r - 1) + 1], c->st));
      }
      CK(cudaEventSynchronize(ev.back()));
      double ms = 0.0;
      for (int r = 0; r < reps; ++r) {
        float m = 0.f;
        CK(cudaEventElapsedTime(&m, ev[2 * r], ev[2 * r + 1]));
        ms += m;
      }
      const double t = 1000.0 * ms / reps;
      if ((int)k < ncand) {
        if (us) us[k] = t;
        if (cand_out) cand_out[k] = cand[k];
      }
      if (win < 0 || t < win_us) { win = (int)k; win_us = t; }
    }
    drop_events();
    // the timing launches summed forces and energies: clear them
    for (auto& L : c->L)
      if (L.present) CK(cudaMemset(L.fsort, 0, accsize(c) * fs_len(L.n)));
    CK(cudaMemset(c->sc->nbacc, 0, sizeof(c->sc->nbacc)));
    CK(cudaMemset(c->sc->work, 0, sizeof(c->sc->work)));
    unsigned bits = 0;
    CK(cudaMemcpy(&bits, &c->sc->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (bits) {
      ibg_set_tuning(c, &keep);
      return check_device(c);
    }
  } catch (CudaError& e) {
    drop_events();
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  int rc = ibg_set_tuning(c, &cand[win]);
  if (best) *best = cand[win];
  return rc ? rc : (int)cand.size();
}

int ibg_set_l2_flush(ibg_ctx* c, long long bytes) {
  if (!c || bytes < 0) return IBG_E_INVALID;
  if (c->flush_buf && (size_t)bytes != c->flush_bytes) {
    cudaFree(c->flush_buf);
    c->flush_buf = nullptr;
  }
  c->flush_bytes = (size_t)bytes;
  return IBG_OK;
}

const char* ibg_last_error(const ibg_ctx* c) { return c ? c->err.c_str() : "null context"; }

long long ibg_device_bytes(const ibg_ctx* c) {
  if (!c) return IBG_E_INVALID;
  return (long long)(c->owned.bytes + (c->flush_buf ? c->flush_bytes : 0));
}

long long ibg_estimate_bytes(const ibg_desc* d, int precision, const float* box) {
  if (!d || !box || d->nitems <= 0) return IBG_E_INVALID;
  const bool f32 = precision == IBG_PREC_FP32_FIXED;
  const double pos = f32 ? 16.0 : 32.0, acc = 8.0, rs = f32 ? 4.0 : 8.0;
  const double vol = (double)box[0] * box[1] * box[2];
  double b = (double)d->nitems * (4 + 8 + 8 + 24 + 2 * 3 * acc + 4 + 80 + 4) + (double)d->natoms * 24;
  long long terms = 0;
  for (int i = 0; i < d->nitems; ++i) {
    terms += d->nbonds ? d->nbonds[i] : 0;
    terms += d->nijk ? d->nijk[i] : 0;
    if (i < d->natoms) terms += (d->nijkl ? d->nijkl[i] : 0) + (d->noopijkl ? d->noopijkl[i] : 0);
  }
  b += (double)terms * 24;
  const int ntab = d->nbtype + d->natype + d->nttype + d->notype;
  b += (double)ntab * 16.0 * 4096;  // bonded table rows, generous
  for (int w = 0; w < 2; ++w) {
    const int n = w == 0 ? d->numatoms : d->ncoarse;
    if (n <= 0) continue;
    const double rl = w == 0 ? d->rlist_atom : d->rlist_bead;
    const double half = (double)n / vol * (2.0 / 3.0) * 3.14159265358979 * rl * rl * rl;
    const double rows = (half * 1.25 + 8.0) * 1.25 + 2.0;  // growth margin and slice padding
    b += (double)n * (7 * 4 + 2 * pos + 3 * acc + rows * 4);
    if (precision == IBG_PREC_FP32_FIXED) b += (double)n * 32 + 16.0 * std::max(4096, n / 32);  // box fractions, cutoff pairs
    if (w == 1 && d->nmts > 0) b += (double)n * 9 * acc;
    const double cells = (box[0] * 1.25 / rl + 2) * (box[1] * 1.25 / rl + 2) * (box[2] * 1.25 / rl + 2);
    b += cells * 12;
    b += (double)d->nnbtype * d->ld_nb * 3 * rs;
  }
  b += 2.0 * 1024 * 1024;  // scalars, partial sums, argument blocks, rounding of allocations
  return (long long)b;
}

int ibg_create(const ibg_desc* d, int precision, ibg_ctx** out) {
  if (!d || !out) return IBG_E_INVALID;
  *out = nullptr;
  if (precision != IBG_PREC_FP32_FIXED && precision != IBG_PREC_FP64_PLAIN) return IBG_E_INVALID;
  if (d->natoms <= 0 || d->nitems != d->natoms + d->nvirta || d->ntype <= 0 || d->nupdate <= 0 || d->halt_drift <= 0)
    return IBG_E_INVALID;
  auto c = std::make_unique<ibg_ctx>();
  try {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    c->dev = dev;
    CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->fork_ev[0], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->fork_ev[1], cudaEventDisableTiming));
    c->prec = precision;
    c->natoms = d->natoms; c->nvirta = d->nvirta; c->nitems = d->nitems; c->ntype = d->ntype;
    c->numatoms = d->numatoms; c->numbeads = d->numbeads; c->ncoarse = d->ncoarse;
    c->ensemble = d->ensemble; c->nupdate = d->nupdate; c->halt_drift = d->halt_drift; c->nmts = d->nmts;
    c->ibrdescr = d->ibrdescr; c->maxnab = d->maxnab > 0 ? d->maxnab : 1000;
    c->dt = d->dt; c->fac = d->fac; c->pfac = d->pfac; c->temp_in = d->temp_in; c->pressure = d->pressure;
    c->mktemp = d->mktemp; c->mktemp_atom = d->mktemp_atom; c->mktemp_bead = d->mktemp_bead;
    c->r2d = 180.0f / 3.14159265358f;  // UNIT.f90:22
    const int N = d->nitems, NA = d->natoms, NT = d->ntype;
    auto& o = c->owned;
    // particles
    std::vector<int> tbits(N), gslot(N, 0);
    std::vector<double> mass(N), inv(N);
    for (int i = 0; i < N; ++i) {
      int t = d->itype[i];
      if (t < 1 || t > NT) return fail(nullptr, IBG_E_INVALID, "");
      int lab = i < NA ? d->type_label[i] : 3;
      tbits[i] = (t - 1) | (lab << 16);
      mass[i] = d->mass[t - 1];
      inv[i] = d->invmass[t - 1];
    }
    c->tbits = dupload(tbits, o);
    c->mass = dupload(mass, o);
    c->invmass = dupload(inv, o);
    c->S = dalloc<double>(3 * (size_t)N, o);
    c->V = dalloc<double>(3 * (size_t)NA, o);
    c->su = c->S;
    c->fnb = dalloc<unsigned char>(accsize(c.get()) * 3 * N, o);
    c->fb = dalloc<unsigned char>(accsize(c.get()) * 3 * N, o);
    // exclusions
    std::vector<int> en(N), ex((size_t)N * 20, -1);
    for (int i = 0; i < N; ++i) {
      en[i] = d->connections[i];
      if (en[i] < 0 || en[i] > 20) return fail(nullptr, IBG_E_INVALID, "");
      for (int k = 0; k < en[i]; ++k) ex[(size_t)i * 20 + k] = d->connected_to[(size_t)k * d->ld_conn + i] - 1;
    }
    c->excl_n = dupload(en, o);
    c->excl = dupload(ex, o);
    // virtual sites
    {
      const int nv = d->nvirta;
      std::vector<int> ctr(std::max(nv, 1), -1), num(std::max(nv, 1), 0), mem((size_t)std::max(nv, 1) * 15, 0);
      std::vector<float> vm((size_t)std::max(nv, 1) * 15, 0.f), vi(std::max(nv, 1), 0.f), vc((size_t)std::max(nv, 1) * 15, 0.f);
      for (int v = 0; v < nv; ++v) {
        int t = d->vitype[v];
        ctr[v] = d->virt_center[v] > 0 ? d->virt_center[v] - 1 : -1;
        num[v] = d->virt_numatoms[t - 1];
        if (num[v] > 15 || num[v] > d->vs_maxatoms) return fail(nullptr, IBG_E_INVALID, "");
        vi[v] = d->virt_invmass[t - 1];
        for (int k = 0; k < num[v]; ++k) {
          int a = d->virt_atm_ind[(size_t)k * d->ld_vs + v];
          if (a < 1 || a > NA) return fail(nullptr, IBG_E_INVALID, "");
          mem[(size_t)v * 15 + k] = a - 1;
          int ta = d->itype[a - 1];
          vm[(size_t)v * 15 + k] = d->mass[ta - 1];
          vc[(size_t)v * 15 + k] = d->virt_masscoeff[(size_t)(t - 1) + (size_t)NT * (ta - 1)];
        }
      }
      c->vcenter = dupload(ctr, o); c->vnum = dupload(num, o); c->vmem = dupload(mem, o);
      c->vmass = dupload(vm, o); c->vinv = dupload(vi, o); c->vcoef = dupload(vc, o);
    }
    // bonded terms in the reference's loop order (BONDED_FORCE.F90:70-91)
    {
      std::vector<int4> bonds, angles, tors, oops;
      std::vector<int2> tors_t, oops_t;
      auto T2 = [&](int a, int b) { return (size_t)(a - 1) + (size_t)NT * (b - 1); };
      auto T3 = [&](int a, int b, int cc) { return T2(a, b) + (size_t)NT * NT * (cc - 1); };
      auto T4 = [&](int a, int b, int cc, int e) { return T3(a, b, cc) + (size_t)NT * NT * NT * (e - 1); };
      for (int I = 1; I <= N; ++I) {
        const int TI = d->itype[I - 1];
        const int nbnd = d->nbonds ? d->nbonds[I - 1] : 0;
        for (int a = 0; a < nbnd; ++a) {
          int J = d->jbond[(size_t)a * d->ld_bond + I - 1];
          if (J > I) {
            int t = d->ibondt[T2(TI, d->itype[J - 1])];
            if (t < 1) return fail(nullptr, IBG_E_INVALID, "");
            bonds.push_back(make_int4(I - 1, J - 1, t - 1, d->bond_type_label[t - 1]));
          }
        }
        const int nang = d->nijk ? d->nijk[I - 1] : 0;
        for (int a = 0; a < nang; ++a) {
          int J = d->jangleijk[(size_t)a * d->ld_angle + I - 1], K = d->kangleijk[(size_t)a * d->ld_angle + I - 1];
          int t = d->iangt[T3(TI, d->itype[J - 1], d->itype[K - 1])];
          if (t < 1) return fail(nullptr, IBG_E_INVALID, "");
          angles.push_back(make_int4(I - 1, J - 1, K - 1, (t - 1) | (d->angle_type_label[t - 1] << 24)));
        }
        if (I <= NA && d->nijkl) {
          for (int a = 0; a < d->nijkl[I - 1]; ++a) {
            int J = d->jtorijkl[(size_t)a * d->ld_torsion + I - 1], K = d->ktorijkl[(size_t)a * d->ld_torsion + I - 1],
                Lq = d->ltorijkl[(size_t)a * d->ld_torsion + I - 1];
            int t = d->itort[T4(TI, d->itype[J - 1], d->itype[K - 1], d->itype[Lq - 1])];
            if (t < 1) return fail(nullptr, IBG_E_INVALID, "");
            tors.push_back(make_int4(I - 1, J - 1, K - 1, Lq - 1));
            tors_t.push_back(make_int2(t - 1, d->torsion_type_label[t - 1]));
          }
        }
        if (I <= NA && d->noopijkl) {
          for (int a = 0; a < d->noopijkl[I - 1]; ++a) {
            int J = d->joopijkl[(size_t)a * d->ld_oop + I - 1], K = d->koopijkl[(size_t)a * d->ld_oop + I - 1],
                Lq = d->loopijkl[(size_t)a * d->ld_oop + I - 1];
            int t = d->ioopt[T4(TI, d->itype[J - 1], d->itype[K - 1], d->itype[Lq - 1])];
            if (t < 1) return fail(nullptr, IBG_E_INVALID, "");
            oops.push_back(make_int4(I - 1, J - 1, K - 1, Lq - 1));
            oops_t.push_back(make_int2(t - 1, d->oop_type_label[t - 1]));
          }
        }
      }
      c->nb = (int)bonds.size(); c->na = (int)angles.size(); c->nt = (int)tors.size(); c->no = (int)oops.size();
      c->bonds = dupload(bonds, o); c->angles = dupload(angles, o); c->tors = dupload(tors, o); c->oops = dupload(oops, o);
      c->tors_t = dupload(tors_t, o); c->oops_t = dupload(oops_t, o);
      // bonded tables: rows {X, F, P, 0}, type-fastest input layout
      auto tables = [&](int ntab, int ld, const int* nd, const float* bin, const float* X, const float* F, const float* P,
                        float4** rows, int** off, int** ndat, float** binout) {
        std::vector<float4> r;
        std::vector<int> of(std::max(ntab, 1), 0), ndv(std::max(ntab, 1), 0);
        std::vector<float> bv(std::max(ntab, 1), 1.f);
        for (int t = 0; t < ntab; ++t) {
          of[t] = (int)r.size();
          ndv[t] = nd[t];
          bv[t] = bin[t];
          for (int k = 0; k < nd[t] + 3; ++k) {
            if (k < ld) {
              size_t at = (size_t)t + (size_t)ntab * k;
              r.push_back(make_float4(X[at], F[at], P[at], 0.f));
            } else {
              r.push_back(make_float4(0.f, 0.f, 0.f, 0.f));
            }
          }
        }
        *rows = dupload(r, o); *off = dupload(of, o); *ndat = dupload(ndv, o); *binout = dupload(bv, o);
      };
      tables(d->nbtype, d->ld_b, d->ndatb, d->binb, d->rbond, d->bond_force, d->bond_pot, &c->tb, &c->tb_off, &c->tb_nd, &c->tb_bin);
      tables(d->natype, d->ld_a, d->ndatan, d->bina, d->angle, d->bend_force, d->bend_pot, &c->ta, &c->ta_off, &c->ta_nd, &c->ta_bin);
      tables(d->nttype, d->ld_t, d->ndatt, d->bint, d->angle_tor, d->tor_force, d->tor_pot, &c->tt, &c->tt_off, &c->tt_nd, &c->tt_bin);
      tables(d->notype, d->ld_o, d->ndato, d->bino, d->angle_oop, d->oop_force, d->oop_pot, &c->to, &c->to_off, &c->to_nd, &c->to_bin);
    }
    // Verlet lists
    build_list(c.get(), d, 0);
    if (d->ibrdescr == 0) build_list(c.get(), d, 1);
    {  // every particle belongs to exactly one list
      std::vector<int> gs(N, -1);
      for (int a = 0; a < c->L[0].n; ++a) gs[d->atom[a] - 1] = a * 2 + 0;
      for (int a = 0; a < c->L[1].n; ++a) gs[d->bead[a] - 1] = a * 2 + 1;
      for (int i = 0; i < N; ++i)
        if (gs[i] < 0) return fail(nullptr, IBG_E_INVALID, "");
      c->gslot = dupload(gs, o);
    }
    // grids and partial sums
    for (auto& L : c->L) {
      if (!L.present) continue;
      // gslot holds slot * 2 + list in an int
      if (L.n >= (1 << 30)) return fail(nullptr, IBG_E_CAPACITY, "");
      if (precision == IBG_PREC_FP32_FIXED) nb_configure<float>(c.get(), L);
      else nb_configure<double>(c.get(), L);
    }
    for (int w = 0; w < 2; ++w) {
      DevList& L = c->L[w];
      if (!L.present) continue;
      c->g_list[w] = grid_for(c.get(), L.n);
      c->g_build[w] = std::max(1, std::min((L.n + 15) / 16, c->nsm * 4));  // blocks take cells
    }
    c->g_dist = grid_for(c.get(), 16LL * std::max(1, c->nvirta));  // 16 lanes per site
    c->g_b = grid_for(c.get(), (long long)c->nb + c->na + c->nt + c->no, 4);
    c->g_mv = grid_for(c.get(), NA, 4);
    c->g_pos = grid_for(c.get(), N, 8);
    c->p_b = dalloc<double>(12 * (size_t)c->g_b, o);
    c->p_mv = dalloc<double>(18 * (size_t)c->g_mv, o);
    c->p_mom = dalloc<double>(3 * (size_t)c->g_mv, o);
    c->sc = dalloc<Scalars>(1, o);
    CK(cudaHostAlloc(&c->hsc, sizeof(Scalars), cudaHostAllocDefault));
    c->ring_cap = 1;
    c->ring = nullptr;
    refresh_args(c.get());
    CK(cudaDeviceSynchronize());
  } catch (CudaError& e) {
    c->owned.free_all();
    return IBG_E_CUDA;
  }
  *out = c.release();
  return IBG_OK;
}

}  // extern "C"

namespace {

// REAL*4 state of the host into the FP64 state: SXYZ(3,NATOMS), the virtual
// sites' rows zero until VIRTUAL_DEF fills them, and VXYZ(3,NATOMS).
__global__ void k_state_in(int natoms, int nitems, const float* s, const float* v, double* S, double* V) {
  const size_t n3 = 3 * (size_t)nitems, a3 = 3 * (size_t)natoms;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n3; k += (size_t)gridDim.x * blockDim.x) {
    S[k] = k < a3 ? (double)s[k] : 0.0;
    if (k < a3) V[k] = (double)v[k];
  }
}

// Slots in list order before the first sort: slot_of = sorted = identity,
// and each listed particle's gslot = slot * 2 + list.
__global__ void k_slots_init(int n, int which, const int* idx, int* slot_of, int* sorted, int* gslot) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    slot_of[a] = a;
    sorted[a] = a;
    gslot[idx[a]] = a * 2 + which;
  }
}

// The state as REAL*4 for ibg_get_state, into staging: SXYZ, RXYZ (wrapped,
// from the slot-ordered positions of the particle's list), VXYZ (NATOMS rows)
// and FXYZ (nonbonded + bonded sums), each 3 x NITEMS floats.
template <typename R, typename A>
__global__ void k_state_out(int natoms, int nitems, const double* S, const double* V, const int* gslot,
                            const void* pos0, const void* pos1, const A* fnb, const A* fb, float* out) {
  using PT = typename Prec<R>::pos_t;
  const size_t n3 = 3 * (size_t)nitems;
  float* s = out;
  float* r = out + n3;
  float* v = out + 2 * n3;
  float* f = out + 3 * n3;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n3; k += (size_t)gridDim.x * blockDim.x) {
    s[k] = (float)S[k];
    if (k < 3 * (size_t)natoms) v[k] = (float)V[k];
    if (sizeof(A) == 8 && sizeof(R) == 4) {
      const long long q = (long long)fnb[k] + (long long)fb[k];
      f[k] = (float)((double)q * kFixInv);
    } else {
      f[k] = (float)((double)fnb[k] + (double)fb[k]);
    }
    const size_t i = k / 3;
    const int c3 = (int)(k - 3 * i);
    const int g = gslot[i];
    const PT p = ((const PT*)((g & 1) ? pos1 : pos0))[g >> 1];
    r[k] = (float)(c3 == 0 ? p.x : (c3 == 1 ? p.y : p.z));
  }
}

float* xfer_buf(ibg_ctx* c) {
  if (!c->xfer) c->xfer = dalloc<float>(12 * (size_t)c->nitems, c->owned);
  return c->xfer;
}

// The argument blocks and launch sizes a captured step graph depends on.
std::vector<unsigned char> graph_key(const ibg_ctx* c) {
  std::vector<unsigned char> k;
  auto add = [&](const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    k.insert(k.end(), b, b + n);
  };
  if (c->prec == IBG_PREC_FP32_FIXED) add(&c->af, sizeof(c->af));
  else add(&c->ad, sizeof(c->ad));
  add(c->g_regrid, sizeof(c->g_regrid));
  return k;
}

}  // namespace

extern "C" {

int ibg_set_state(ibg_ctx* c, const float* sxyz, const float* vxyz, const float* box) {
  if (!c || !sxyz || !vxyz || !box) return IBG_E_INVALID;
  try {
    const int NA = c->natoms;
    const std::vector<unsigned char> key0 = graph_key(c);
    {  // REAL*4 arrays to the device, widened to the FP64 state there
      float* x = xfer_buf(c);
      CK(cudaMemcpyAsync(x, sxyz, sizeof(float) * 3 * (size_t)NA, cudaMemcpyHostToDevice, c->st));
      CK(cudaMemcpyAsync(x + 3 * (size_t)NA, vxyz, sizeof(float) * 3 * (size_t)NA, cudaMemcpyHostToDevice, c->st));
      k_state_in<<<grid_for(c, 3LL * c->nitems), 256, 0, c->st>>>(NA, c->nitems, x, x + 3 * (size_t)NA, c->S, c->V);
      CK(cudaGetLastError());
    }
    Scalars h;
    std::memset(&h, 0, sizeof(h));
    for (int k = 0; k < 3; ++k) {
      h.boxf[k] = box[k];
      h.boxinvf[k] = 1.0f / box[k];       // RDCOOR.f90:70-71
      h.box2f[k] = box[k] / 2.0f;
      h.box[k] = (double)box[k];
      h.boxinv[k] = 1.0 / h.box[k];
      h.box2[k] = h.box[k] / 2.0;
    }
    h.step = 0;
    h.mts_m = -1;
    h.miu = 1.0;
    h.stop_at = INT_MAX;
    h.lam[0] = h.lam[1] = 1.0;
    CK(cudaMemcpy(c->sc, &h, sizeof(h), cudaMemcpyHostToDevice));
    for (auto& L : c->L) {
      if (!L.present) continue;
      alloc_cells(c, L, box);
      CK(cudaMemsetAsync(L.fsort, 0, accsize(c) * fs_len(L.n), c->st));
      if (L.mtsf) CK(cudaMemsetAsync(L.mtsf, 0, accsize(c) * 9 * (size_t)L.n, c->st));
      c->g_regrid[L.which] = grid_for(c, L.cell_cap, 2);
    }
    CK(cudaMemsetAsync(c->fnb, 0, accsize(c) * 3 * (size_t)c->nitems, c->st));
    CK(cudaMemsetAsync(c->fb, 0, accsize(c) * 3 * (size_t)c->nitems, c->st));
    refresh_args(c);
    // slots = list order before the first sort
    CK(cudaMemsetAsync(c->gslot, 0, sizeof(int) * (size_t)c->nitems, c->st));
    for (auto& L : c->L)
      if (L.present)
        k_slots_init<<<grid_for(c, L.n), 256, 0, c->st>>>(L.n, L.which, L.idx, L.slot_of, L.sorted, c->gslot);
    CK(cudaGetLastError());
    // the step graphs hold the argument blocks by value: they are kept when
    // this state left every array where it was
    if (graph_key(c) != key0) {
      for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
      c->graphs.clear();
    }
    // main.F90:150-234: virtual sites, SHIFT, initial temperatures, first lists
    if (c->prec == IBG_PREC_FP32_FIXED) enq_positions<float>(c);
    else enq_positions<double>(c);
    k_kinetic<<<c->g_mv, 256, 0, c->st>>>(NA, c->V, c->tbits, c->mass, c->p_mv, c->g_mv);
    k_init_temps<<<1, 64, 0, c->st>>>(c->p_mv, c->g_mv, c->sc, c->mktemp, c->mktemp_atom, c->mktemp_bead, c->temp_in, c->fac,
                                      c->ensemble);
    int grew = 1;
    for (int pass = 0; pass < 4 && grew; ++pass) {
      if (c->prec == IBG_PREC_FP32_FIXED) rebuild_now<float>(c);
      else rebuild_now<double>(c);
      CK(cudaStreamSynchronize(c->st));
      unsigned bits = 0;
      CK(cudaMemcpy(&bits, &c->sc->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
      if (bits) return check_device(c);
      grew = grow_lists(c);
      // a repeated build sorts already sorted slots and yields the same lists
    }
    if (grew) return fail(c, IBG_E_CAPACITY, "neighbour-list storage could not be sized");
    int rc = check_device(c);
    if (rc) return rc;
    c->state_set = true;
    c->step_now = 0;
    c->fb_dirty = false;
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return IBG_OK;
}

static int run_steps(ibg_ctx* c, int first, int nsteps, ibg_obs* per_step, bool force_only, bool use_graphs) {
  if (!c) return IBG_E_INVALID;
  if (!c->state_set) return fail(c, IBG_E_INVALID, "ibg_set_state has not been called");
  try {
    if (per_step && nsteps > c->ring_cap) {
      if (c->ring) c->owned.release(c->ring);
      c->ring_cap = std::max(nsteps, 64);
      c->ring = dalloc<ObsD>(c->ring_cap, c->owned);
      refresh_args(c);
      for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
      c->graphs.clear();
    }
    int done = 0;
    float run_ms_total = 0.f;
    for (int attempt = 0; attempt < 8 && done < nsteps; ++attempt) {
      set_step_counter(c, first + done - 1, first, first + nsteps - 1, false);
      if (c->flush_bytes) {
        if (!c->flush_buf) CK(cudaMalloc(&c->flush_buf, c->flush_bytes));
        while ((int)c->step_ev.size() < 2 * nsteps) {
          cudaEvent_t e;
          CK(cudaEventCreate(&e));
          c->step_ev.push_back(e);
        }
      }
      if (!c->run_ev[0]) {
        CK(cudaEventCreate(&c->run_ev[0]));
        CK(cudaEventCreate(&c->run_ev[1]));
      }
      CK(cudaEventRecord(c->run_ev[0], c->st));
      const int begin = done;
      for (int k = begin; k < nsteps; ++k) {
        const int step = first + k;
        const unsigned v = variant_of(c, step, force_only);
        const bool flush = c->flush_bytes && c->flush_buf;
        if (flush) {
          CK(cudaMemsetAsync(c->flush_buf, k & 0xff, c->flush_bytes, c->st));
          CK(cudaEventRecord(c->step_ev[2 * k], c->st));
        }
        if (use_graphs && !c->timing) {
          auto it = c->graphs.find(v);
          if (it == c->graphs.end()) {
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
            long long l0 = c->launches;
            enqueue(c, v);
            CK(cudaStreamEndCapture(c->st, &g));
            c->launches_per_variant[v & 31] = c->launches - l0;
            cudaGraphExec_t ge;
            CK(cudaGraphInstantiate(&ge, g, 0));
            CK(cudaGraphDestroy(g));
            it = c->graphs.emplace(v, ge).first;
          }
          CK(cudaGraphLaunch(it->second, c->st));
          c->launches += c->launches_per_variant[v & 31];
        } else {
          enqueue(c, v);
        }
        if (flush) CK(cudaEventRecord(c->step_ev[2 * k + 1], c->st));
      }
      CK(cudaEventRecord(c->run_ev[1], c->st));
      // one read-back per run: step, abort and error flags, observables
      CK(cudaMemcpyAsync(c->hsc, c->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, c->st));
      collect_marks(c);
      CK(cudaStreamSynchronize(c->st));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, c->run_ev[0], c->run_ev[1]));
      if (c->flush_bytes && c->flush_buf) {  // only the steps, not the flushes
        ms = 0.f;
        for (int k = begin; k < nsteps; ++k) {
          float m = 0.f;
          CK(cudaEventElapsedTime(&m, c->step_ev[2 * k], c->step_ev[2 * k + 1]));
          ms += m;
        }
      }
      run_ms_total += ms;
      if (c->hsc->abort && grow_lists(c)) {
        done = c->hsc->step - first;  // the step that aborted did not complete
        continue;
      }
      done = nsteps;
    }
    c->stage_ms[5] = run_ms_total;
    c->step_now = first + done - 1;
    if (done < nsteps) return fail(c, IBG_E_CAPACITY, "neighbour-list storage could not be sized");
    int rc = check_bits(c, c->hsc->err);
    if (rc) return rc;
    if (per_step) {
      std::vector<ObsD> h(nsteps);
      CK(cudaMemcpy(h.data(), c->ring, sizeof(ObsD) * nsteps, cudaMemcpyDeviceToHost));
      for (int k = 0; k < nsteps; ++k) obs_to_c(h[k], &per_step[k]);
    }
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return IBG_OK;
}

int ibg_step(ibg_ctx* c, int step, ibg_obs* out) {
  int rc = run_steps(c, step, 1, nullptr, false, true);
  if (rc) return rc;
  if (out) obs_to_c(c->hsc->obs, out);  // read back by run_steps
  return IBG_OK;
}

int ibg_forces(ibg_ctx* c, int step, ibg_obs* out) {
  int rc = run_steps(c, step, 1, nullptr, true, false);
  if (rc) return rc;
  if (out) obs_to_c(c->hsc->obs, out);
  return IBG_OK;
}

int ibg_run(ibg_ctx* c, int first_step, int nsteps, ibg_obs* per_step) {
  if (nsteps < 0) return IBG_E_INVALID;
  return run_steps(c, first_step, nsteps, per_step, false, true);
}

int ibg_get_state(ibg_ctx* c, float* sxyz, float* rxyz, float* vxyz, float* fxyz) {
  if (!c) return IBG_E_INVALID;
  try {
    // narrowed to REAL*4 on the device, then one copy per requested array
    const size_t N = c->nitems, NA = c->natoms, n3 = 3 * N;
    float* x = xfer_buf(c);
    const void* p0 = c->L[0].present ? c->L[0].pos4 : c->L[1].pos4;
    const void* p1 = c->L[1].present ? c->L[1].pos4 : p0;
    const int g = grid_for(c, (long long)n3);
    if (c->prec == IBG_PREC_FP32_FIXED)
      k_state_out<float, unsigned long long><<<g, 256, 0, c->st>>>(
          c->natoms, c->nitems, c->S, c->V, c->gslot, p0, p1, (const unsigned long long*)c->fnb,
          (const unsigned long long*)c->fb, x);
    else
      k_state_out<double, double><<<g, 256, 0, c->st>>>(c->natoms, c->nitems, c->S, c->V, c->gslot, p0, p1,
                                                          (const double*)c->fnb, (const double*)c->fb, x);
    CK(cudaGetLastError());
    if (sxyz) CK(cudaMemcpyAsync(sxyz, x, sizeof(float) * n3, cudaMemcpyDeviceToHost, c->st));
    if (rxyz) CK(cudaMemcpyAsync(rxyz, x + n3, sizeof(float) * n3, cudaMemcpyDeviceToHost, c->st));
    if (vxyz) CK(cudaMemcpyAsync(vxyz, x + 2 * n3, sizeof(float) * 3 * NA, cudaMemcpyDeviceToHost, c->st));
    if (fxyz) CK(cudaMemcpyAsync(fxyz, x + 3 * n3, sizeof(float) * n3, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return IBG_OK;
}

int ibg_get_state_f64(ibg_ctx* c, double* sxyz, double* vxyz, double* fxyz) {
  if (!c) return IBG_E_INVALID;
  try {
    CK(cudaStreamSynchronize(c->st));
    const size_t N = c->nitems, NA = c->natoms;
    if (sxyz) CK(cudaMemcpy(sxyz, c->S, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
    if (vxyz) CK(cudaMemcpy(vxyz, c->V, sizeof(double) * 3 * NA, cudaMemcpyDeviceToHost));
    if (fxyz) {
      if (c->prec == IBG_PREC_FP32_FIXED) {
        std::vector<long long> a(3 * N), b(3 * N);
        CK(cudaMemcpy(a.data(), c->fnb, sizeof(long long) * 3 * N, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(b.data(), c->fb, sizeof(long long) * 3 * N, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < 3 * N; ++k) fxyz[k] = (double)(a[k] + b[k]) * kFixInv;
      } else {
        std::vector<double> a(3 * N), b(3 * N);
        CK(cudaMemcpy(a.data(), c->fnb, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(b.data(), c->fb, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < 3 * N; ++k) fxyz[k] = a[k] + b[k];
      }
    }
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return IBG_OK;
}

int ibg_get_neighbour_list(ibg_ctx* c, int which, int* list, int maxnab, int* nnebs) {
  if (!c || which < 0 || which > 1) return IBG_E_INVALID;
  DevList& L = c->L[which];
  if (!L.present) return 0;
  try {
    CK(cudaStreamSynchronize(c->st));
    std::vector<int> counts(L.n), sorted(L.n), idx(L.n);
    CK(cudaMemcpy(counts.data(), L.counts, sizeof(int) * L.n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(sorted.data(), L.sorted, sizeof(int) * L.n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(idx.data(), L.idx, sizeof(int) * L.n, cudaMemcpyDeviceToHost));
    std::vector<int> e(list ? (size_t)L.nslices * 32 * L.w_cap : 0);
    if (!e.empty()) CK(cudaMemcpy(e.data(), L.entries, sizeof(int) * e.size(), cudaMemcpyDeviceToHost));
    // lists stored in two groups (rgroupsq), and slice lists, are put back in
    // the reference's order: the own cell, then the 13 stencil cells, each by
    // decreasing slot
    const bool regroup = list && (L.rgroupsq > 0.f || L.form == 1);
    std::vector<int> cell_of;
    int nc[3] = {0, 0, 0};
    if (regroup) {
      cell_of.resize(L.n);
      CK(cudaMemcpy(cell_of.data(), L.cell_of, sizeof(int) * L.n, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(nc, c->sc->ncell[which], sizeof(nc), cudaMemcpyDeviceToHost));
    }
    auto run_of = [&](int s, int t) {
      const int ci = cell_of[sorted[s]], cj = cell_of[sorted[t]];
      if (ci == cj) return 0;
      const int a[3] = {ci / (nc[2] * nc[1]), (ci / nc[2]) % nc[1], ci % nc[2]};
      const int b[3] = {cj / (nc[2] * nc[1]), (cj / nc[2]) % nc[1], cj % nc[2]};
      int d[3];
      for (int q = 0; q < 3; ++q) {
        d[q] = b[q] - a[q];
        if (d[q] > 1) d[q] -= nc[q];
        if (d[q] < -1) d[q] += nc[q];
      }
      for (int u = 0; u < 13; ++u)
        if (d[0] == kStencilHost[u][0] && d[1] == kStencilHost[u][1] && d[2] == kStencilHost[u][2]) return u + 1;
      return 14;  // not a stencil cell: cannot happen for a list built on this grid
    };
    const int T = L.T, P = 32 / L.T;
    std::vector<int> slice_w;
    if (list && L.form == 1) {
      slice_w.resize(L.nslices);
      CK(cudaMemcpy(slice_w.data(), L.slice_w, sizeof(int) * L.nslices, cudaMemcpyDeviceToHost));
    }
    std::vector<std::pair<int, int>> keyed;
    for (int s = 0; s < L.n; ++s) {
      const int a = sorted[s];
      const int g = s / P, lane0 = (s % P) * T;
      if (nnebs) nnebs[a] = counts[s];
      if (!list) continue;
      if (counts[s] >= maxnab) return fail(c, IBG_E_INVALID, "maxnab smaller than a list");
      int* col = list + (size_t)a * maxnab;
      keyed.clear();
      if (L.form == 1) {  // the entries of slot s's slice whose mask holds s
        const unsigned bit = 1u << (s % kUSlots);
        const size_t base = (size_t)(s / kUSlots) * L.w_cap * 32;
        const int ne = std::min(slice_w[s / kUSlots], L.w_cap) * 32;
        for (int k = 0; k < ne; ++k) {
          const unsigned u = (unsigned)e[base + k];
          if (((u >> 28) & bit) == 0) continue;
          const int t = (int)(u & kUSlotMask);
          keyed.emplace_back(run_of(s, t), -t);
        }
        if ((int)keyed.size() != counts[s]) return fail(c, IBG_E_INVALID, "slice list and pair count disagree");
      } else {
        for (int k = 0; k < counts[s]; ++k) {
          const int t = e[((size_t)g * L.w_cap + (size_t)(k / T)) * 32 + lane0 + (k % T)];
          keyed.emplace_back(regroup ? run_of(s, t) : 0, regroup ? -t : k);
        }
      }
      if (regroup) std::sort(keyed.begin(), keyed.end());
      for (int k = 0; k < maxnab; ++k) {
        if (k < counts[s]) {
          const int t = regroup ? -keyed[k].second
                                : e[((size_t)g * L.w_cap + (size_t)(k / T)) * 32 + lane0 + (k % T)];
          col[k] = idx[sorted[t]] + 1;
        } else {
          col[k] = 0;
        }
      }
    }
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return L.n;
}

int ibg_get_exclusions(ibg_ctx* c, int* connections, int* connected_to) {
  if (!c) return IBG_E_INVALID;
  try {
    const int N = c->nitems;
    std::vector<int> en(N), ex((size_t)N * 20);
    CK(cudaMemcpy(en.data(), c->excl_n, sizeof(int) * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ex.data(), c->excl, sizeof(int) * ex.size(), cudaMemcpyDeviceToHost));
    for (int i = 0; i < N; ++i) {
      if (connections) connections[i] = en[i];
      if (connected_to)
        for (int k = 0; k < 20; ++k) connected_to[(size_t)k * N + i] = k < en[i] ? ex[(size_t)i * 20 + k] + 1 : 0;
    }
  } catch (CudaError& e) {
    return fail(c, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
  return IBG_OK;
}

int ibg_set_timing(ibg_ctx* c, int on) {
  if (!c) return IBG_E_INVALID;
  c->timing = on != 0;
  for (double& x : c->stage_ms) x = 0.0;
  return IBG_OK;
}

int ibg_get_timing(ibg_ctx* c, double* stage_ms, int nstage, long long* launches) {
  if (!c) return IBG_E_INVALID;
  c->stage_ms[7] = (double)c->list_growths;
  for (int k = 0; k < nstage && k < 9; ++k) stage_ms[k] = c->stage_ms[k];
  if (launches) *launches = c->launches;
  return IBG_OK;
}

void ibg_destroy(ibg_ctx* c) {
  if (!c) return;
  cudaStreamSynchronize(c->st);
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
  c->owned.free_all();
  for (auto* e : c->run_ev)
    if (e) cudaEventDestroy(e);
  for (auto* e : c->step_ev) cudaEventDestroy(e);
  if (c->flush_buf) cudaFree(c->flush_buf);
  if (c->hsc) cudaFreeHost(c->hsc);
  for (auto* e : c->fork_ev)
    if (e) cudaEventDestroy(e);
  if (c->st2) cudaStreamDestroy(c->st2);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

}  // extern "C"

// ===================================================================== batch
// Many independent systems stepped together: one launch per stage covers
// every system (blocks map to systems through a block map, arguments come
// from each system's device argument block), and the whole batch step is one
// CUDA graph.  Each system keeps its own step counter, list schedule, MTS
// phase, thermostat and barostat; device-side flags make a stage a no-op for
// the systems it does not concern this step.  Integer force and energy sums
// and per-system launch shapes for the statically scheduled kernels make every
// system's result bitwise the same alone and in any batch.

struct BMap {
  int* sys_of = nullptr;
  int* start = nullptr;
  int grid = 0;
  BlockMap m() const { return BlockMap{sys_of, start}; }
};

struct NBGroup {
  int T = 1;
  int form = 0;  // list form (DevList::form)
  bool smem = false;
  bool mixed = true;  // nonbonded groups: lists of more than one label
  size_t sm = 0;
  BMap map;
};

struct ibg_batch {
  int prec = 0, dev = 0, nsm = 148;
  std::vector<ibg_ctx*> sys;
  Owned owned;
  cudaStream_t st = nullptr, st2 = nullptr;
  cudaEvent_t fork_ev[2] = {nullptr, nullptr}, run_ev[2] = {nullptr, nullptr};
  // per-system pointers to the argument blocks, by kind
  void** t_pos = nullptr;
  void** t_list[2] = {nullptr, nullptr};
  void** t_nb[2] = {nullptr, nullptr};
  void** t_col[2] = {nullptr, nullptr};
  void** t_dist = nullptr;
  void** t_bond = nullptr;
  void** t_move = nullptr;
  void** t_mom = nullptr;
  void** t_fin = nullptr;
  BMap m_pos, m_regrid[2], m_list[2], m_scan[2], m_dist, m_bond, m_move, m_fin;
  std::vector<NBGroup> lb[2];  // list build, by T (smem unused)
  std::vector<NBGroup> nb[2];  // nonbonded, by (T, smem)
  bool any_vs = false, any_list[2] = {false, false};
  bool any_com_carry = false;  // a system with the reference's centre-of-mass chain
  std::map<unsigned, cudaGraphExec_t> graphs;
  long long launches = 0, launches_per_variant[8] = {0};
  double run_ms = 0.0;
  std::string err;
};

namespace {

int bfail(ibg_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  return code;
}

// Block map from per-system block counts (0: the system takes no part).
BMap make_map(ibg_batch* b, const std::vector<int>& g) {
  BMap m;
  std::vector<int> start(g.size() + 1, 0), sys_of;
  for (size_t s = 0; s < g.size(); ++s) {
    start[s + 1] = start[s] + g[s];
    for (int k = 0; k < g[s]; ++k) sys_of.push_back((int)s);
  }
  m.grid = start.back();
  m.start = dupload(start, b->owned);
  m.sys_of = dupload(sys_of.empty() ? std::vector<int>{0} : sys_of, b->owned);
  return m;
}

template <typename R>
void** make_table(ibg_batch* b, size_t offset) {
  std::vector<void*> p(b->sys.size());
  for (size_t s = 0; s < b->sys.size(); ++s) p[s] = (char*)b->sys[s]->dargs + offset;
  return dupload(p, b->owned);
}

template <typename R>
void batch_layout(ibg_batch* b) {
  using SA = SysArgs<R>;
  const size_t n = b->sys.size();
  b->t_pos = make_table<R>(b, offsetof(SA, pos));
  for (int w = 0; w < 2; ++w) {
    b->t_list[w] = make_table<R>(b, offsetof(SA, list) + w * sizeof(ListArgs));
    b->t_nb[w] = make_table<R>(b, offsetof(SA, nb) + w * sizeof(NBArgs<R>));
    b->t_col[w] = make_table<R>(b, offsetof(SA, col) + w * sizeof(CollectArgs<R>));
  }
  b->t_dist = make_table<R>(b, offsetof(SA, dist));
  b->t_bond = make_table<R>(b, offsetof(SA, bond));
  b->t_move = make_table<R>(b, offsetof(SA, move));
  b->t_mom = make_table<R>(b, offsetof(SA, mom));
  b->t_fin = make_table<R>(b, offsetof(SA, fin));
  std::vector<int> g(n);
  for (size_t s = 0; s < n; ++s) g[s] = b->sys[s]->g_pos;
  b->m_pos = make_map(b, g);
  for (size_t s = 0; s < n; ++s) g[s] = b->sys[s]->nvirta ? b->sys[s]->g_dist : 0;
  b->m_dist = make_map(b, g);
  for (size_t s = 0; s < n; ++s) b->any_vs |= b->sys[s]->nvirta > 0;
  for (size_t s = 0; s < n; ++s) b->any_com_carry |= b->sys[s]->vs_com_form == IBG_VS_COM_REFERENCE;
  for (size_t s = 0; s < n; ++s) g[s] = b->sys[s]->g_b;
  b->m_bond = make_map(b, g);
  for (size_t s = 0; s < n; ++s) g[s] = b->sys[s]->g_mv;
  b->m_move = make_map(b, g);
  for (size_t s = 0; s < n; ++s) g[s] = 1;
  b->m_fin = make_map(b, g);
  for (int w = 0; w < 2; ++w) {
    for (size_t s = 0; s < n; ++s) b->any_list[w] |= b->sys[s]->L[w].present;
    for (size_t s = 0; s < n; ++s) g[s] = b->sys[s]->L[w].present ? b->sys[s]->g_regrid[w] : 0;
    b->m_regrid[w] = make_map(b, g);
    for (size_t s = 0; s < n; ++s) g[s] = b->sys[s]->L[w].present ? b->sys[s]->g_list[w] : 0;
    b->m_list[w] = make_map(b, g);
    for (size_t s = 0; s < n; ++s) g[s] = b->sys[s]->L[w].present ? 1 : 0;
    b->m_scan[w] = make_map(b, g);
    // list build: one group per list form, each system with its own grid
    std::set<int> forms;
    for (size_t s = 0; s < n; ++s)
      if (b->sys[s]->L[w].present) forms.insert(b->sys[s]->L[w].form);
    for (int f : forms) {
      NBGroup grp;
      grp.T = 8;
      grp.form = f;
      for (size_t s = 0; s < n; ++s) {
        const DevList& L = b->sys[s]->L[w];
        g[s] = (L.present && L.form == f) ? b->sys[s]->g_build[w] : 0;
      }
      grp.map = make_map(b, g);
      b->lb[w].push_back(grp);
    }
    // nonbonded: one group per (labels mixed, smem, list form); the group's
    // resident blocks are shared among its systems in proportion to their
    // work units
    std::set<std::array<int, 3>> keys;
    auto key_of = [](const DevList& L) { return std::array<int, 3>{(int)L.mixed, (int)L.use_smem, L.form}; };
    for (size_t s = 0; s < n; ++s)
      if (b->sys[s]->L[w].present) keys.insert(key_of(b->sys[s]->L[w]));
    for (auto key : keys) {
      NBGroup grp;
      grp.mixed = key[0] != 0;
      grp.smem = key[1] != 0;
      grp.form = key[2];
      double units = 0;
      for (size_t s = 0; s < n; ++s) {
        const DevList& L = b->sys[s]->L[w];
        if (!(L.present && key_of(L) == key)) continue;
        grp.sm = std::max(grp.sm, nb_smem(b->sys[s], L));
        units += (double)L.nslices * ((L.w_cap + 7) / 8);
      }
      int per = 1;
      for (size_t s = 0; s < n; ++s) {
        const DevList& L = b->sys[s]->L[w];
        if (L.present && key_of(L) == key) {
          per = nb_occupancy<R, true>(b->sys[s], L, grp.sm);
          break;
        }
      }
      const double resident = (double)b->nsm * per;
      for (size_t s = 0; s < n; ++s) {
        const DevList& L = b->sys[s]->L[w];
        if (!(L.present && key_of(L) == key)) { g[s] = 0; continue; }
        const double u = (double)L.nslices * ((L.w_cap + 7) / 8);
        g[s] = std::max(1, std::min(L.grid_nb, (int)std::lround(resident * u / std::max(units, 1.0))));
      }
      grp.map = make_map(b, g);
      b->nb[w].push_back(grp);
    }
  }
}

enum BatchVariant : unsigned { BV_REBUILD = 1u, BV_MOMENTUM = 2u, BV_SCALE = 4u };

template <typename R>
void batch_enqueue(ibg_batch* b, unsigned v) {
  cudaStream_t st = b->st, st2 = b->st2;
  long long& n = b->launches;
  k_positions<R, true><<<b->m_pos.grid, 256, 0, st>>>(PosArgs{}, (const PosArgs* const*)b->t_pos, b->m_pos.m(), 1);
  ++n;
  if (b->any_com_carry) {
    k_vsite_chain<R, true><<<b->m_fin.grid, 256, 0, st>>>(PosArgs{}, (const PosArgs* const*)b->t_pos, b->m_fin.m());
    ++n;
  }
  // bonded branch
  CK(cudaEventRecord(b->fork_ev[0], st));
  CK(cudaStreamWaitEvent(st2, b->fork_ev[0], 0));
  k_bonded<R, true><<<b->m_bond.grid, 256, 0, st2>>>(BondedArgs<R>{}, (const BondedArgs<R>* const*)b->t_bond,
                                                     b->m_bond.m());
  ++n;
  // launches that follow a kernel of the same stream start by programmatic
  // dependent launch, as in one system's step
  using DA = const DistArgs<R>* const*;
  if (b->any_vs) {
    launch_on(st2, true, k_distribute<R, true>, b->m_dist.grid, 256, 0, DistArgs<R>{}, (DA)b->t_dist, b->m_dist.m(), 1);
    ++n;
  }
  CK(cudaEventRecord(b->fork_ev[1], st2));
  // list rebuild of the systems whose step rebuilds
  if (v & BV_REBUILD) {
    for (int w = 0; w < 2; ++w) {
      if (!b->any_list[w]) continue;
      const ListArgs* const* t = (const ListArgs* const*)b->t_list[w];
      const BMap& ml = b->m_list[w];
      k_regrid<R, true><<<b->m_regrid[w].grid, 256, 0, st>>>(ListArgs{}, t, b->m_regrid[w].m(), 0);
      launch_on(st, true, k_cell_assign<R, true>, ml.grid, 256, 0, ListArgs{}, t, ml.m(), 0);
      launch_on(st, true, k_scan_cells<true>, b->m_scan[w].grid, 1024, 0, ListArgs{}, t, b->m_scan[w].m(), 0);
      launch_on(st, true, k_cell_fill<true>, ml.grid, 256, 0, ListArgs{}, t, ml.m(), 0);
      launch_on(st, true, k_cell_rank<true>, ml.grid, 256, 0, ListArgs{}, t, ml.m(), 0);
      launch_on(st, true, k_reslot<R, true>, ml.grid, 256, 0, ListArgs{}, t, ml.m(), 0);
      launch_on(st, true, k_slot_of<R, true>, ml.grid, 256, 0, ListArgs{}, t, ml.m(), 0);
      n += 7;
      for (const NBGroup& grp : b->lb[w]) {
        const BlockMap bm = grp.map.m();
        if (grp.form == 1)
          launch_on(st, true, k_list_build_slices<true>, grp.map.grid, 256, 0, ListArgs{}, t, bm, 0);
        else
          launch_on(st, true, k_list_build_warp<R, 8, true>, grp.map.grid, 256, 0, ListArgs{}, t, bm, 0);
        ++n;
      }
    }
  }
  // nonbonded, bead list first; the FP32 path's pairs at the cutoff after
  // each list (one block per system with the list, as the cell scan)
  for (int w : {1, 0}) {
    for (const NBGroup& grp : b->nb[w]) {
      launch_on(st, true, nb_kernel<R, true>(grp.smem, grp.mixed, grp.form), grp.map.grid, 256, grp.sm, NBArgs<R>{},
                (const NBArgs<R>* const*)b->t_nb[w], grp.map.m());
      ++n;
    }
    if (b->prec == IBG_PREC_FP32_FIXED && b->any_list[w]) {
      launch_on(st, true, k_nb_near<true>, b->m_scan[w].grid, 256, 0, NBArgs<float>{},
                (const NBArgs<float>* const*)b->t_nb[w], b->m_scan[w].m());
      ++n;
    }
  }
  for (int w : {1, 0}) {
    if (!b->any_list[w]) continue;
    launch_on(st, true, k_nb_collect<R, true>, b->m_list[w].grid, 256, 0, CollectArgs<R>{},
              (const CollectArgs<R>* const*)b->t_col[w], b->m_list[w].m());
    ++n;
  }
  if (b->any_vs) {
    launch_on(st, true, k_distribute<R, true>, b->m_dist.grid, 256, 0, DistArgs<R>{}, (DA)b->t_dist, b->m_dist.m(), 0);
    ++n;
  }
  CK(cudaStreamWaitEvent(st, b->fork_ev[1], 0));
  k_move<R, true><<<b->m_move.grid, 256, 0, st>>>(MoveArgs<R>{}, (const MoveArgs<R>* const*)b->t_move, b->m_move.m());
  ++n;
  if (v & BV_MOMENTUM) {
    k_mom_sum<true><<<b->m_move.grid, 256, 0, st>>>(MomArgs{}, (const MomArgs* const*)b->t_mom, b->m_move.m());
    k_mom_apply<true><<<b->m_move.grid, 256, 0, st>>>(MomArgs{}, (const MomArgs* const*)b->t_mom, b->m_move.m());
    n += 2;
  }
  launch_on(st, true, k_finalize<true>, b->m_fin.grid, 1024, 0, FinalArgs{}, (const FinalArgs* const*)b->t_fin,
            b->m_fin.m());
  ++n;
  if (v & BV_SCALE) {
    k_scale_positions<R, true><<<b->m_move.grid, 256, 0, st>>>(MoveArgs<R>{}, (const MoveArgs<R>* const*)b->t_move,
                                                               b->m_move.m());
    ++n;
  }
}

void batch_enqueue_any(ibg_batch* b, unsigned v) {
  if (b->prec == IBG_PREC_FP32_FIXED) batch_enqueue<float>(b, v);
  else batch_enqueue<double>(b, v);
}

// Variant of batch step k: which optional stages some system needs.
unsigned batch_variant(const ibg_batch* b, const std::vector<int>& from, const std::vector<int>& last, int k) {
  unsigned v = 0;
  for (size_t s = 0; s < b->sys.size(); ++s) {
    const ibg_ctx* c = b->sys[s];
    const int step = from[s] + 1 + k;
    if (step > last[s]) continue;
    if (step % c->nupdate == 0) v |= BV_REBUILD;
    if (step % c->halt_drift == 0) v |= BV_MOMENTUM;
    if (c->ensemble == 2 && step % 10 == 0) v |= BV_SCALE;
  }
  return v;
}

}  // namespace

extern "C" {

int ibg_batch_create(ibg_ctx* const* ctxs, int n, ibg_batch** out) {
  if (!ctxs || n <= 0 || !out) return IBG_E_INVALID;
  *out = nullptr;
  auto b = std::make_unique<ibg_batch>();
  try {
    CK(cudaGetDevice(&b->dev));
    CK(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->dev));
    std::set<const ibg_ctx*> seen;
    for (int s = 0; s < n; ++s) {
      ibg_ctx* c = ctxs[s];
      if (!c || !c->state_set || c->in_batch || seen.count(c)) return IBG_E_INVALID;
      if (s > 0 && (c->prec != ctxs[0]->prec || c->dev != ctxs[0]->dev)) return IBG_E_INVALID;
      seen.insert(c);
      CK(cudaStreamSynchronize(c->st));
      b->sys.push_back(c);
    }
    b->prec = ctxs[0]->prec;
    CK(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&b->st2, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
      CK(cudaEventCreateWithFlags(&b->fork_ev[k], cudaEventDisableTiming));
      CK(cudaEventCreate(&b->run_ev[k]));
    }
    if (b->prec == IBG_PREC_FP32_FIXED) batch_layout<float>(b.get());
    else batch_layout<double>(b.get());
    for (ibg_ctx* c : b->sys) c->in_batch = true;
    CK(cudaDeviceSynchronize());
  } catch (CudaError& e) {
    b->owned.free_all();
    return IBG_E_CUDA;
  }
  *out = b.release();
  return IBG_OK;
}

int ibg_batch_run(ibg_batch* b, int nsteps, const int* last_step, ibg_obs* last_obs) {
  if (!b || nsteps < 0) return IBG_E_INVALID;
  const size_t n = b->sys.size();
  try {
    std::vector<int> last(n), from(n);
    for (size_t s = 0; s < n; ++s) {
      ibg_ctx* c = b->sys[s];
      from[s] = c->step_now;
      last[s] = c->step_now + nsteps;
      if (last_step) last[s] = std::max(c->step_now, std::min(last[s], last_step[s]));
    }
    float total_ms = 0.f;
    for (int attempt = 0; attempt < 8; ++attempt) {
      int need = 0;
      for (size_t s = 0; s < n; ++s) need = std::max(need, last[s] - from[s]);
      if (need == 0) break;
      for (size_t s = 0; s < n; ++s) set_step_counter(b->sys[s], from[s], INT_MAX, last[s], true);
      CK(cudaEventRecord(b->run_ev[0], b->st));
      for (int k = 0; k < need; ++k) {
        const unsigned v = batch_variant(b, from, last, k);
        auto it = b->graphs.find(v);
        if (it == b->graphs.end()) {
          cudaGraph_t g;
          CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
          const long long l0 = b->launches;
          batch_enqueue_any(b, v);
          CK(cudaStreamEndCapture(b->st, &g));
          b->launches_per_variant[v & 7] = b->launches - l0;
          b->launches = l0;
          cudaGraphExec_t ge;
          CK(cudaGraphInstantiate(&ge, g, 0));
          CK(cudaGraphDestroy(g));
          it = b->graphs.emplace(v, ge).first;
        }
        CK(cudaGraphLaunch(it->second, b->st));
        b->launches += b->launches_per_variant[v & 7];
      }
      CK(cudaEventRecord(b->run_ev[1], b->st));
      CK(cudaStreamSynchronize(b->st));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, b->run_ev[0], b->run_ev[1]));
      total_ms += ms;
      // systems whose list storage overflowed: grow it and repeat from the
      // step that aborted; the others are done
      bool again = false;
      for (size_t s = 0; s < n; ++s) {
        ibg_ctx* c = b->sys[s];
        if (grow_lists(c)) {
          int st = 0;
          CK(cudaMemcpy(&st, &c->sc->step, sizeof(int), cudaMemcpyDeviceToHost));
          from[s] = st - 1;
          again = true;
        } else {
          from[s] = last[s];
        }
      }
      if (!again) break;
    }
    b->run_ms = total_ms;
    // every system's status: a failing system does not hide the others'
    int first_rc = IBG_OK;
    for (size_t s = 0; s < n; ++s) {
      ibg_ctx* c = b->sys[s];
      int rc = IBG_OK;
      if (from[s] < last[s]) rc = fail(c, IBG_E_CAPACITY, "neighbour-list storage could not be sized");
      c->step_now = from[s];
      if (!rc) rc = check_device(c);
      if (last_obs) {
        read_obs(c, &last_obs[s]);
        last_obs[s].status = rc;
      }
      if (rc && !first_rc) {
        first_rc = rc;
        bfail(b, rc, "system " + std::to_string(s) + ": " + c->err);
      }
    }
    return first_rc;
  } catch (CudaError& e) {
    return bfail(b, IBG_E_CUDA, cudaGetErrorString(e.e));
  }
}

int ibg_batch_size(const ibg_batch* b) { return b ? (int)b->sys.size() : 0; }

int ibg_batch_get_timing(const ibg_batch* b, double* run_ms, long long* launches) {
  if (!b) return IBG_E_INVALID;
  if (run_ms) *run_ms = b->run_ms;
  if (launches) *launches = b->launches;
  return IBG_OK;
}

const char* ibg_batch_last_error(const ibg_batch* b) { return b ? b->err.c_str() : "null batch"; }

void ibg_batch_destroy(ibg_batch* b) {
  if (!b) return;
  cudaStreamSynchronize(b->st);
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->owned.free_all();
  for (int k = 0; k < 2; ++k) {
    if (b->fork_ev[k]) cudaEventDestroy(b->fork_ev[k]);
    if (b->run_ev[k]) cudaEventDestroy(b->run_ev[k]);
  }
  if (b->st2) cudaStreamDestroy(b->st2);
  if (b->st) cudaStreamDestroy(b->st);
  for (ibg_ctx* c : b->sys) c->in_batch = false;
  delete b;
}

}  // extern "C"
