// Kernels of the B200 force-and-integrate step.  Each kernel names the
// reference routine whose arithmetic it restates.  The file is compiled with
// --fmad=false, IEEE division and square root, so every REAL*4 expression is
// evaluated with the same roundings as gfortran -O2 on x86-64 (no FMA).
#pragma once
#include "ibg_common.cuh"

namespace ibg {

// ------------------------------------------------------------ precision policy
// FP32 path: REAL*4 geometry and table math, forces summed as 64-bit
// fixed-point integers (order independent, reproducible run to run).
// FP64 path: the same algorithm in double with double atomics.
template <typename R>
struct Prec;

template <>
struct Prec<float> {
  using pos_t = float4;
  using acc_t = unsigned long long;  // global accumulator element
  using reg_t = long long;           // per-thread partial sum
  static __device__ __forceinline__ reg_t q(float v, unsigned* err) {
    if (!(fabsf(v) < kFixMax)) {  // also catches NaN
      atomicOr(err, EB_FIXED);
      v = (v == v) ? copysignf(kFixMax, v) : 0.0f;
    }
    return __float2ll_rn(v * kFixScale);
  }
  static __device__ __forceinline__ void add(acc_t* p, reg_t v) { atomicAdd(p, (unsigned long long)v); }
  static __device__ __forceinline__ double get(acc_t v) { return (double)(long long)v * kFixInv; }
  static __device__ __forceinline__ reg_t from_double(double v, unsigned* err) {
    double s = v * 4294967296.0;
    if (!(fabs(s) < 9.2e18)) {
      atomicOr(err, EB_FIXED);
      s = (s == s) ? copysign(9.2e18, s) : 0.0;
    }
    return __double2ll_rn(s);
  }
  static __device__ __forceinline__ float tbits(int b) { return __int_as_float(b); }
  static __device__ __forceinline__ int bits(float w) { return __float_as_int(w); }
};

template <>
struct Prec<double> {
  using pos_t = double4;
  using acc_t = double;
  using reg_t = double;
  static __device__ __forceinline__ reg_t q(double v, unsigned*) { return v; }
  static __device__ __forceinline__ void add(acc_t* p, reg_t v) { atomicAdd(p, v); }
  static __device__ __forceinline__ double get(acc_t v) { return v; }
  static __device__ __forceinline__ reg_t from_double(double v, unsigned*) { return v; }
  static __device__ __forceinline__ double tbits(int b) { return __longlong_as_double((long long)b); }
  static __device__ __forceinline__ int bits(double w) { return (int)__double_as_longlong(w); }
};

__device__ __forceinline__ float r_round(float x) { return roundf(x); }
__device__ __forceinline__ double r_round(double x) { return round(x); }
__device__ __forceinline__ float r_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double r_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float r_acos(float x) { return acosf(x); }
__device__ __forceinline__ double r_acos(double x) { return acos(x); }
__device__ __forceinline__ float r_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double r_abs(double x) { return fabs(x); }

// Fortran INT: truncation; values outside the int range saturate.
template <typename R>
__device__ __forceinline__ int fint(R x) {
  if (!(x == x)) return INT_MIN;
  if (x >= (R)2147483647.0) return INT_MAX;
  if (x <= (R)-2147483647.0) return -INT_MAX;
  return (int)x;
}

template <typename R>
__device__ __forceinline__ void box_of(const Scalars* sc, R* b, R* bi, R* b2);
template <>
__device__ __forceinline__ void box_of<float>(const Scalars* sc, float* b, float* bi, float* b2) {
  for (int c = 0; c < 3; ++c) { b[c] = sc->boxf[c]; bi[c] = sc->boxinvf[c]; b2[c] = sc->box2f[c]; }
}
template <>
__device__ __forceinline__ void box_of<double>(const Scalars* sc, double* b, double* bi, double* b2) {
  for (int c = 0; c < 3; ++c) { b[c] = sc->box[c]; bi[c] = sc->boxinv[c]; b2[c] = sc->box2[c]; }
}

// ------------------------------------------------------------------ per step
// Fold into the primary box (SHIFT.f90:37-43): applied to all three
// components when any one lies outside [-L/2, L/2].
template <typename R>
__device__ __forceinline__ void fold3(R* r, const R* b2) {
  bool out = false;
#pragma unroll
  for (int c = 0; c < 3; ++c) out |= (r[c] > b2[c]) || (r[c] < -b2[c]);
  if (!out) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    R x = r[c] / b2[c];
    R sp = x - (R)2.0 * (R)fint(x / (R)2.0);
    r[c] = (sp - (R)2.0 * (R)fint(sp)) * b2[c];
  }
}

// A position as 32-bit fractions of the box per axis: round(x/L * 2^32)
// modulo 2^32, in FP64.  The wrapped difference of two of them, read as a
// signed integer, is the nearest-image displacement in units of L/2^32, exact
// to one unit (L/2^32: 3e-9 nm for a 12.6 nm box), whatever the particles'
// distance from the box centre.
__device__ __forceinline__ int4 box_fraction(const double* x, const double* boxinv, int w) {
  int q[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double t = x[c] * boxinv[c];
    t -= floor(t + 0.5);
    q[c] = (int)(unsigned)(long long)llrint(t * 4294967296.0);
  }
  return make_int4(q[0], q[1], q[2], w);
}

struct PosArgs {
  Scalars* sc;
  int natoms, nvirta;
  int nupdate, nmts;
  const double* S;     // unwrapped positions (3,NITEMS), FP64 state
  double* Svs;         // VS rows of S (written for the FP64 path and output)
  const int* tbits;    // type | label<<16 per particle
  const int* gslot;    // slot*2 + list per particle
  void* pos4[2];       // per-list wrapped positions, slot order
  int4* posq[2];       // FP32 path: per-list positions as 32-bit fractions of the box, slot order
  const int* vcenter;  // VIRT_CENTER (0-based atom id or -1 for COM)
  const int* vnum;     // members per VS
  const int* vmem;     // members, [v*15 + k], 0-based
  const float* vmass;  // member masses per [v*15 + k]
  const float* vinv;   // VIRT_INVMASS per VS
  int com_carry;       // 1: the reference's centre-of-mass form (VIRTUAL_DEF.f90:31)
  // com_carry: per site the mass-weighted y and z member terms (R[32]: y at
  // 0..14, z at 16..30), then the x coordinates (R[nvirta]), then the member
  // counts (int[nvirta], -1 for a centre-atom site), for k_vsite_chain
  void* chain;
};

template <typename R>
struct ChainView {
  R* terms;
  R* xs;
  int* n;
  __device__ ChainView(const PosArgs& a)
      : terms((R*)a.chain), xs((R*)a.chain + 32 * (size_t)a.nvirta), n((int*)(xs + a.nvirta)) {}
};

// Bytes of the com_carry scratch for nvirta sites.
template <typename R>
constexpr size_t chain_bytes(long long nvirta) {
  return (size_t)nvirta * (33 * sizeof(R) + sizeof(int));
}

// A particle's wrapped position into its list's slot: the FP32/FP64 record
// with its type/label word, and on the FP32 path the 32-bit box fractions
// from the FP64 value sd.
template <typename R>
__device__ __forceinline__ void store_position(const PosArgs& a, const R* b2, const double* boxinv, int i, const R* s,
                                               const double* sd) {
  using PT = typename Prec<R>::pos_t;
  const int g = a.gslot[i];
  const int tb = a.tbits[i];
  R r[3] = {s[0], s[1], s[2]};
  fold3<R>(r, b2);
  PT p;
  p.x = r[0]; p.y = r[1]; p.z = r[2];
  p.w = Prec<R>::tbits(tb);
  ((PT*)a.pos4[g & 1])[g >> 1] = p;
  if (a.posq[g & 1]) a.posq[g & 1][g >> 1] = box_fraction(sd, boxinv, tb);
}

// SHIFT.f90:33-45 for atoms and VIRTUAL_DEF.f90:19-47 for virtual sites
// (centre-of-mass sums with all three components reset per site, or the
// reference's form, where only the x sum is reset: com_carry).
// begin: when set, block 0 first starts the step: it advances the step
// counter and sets this step's flags, or marks the step skipped when the run
// aborted.  A system that has run its last step (done) is left as it is, so
// its virtual-site rows keep the values of its last step.
template <typename R, bool B>
__global__ void k_positions(__grid_constant__ const PosArgs a0, const PosArgs* const* tab, const BlockMap bm,
                            int begin) {
  using PT = typename Prec<R>::pos_t;
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  const PosArgs& a = B ? *tab[bk.sys] : a0;
  Scalars* sc = a.sc;
  if (sc->done) {
    if (begin && bk.b == 0 && threadIdx.x == 0) sc->skip = 1;
    return;
  }
  if (begin && bk.b == 0 && threadIdx.x == 0) {
    if (sc->abort) {
      sc->skip = 1;
    } else {
      sc->skip = 0;
      for (int q = 0; q < 4; ++q) sc->work[q] = 0u;
      const int st = ++sc->step;
      sc->rebuild = (st % a.nupdate) == 0;
      sc->mts_m = a.nmts > 0 ? st % (3 + a.nmts) : -1;
      sc->miu = 1.0;
    }
  }
  R b[3], bi[3], b2[3];
  box_of<R>(sc, b, bi, b2);
  const double boxinv[3] = {sc->boxinv[0], sc->boxinv[1], sc->boxinv[2]};
  // sd: the position in FP64 for the fixed-point copy (FP32 path).  The slot
  // and label are loaded before the first store (the arrays may alias as far
  // as the compiler knows, and a load after a store would wait for it).
  auto store = [&](int i, const R* s, const double* sd) { store_position<R>(a, b2, boxinv, i, s, sd); };
  for (int i = bk.b * blockDim.x + threadIdx.x; i < a.natoms; i += bk.g * blockDim.x) {
    R s[3];
    double sd[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      sd[c] = a.S[3 * (size_t)i + c];
      s[c] = (R)sd[c];
    }
    store(i, s, sd);
  }
  const int hl = threadIdx.x & 15;
  // VIRTUAL_DEF.f90:30-39 with all three sums reset per site: 16 lanes per
  // site (half a warp), lane k holding member k's mass-weighted position; the
  // sum runs over the members in order (0 + p0 + p1 + ...), as the
  // reference's loop does.  The loop over sites is uniform within a warp, so
  // its shuffles see all 32 lanes.  In the reference's form (com_carry) only
  // the x sum is reset per site (:31): the x coordinate is formed here, and
  // the y and z member terms go to the chain scratch, whose sums
  // k_vsite_chain runs on from site to site.
  const ChainView<R> cv(a);
  const int w0 = (bk.b * blockDim.x + threadIdx.x) >> 5, nw = (bk.g * blockDim.x) >> 5;
  for (int w = w0; 2 * w < a.nvirta; w += nw) {
    const int v = 2 * w + ((threadIdx.x >> 4) & 1);
    const bool valid = v < a.nvirta;
    const int ctr = valid ? a.vcenter[v] : 0;
    const int nm = valid && ctr < 0 ? a.vnum[v] : 0;
    R pm[3] = {0, 0, 0};
    if (hl < nm) {
      const int m = a.vmem[v * 15 + hl];
      const R mm = (R)a.vmass[v * 15 + hl];
#pragma unroll
      for (int c = 0; c < 3; ++c) pm[c] = mm * (R)a.S[3 * (size_t)m + c];
    }
    if (a.com_carry && hl < nm) {
      cv.terms[32 * (size_t)v + hl] = pm[1];
      cv.terms[32 * (size_t)v + 16 + hl] = pm[2];
    }
    R acc[3] = {0, 0, 0};
#pragma unroll
    for (int q = 0; q < 15; ++q) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const R x = __shfl_sync(0xffffffffu, pm[c], q, 16);
        if (q < nm) acc[c] = acc[c] + x;
      }
    }
    if (!valid || hl != 0) continue;
    if (a.com_carry) {
      cv.n[v] = ctr >= 0 ? -1 : nm;  // -1: a centre-atom site, outside the sums
      if (ctr < 0) {  // finished by k_vsite_chain
        cv.xs[v] = acc[0] * (R)a.vinv[v];
        continue;
      }
    }
    R s[3];
    if (ctr >= 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) s[c] = (R)a.S[3 * (size_t)ctr + c];
    } else {
      const R inv = (R)a.vinv[v];
#pragma unroll
      for (int c = 0; c < 3; ++c) s[c] = acc[c] * inv;
    }
    double sd[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      sd[c] = (double)s[c];
      a.Svs[3 * (size_t)v + c] = sd[c];
    }
    store(a.natoms + v, s, sd);
  }
}

// VIRTUAL_DEF.f90:30-39 as the reference runs it (com_carry): SUMTOTXYZ(2)
// and (3) are not reset before a centre-of-mass site (only (1) is, :31), so
// the y and z sums run on from one such site to the next, from zero at the
// start of the pass.  k_positions has formed each site's x coordinate and its
// mass-weighted y and z member terms; one block per system adds the terms in
// the reference's order.  The sites go through shared memory in chunks, two
// buffers: thread 0 runs the sums over one chunk while warps 1..7 load the
// next and finish the one before (the sums times VIRT_INVMASS, the FP64 row
// and the list record).
// A row of 32 values from shared memory in 16-byte loads issued back to back
// (asm volatile keeps them together, ahead of the arithmetic that uses them).
__device__ __forceinline__ void lds_row(float* t, const float* row) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(row);
#pragma unroll
  for (int k = 0; k < 8; ++k)
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(t[4 * k]), "=f"(t[4 * k + 1]), "=f"(t[4 * k + 2]), "=f"(t[4 * k + 3])
                 : "r"(a + 16 * k));
}
__device__ __forceinline__ void lds_row(double* t, const double* row) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(row);
#pragma unroll
  for (int k = 0; k < 16; ++k)
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(t[2 * k]), "=d"(t[2 * k + 1]) : "r"(a + 16 * k));
}

template <typename R, bool B>
__global__ void __launch_bounds__(256) k_vsite_chain(__grid_constant__ const PosArgs a0, const PosArgs* const* tab,
                                                     const BlockMap bm) {
  constexpr int kC = sizeof(R) == 4 ? 128 : 64;  // sites per chunk
  __shared__ __align__(16) R s_t[2][kC][32];
  __shared__ int s_n[2][kC];
  __shared__ R s_c[2][kC][2];
  const Blk bk = blk<B>(bm);
  const PosArgs& a = B ? *tab[bk.sys] : a0;
  Scalars* sc = a.sc;
  if (!a.com_carry || bk.b != 0 || sc->done) return;
  const ChainView<R> cv(a);
  R b[3], bi[3], b2[3];
  box_of<R>(sc, b, bi, b2);
  const double boxinv[3] = {sc->boxinv[0], sc->boxinv[1], sc->boxinv[2]};
  const int nv = a.nvirta;
  // chunk c0 into buffer q, by the threads from t0 on
  auto load = [&](int c0, int q, int t0) {
    const int nc = min(kC, nv - c0);
    for (int k = (int)threadIdx.x - t0; k < nc * 32; k += (int)blockDim.x - t0)
      s_t[q][k >> 5][k & 31] = cv.terms[32 * (size_t)c0 + k];
    for (int k = (int)threadIdx.x - t0; k < nc; k += (int)blockDim.x - t0) s_n[q][k] = cv.n[c0 + k];
  };
  // the sites of chunk c0 from the sums in s_c[q], by the threads from t0 on:
  // the sums times VIRT_INVMASS, the FP64 row and the list record
  auto finish = [&](int c0, int q, int t0) {
    const int nc = min(kC, nv - c0);
    for (int u = (int)threadIdx.x - t0; u < nc; u += (int)blockDim.x - t0) {
      const int v = c0 + u;
      if (cv.n[v] < 0) continue;  // a centre-atom site: k_positions placed it
      const R inv = (R)a.vinv[v];
      R sv[3] = {cv.xs[v], s_c[q][u][0] * inv, s_c[q][u][1] * inv};
      double sd[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sd[c] = (double)sv[c];
        a.Svs[3 * (size_t)v + c] = sd[c];
      }
      store_position<R>(a, b2, boxinv, a.natoms + v, sv, sd);
    }
  };
  if (nv > 0) load(0, 0, 0);
  __syncthreads();
  // step j: thread 0 sums chunk j (buffer j&1) while warps 1..7 load chunk
  // j+1 into the other buffer and finish chunk j-1 from its sums
  R cy = 0, cz = 0;  // the running sums, held by thread 0
  int last = -1;     // the chunk summed last, still to be finished
  for (int c0 = 0, q = 0; c0 < nv; c0 += kC, q ^= 1) {
    const int nc = min(kC, nv - c0);
    if (threadIdx.x == 0) {
      // two sites at a time: both sites' terms are loaded (whole rows, the
      // unused slots included) before the first addition, so the additions
      // wait on one another only
      for (int u = 0; u < nc; u += 2) {
        const int u1 = min(u + 1, nc - 1);
        R t0[32], t1[32];
        lds_row(t0, s_t[q][u]);
        lds_row(t1, s_t[q][u1]);
        const int n0 = s_n[q][u], n1 = s_n[q][u1];
#pragma unroll
        for (int k = 0; k < 15; ++k) {
          if (k < n0) {
            cy = cy + t0[k];
            cz = cz + t0[16 + k];
          }
        }
        s_c[q][u][0] = cy;
        s_c[q][u][1] = cz;
        if (u1 == u) break;
#pragma unroll
        for (int k = 0; k < 15; ++k) {
          if (k < n1) {
            cy = cy + t1[k];
            cz = cz + t1[16 + k];
          }
        }
        s_c[q][u1][0] = cy;
        s_c[q][u1][1] = cz;
      }
    } else if (threadIdx.x >= 32) {
      if (c0 + kC < nv) load(c0 + kC, q ^ 1, 32);
      if (last >= 0) finish(last, q ^ 1, 32);
    }
    __syncthreads();  // buffer q is summed, q^1 loaded and its sums used
    last = c0;
  }
  if (last >= 0) finish(last, ((last / kC) & 1), 0);
}

// ------------------------------------------------------------ cell lists
struct ListArgs {
  Scalars* sc;
  int n;             // particles in the list
  int which;         // 0 atoms, 1 beads
  int natoms;        // NATOMS (VS-VS exclusion)
  int hybrid;        // IBRDESCR == 0
  int maxnab;        // reference STOP threshold
  int cell_cap;      // capacity of the cell arrays
  int nslices;       // slices of the list storage
  float rlist, rlistsq;
  double rlistd, rlistsqd;
  // FP32 path: accepted pairs at r^2 >= rgroupsq (rc + skin/4, squared) are
  // stored after the others, each group in the reference's order, so that
  // list rows far beyond the cutoff are mostly skipped whole by the
  // nonbonded kernel's warps; 0 keeps the reference's order throughout
  float rgroupsq;
  const int* idx;    // INDEX_LIST, 0-based global ids
  int* cell_of;      // [n] cell of list entry A
  int* cell_count;   // [cell_cap]
  int* cell_start;   // [cell_cap + 1]
  int* cell_fill;    // [cell_cap]
  int* sorted;       // [n] slot -> A
  int* sorted_new;   // [n]
  int* slot_of;      // [n] A -> slot
  int* slot_of_new;  // [n]
  int* gslot;        // [NITEMS]
  void* pos4;        // [n]
  void* pos4_new;    // [n]
  int4* posq;        // [n] FP32 path: fixed-point positions (box fractions), or null
  int4* posq_new;    // [n]
  int* counts;       // [n] per slot
  int* slice_w;      // [nslices] rows of 32 entries used by each slice
  int* entries;      // list storage: slice g owns rows [g*w_cap, (g+1)*w_cap) of 32 entries
  int w_cap;         // rows of 32 entries per slice
  const int* excl_n; // CONNECTIONS, by global id
  const int* excl;   // CONNECTED_TO, [i*20 + c], 0-based
};

// List-rebuild kernels run when the step rebuilds its lists (or always, for
// the rebuild of ibg_set_state) and the step is not skipped.
//
// UPDATE_NEIGHBOURLIST.F90:14-48 / ALLOCATEVAR2.f90:19-42: cells per
// dimension = INT(BOX/RLIST).  The grid also clears the cell counters.
template <typename R, bool B>
__global__ void k_regrid(__grid_constant__ const ListArgs L0, const ListArgs* const* tab, const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  const ListArgs& L = B ? *tab[bk.sys] : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  for (int c = bk.b * blockDim.x + threadIdx.x; c < L.cell_cap; c += bk.g * blockDim.x) L.cell_count[c] = 0;
  for (int g = bk.b * blockDim.x + threadIdx.x; g < L.nslices; g += bk.g * blockDim.x) L.slice_w[g] = 0;
  if (threadIdx.x || bk.b) return;
  int nc[3];
  for (int c = 0; c < 3; ++c) {
    if (sizeof(R) == 4) nc[c] = fint(sc->boxf[c] / L.rlist);
    else nc[c] = fint(sc->box[c] / L.rlistd);
  }
  bool bad = nc[0] < 3 || nc[1] < 3 || nc[2] < 3;
  long long tot = (long long)nc[0] * nc[1] * nc[2];
  if (bad) atomicOr(&sc->err, EB_CELL_GRID);
  if (tot > L.cell_cap) atomicOr(&sc->err, EB_CAPACITY);
  if (bad || tot > L.cell_cap) nc[0] = nc[1] = nc[2] = 1;
  for (int c = 0; c < 3; ++c) sc->ncell[L.which][c] = nc[c];
}

// LINKS.f90:16-18.  A component equal to NCELL (coordinate at +L/2 after
// rounding) would address a cell outside the grid; it is clamped and counted.
template <typename R, bool B>
__global__ void k_cell_assign(__grid_constant__ const ListArgs L0, const ListArgs* const* tab, const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  using PT = typename Prec<R>::pos_t;
  const Blk bk = blk<B>(bm);
  const ListArgs& L = B ? *tab[bk.sys] : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  const int nx = sc->ncell[L.which][0], ny = sc->ncell[L.which][1], nz = sc->ncell[L.which][2];
  R b[3], bi[3], b2[3];
  box_of<R>(sc, b, bi, b2);
  const PT* pos = (const PT*)L.pos4;
  for (int a = bk.b * blockDim.x + threadIdx.x; a < L.n; a += bk.g * blockDim.x) {
    PT p = pos[L.slot_of[a]];
    R x[3] = {p.x, p.y, p.z};
    int nc[3] = {nx, ny, nz}, k[3];
    int clamps = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      k[c] = fint((x[c] * bi[c] + (R)0.5) * (R)nc[c]);
      if (k[c] >= nc[c]) { k[c] = nc[c] - 1; ++clamps; }
      if (k[c] < 0) { k[c] = 0; ++clamps; }
    }
    if (clamps) atomicAdd(&sc->cell_clamps, (unsigned long long)clamps);
    int cell = k[0] * nz * ny + k[1] * nz + k[2];
    L.cell_of[a] = cell;
    atomicAdd(&L.cell_count[cell], 1);
  }
}

// Exclusive scan of the cell counts by one block per system (cell_start has
// cell_cap + 1 entries); clears the fill counters.
template <bool B>
__global__ void k_scan_cells(__grid_constant__ const ListArgs L0, const ListArgs* const* tab, const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  const ListArgs& L = B ? *tab[bk.sys] : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  const int* in = L.cell_count;
  int* out = L.cell_start;
  int* zero = L.cell_fill;
  const int m = L.cell_cap;
  __shared__ int wsum[32];
  const int t = threadIdx.x, T = blockDim.x, lane = t & 31, warp = t >> 5, nw = (T + 31) >> 5;
  // tiles of V*T consecutive cells, thread t holding cells V*t..V*t+V-1 of
  // the tile (read and written as int4 where the tile is whole), the tiles in
  // order with the running total carried from one to the next
  constexpr int V = 16;
  int carry = 0;
  for (int base = 0; base < m; base += V * T) {
    const int i0 = base + V * t;
    const bool whole = i0 + V <= m;
    int x[V], s = 0;
    if (whole) {
#pragma unroll
      for (int j = 0; j < V / 4; ++j) {
        const int4 q = ((const int4*)(in + i0))[j];
        x[4 * j] = q.x; x[4 * j + 1] = q.y; x[4 * j + 2] = q.z; x[4 * j + 3] = q.w;
      }
    } else {
#pragma unroll
      for (int j = 0; j < V; ++j) x[j] = i0 + j < m ? in[i0 + j] : 0;
    }
#pragma unroll
    for (int j = 0; j < V; ++j) s += x[j];
    int v = s;  // inclusive scan of the threads' sums: warps, then warp totals
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    if (lane == 31) wsum[warp] = v;
    __syncthreads();
    if (warp == 0) {
      int w = lane < nw ? wsum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    int run = carry + v - s + (warp ? wsum[warp - 1] : 0);
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int e = run;
      run += x[j];
      x[j] = e;
    }
    if (whole) {
#pragma unroll
      for (int j = 0; j < V / 4; ++j) {
        ((int4*)(out + i0))[j] = make_int4(x[4 * j], x[4 * j + 1], x[4 * j + 2], x[4 * j + 3]);
        ((int4*)(zero + i0))[j] = make_int4(0, 0, 0, 0);
      }
    } else {
#pragma unroll
      for (int j = 0; j < V; ++j)
        if (i0 + j < m) {
          out[i0 + j] = x[j];
          zero[i0 + j] = 0;
        }
    }
    carry += wsum[nw - 1];
    __syncthreads();  // wsum is rewritten by the next tile
  }
  if (t == 0) out[m] = carry;
}

template <bool B>
__global__ void k_cell_fill(__grid_constant__ const ListArgs L0, const ListArgs* const* tab, const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  const ListArgs& L = B ? *tab[bk.sys] : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  for (int a = bk.b * blockDim.x + threadIdx.x; a < L.n; a += bk.g * blockDim.x) {
    int c = L.cell_of[a];
    int s = L.cell_start[c] + atomicAdd(&L.cell_fill[c], 1);
    L.sorted_new[s] = a;
  }
}

// Within a cell the reference's linked list visits entries by decreasing A
// (LINKS.f90:19-20); slots are kept in increasing A so the list build can
// walk them backwards.  k_cell_fill placed a cell's entries in arbitrary order
// (atomics); here each entry finds its rank among its cell's entries.
template <bool B>
__global__ void k_cell_rank(__grid_constant__ const ListArgs L0, const ListArgs* const* tab, const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  const ListArgs& L = B ? *tab[bk.sys] : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  for (int s = bk.b * blockDim.x + threadIdx.x; s < L.n; s += bk.g * blockDim.x) {
    const int a = L.sorted_new[s];
    const int c = L.cell_of[a];
    const int b = L.cell_start[c], e = L.cell_start[c + 1];
    int rank = 0;
    for (int k = b; k < e; ++k) rank += L.sorted_new[k] < a;
    L.slot_of_new[b + rank] = a;  // scratch: the ordered cell segment
  }
}

// New slot order: positions move to their new slots, and the slot of every
// entry (and of its global particle) is updated.  Reads the ordered cells from
// the scratch k_cell_rank wrote; writes the new order to sorted.
template <typename R, bool B>
__global__ void k_reslot(__grid_constant__ const ListArgs L0, const ListArgs* const* tab, const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  using PT = typename Prec<R>::pos_t;
  const Blk bk = blk<B>(bm);
  const ListArgs& L = B ? *tab[bk.sys] : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  for (int s = bk.b * blockDim.x + threadIdx.x; s < L.n; s += bk.g * blockDim.x) {
    int a = L.slot_of_new[s];
    ((PT*)L.pos4_new)[s] = ((const PT*)L.pos4)[L.slot_of[a]];
    if (L.posq) L.posq_new[s] = L.posq[L.slot_of[a]];
    L.sorted[s] = a;
    L.gslot[L.idx[a]] = s * 2 + L.which;
  }
}

// slot_of from the new order, and the positions into their new slots (after
// k_reslot).
template <typename R, bool B>
__global__ void k_slot_of(__grid_constant__ const ListArgs L0, const ListArgs* const* tab, const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  using PT = typename Prec<R>::pos_t;
  const Blk bk = blk<B>(bm);
  const ListArgs& L = B ? *tab[bk.sys] : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  for (int s = bk.b * blockDim.x + threadIdx.x; s < L.n; s += bk.g * blockDim.x) {
    L.slot_of[L.sorted[s]] = s;
    ((PT*)L.pos4)[s] = ((const PT*)L.pos4_new)[s];
    if (L.posq) L.posq[s] = L.posq_new[s];
  }
}

// NEW_NEIGHBOUR_WITHLIST.f90:34-123 for lists of up to a few hundred
// thousand particles.  A block builds the lists of one cell's
// particles at a time (cells taken dynamically).  The candidates of the cell --
// its own slots, then the slots of the 13 cells of the MAPS.f90:39-51
// stencil, each run by decreasing A -- are staged once in shared memory, in
// that order, with their slot numbers; every particle of the cell then reads
// them from there.  A warp builds one particle's list: its candidates are the
// staged ones from just below its own slot to the end, which is the
// reference's order (its own cell below it by decreasing A, then the stencil
// cells), visited 32 at a time, one per lane; a ballot and a prefix count keep
// the accepted ones in that order.  A cell whose candidates do not fit the
// staging buffer reads them from global memory instead (same order).  The
// distance test runs first and the exclusion test only for candidates inside
// RLIST (the accepted set is the same); exclusions are compared as slots of
// this list, and a virtual site is recognised by its label in the position's
// w, so no candidate's global id is loaded.  The list is stored in the
// nonbonded kernel's layout: T lanes per slot, slices of P = 32/T slots, entry
// k of slot s (slice g) at (g*w_cap + k/T)*32 + (s%P)*T + k%T.  A slot that
// needs more than w_cap rows records its need and raises the abort flag (the
// host enlarges the storage and repeats the step).
// The 13 neighbour cells of the half stencil in MAPS.f90:39-51 order.
#define IBG_HALF_STENCIL                                                                                    \
  {{1, 0, 0}, {1, 1, 0},  {0, 1, 0},  {-1, 1, 0}, {1, 0, -1}, {1, 1, -1}, {0, 1, -1},                        \
   {-1, 1, -1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}, {-1, 1, 1}, {0, 0, 1}}
__constant__ int kStencil[13][3] = IBG_HALF_STENCIL;
static const int kStencilHost[13][3] = IBG_HALF_STENCIL;  // the same, for host code

// Candidates one block stages (positions and slots): 2,304 in FP32 (about 160
// particles per cell), 1,152 in FP64, within 48 KB of static shared memory.
// A staged slot carries its run (0..13) in bits 27..30, so lists hold fewer
// than 2^27 particles.
constexpr int kSlotMask = (1 << 27) - 1;
// Entries of the outer group (ListArgs::rgroupsq) a list build holds back to
// append after the others: per warp in the warp-per-particle build, per
// thread in the thread-per-particle build.
constexpr int kLateWarp = 48;
constexpr int kLateThread = 24;
template <typename R>
struct ListStage {
  static constexpr int cap = sizeof(R) == 4 ? 2304 : 1152;
};

template <typename R, int T, bool B>
__global__ void __launch_bounds__(256, 4) k_list_build_warp(__grid_constant__ const ListArgs L0, const ListArgs* const* tab,
                                                       const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  using PT = typename Prec<R>::pos_t;
  constexpr int kCap = ListStage<R>::cap;
  constexpr int kWarps = 8;  // blockDim.x = 256
  const Blk bk = blk<B>(bm);
  __shared__ ListArgs s_args;
  if (B) stage_args(&s_args, tab[bk.sys]);
  const ListArgs& L = B ? s_args : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  constexpr int P = 32 / T;
  __shared__ PT s_pos[kCap];
  __shared__ int s_slot[kCap];          // slot | run << 27
  __shared__ int s_hi[14], s_pre[15];  // run u: slots s_hi[u] down, staged from s_pre[u]
  __shared__ R s_sh[14][3];            // run u: periodic image shift, 0 or +-L per axis
  __shared__ int s_exs[kWarps][20];    // each warp's particle's exclusions, as slots of this list
  __shared__ int s_late[kWarps][kLateWarp];  // each warp's entries of the outer group (rgroupsq), in order
  __shared__ int s_cell;
  const int nx = sc->ncell[L.which][0], ny = sc->ncell[L.which][1], nz = sc->ncell[L.which][2];
  const int ncells = nx * ny * nz;
  R b[3], bi[3], b2[3];
  box_of<R>(sc, b, bi, b2);
  const R rlsq = sizeof(R) == 4 ? (R)L.rlistsq : (R)L.rlistsqd;
  const R rg = L.rgroupsq > 0.f ? (R)L.rgroupsq : rlsq;
  const PT* pos = (const PT*)L.pos4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  int* late = s_late[warp];
  const int cap = L.w_cap * T;  // entries a slot may hold
  int* exs = s_exs[warp];
  for (;;) {
    __syncthreads();  // the previous cell's staging is no longer read
    if (threadIdx.x == 0) s_cell = (int)atomicAdd(&sc->work[2 + L.which], 1u);
    __syncthreads();
    const int c0 = s_cell;
    if (c0 >= ncells) break;
    const int first = L.cell_start[c0], last = L.cell_start[c0 + 1];
    if (first == last) continue;
    if (warp == 0) {
      // run 0: the own cell from its last slot down; runs 1..13: the stencil
      // cells, each from its last slot down; exclusive prefix of the lengths
      int hi = 0, len = 0;
      int w[3] = {0, 0, 0};  // the neighbour cell wraps past the box's +L/2 (1) or -L/2 (-1) face
      if (lane == 0) {
        hi = last - 1;
        len = last - first;
      } else if (lane < 14) {
        const int ic[3] = {c0 / (nz * ny), (c0 / nz) % ny, c0 % nz}, nc[3] = {nx, ny, nz};
        int jc[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int j = ic[q] + kStencil[lane - 1][q];
          w[q] = j >= nc[q] ? 1 : (j < 0 ? -1 : 0);
          jc[q] = j - w[q] * nc[q];
        }
        const int c = jc[0] * nz * ny + jc[1] * nz + jc[2];
        const int lo = L.cell_start[c];
        hi = L.cell_start[c + 1] - 1;
        len = hi - lo + 1;
      }
      int incl = len;
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane < 14) {
        s_hi[lane] = hi;
        s_pre[lane] = incl - len;
#pragma unroll
        for (int q = 0; q < 3; ++q) s_sh[lane][q] = w[q] > 0 ? b[q] : (w[q] < 0 ? -b[q] : (R)0);
      }
      if (lane == 13) s_pre[14] = incl;
    }
    __syncthreads();
    const int total = s_pre[14];
    // staged index v -> slot | run << 27, the run being the largest u with
    // s_pre[u] <= v (that run is not empty)
    auto slot_at = [&](int v) {
      int lo = 0, hi = 13;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_pre[mid] <= v) lo = mid;
        else hi = mid - 1;
      }
      return (s_hi[lo] - (v - s_pre[lo])) | (lo << 27);
    };
    const bool staged = total <= kCap;
    if (staged) {
      for (int v = threadIdx.x; v < total; v += blockDim.x) {
        const int tu = slot_at(v);
        s_slot[v] = tu;
        s_pos[v] = pos[tu & kSlotMask];
      }
    }
    __syncthreads();
    for (int s = first + warp; s < last; s += kWarps) {
      const int g = s / P;
      const long long base = (long long)g * L.w_cap * 32 + (s % P) * T;
      const int a = L.sorted[s];
      const int i = L.idx[a];
      const PT pi = staged ? s_pos[last - 1 - s] : pos[s];
      const int ne = L.excl_n[i];
      if (lane < ne) {
        const int gs = L.gslot[L.excl[(size_t)i * 20 + lane]];
        exs[lane] = (gs & 1) == L.which ? gs >> 1 : -1;
      }
      __syncwarp();
      // the first four exclusions in registers (a bead of a chain has four
      // 1-2 and 1-3 partners), the rest from shared memory
      const int e0 = ne > 0 ? exs[0] : -1, e1 = ne > 1 ? exs[1] : -1, e2 = ne > 2 ? exs[2] : -1,
                e3 = ne > 3 ? exs[3] : -1;
      const bool i_vs = L.hybrid && i >= L.natoms;
      int cnt = 0, nlate = 0;
      // minimum image: d - s with s the run's image shift.  For a pair inside
      // RLIST <= L/3 that shift is the nearest image, so s = ANINT(d/L)*L
      // exactly and d - s is the reference's d - ANINT(d/L)*L bit for bit;
      // with any other shift the distance is above RLIST either way.
      for (int v0 = last - s; v0 < total; v0 += 32) {
        const int v = v0 + lane;
        bool ok = false;
        int t = -1;
        R r2 = (R)0;
        if (v < total) {
          PT pj;
          int tu;
          if (staged) {
            tu = s_slot[v];
            pj = s_pos[v];
          } else {
            tu = slot_at(v);
            pj = pos[tu & kSlotMask];
          }
          t = tu & kSlotMask;
          const R* sh = s_sh[tu >> 27];
          R d0 = pi.x - pj.x, d1 = pi.y - pj.y, d2 = pi.z - pj.z;
          d0 = d0 - sh[0];
          d1 = d1 - sh[1];
          d2 = d2 - sh[2];
          r2 = d0 * d0;
          r2 = r2 + d1 * d1;
          r2 = r2 + d2 * d2;
          ok = r2 < rlsq && !(i_vs && (Prec<R>::bits(pj.w) >> 16) == 3) && t != e0 && t != e1 && t != e2 &&
               t != e3;
          if (ok && ne > 4)
            for (int e = 4; e < ne; ++e) ok &= exs[e] != t;
        }
        // entries of the outer group go to the warp's stage while it has
        // room (the rest are written in place, which only mixes the groups)
        const bool outer = ok && r2 >= rg;
        const unsigned mo = __ballot_sync(0xffffffffu, outer);
        const int po = __popc(mo & below), room = kLateWarp - nlate;
        const bool staged_late = outer && po < room;
        const bool now = ok && !staged_late;
        const unsigned m = __ballot_sync(0xffffffffu, now);
        if (now) {
          const int k = cnt + __popc(m & below);
          if (k < cap) ((int*)L.entries)[base + (long long)(k / T) * 32 + (k % T)] = t;
        }
        if (staged_late) late[nlate + po] = t;
        cnt += __popc(m);
        nlate += min(__popc(mo), room);
      }
      __syncwarp();
      for (int q = lane; q < nlate; q += 32) {
        const int k = cnt + q;
        if (k < cap) ((int*)L.entries)[base + (long long)(k / T) * 32 + (k % T)] = late[q];
      }
      cnt += nlate;
      if (lane == 0) {
        L.counts[s] = cnt;
        if (cnt >= L.maxnab) atomicOr(&sc->err, EB_LIST_OVERFLOW);
        const int rows = (cnt + T - 1) / T;
        atomicMax(&L.slice_w[g], rows);
        if (rows > L.w_cap) {
          atomicMax(&sc->need_rows[L.which], rows);
          sc->abort = 1;
          sc->skip = 1;
        }
      }
      __syncwarp();  // exs is rewritten for the next particle
    }
  }
}

// NEW_NEIGHBOUR_WITHLIST.f90:34-123 for large lists: a thread builds one
// particle's list (k_list_build_warp, above, gives a warp to each particle and
// suits lists too short to fill the GPU with one thread per particle).
// A warp takes 32 consecutive slots at a time (dynamically), so its lanes
// mostly share a cell and walk the same candidates in step: a candidate's
// position is one load that the lanes share, and each lane appends what it
// accepts to its own list in the order it visits the candidates.  That order
// is the reference's: the particle's own cell below it by decreasing A (slots
// keep increasing A within a cell), then the 13 cells of the MAPS.f90:39-51
// stencil, each by decreasing A.  The distance test runs first and the
// exclusion test only for candidates inside RLIST (the accepted set is the
// same); exclusions are compared as slots of this list (the first four in
// registers, the rest in shared memory), and a virtual site is recognised by
// its label in the position's w, so no candidate's global id is loaded.
//
// The minimum image needs no per-candidate test: each stencil cell carries
// its periodic shift s (0 or +-L per axis, from whether it wrapped around the
// box), and a candidate's displacement is (x_i - x_j) - s.  For a pair inside
// RLIST <= L/3 that shift is the nearest image, so s = ANINT(d/L)*L exactly
// and d - s is the reference's d - ANINT(d*BOXINV)*BOX
// (NEW_NEIGHBOUR_WITHLIST.f90:65) bit for bit; with any other shift the
// distance is above RLIST either way.
//
// The list is stored in the nonbonded kernel's layout: T lanes per slot,
// slices of P = 32/T slots, entry k of slot s (slice g) at
// (g*w_cap + k/T)*32 + (s%P)*T + k%T.  A slot that needs more than w_cap rows
// records its need and raises the abort flag (the host enlarges the storage
// and repeats the step).
template <typename R, int T, bool B>
__global__ void __launch_bounds__(256) k_list_build_thread(__grid_constant__ const ListArgs L0, const ListArgs* const* tab,
                                                    const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  using PT = typename Prec<R>::pos_t;
  const Blk bk = blk<B>(bm);
  __shared__ ListArgs s_args;
  if (B) stage_args(&s_args, tab[bk.sys]);
  const ListArgs& L = B ? s_args : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  constexpr int P = 32 / T;
  __shared__ int s_ex[16][256];  // exclusions 5..20 of each thread's particle, as slots of this list
  __shared__ int s_late[kLateThread][256];  // each thread's entries of the outer group (rgroupsq), in order
  const int nx = sc->ncell[L.which][0], ny = sc->ncell[L.which][1], nz = sc->ncell[L.which][2];
  const int nc[3] = {nx, ny, nz};
  R b[3], bi[3], b2[3];
  box_of<R>(sc, b, bi, b2);
  const R rlsq = sizeof(R) == 4 ? (R)L.rlistsq : (R)L.rlistsqd;
  const R rg = L.rgroupsq > 0.f ? (R)L.rgroupsq : rlsq;
  const PT* pos = (const PT*)L.pos4;
  const int lane = threadIdx.x & 31;
  const int cap = L.w_cap * T;  // entries a slot may hold
  const int nchunks = (L.n + 31) / 32;
  for (;;) {
    int ch = 0;
    if (lane == 0) ch = (int)atomicAdd(&sc->work[2 + L.which], 1u);
    ch = __shfl_sync(0xffffffffu, ch, 0);
    if (ch >= nchunks) break;
    const int s = ch * 32 + lane;
    if (s >= L.n) continue;
    const int a = L.sorted[s];
    const int i = L.idx[a];
    const int c0 = L.cell_of[a];
    const PT pi = pos[s];
    const int ne = min(L.excl_n[i], 20);
    int e0 = -1, e1 = -1, e2 = -1, e3 = -1;
    for (int e = 0; e < ne; ++e) {
      const int gs = L.gslot[L.excl[(size_t)i * 20 + e]];
      const int t = (gs & 1) == L.which ? gs >> 1 : -1;
      if (e == 0) e0 = t;
      else if (e == 1) e1 = t;
      else if (e == 2) e2 = t;
      else if (e == 3) e3 = t;
      else s_ex[e - 4][threadIdx.x] = t;
    }
    const bool i_vs = L.hybrid && i >= L.natoms;
    const int g = s / P;
    int* row = L.entries + (long long)g * L.w_cap * 32 + (s % P) * T;
    int cnt = 0, nlate = 0;
    // candidates slot hi down to lo, displaced by the run's image shift
    // a candidate inside RLIST: exclusions, the site-site rule, then stored
    auto accept = [&](int t, R r2, const PT& pj) {
      bool ok = !(i_vs && (Prec<R>::bits(pj.w) >> 16) == 3) && t != e0 && t != e1 && t != e2 && t != e3;
      if (ok && ne > 4)
        for (int e = 4; e < ne; ++e) ok &= s_ex[e - 4][threadIdx.x] != t;
      if (ok) {
        if (r2 >= rg && nlate < kLateThread) {
          s_late[nlate++][threadIdx.x] = t;  // the outer group, appended below
        } else {
          if (cnt < cap) row[(cnt / T) * 32 + cnt % T] = t;
          ++cnt;
        }
      }
    };
    auto scan = [&](int hi, int lo, R sh0, R sh1, R sh2) {
#pragma unroll 4
      for (int t = hi; t >= lo; --t) {
        const PT pj = pos[t];
        R d0 = pi.x - pj.x, d1 = pi.y - pj.y, d2 = pi.z - pj.z;
        d0 = d0 - sh0;
        d1 = d1 - sh1;
        d2 = d2 - sh2;
        R r2 = d0 * d0;
        r2 = r2 + d1 * d1;
        r2 = r2 + d2 * d2;
        if (r2 < rlsq) accept(t, r2, pj);
      }
    };
    scan(s - 1, L.cell_start[c0], (R)0, (R)0, (R)0);  // the own cell below this particle
    const int ic[3] = {c0 / (nz * ny), (c0 / nz) % ny, c0 % nz};
    for (int u = 0; u < 13; ++u) {
      int jc[3];
      R sh[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int j = ic[q] + kStencil[u][q];
        const int w = j >= nc[q] ? 1 : (j < 0 ? -1 : 0);
        jc[q] = j - w * nc[q];
        sh[q] = w > 0 ? b[q] : (w < 0 ? -b[q] : (R)0);
      }
      const int c = jc[0] * nz * ny + jc[1] * nz + jc[2];
      scan(L.cell_start[c + 1] - 1, L.cell_start[c], sh[0], sh[1], sh[2]);
    }
    for (int q = 0; q < nlate; ++q, ++cnt)
      if (cnt < cap) row[(cnt / T) * 32 + cnt % T] = s_late[q][threadIdx.x];
    L.counts[s] = cnt;
    if (cnt >= L.maxnab) atomicOr(&sc->err, EB_LIST_OVERFLOW);
    const int rows = (cnt + T - 1) / T;
    atomicMax(&L.slice_w[g], rows);
    if (rows > L.w_cap) {
      atomicMax(&sc->need_rows[L.which], rows);
      sc->abort = 1;
      sc->skip = 1;
    }
  }
}

// Slice lists (FP32 path, ListArgs/NBArgs form 1).  Slice g is the four
// slots 4g..4g+3.  Its list holds each neighbour once, as the entry
// slot | mask << 28, where bit k of the mask says that slot 4g+k pairs with
// it: the union of the four half lists, with no pair added or lost.  The
// four slots are consecutive in the cell order, so their lists share most of
// their neighbours (a stored entry stands for ~1.9 pairs on the melts), and
// the nonbonded kernel gathers each neighbour's position and adds its force
// once per slice instead of once per pair.  Entry e of slice g lives at
// g*w_cap*32 + e; the last row is filled up with empty entries (mask 0).
constexpr int kUSlots = 4;
constexpr unsigned kUSlotMask = (1u << 28) - 1u;
constexpr int kUBuf = 256;  // entries of a slice each warp sorts in shared memory

// NEW_NEIGHBOUR_WITHLIST.f90:34-123 in the slice form: a warp builds one
// slice's list.  For each cell that holds particles of the slice (one, or two
// when the slice straddles a cell boundary) it walks that cell's candidates,
// 32 at a time, one per lane: the own cell below the slice's last particle
// there, then the 13 stencil cells of MAPS.f90:39-51, each by decreasing slot.
// A lane tests its candidate against each particle of the slice in that cell
// with the reference's REAL*4 distance (the run's image shift gives the
// nearest image, as in k_list_build_thread), the own-cell rule (only slots
// below the particle), the virtual-site rule and the particle's exclusions.
// A candidate that two cells of a slice both reach is stored once per cell,
// with disjoint masks, so every pair is stored exactly once.
//
// The accepted entries are gathered in shared memory and stored sorted by
// the key (outer group, mask), stably: first the entries with a pair inside
// rgroupsq, by mask, then the rest, by mask.  So a row of 32 entries mostly
// shares one mask, and the nonbonded kernel's warp runs the pair arithmetic
// once per bit of that mask with all its lanes busy, instead of once per
// particle of the slice with the lanes whose masks hold it.  Entries beyond
// the first kUBuf of a slice are stored unsorted after them.  counts[s] is the
// number of pairs of slot s (its reference NNEBS).
template <bool B>
__global__ void __launch_bounds__(256) k_list_build_slices(__grid_constant__ const ListArgs L0,
                                                          const ListArgs* const* tab, const BlockMap bm, int always) {
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  __shared__ ListArgs s_args;
  if (B) stage_args(&s_args, tab[bk.sys]);
  const ListArgs& L = B ? s_args : L0;
  Scalars* sc = L.sc;
  if (sc->skip || !(always || sc->rebuild)) return;
  constexpr int kWarps = 8;
  __shared__ int s_ex[kWarps][kUSlots][20];  // each particle's exclusions as slots of this list
  __shared__ int s_buf[kWarps][kUBuf];       // the slice's entries, in the order accepted
  __shared__ unsigned char s_key[kWarps][kUBuf];  // their keys: mask | 16 for the outer group
  __shared__ int s_off[kWarps][32];          // per key: count, then next position
  __shared__ int2 s_run[kWarps][14];         // each candidate run: highest slot, first index
  __shared__ float s_sh[kWarps][14][3];      // each candidate run: image shift
  const int nx = sc->ncell[L.which][0], ny = sc->ncell[L.which][1], nz = sc->ncell[L.which][2];
  const int nc[3] = {nx, ny, nz};
  float b[3], bi[3], b2[3];
  box_of<float>(sc, b, bi, b2);
  const float rlsq = L.rlistsq;
  const float rg = L.rgroupsq > 0.f ? L.rgroupsq : rlsq;
  const float4* pos = (const float4*)L.pos4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  int* buf = s_buf[warp];
  unsigned char* keys = s_key[warp];
  int* off = s_off[warp];
  const int cap = L.w_cap * 32;  // entries a slice may hold
  for (;;) {
    int g = 0;
    if (lane == 0) g = (int)atomicAdd(&sc->work[2 + L.which], 1u);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= L.nslices) break;
    // the slice's particles: slot, cell, position, exclusions, site flag
    int my_cell = INT_MAX, my_ne = 0, my_vs = 0;
    float4 my_pos = make_float4(0.f, 0.f, 0.f, 0.f);
    int my_i = 0;
    if (lane < kUSlots && kUSlots * g + lane < L.n) {
      const int s = kUSlots * g + lane;
      const int a = L.sorted[s];
      my_i = L.idx[a];
      my_cell = L.cell_of[a];
      my_pos = pos[s];
      my_ne = min(L.excl_n[my_i], 20);
      my_vs = L.hybrid && my_i >= L.natoms;
    }
    float4 pi[kUSlots];
    int ci[kUSlots], ne[kUSlots];
    unsigned vsm = 0;
#pragma unroll
    for (int k = 0; k < kUSlots; ++k) {
      pi[k].x = __shfl_sync(0xffffffffu, my_pos.x, k);
      pi[k].y = __shfl_sync(0xffffffffu, my_pos.y, k);
      pi[k].z = __shfl_sync(0xffffffffu, my_pos.z, k);
      ci[k] = __shfl_sync(0xffffffffu, my_cell, k);
      ne[k] = __shfl_sync(0xffffffffu, my_ne, k);
      vsm |= (unsigned)__shfl_sync(0xffffffffu, my_vs, k) << k;
      const int ik = __shfl_sync(0xffffffffu, my_i, k);
      if (lane < ne[k]) {
        const int gs = L.gslot[L.excl[(size_t)ik * 20 + lane]];
        s_ex[warp][k][lane] = (gs & 1) == L.which ? gs >> 1 : -1;
      }
    }
    __syncwarp();
    const long long base = (long long)g * cap;
    int cnt = 0;
    int npair[kUSlots] = {0, 0, 0, 0};  // this lane's accepted pairs of each particle
    // each cell of the slice in turn (slots are in cell order, so the
    // particles of one cell are consecutive).  Its 14 runs (the own cell
    // below the group's last particle, then the 13 stencil cells) are walked
    // as one sequence of candidates, 32 at a time: lane u < 14 describes run
    // u (highest slot, image shift), a prefix sum gives each run's first index
    for (int k0 = 0; k0 < kUSlots && ci[k0] != INT_MAX;) {
      const int c0 = ci[k0];
      unsigned gm = 0;
      int k1 = k0;
      while (k1 < kUSlots && ci[k1] == c0) gm |= 1u << k1++;
      int hi = -1, len = 0;
      float sh[3] = {0.f, 0.f, 0.f};
      if (lane == 0) {
        hi = kUSlots * g + k1 - 2;
        len = max(0, hi - L.cell_start[c0] + 1);
      } else if (lane < 14) {
        const int ic[3] = {c0 / (nz * ny), (c0 / nz) % ny, c0 % nz};
        int jc[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int j = ic[q] + kStencil[lane - 1][q];
          const int w = j >= nc[q] ? 1 : (j < 0 ? -1 : 0);
          jc[q] = j - w * nc[q];
          sh[q] = w > 0 ? b[q] : (w < 0 ? -b[q] : 0.f);
        }
        const int c = jc[0] * nz * ny + jc[1] * nz + jc[2];
        hi = L.cell_start[c + 1] - 1;
        len = hi - L.cell_start[c] + 1;
      }
      int incl = len;
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 13);
      __syncwarp();  // the previous cell's run table is no longer read
      if (lane < 14) {
        s_run[warp][lane] = make_int2(hi, incl - len);
        s_sh[warp][lane][0] = sh[0];
        s_sh[warp][lane][1] = sh[1];
        s_sh[warp][lane][2] = sh[2];
      }
      __syncwarp();
      for (int v0 = 0; v0 < total; v0 += 32) {
        const int v = v0 + lane;
        unsigned m = 0;
        bool inner = false;
        int t = 0;
        if (v < total) {
          // the run of candidate v: the last run that starts at or before v
          // (empty runs start where the next one does, and are skipped)
          int u = 0;
#pragma unroll
          for (int step = 8; step > 0; step >>= 1)
            if (u + step < 14 && s_run[warp][u + step].y <= v) u += step;
          const int2 run = s_run[warp][u];
          t = run.x - (v - run.y);
          const float sh0 = s_sh[warp][u][0], sh1 = s_sh[warp][u][1], sh2 = s_sh[warp][u][2];
          const bool own = u == 0;
          const float4 pj = pos[t];
          const bool j_vs = (__float_as_int(pj.w) >> 16) == 3;
#pragma unroll
          for (int k = 0; k < kUSlots; ++k) {
            if (!((gm >> k) & 1u)) continue;
            // the reference's REAL*4 distance, scalar and uncontracted
            float d0 = pi[k].x - pj.x, d1 = pi[k].y - pj.y, d2 = pi[k].z - pj.z;
            d0 = d0 - sh0;
            d1 = d1 - sh1;
            d2 = d2 - sh2;
            float r2 = d0 * d0;
            r2 = r2 + d1 * d1;
            r2 = r2 + d2 * d2;
            if (!(r2 < rlsq)) continue;
            if (own && t >= kUSlots * g + k) continue;  // the own cell: only slots below the particle
            if (((vsm >> k) & 1u) && j_vs) continue;    // no site-site pair
            bool ok = true;
            for (int e = 0; e < ne[k]; ++e) ok &= s_ex[warp][k][e] != t;
            if (!ok) continue;
            m |= 1u << k;
            ++npair[k];
            inner |= r2 < rg;
          }
        }
        const unsigned ma = __ballot_sync(0xffffffffu, m != 0);
        if (m != 0) {
          const int k = cnt + __popc(ma & below);
          const int entry = t | (int)(m << 28);
          if (k < kUBuf) {
            buf[k] = entry;
            keys[k] = (unsigned char)(m | (inner ? 0u : 16u));
          } else if (k < cap) {
            L.entries[base + k] = entry;  // beyond the sort buffer: stored as found
          }
        }
        cnt += __popc(ma);
      }
      k0 = k1;
    }
#pragma unroll
    for (int k = 0; k < kUSlots; ++k)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) npair[k] += __shfl_xor_sync(0xffffffffu, npair[k], o);
    // stable counting sort of the buffered entries by key
    __syncwarp();
    const int nb = min(cnt, kUBuf);
    off[lane] = 0;
    __syncwarp();
    for (int c = 0; c < nb; c += 32) {
      const int q = c + lane;
      const int key = q < nb ? keys[q] : 32 + lane;  // unique keys for the idle lanes
      const unsigned same = __match_any_sync(0xffffffffu, key);
      if (q < nb && (same & below) == 0) off[key] += __popc(same);
      __syncwarp();
    }
    {
      const int n_key = off[lane];
      int incl = n_key;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      __syncwarp();
      off[lane] = incl - n_key;  // first position of key `lane`
      __syncwarp();
    }
    for (int c = 0; c < nb; c += 32) {
      const int q = c + lane;
      const int key = q < nb ? keys[q] : 32 + lane;
      const unsigned same = __match_any_sync(0xffffffffu, key);
      int at = 0;
      if (q < nb) at = off[key] + __popc(same & below);
      __syncwarp();
      if (q < nb && (same & below) == 0) off[key] += __popc(same);
      if (q < nb && at < cap) L.entries[base + at] = buf[q];
      __syncwarp();
    }
    // empty entries up to the end of the last row
    const int rows = (cnt + 31) / 32;
    if (cnt + lane < rows * 32 && cnt + lane < cap) L.entries[base + cnt + lane] = 0;
    if (lane < kUSlots && kUSlots * g + lane < L.n) {
      int np = npair[0];
#pragma unroll
      for (int k = 1; k < kUSlots; ++k) np = lane == k ? npair[k] : np;
      L.counts[kUSlots * g + lane] = np;
      if (np >= L.maxnab) atomicOr(&sc->err, EB_LIST_OVERFLOW);
    }
    if (lane == 0) {
      L.slice_w[g] = rows;
      if (rows > L.w_cap) {
        atomicMax(&sc->need_rows[L.which], rows);
        sc->abort = 1;
        sc->skip = 1;
      }
    }
    __syncwarp();  // s_ex, buf and keys are rewritten for the next slice
  }
}

// ------------------------------------------------------------- nonbonded
// FP32 nonbonded energies and virials are summed in FP32 over this many list
// rows of a slice, then in fixed point.
constexpr int kEnergyRows = 8;

template <typename R>
struct NBArgs {
  Scalars* sc;
  int mts;                         // bead list of an MTS run: only steps m = 1..3 evaluate it
  int n, nslices, ntype;
  const void* pos4;
  const int4* posq;                // FP32 kernel: positions as box fractions
  const int* counts;
  const int* slice_w;
  const int* entries;
  int w_cap;                       // rows of 32 entries per slice
  int work;                        // index of this launch's work counter
  typename Prec<R>::acc_t* fsort;  // per slot, in blocks of 32 slots (fs_at)
  // tables of this list: ltab[ti*ntype+tj] = local table or -1; rows of table
  // t are [toff[t], toff[t+1]); fp = {F,P} per row, x = RNBOND per row
  const int* ltab;
  const int* toff;
  const int* tndat;
  const R* tbin;
  const R* tinv; // 1/bin per table (FP32 force kernel)
  const int4* ptab;  // FP32 kernel: per type pair {first row, NDAT, 1/bin bits, 1 if a table}
  int chunk;         // FP32 kernel: 256ths of the units taken dynamically after the blocks' own ranges (0: all, per warp)
  int window;        // FP32 kernel, chunk > 0: 0 = each block one contiguous range of units; W > 0 = runs of W
                     // consecutive units dealt to the blocks in turn (block b takes runs b, b + G, b + 2G, ...)
  int rows;          // list rows per work unit, a multiple of kEnergyRows
  // FP32 kernel: pairs whose r^2 lies within a relative 1e-6 of the cutoff
  // are left to k_nb_near, which decides them as the FP64 path does from the
  // FP64 state (global ids from slot -> A -> global id)
  float rcut_lo, rcut_hi;
  int4* near;          // (i slot, j slot, i global id, j global id) of those pairs
  int near_cap;
  const int* sorted;
  const int* idx;
  const double* S;
  int natoms;
  const R* tfp;  // 2 per row
  // FP32 kernel: per row {A, C, B, D}, F = A + B u and P = C + D u with
  // u = r/bin - (row within the table); one 16-byte read per pair
  const float4* tcoef;
  const R* tx;
  int ntab, nrows;
  R rcutsq;
};

// A nonbonded launch does nothing on a skipped step, and for the bead list
// of an MTS run on the steps MTS_APPROX extrapolates (MTS_LOOP.f90:100-110).
template <typename R>
__device__ __forceinline__ bool nb_idle(const NBArgs<R>& A) {
  const Scalars* sc = A.sc;
  if (sc->skip) return true;
  if (A.mts) {
    const int m = sc->mts_m;
    return !(m >= 1 && m <= 3);
  }
  return false;
}

// NONBONDED_FORCE.F90:45-104.  Persistent grid; a warp owns one slice of
// P = 32/T slots at a time and T lanes walk each slot's list; list reads are
// coalesced 128-byte rows, neighbour positions are float4 gathers from the
// cell-ordered array.  i-forces are summed in registers and reduced exactly
// over the slot's lanes (integer shuffles); j-forces are 64-bit integer
// atomics.  Tables are staged in shared memory when SMEM.
template <typename R, bool SMEM, int T, bool B>
__global__ void __launch_bounds__(256, 4) k_nonbonded(__grid_constant__ const NBArgs<R> A0, const NBArgs<R>* const* tab,
                                                      const BlockMap bm) {
  using P = Prec<R>;
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  __shared__ NBArgs<R> s_args;
  if (B) stage_args(&s_args, tab[bk.sys]);
  const NBArgs<R>& A = B ? s_args : A0;
  Scalars* sc = A.sc;
  if (nb_idle(A)) return;
  using PT = typename P::pos_t;
  using reg_t = typename P::reg_t;
  constexpr int PS = 32 / T;
  extern __shared__ unsigned char smem_raw[];
  const int* ltab = A.ltab;
  const int* toff = A.toff;
  const int* tndat = A.tndat;
  const R* tbin = A.tbin;
  const R* tfp = A.tfp;
  const R* tx = A.tx;
  double* red = (double*)smem_raw;  // 9 * 8 doubles, reused at the end
  if (SMEM) {
    unsigned char* p = smem_raw + 9 * 8 * sizeof(double);
    R* s_fp = (R*)p;               p += sizeof(R) * 2 * A.nrows;
    R* s_x = (R*)p;                p += sizeof(R) * A.nrows;
    R* s_bin = (R*)p;              p += sizeof(R) * A.ntab;
    int* s_ltab = (int*)p;         p += sizeof(int) * A.ntype * A.ntype;
    int* s_toff = (int*)p;         p += sizeof(int) * (A.ntab + 1);
    int* s_ndat = (int*)p;
    for (int k = threadIdx.x; k < 2 * A.nrows; k += blockDim.x) s_fp[k] = A.tfp[k];
    for (int k = threadIdx.x; k < A.nrows; k += blockDim.x) s_x[k] = A.tx[k];
    for (int k = threadIdx.x; k < A.ntab; k += blockDim.x) { s_bin[k] = A.tbin[k]; s_ndat[k] = A.tndat[k]; }
    for (int k = threadIdx.x; k < A.ntype * A.ntype; k += blockDim.x) s_ltab[k] = A.ltab[k];
    for (int k = threadIdx.x; k <= A.ntab; k += blockDim.x) s_toff[k] = A.toff[k];
    __syncthreads();
    ltab = s_ltab; toff = s_toff; tndat = s_ndat; tbin = s_bin; tfp = s_fp; tx = s_x;
  }
  R b[3], bi[3], b2[3];
  box_of<R>(sc, b, bi, b2);
  const PT* pos = (const PT*)A.pos4;
  const int lane = threadIdx.x & 31, grp = lane / T, q = lane % T;
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) acc[k] = 0.0;
  unsigned err = 0;
  const bool run = true;
  // work unit = up to ROWS rows of 32 entries of one slice; units are taken
  // dynamically so that warps finish within one unit of each other
  const int ROWS = A.rows;
  const int U = (A.w_cap + ROWS - 1) / ROWS;
  const int nunits = A.nslices * U;
  for (;;) {
    int u = 0;
    if (lane == 0) u = run ? (int)atomicAdd(&sc->work[A.work], 1u) : nunits;
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= nunits) break;
    const int g = u / U;
    const int r0 = (u - g * U) * ROWS;
    const int w = min(A.slice_w[g], A.w_cap);
    if (r0 >= w) continue;
    const int r1 = min(w, r0 + ROWS);
    const int s = g * PS + grp;
    const bool valid = s < A.n;
    const int cnt = valid ? A.counts[s] : 0;
    const int* ent = A.entries + (long long)g * A.w_cap * 32 + lane;
    PT pi;
    if (valid) pi = pos[s];
    else { pi.x = pi.y = pi.z = 0; pi.w = P::tbits(0); }
    const int wi = P::bits(pi.w);
    const int ti = wi & 0xffff, li = wi >> 16;
    reg_t fi0 = 0, fi1 = 0, fi2 = 0;
    auto pair = [&](int t, const PT& pj) {
      R d0 = pi.x - pj.x, d1 = pi.y - pj.y, d2 = pi.z - pj.z;
      d0 = d0 - r_round(d0 * bi[0]) * b[0];
      d1 = d1 - r_round(d1 * bi[1]) * b[1];
      d2 = d2 - r_round(d2 * bi[2]) * b[2];
      R r2 = d0 * d0;
      r2 = r2 + d1 * d1;
      r2 = r2 + d2 * d2;
      if (!(r2 < A.rcutsq)) return;
      const int wj = P::bits(pj.w);
      const int tj = wj & 0xffff, lj = wj >> 16;
      const int tab = ltab[ti * A.ntype + tj];
      if (tab < 0) { err |= EB_MISSING_TABLE; return; }
      const R r = r_sqrt(r2);
      const R bin = tbin[tab];
      const int ni = fint(r / bin);
      if (ni < 0 || ni > tndat[tab]) { err |= EB_TABLE_RANGE; return; }
      const int row = toff[tab] + ni;
      const R alpha = (r - tx[row]) / bin;
      const R f0 = tfp[2 * row], p0 = tfp[2 * row + 1], f1 = tfp[2 * row + 2], p1 = tfp[2 * row + 3];
      const R one_a = (R)1.0 - alpha;
      const R fij = f0 * one_a + f1 * alpha;
      const R vij = p0 * one_a + p1 * alpha;
      if (li == 1) acc[0] += (double)vij;
      else if (li == 2) {
        if (lj == 2) acc[1] += (double)vij;
        else if (lj == 3) acc[2] += (double)vij;
      } else if (li == 3) acc[2] += (double)vij;
      const R fx = fij * d0, fy = fij * d1, fz = fij * d2;
      const reg_t qx = P::q(fx, &sc->err), qy = P::q(fy, &sc->err), qz = P::q(fz, &sc->err);
      fi0 += qx; fi1 += qy; fi2 += qz;
      typename P::acc_t* fj = A.fsort + fs_at(t);
      P::add(fj, -qx);
      P::add(fj + 32, -qy);
      P::add(fj + 64, -qz);
      acc[3] += (double)(fx * d0);
      acc[4] += (double)(fy * d1);
      acc[5] += (double)(fz * d2);
      acc[6] += (double)(fy * d0);
      acc[7] += (double)(fz * d0);
      acc[8] += (double)(fz * d1);
    };
    // two rows per iteration: both entry loads and both position gathers are
    // in flight before either pair is evaluated
    for (int it = r0; it < r1; it += 2) {
      const bool v0 = it * T + q < cnt;
      const bool v1 = it + 1 < r1 && (it + 1) * T + q < cnt;
      const int t0 = v0 ? __ldcs(ent + it * 32) : 0;
      const int t1 = v1 ? __ldcs(ent + (it + 1) * 32) : 0;
      const PT p0 = pos[t0];
      const PT p1 = pos[t1];
      if (v0) pair(t0, p0);
      if (v1) pair(t1, p1);
    }
#pragma unroll
    for (int o = T / 2; o > 0; o >>= 1) {
      fi0 += __shfl_down_sync(0xffffffffu, fi0, o, T);
      fi1 += __shfl_down_sync(0xffffffffu, fi1, o, T);
      fi2 += __shfl_down_sync(0xffffffffu, fi2, o, T);
    }
    if (q == 0 && valid && r0 * T < cnt) {
      typename P::acc_t* fo = A.fsort + fs_at(s);
      P::add(fo, fi0);
      P::add(fo + 32, fi1);
      P::add(fo + 64, fi2);
    }
  }
  if (err) atomicOr(&sc->err, err);
  __syncthreads();
  double out[9];
  block_sum<9>(acc, red, out);
  if (threadIdx.x == 0)
    for (int k = 0; k < 9; ++k) atomicAdd((double*)&sc->nbacc[A.work][k], out[k]);
}

// round(v * 2^S) to the nearest 64-bit integer: the scaling by a power of two
// is exact and the conversion rounds to nearest.  Values of magnitude
// 2^(63-S) and above (and Inf/NaN) raise EB_FIXED and count as 0.
// fabsf(fij) r below 0.99 kFixMax, tested on the force scaled by 2^32
constexpr float kFixLimScaled = 0.99f * kFixMax * kFixScale;
// The FP32 nonbonded kernel's energy and virial sums: 9 per pair of lanes of
// its 256-thread blocks, at the start of its dynamic shared memory.
constexpr int kNbPairs = 128;
constexpr int kNbAccBytes = 9 * kNbPairs * (int)sizeof(long long);

template <int S>
__device__ __forceinline__ long long fixq(float v, unsigned& err) {
  const float s = v * (float)(1ull << S);
  if (!(fabsf(s) < 0x1p63f)) { err |= EB_FIXED; return 0; }
  return __float2ll_rn(s);
}

// The work units of an FP32 nonbonded launch handed to the warps of a block
// (NBArgs::chunk, NBArgs::window); unit(u) is called for each of them.
template <typename F>
__device__ __forceinline__ void nb_schedule(const NBArgs<float>& A, const Blk& bk, int nunits, F&& unit) {
  const int lane = threadIdx.x & 31;
  if (A.chunk > 0) {
    // each block a contiguous range of units (neighbouring slices), its warps
    // taking them through a shared counter, so they gather from one region of
    // space and share it in L1, with no barrier between them; the last
    // chunk/256 of the units are taken from the global counter by whichever
    // warps finish their block's range first
    __shared__ int s_next;
    if (threadIdx.x == 0) s_next = 0;
    __syncthreads();
    const int tail = (int)((long long)nunits * min(A.chunk, 256) / 256);
    const int nstat = nunits - tail;
    if (A.window > 0) {
      // runs of W consecutive units dealt to the blocks in turn: the blocks
      // advance together through one window of space, whose positions and
      // force sums then stay in L2, while a block's warps still share a run
      const int W = A.window;
      for (;;) {
        int k = 0;
        if (lane == 0) k = atomicAdd(&s_next, 1);
        k = __shfl_sync(0xffffffffu, k, 0);
        const long long u = ((long long)(k / W) * bk.g + bk.b) * W + k % W;
        if (u >= nstat) break;
        unit((int)u);
      }
    } else {
      const int lo = (int)((long long)nstat * bk.b / bk.g), hi = (int)((long long)nstat * (bk.b + 1) / bk.g);
      for (;;) {
        int k = 0;
        if (lane == 0) k = atomicAdd(&s_next, 1);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (lo + k >= hi) break;
        unit(lo + k);
      }
    }
    for (;;) {
      int u = 0;
      if (lane == 0) u = nstat + (int)atomicAdd(&A.sc->work[A.work], 1u);
      u = __shfl_sync(0xffffffffu, u, 0);
      if (u >= nunits) break;
      unit(u);
    }
  } else {
    for (;;) {
      int u = 0;
      if (lane == 0) u = (int)atomicAdd(&A.sc->work[A.work], 1u);
      u = __shfl_sync(0xffffffffu, u, 0);
      if (u >= nunits) break;
      unit(u);
    }
  }
}

// NONBONDED_FORCE.F90:45-104, FP32 force path.  Same structure as
// k_nonbonded (slices of P = 32/T slots, T lanes per slot, dynamic units of
// `rows` list rows).  The arithmetic is REAL*4 as in the reference, with
// cheaper equivalents where only the force value (not a bit pattern) is
// compared: positions as 32-bit box fractions, whose wrapped difference is
// the nearest-image displacement at full precision anywhere in the box (a
// REAL*4 coordinate near the box edge carries only 24 bits), r from rsqrt,
// the table row and interpolation weight from a precomputed 1/bin,
// float-to-fixed by the hardware conversion of the exactly scaled value.  Energies and virials are
// summed in FP32 over kEnergyRows list rows, then as 64-bit fixed point
// (2^-24) per lane and per block, and added to the system's accumulators:
// integer sums depend neither on which warp took which unit nor on the rows
// per unit, so they are reproducible and the same alone or in a batch.
// MIXED: the list holds particles of more than one label, so each pair's
// energy term depends on j's label; otherwise every pair adds to the term of
// the list's one label.
template <bool SMEM, bool MIXED, bool B>
__global__ void __launch_bounds__(256, 4) k_nonbonded_f32(__grid_constant__ const NBArgs<float> A0,
                                                          const NBArgs<float>* const* tab, const BlockMap bm) {
  constexpr int T = 8;  // lanes per particle (the lists are built for eight)
  constexpr int PS = 32 / T;
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  __shared__ NBArgs<float> s_args;
  if (B) stage_args(&s_args, tab[bk.sys]);
  const NBArgs<float>& A = B ? s_args : A0;
  Scalars* sc = A.sc;
  if (nb_idle(A)) return;
  extern __shared__ unsigned char smem_raw[];
  // [9][kNbPairs] sums of each pair of lanes (the two lanes of a pair serve
  // the same particle): half the shared memory of per-lane sums, which leaves
  // more of the SM's 256 KB to L1
  long long* lacc = (long long*)smem_raw;
  // per type pair {first row, last row index, 1/bin bits, has a table}
  const int4* ptab = A.ptab;
  const float4* tco = A.tcoef;
  {
    unsigned char* p = smem_raw + kNbAccBytes;
    if (SMEM) {
      int4* s_ptab = (int4*)p;       p += sizeof(int4) * A.ntype * A.ntype;
      float4* s_co = (float4*)p;
      for (int k = threadIdx.x; k < A.nrows; k += blockDim.x) s_co[k] = A.tcoef[k];
      for (int k = threadIdx.x; k < A.ntype * A.ntype; k += blockDim.x) s_ptab[k] = A.ptab[k];
      ptab = s_ptab; tco = s_co;
    }
  }
  if (!(threadIdx.x & 1))
    for (int k = 0; k < 9; ++k) lacc[k * kNbPairs + (threadIdx.x >> 1)] = 0;
  __syncthreads();
  // displacement unit per axis: L / 2^32
  const float ux = (float)(sc->box[0] * 0x1p-32), uy = (float)(sc->box[1] * 0x1p-32), uz = (float)(sc->box[2] * 0x1p-32);
  const float2 uxy = make_float2(ux, uy);
  const int4* pos = A.posq;
  const int lane = threadIdx.x & 31, grp = lane / T, q = lane % T;
  unsigned err = 0;
  // a work unit is `rows` list rows of one slice (a multiple of kEnergyRows)
  const int rows = A.rows;
  const int U = (A.w_cap + rows - 1) / rows;
  const int nunits = A.nslices * U;
  long long* la = lacc + (threadIdx.x >> 1);
  auto unit = [&](int u) {
    const int g = u / U;
    const int r0 = (u - g * U) * rows;
    const int w = min(A.slice_w[g], A.w_cap);
    if (r0 >= w) return;
    const int r1 = min(w, r0 + rows);
    const int s = g * PS + grp;
    const bool valid = s < A.n;
    const int cnt = valid ? A.counts[s] : 0;
    const int* ent = A.entries + (long long)g * A.w_cap * 32 + lane;
    const int4 pi = valid ? pos[s] : make_int4(0, 0, 0, 0);
    const int wi = pi.w;
    const int ti = wi & 0xffff, li = wi >> 16;
    const int4* pti = ptab + ti * A.ntype;  // descriptors of (ti, tj) for every tj
    // the energy term of a pair follows from j's label once i's is fixed:
    // V_NB(1) when i is an atom, V_NB(3) when i is a virtual site; when i is
    // a bead, V_NB(2) for a bead j and V_NB(3) for a site j
    const bool i_bead = li == 2;
    long long fi0 = 0, fi1 = 0, fi2 = 0;
    // energies and virials: FP32 over kEnergyRows rows (aligned to multiples of
    // kEnergyRows), then fixed point, so that their sums depend neither on the
    // rows per unit nor on which warp took which unit
    for (int b0 = r0; b0 < r1; b0 += kEnergyRows) {
      const int b1 = min(r1, b0 + kEnergyRows);
      // em: the term of i's label (and bead-bead); e3: bead i with site j.
      // The virials are summed scaled by -2^32 (exact: a power of two).
      float em = 0.f, e3 = 0.f;
      float2 v03 = make_float2(0.f, 0.f), v15 = v03, v24 = v03;  // virial pairs (0,3), (1,5), (2,4)
      auto pair = [&](int t, const int4& pj) {
        // nearest image: the wrapped difference of the box fractions (it and
        // ANINT could choose differently only at |d| = L/2, beyond the cutoff)
        // packed FP32 pairs (fmul/ffma .f32x2) round each element as the
        // scalar instructions do
        const float2 d01 = __fmul2_rn(make_float2((float)(int)((unsigned)pi.x - (unsigned)pj.x),
                                                  (float)(int)((unsigned)pi.y - (unsigned)pj.y)),
                                      uxy);
        const float d0 = d01.x, d1 = d01.y;
        const float d2 = (float)(int)((unsigned)pi.z - (unsigned)pj.z) * uz;
        const float r2 = __fmaf_rn(d2, d2, __fmaf_rn(d1, d1, d0 * d0));
        if (!(r2 < A.rcut_hi)) return;
        if (r2 > A.rcut_lo) {  // at the cutoff: k_nb_near decides and computes it
          const unsigned k = atomicAdd(&sc->near_n[A.work], 1u);
          if (k < (unsigned)A.near_cap) A.near[k] = make_int4(s, t, A.idx[A.sorted[s]], A.idx[A.sorted[t]]);
          return;  // beyond the buffer: k_nb_near has the step repeated with a larger one
        }
        const int wj = pj.w;
        const int tj = wj & 0xffff, lj = wj >> 16;
        const int4 pt = pti[tj];
        const float r = r2 * rsqrtf(r2);
        const float rb = r * __int_as_float(pt.z);  // r / bin
        int ni = (int)rb;
        // a missing table (all-zero descriptor) or a distance beyond the table
        // stops the step with an error; the row read stays inside the array
        // (it holds at least two rows), so no branch is needed here
        err |= pt.w ? 0u : (unsigned)EB_MISSING_TABLE;
        err |= ni > pt.y ? (unsigned)EB_TABLE_RANGE : 0u;
        ni = min(ni, pt.y);
        // linear interpolation between rows ni and ni + 1 (NONBONDED_FORCE.F90:66-74)
        const float u = rb - (float)ni;
        const float4 co = tco[pt.x + ni];  // {F base, P base, dF, dP}
        const float2 fv = __ffma2_rn(make_float2(co.z, co.w), make_float2(u, u), make_float2(co.x, co.y));
        const float fij = fv.x, vij = fv.y;
        if (MIXED) {
          em += (!i_bead || lj == 2) ? vij : 0.f;
          e3 += (i_bead && lj == 3) ? vij : 0.f;
        } else {
          em += vij;
        }
        // j's share in fixed point, round(-f * 2^32): fs * d equals the
        // product f_c * -2^32 exactly (scaling by a power of two), and
        // round-to-nearest is symmetric, so i's share is exactly its negation.
        // |f component| <= |fij| r (to rounding): one test keeps every
        // component in range
        const float fs = fij * -kFixScale;
        err |= fabsf(fs) * r < kFixLimScaled ? 0u : (unsigned)EB_FIXED;
        const float2 sxy = __fmul2_rn(make_float2(fs, fs), d01);
        const float sx = sxy.x, sy = sxy.y, sz = fs * d2;
        const long long qx = __float2ll_rn(sx), qy = __float2ll_rn(sy), qz = __float2ll_rn(sz);
        fi0 -= qx; fi1 -= qy; fi2 -= qz;
        unsigned long long* fj = (unsigned long long*)A.fsort + fs_at(t);
        atomicAdd(fj, (unsigned long long)qx);
        atomicAdd(fj + 32, (unsigned long long)qy);
        atomicAdd(fj + 64, (unsigned long long)qz);
        // (xx, yx) += (sx, sy) d0; (yy, zy) += (sy, sz) d1; (zz, zx) += sz (d2, d0)
        v03 = __ffma2_rn(sxy, make_float2(d0, d0), v03);
        v15 = __ffma2_rn(make_float2(sy, sz), make_float2(d1, d1), v15);
        v24 = __ffma2_rn(make_float2(sz, sz), make_float2(d2, d0), v24);
      };
      // list entries are read once per launch: loaded evict-first (__ldcs),
      // so that the streamed list does not push the positions and force sums
      // it points into out of L2
      for (int it = b0; it < b1; it += 2) {
        const bool v0 = it * T + q < cnt;
        const bool v1 = it + 1 < b1 && (it + 1) * T + q < cnt;
        const int t0 = v0 ? __ldcs(ent + it * 32) : 0;
        const int t1 = v1 ? __ldcs(ent + (it + 1) * 32) : 0;
        const int4 p0 = pos[t0];
        const int4 p1 = pos[t1];
        if (v0) pair(t0, p0);
        if (v1) pair(t1, p1);
      }
      long long v[8];
      v[0] = fixq<24>(em, err);
      v[1] = fixq<24>(e3, err);
      {
        const float vir[6] = {v03.x, v15.x, v24.x, v03.y, v24.y, v15.y};
#pragma unroll
        for (int k = 0; k < 6; ++k) v[2 + k] = fixq<24>(vir[k] * -0x1p-32f, err);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], 1);
      if (!(lane & 1)) {
        la[(li == 1 ? 0 : (i_bead ? 1 : 2)) * kNbPairs] += v[0];
        la[2 * kNbPairs] += v[1];
#pragma unroll
        for (int k = 0; k < 6; ++k) la[(3 + k) * kNbPairs] += v[2 + k];
      }
    }
#pragma unroll
    for (int o = T / 2; o > 0; o >>= 1) {
      fi0 += __shfl_down_sync(0xffffffffu, fi0, o, T);
      fi1 += __shfl_down_sync(0xffffffffu, fi1, o, T);
      fi2 += __shfl_down_sync(0xffffffffu, fi2, o, T);
    }
    if (q == 0 && valid && r0 * T < cnt) {
      unsigned long long* fo = (unsigned long long*)A.fsort + fs_at(s);
      atomicAdd(fo, (unsigned long long)fi0);
      atomicAdd(fo + 32, (unsigned long long)fi1);
      atomicAdd(fo + 64, (unsigned long long)fi2);
    }
  };
  nb_schedule(A, bk, nunits, unit);
  if (err) atomicOr(&sc->err, err);
  long long acc[9];
  for (int k = 0; k < 9; ++k) acc[k] = (threadIdx.x & 1) ? 0 : lacc[k * kNbPairs + (threadIdx.x >> 1)];
  __syncthreads();
  block_sum_i64<9>(acc, lacc);
  if (threadIdx.x < 9 && lacc[threadIdx.x] != 0)
    atomicAdd(&sc->nbacc[A.work][threadIdx.x], (unsigned long long)lacc[threadIdx.x]);
}

// NONBONDED_FORCE.F90:45-104 over slice lists (k_list_build_slices), FP32
// force path.  A warp takes a unit of `rows` rows of one slice: its 32 lanes
// take 32 entries of the slice's list at a time, and each lane evaluates the
// pairs of its entry's neighbour with the (up to four) particles of its mask,
// holding the four particles' positions in registers.  The pair arithmetic,
// cutoff handling, error bits, fixed-point conversion and energy/virial
// grouping are those of k_nonbonded_f32, so every pair's force
// contribution is the same integer and the force sums are bit for bit those
// of the per-particle form.  What changes is what a pair costs in memory
// traffic: one list entry, one position gather and one set of three j-force
// atomics serve all the pairs of an entry, and the slice's i-forces are
// summed over the warp once per unit (a butterfly that leaves each of the
// twelve sums on one pair of lanes) before one atomic each.
template <bool SMEM, bool MIXED, bool B>
__global__ void __launch_bounds__(256, 3) k_nonbonded_slices(__grid_constant__ const NBArgs<float> A0,
                                                             const NBArgs<float>* const* tab, const BlockMap bm) {
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  __shared__ NBArgs<float> s_args;
  if (B) stage_args(&s_args, tab[bk.sys]);
  const NBArgs<float>& A = B ? s_args : A0;
  Scalars* sc = A.sc;
  if (nb_idle(A)) return;
  extern __shared__ unsigned char smem_raw[];
  long long* lacc = (long long*)smem_raw;  // [9][kNbPairs] sums of each pair of lanes
  const int4* ptab = A.ptab;
  const float4* tco = A.tcoef;
  {
    unsigned char* p = smem_raw + kNbAccBytes;
    if (SMEM) {
      int4* s_ptab = (int4*)p;       p += sizeof(int4) * A.ntype * A.ntype;
      float4* s_co = (float4*)p;
      for (int k = threadIdx.x; k < A.nrows; k += blockDim.x) s_co[k] = A.tcoef[k];
      for (int k = threadIdx.x; k < A.ntype * A.ntype; k += blockDim.x) s_ptab[k] = A.ptab[k];
      ptab = s_ptab; tco = s_co;
    }
  }
  if (!(threadIdx.x & 1))
    for (int k = 0; k < 9; ++k) lacc[k * kNbPairs + (threadIdx.x >> 1)] = 0;
  __syncthreads();
  const float ux = (float)(sc->box[0] * 0x1p-32), uy = (float)(sc->box[1] * 0x1p-32), uz = (float)(sc->box[2] * 0x1p-32);
  const float2 uxy = make_float2(ux, uy);
  const int4* pos = A.posq;
  const int lane = threadIdx.x & 31;
  unsigned err = 0;
  const int rows = A.rows;
  const int U = (A.w_cap + rows - 1) / rows;
  const int nunits = A.nslices * U;
  long long* la = lacc + (threadIdx.x >> 1);
  // each warp's slice: the positions of its four particles, read from shared
  // memory by the pair passes (held in registers they push the kernel past
  // its 80-register bound into spills)
  __shared__ int4 s_pi[8][kUSlots];
  auto unit = [&](int u) {
    const int g = u / U;
    const int r0 = (u - g * U) * rows;
    const int w = min(A.slice_w[g], A.w_cap);
    if (r0 >= w) return;
    const int r1 = min(w, r0 + rows);
    const int s0 = kUSlots * g;
    int4* pi = s_pi[threadIdx.x >> 5];
    if (lane < kUSlots) pi[lane] = s0 + lane < A.n ? pos[s0 + lane] : make_int4(0, 0, 0, 0);
    __syncwarp();
    const int* ent = A.entries + (long long)g * A.w_cap * 32 + lane;
    long long fi[kUSlots][3];
#pragma unroll
    for (int k = 0; k < kUSlots; ++k) fi[k][0] = fi[k][1] = fi[k][2] = 0;
    // energies and virials: FP32 over kEnergyRows rows, then fixed point
    for (int b0 = r0; b0 < r1; b0 += kEnergyRows) {
      const int b1 = min(r1, b0 + kEnergyRows);
      // V_NB(1), V_NB(2), V_NB(3) terms (MIXED); e1 alone otherwise.  The
      // virials are summed scaled by -2^32 (exact: a power of two).
      float e1 = 0.f, e2 = 0.f, e3 = 0.f;
      float2 v03 = make_float2(0.f, 0.f), v15 = v03, v24 = v03;
      auto entry = [&](int e, const int4& pj) {
        const int t = (int)((unsigned)e & kUSlotMask);
        const unsigned m = (unsigned)e >> 28;
        const int wj = pj.w;
        const int tj = wj & 0xffff, lj = wj >> 16;
        long long qj0 = 0, qj1 = 0, qj2 = 0;
        bool hit = false;
#pragma unroll
        for (int k = 0; k < kUSlots; ++k) {
          if (!((m >> k) & 1u)) continue;
          const int4 pik = pi[k];
          const float2 d01 = __fmul2_rn(make_float2((float)(int)((unsigned)pik.x - (unsigned)pj.x),
                                                    (float)(int)((unsigned)pik.y - (unsigned)pj.y)),
                                        uxy);
          const float d0 = d01.x, d1 = d01.y;
          const float d2 = (float)(int)((unsigned)pik.z - (unsigned)pj.z) * uz;
          const float r2 = __fmaf_rn(d2, d2, __fmaf_rn(d1, d1, d0 * d0));
          if (!(r2 < A.rcut_hi)) continue;
          if (r2 > A.rcut_lo) {  // at the cutoff: k_nb_near decides and computes it
            const unsigned kk = atomicAdd(&sc->near_n[A.work], 1u);
            if (kk < (unsigned)A.near_cap)
              A.near[kk] = make_int4(s0 + k, t, A.idx[A.sorted[s0 + k]], A.idx[A.sorted[t]]);
            continue;  // beyond the buffer: k_nb_near has the step repeated with a larger one
          }
          const int wi = pik.w;
          const int ti = wi & 0xffff, li = wi >> 16;
          const int4 pt = ptab[ti * A.ntype + tj];
          const float r = r2 * rsqrtf(r2);
          const float rb = r * __int_as_float(pt.z);  // r / bin
          int ni = (int)rb;
          err |= pt.w ? 0u : (unsigned)EB_MISSING_TABLE;
          err |= ni > pt.y ? (unsigned)EB_TABLE_RANGE : 0u;
          ni = min(ni, pt.y);
          const float uu = rb - (float)ni;
          const float4 co = tco[pt.x + ni];  // {F base, P base, dF, dP}
          const float2 fv = __ffma2_rn(make_float2(co.z, co.w), make_float2(uu, uu), make_float2(co.x, co.y));
          const float fij = fv.x, vij = fv.y;
          if (MIXED) {
            // V_NB(1) for an atom i, V_NB(3) for a site i or a bead i with a
            // site j, V_NB(2) for two beads
            if (li == 1) e1 += vij;
            else if (li == 3 || lj == 3) e3 += vij;
            else if (lj == 2) e2 += vij;
          } else {
            e1 += vij;
          }
          const float fs = fij * -kFixScale;
          err |= fabsf(fs) * r < kFixLimScaled ? 0u : (unsigned)EB_FIXED;
          const float2 sxy = __fmul2_rn(make_float2(fs, fs), d01);
          const float sx = sxy.x, sy = sxy.y, sz = fs * d2;
          const long long qx = __float2ll_rn(sx), qy = __float2ll_rn(sy), qz = __float2ll_rn(sz);
          fi[k][0] -= qx; fi[k][1] -= qy; fi[k][2] -= qz;
          qj0 += qx; qj1 += qy; qj2 += qz;
          hit = true;
          v03 = __ffma2_rn(sxy, make_float2(d0, d0), v03);
          v15 = __ffma2_rn(make_float2(sy, sz), make_float2(d1, d1), v15);
          v24 = __ffma2_rn(make_float2(sz, sz), make_float2(d2, d0), v24);
        }
        if (hit) {
          unsigned long long* fj = (unsigned long long*)A.fsort + fs_at(t);
          atomicAdd(fj, (unsigned long long)qj0);
          atomicAdd(fj + 32, (unsigned long long)qj1);
          atomicAdd(fj + 64, (unsigned long long)qj2);
        }
      };
      // two rows per iteration: both entry loads and both position gathers
      // in flight before either is evaluated; entries are read once per
      // launch (evict-first), empty ones (mask 0) point at slot 0
      for (int it = b0; it < b1; it += 2) {
        const bool has1 = it + 1 < b1;
        const int ea = __ldcs(ent + it * 32);
        const int eb = has1 ? __ldcs(ent + (it + 1) * 32) : 0;
        const int4 pa = pos[(unsigned)ea & kUSlotMask];
        const int4 pb = pos[(unsigned)eb & kUSlotMask];
        entry(ea, pa);
        if (has1) entry(eb, pb);
      }
      long long v[9];
      v[0] = fixq<24>(e1, err);
      v[1] = MIXED ? fixq<24>(e2, err) : 0;
      v[2] = MIXED ? fixq<24>(e3, err) : 0;
      {
        const float vir[6] = {v03.x, v15.x, v24.x, v03.y, v24.y, v15.y};
#pragma unroll
        for (int k = 0; k < 6; ++k) v[3 + k] = fixq<24>(vir[k] * -0x1p-32f, err);
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], 1);
      if (!(lane & 1)) {
        if (MIXED) {
#pragma unroll
          for (int k = 0; k < 3; ++k) la[k * kNbPairs] += v[k];
        } else {
          const int li = pi[0].w >> 16;  // the list's one label
          la[(li == 1 ? 0 : (li == 2 ? 1 : 2)) * kNbPairs] += v[0];
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) la[(3 + k) * kNbPairs] += v[3 + k];
      }
    }
    // the twelve i-force sums over the warp: at each level a lane keeps one
    // half of its values and adds the partner's share of that half, which
    // leaves sum 8 b4 + 4 b3 + 2 b2 + b1 (b: the lane's bits) on lanes 2m, 2m+1
    long long v[16];
#pragma unroll
    for (int k = 0; k < kUSlots; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) v[3 * k + c] = fi[k][c];
#pragma unroll
    for (int k = 12; k < 16; ++k) v[k] = 0;
#pragma unroll
    for (int h = 8, o = 16; h >= 1; h >>= 1, o >>= 1) {
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int j = 0; j < h; ++j) {
        const long long send = up ? v[j] : v[j + h];
        const long long keep = up ? v[j + h] : v[j];
        v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
    const long long tot = v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
    const int vi = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
    if (!(lane & 1) && vi < 3 * kUSlots && tot != 0) {
      const int s = s0 + vi / 3;
      if (s < A.n) atomicAdd((unsigned long long*)A.fsort + fs_at(s) + 32 * (vi % 3), (unsigned long long)tot);
    }
    __syncwarp();  // pi is rewritten by the next unit
  };
  nb_schedule(A, bk, nunits, unit);
  if (err) atomicOr(&sc->err, err);
  long long acc[9];
  for (int k = 0; k < 9; ++k) acc[k] = (threadIdx.x & 1) ? 0 : lacc[k * kNbPairs + (threadIdx.x >> 1)];
  __syncthreads();
  block_sum_i64<9>(acc, lacc);
  if (threadIdx.x < 9 && lacc[threadIdx.x] != 0)
    atomicAdd(&sc->nbacc[A.work][threadIdx.x], (unsigned long long)lacc[threadIdx.x]);
}

// Whether the pair of particles gi, gj (FP32 r^2 = r2) lies inside the cutoff as
// the FP64 path decides it: the same fold of the FP64 state into the box
// (SHIFT), nearest image and sum of squares as k_positions<double> and
// k_nonbonded<double>.  FP32 rounding of r^2 (a relative ~5e-7) would
// otherwise take pairs that sit at the cutoff in or out against that path,
// each a jump of F(rc) r_c in the force (1.3e-5 of the largest force on the
// 40,000-bead melt).  A pair with a virtual site keeps the FP32 decision: its
// FP64 position is not kept on this path.
__device__ bool inside_as_fp64(const NBArgs<float>& A, const Scalars* sc, int gi, int gj, float r2) {
  if (gi >= A.natoms || gj >= A.natoms) return r2 < A.rcutsq;
  double b[3], bi[3], b2[3];
  box_of<double>(sc, b, bi, b2);
  double ri[3], rj[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    ri[c] = A.S[3 * (size_t)gi + c];
    rj[c] = A.S[3 * (size_t)gj + c];
  }
  fold3<double>(ri, b2);
  fold3<double>(rj, b2);
  double d[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    d[c] = ri[c] - rj[c];
    d[c] = d[c] - r_round(d[c] * bi[c]) * b[c];
  }
  double q = d[0] * d[0];
  q = q + d[1] * d[1];
  q = q + d[2] * d[2];
  return q < (double)A.rcutsq;
}

// The pairs the FP32 kernel left at the cutoff: each is decided as the FP64
// path decides it (inside_as_fp64) and, when inside, computed with the FP32
// kernel's pair arithmetic; its energy and virial terms go to the system's
// fixed-point sums one pair at a time.  One block per system and list; the
// block clears the list's pair count for the next launch.  When more pairs came
// than the buffer holds, the step is aborted and repeated with a larger one.
template <bool B>
__global__ void __launch_bounds__(256) k_nb_near(__grid_constant__ const NBArgs<float> A0,
                                                 const NBArgs<float>* const* tab, const BlockMap bm) {
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  const NBArgs<float>& A = B ? *tab[bk.sys] : A0;
  Scalars* sc = A.sc;
  if (nb_idle(A)) return;
  __shared__ long long red[32 + 9 * 8];  // block_sum_i64: 32 results + 9 per warp
  const unsigned n = sc->near_n[A.work];
  if (n > (unsigned)A.near_cap) {
    // the pairs did not fit: record the need and abort the step, which the
    // host repeats with a larger buffer (as for the Verlet-list storage)
    __syncthreads();  // every thread has read the count
    if (threadIdx.x == 0) {
      sc->need_near[A.work] = (int)n;
      sc->near_n[A.work] = 0u;
      sc->abort = 1;
      sc->skip = 1;
    }
    return;
  }
  const float ux = (float)(sc->box[0] * 0x1p-32), uy = (float)(sc->box[1] * 0x1p-32), uz = (float)(sc->box[2] * 0x1p-32);
  unsigned err = 0;
  long long acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (unsigned k = threadIdx.x; k < n; k += blockDim.x) {
    const int4 nk = A.near[k];
    const int s = nk.x, t = nk.y;
    const int4 pi = A.posq[s], pj = A.posq[t];
    const float d0 = (float)(int)((unsigned)pi.x - (unsigned)pj.x) * ux;
    const float d1 = (float)(int)((unsigned)pi.y - (unsigned)pj.y) * uy;
    const float d2 = (float)(int)((unsigned)pi.z - (unsigned)pj.z) * uz;
    const float r2 = __fmaf_rn(d2, d2, __fmaf_rn(d1, d1, d0 * d0));
    if (!inside_as_fp64(A, sc, nk.z, nk.w, r2)) continue;
    const int ti = pi.w & 0xffff, li = pi.w >> 16, tj = pj.w & 0xffff, lj = pj.w >> 16;
    const int4 pt = A.ptab[ti * A.ntype + tj];
    if (!pt.w) { err |= EB_MISSING_TABLE; continue; }
    const float r = r2 * rsqrtf(r2);
    const float ib = __int_as_float(pt.z);
    const int ni = (int)(r * ib);
    if (ni > pt.y) { err |= EB_TABLE_RANGE; continue; }
    const int row = pt.x + ni;
    const float alpha = (r - A.tx[row]) * ib;
    const float2 a0 = ((const float2*)A.tfp)[row], a1 = ((const float2*)A.tfp)[row + 1];
    const float fij = __fmaf_rn(a1.x - a0.x, alpha, a0.x);
    const float vij = __fmaf_rn(a1.y - a0.y, alpha, a0.y);
    if (!(fabsf(fij) * r < 0.99f * kFixMax)) { err |= EB_FIXED; continue; }
    const float fx = fij * d0, fy = fij * d1, fz = fij * d2;
    const long long qx = __float2ll_rn(fx * kFixScale), qy = __float2ll_rn(fy * kFixScale),
                    qz = __float2ll_rn(fz * kFixScale);
    unsigned long long* fsi = (unsigned long long*)A.fsort + fs_at(s);
    unsigned long long* fsj = (unsigned long long*)A.fsort + fs_at(t);
    atomicAdd(fsi, (unsigned long long)qx);
    atomicAdd(fsi + 32, (unsigned long long)qy);
    atomicAdd(fsi + 64, (unsigned long long)qz);
    atomicAdd(fsj, (unsigned long long)(-qx));
    atomicAdd(fsj + 32, (unsigned long long)(-qy));
    atomicAdd(fsj + 64, (unsigned long long)(-qz));
    const bool lab3 = li == 3 || lj == 3;
    const long long qe = fixq<24>(vij, err);
    if (li == 1) acc[0] += qe;
    if (li == 2 && lj == 2) acc[1] += qe;
    if (li != 1 && lab3) acc[2] += qe;
    acc[3] += fixq<24>(fx * d0, err);
    acc[4] += fixq<24>(fy * d1, err);
    acc[5] += fixq<24>(fz * d2, err);
    acc[6] += fixq<24>(fy * d0, err);
    acc[7] += fixq<24>(fz * d0, err);
    acc[8] += fixq<24>(fz * d1, err);
  }
  if (err) atomicOr(&sc->err, err);
  block_sum_i64<9>(acc, red);
  if (threadIdx.x < 9 && red[threadIdx.x] != 0)
    atomicAdd(&sc->nbacc[A.work][threadIdx.x], (unsigned long long)red[threadIdx.x]);
  __syncthreads();
  if (threadIdx.x == 0) sc->near_n[A.work] = 0u;
}

// Per-slot forces of both lists into the global-order nonbonded force
// array; the bead list's MTS history is saved (MTS_SAVEFORCE, explicit steps)
// or used for the extrapolation F = F3 + (m-3)/2 (F3 - F1) (MTS_APPROX,
// MTS_LOOP.f90:176).  The slot buffer is cleared for the next step.
template <typename R>
struct CollectArgs {
  Scalars* sc;
  int n;                         // slots in this list
  int mts;                       // 1 for the bead list of an MTS run
  const int* sorted;             // slot -> A
  const int* idx;                // A -> global id
  typename Prec<R>::acc_t* fsort;
  typename Prec<R>::acc_t* fnb;  // (3,NITEMS) global order
  typename Prec<R>::acc_t* mtsf; // [3][n][3] by A
};

template <typename R, bool B>
__global__ void k_nb_collect(__grid_constant__ const CollectArgs<R> C0, const CollectArgs<R>* const* tab,
                             const BlockMap bm) {
  using P = Prec<R>;
  pdl_wait();
  const Blk bk = blk<B>(bm);
  const CollectArgs<R>& C = B ? *tab[bk.sys] : C0;
  Scalars* sc = C.sc;
  if (sc->skip) return;
  const int m = sc->mts_m;
  const bool explicit_step = !C.mts || (m >= 1 && m <= 3);
  for (int s = bk.b * blockDim.x + threadIdx.x; s < C.n; s += bk.g * blockDim.x) {
    const int a = C.sorted[s];
    const int gi = C.idx[a];
    if (explicit_step) {
      // all three loads before the first store (the arrays may alias as far
      // as the compiler knows)
      typename P::acc_t v[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) v[c] = C.fsort[fs_at(s) + 32 * c];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        C.fnb[3 * (size_t)gi + c] = v[c];
        if (C.mts) C.mtsf[((size_t)(m - 1) * C.n + a) * 3 + c] = v[c];
        C.fsort[fs_at(s) + 32 * c] = 0;
      }
    } else {
      const double coef = (double)(m - 3) * 0.5;
      double f3[3], f1[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        f3[c] = P::get(C.mtsf[((size_t)2 * C.n + a) * 3 + c]);
        f1[c] = P::get(C.mtsf[((size_t)0 * C.n + a) * 3 + c]);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
        C.fnb[3 * (size_t)gi + c] = (typename P::acc_t)P::from_double(f3[c] + coef * (f3[c] - f1[c]), &sc->err);
    }
  }
}

template <typename R>
struct DistArgs {
  Scalars* sc;
  typename Prec<R>::acc_t* F[2];  // nonbonded / bonded forces (3,NITEMS)
  int natoms, nvirta;
  const int* vnum;
  const int* vmem;
  const float* vcoef;
};

// DISTRIBUTE_VSFORCE.f90:27-37: F(atom) += F(vs) * VIRT_MASSCOEFF; F(vs) = 0,
// on the nonbonded (which = 0) or bonded (which = 1) forces.
template <typename R, bool B>
__global__ void k_distribute(__grid_constant__ const DistArgs<R> D0, const DistArgs<R>* const* tab, const BlockMap bm,
                             int which) {
  pdl_wait();
  pdl_trigger();
  using P = Prec<R>;
  const Blk bk = blk<B>(bm);
  const DistArgs<R>& D = B ? *tab[bk.sys] : D0;
  Scalars* sc = D.sc;
  if (sc->skip) return;
  typename P::acc_t* F = D.F[which];
  const int natoms = D.natoms, nvirta = D.nvirta;
  const int* vnum = D.vnum;
  const int* vmem = D.vmem;
  const float* vcoef = D.vcoef;
  // 16 lanes per site (half a warp), one member each (VIRT_NUMATOMS <= 15)
  const int hl = threadIdx.x & 15;
  const unsigned half = 0xffffu << (threadIdx.x & 16);
  const int h0 = (bk.b * blockDim.x + threadIdx.x) >> 4, nh = (bk.g * blockDim.x) >> 4;
  for (int v = h0; v < nvirta; v += nh) {
    const size_t vs = (size_t)(natoms + v);
    double f[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) f[c] = P::get(F[3 * vs + c]);
    if (hl < vnum[v]) {
      const int j = vmem[v * 15 + hl];
      const double cf = (double)vcoef[v * 15 + hl];
#pragma unroll
      for (int c = 0; c < 3; ++c) P::add(&F[3 * (size_t)j + c], P::from_double(f[c] * cf, &sc->err));
    }
    __syncwarp(half);  // the site's 16 lanes have read F(vs)
    if (hl == 0)
#pragma unroll
      for (int c = 0; c < 3; ++c) F[3 * vs + c] = 0;
  }
}

// --------------------------------------------------------------- bonded
template <typename A>
struct BondedArgs {
  Scalars* sc;
  const double* su;                // unwrapped positions (3,NITEMS), FP64
  typename Prec<A>::acc_t* fb;     // bonded forces (3,NITEMS)
  int nb, na, nt, no;
  const int4* bonds;               // i, j, table, label
  const int4* angles;              // i, j, k, table | label<<24
  const int4* tors;                // i, j, k, l
  const int2* tors_t;              // table, label
  const int4* oops;
  const int2* oops_t;
  // tables: rows {X, F, P, 0}; table t starts at off[t]
  const float4* tb; const int* tb_off; const int* tb_ndat; const float* tb_bin;
  const float4* ta; const int* ta_off; const int* ta_ndat; const float* ta_bin;
  const float4* tt; const int* tt_off; const int* tt_ndat; const float* tt_bin;
  const float4* to; const int* to_off; const int* to_ndat; const float* to_bin;
  float r2d;
  double* part;   // 12 per block: V_BOND(3), V_ANGLE(3), V_TORSION(3), V_OOP(3)
  int part_stride;
};

template <typename R>
__device__ __forceinline__ R lerp_mixed(R y0, R y1, R alpha) {
  // y0*(1.0D0-alpha) + alpha*y1 with the FP64 promotion of BONDS.inc:36-40
  return (R)((double)y0 * (1.0 - (double)alpha) + (double)(alpha * y1));
}

template <typename A>
__device__ __forceinline__ void addf(typename Prec<A>::acc_t* F, int i, const double* f, unsigned* err) {
  using P = Prec<A>;
  P::add(&F[3 * (size_t)i + 0], P::from_double(f[0], err));
  P::add(&F[3 * (size_t)i + 1], P::from_double(f[1], err));
  P::add(&F[3 * (size_t)i + 2], P::from_double(f[2], err));
}

// BONDS.inc:3-57, ANGLES.inc:2-75, TORSIONS.inc:1-152, OUTOFPLANES.inc:1-141
// with one thread per term; the four term kinds share the grid.  The bonded
// geometry is evaluated in FP64 on both paths: acos near straight angles and
// trans dihedrals amplifies REAL*4 rounding (about 1e-5 of the largest force
// in a strained chain), while the terms are few; the forces are summed in the
// path's accumulator (64-bit fixed point on the FP32 path).
template <typename A, bool BA>
__global__ void __launch_bounds__(256) k_bonded(__grid_constant__ const BondedArgs<A> B0, const BondedArgs<A>* const* tab,
                                                const BlockMap bm) {
  using R = double;
  const Blk bk = blk<BA>(bm);
  const BondedArgs<A>& B = BA ? *tab[bk.sys] : B0;
  Scalars* sc = B.sc;
  __shared__ double red[12 * 8];
  double acc[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) acc[k] = 0.0;
  unsigned long long overext = 0;
  unsigned* err = &sc->err;
  const R* S = B.su;
  const int total = sc->skip ? 0 : B.nb + B.na + B.nt + B.no;
  auto pos = [&](int i, R* o) { o[0] = S[3 * (size_t)i]; o[1] = S[3 * (size_t)i + 1]; o[2] = S[3 * (size_t)i + 2]; };
  for (int u = bk.b * blockDim.x + threadIdx.x; u < total; u += bk.g * blockDim.x) {
    if (u < B.nb) {  // -------------------------------- bond
      const int4 e = B.bonds[u];
      R ri[3], rj[3], d[3];
      pos(e.x, ri); pos(e.y, rj);
      for (int c = 0; c < 3; ++c) d[c] = ri[c] - rj[c];
      R rsq = d[0] * d[0] + d[1] * d[1];
      rsq = rsq + d[2] * d[2];
      const R rij = r_sqrt(rsq);
      const int t = e.z;
      const float4* T = B.tb + B.tb_off[t];
      const R bin = (R)B.tb_bin[t];
      int k = fint((rij - (R)T[0].x) / bin);
      if (k > B.tb_ndat[t]) { ++overext; k = B.tb_ndat[t]; }
      else if (k < 0) k = 0;
      const float4 r0 = T[k], r1 = T[k + 1];
      const R alpha = (rij - (R)r0.x) / bin;
      const R fij = lerp_mixed<R>((R)r0.y, (R)r1.y, alpha);
      const R vij = lerp_mixed<R>((R)r0.z, (R)r1.z, alpha);
      acc[e.w - 1] += (double)vij;
      R f[3], mf[3];
      for (int c = 0; c < 3; ++c) { f[c] = fij * d[c]; mf[c] = -f[c]; }
      addf<A>(B.fb, e.x, f, err);
      addf<A>(B.fb, e.y, mf, err);
    } else if (u < B.nb + B.na) {  // ---------------- angle
      const int4 e = B.angles[u - B.nb];
      const int t = e.w & 0xffffff, lab = e.w >> 24;
      R ri[3], rj[3], rk[3], ij[3], kj[3];
      pos(e.x, ri); pos(e.y, rj); pos(e.z, rk);
      for (int c = 0; c < 3; ++c) { ij[c] = ri[c] - rj[c]; kj[c] = rk[c] - rj[c]; }
      const R rij = r_sqrt((ij[0] * ij[0] + ij[1] * ij[1]) + ij[2] * ij[2]);
      const R rkj = r_sqrt((kj[0] * kj[0] + kj[1] * kj[1]) + kj[2] * kj[2]);
      R ct = ((ij[0] * kj[0] + ij[1] * kj[1]) + ij[2] * kj[2]) / rij / rkj;
      ct = ct > (R)1 ? (R)1 : (ct < (R)-1 ? (R)-1 : ct);  // rounding of a straight angle (the oracle clamps too)
      const R theta = r_acos(ct) * (R)B.r2d;
      R m[3];
      m[0] = -(ij[1] * kj[2] - ij[2] * kj[1]);
      m[1] = -(-ij[0] * kj[2] + ij[2] * kj[0]);
      m[2] = -(ij[0] * kj[1] - ij[1] * kj[0]);
      const R rm = r_sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
      for (int c = 0; c < 3; ++c) m[c] = m[c] / rm;
      R nn[3], ss[3];
      nn[0] = (m[1] * ij[2] - m[2] * ij[1]) / rij;
      nn[1] = (-m[0] * ij[2] + m[2] * ij[0]) / rij;
      nn[2] = (m[0] * ij[1] - m[1] * ij[0]) / rij;
      ss[0] = -(m[1] * kj[2] - m[2] * kj[1]) / rkj;
      ss[1] = -(-m[0] * kj[2] + m[2] * kj[0]) / rkj;
      ss[2] = -(m[0] * kj[1] - m[1] * kj[0]) / rkj;
      const float4* T = B.ta + B.ta_off[t];
      const R bin = (R)B.ta_bin[t];
      int k = fint(theta / bin);
      if (k < 0 || k > B.ta_ndat[t] + 1) { atomicOr(err, EB_TABLE_RANGE); continue; }
      R fijk, vijk;
      const float4 r0 = T[k];
      if (theta == (R)180.0) {
        fijk = (R)r0.y; vijk = (R)r0.z;
      } else {
        const float4 r1 = T[k + 1];
        const R alpha = (theta - (R)r0.x) / bin;
        fijk = lerp_mixed<R>((R)r0.y, (R)r1.y, alpha);
        vijk = lerp_mixed<R>((R)r0.z, (R)r1.z, alpha);
      }
      acc[3 + lab - 1] += (double)vijk;
      R fI[3], fK[3], mI[3], mK[3];
      for (int c = 0; c < 3; ++c) {
        fI[c] = fijk * nn[c] / rij;
        fK[c] = fijk * ss[c] / rkj;
        mI[c] = -fI[c]; mK[c] = -fK[c];
      }
      addf<A>(B.fb, e.x, fI, err);
      addf<A>(B.fb, e.z, fK, err);
      addf<A>(B.fb, e.y, mK, err);
      addf<A>(B.fb, e.y, mI, err);
    } else if (u < B.nb + B.na + B.nt) {  // -------- torsion
      const int q = u - B.nb - B.na;
      const int4 e = B.tors[q];
      const int2 tl = B.tors_t[q];
      R ri[3], rj[3], rk[3], rl[3], ij[3], jk[3], kl[3];
      pos(e.x, ri); pos(e.y, rj); pos(e.z, rk); pos(e.w, rl);
      for (int c = 0; c < 3; ++c) { ij[c] = ri[c] - rj[c]; jk[c] = rj[c] - rk[c]; kl[c] = rk[c] - rl[c]; }
      R rij = r_sqrt((ij[0] * ij[0] + ij[1] * ij[1]) + ij[2] * ij[2]);
      const R rjk = r_sqrt((jk[0] * jk[0] + jk[1] * jk[1]) + jk[2] * jk[2]);
      R rkl = r_sqrt((kl[0] * kl[0] + kl[1] * kl[1]) + kl[2] * kl[2]);
      R m[3], nn[3], cosm = 0, sinm = 0, cotanm = 0, cosn = 0, sinn = 0, cotann = 0;
      auto crossm = [&]() {
        m[0] = ij[1] * jk[2] - ij[2] * jk[1];
        m[1] = -ij[0] * jk[2] + ij[2] * jk[0];
        m[2] = ij[0] * jk[1] - ij[1] * jk[0];
      };
      auto crossn = [&]() {
        nn[0] = jk[1] * kl[2] - jk[2] * kl[1];
        nn[1] = -jk[0] * kl[2] + jk[2] * kl[0];
        nn[2] = jk[0] * kl[1] - jk[1] * kl[0];
      };
      crossm();
      R rm = r_sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
      if (rm == (R)0) {  // TORSIONS.inc:47-60: perturb collinear i-j-k
        ij[0] = ri[0] * (R)0.99f - rj[0];
        rij = r_sqrt((ij[0] * ij[0] + ij[1] * ij[1]) + ij[2] * ij[2]);
        crossm();
        rm = r_sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
      }
      if (rm > (R)0 || rm == (R)0) {
        for (int c = 0; c < 3; ++c) m[c] = m[c] / rm;
        cosm = ((ij[0] * jk[0] + ij[1] * jk[1]) + ij[2] * jk[2]) / rij / rjk;
        sinm = r_sqrt((R)1 - cosm * cosm);
        cotanm = cosm / sinm;
      }
      crossn();
      R rn = r_sqrt((nn[0] * nn[0] + nn[1] * nn[1]) + nn[2] * nn[2]);
      if (rn == (R)0) {  // TORSIONS.inc:75-88
        kl[0] = rk[0] - rl[0] * (R)0.99f;
        rkl = r_sqrt((kl[0] * kl[0] + kl[1] * kl[1]) + kl[2] * kl[2]);
        crossn();
        rn = r_sqrt((nn[0] * nn[0] + nn[1] * nn[1]) + nn[2] * nn[2]);
      }
      if (rn > (R)0 || rn == (R)0) {
        for (int c = 0; c < 3; ++c) nn[c] = nn[c] / rn;
        cosn = ((jk[0] * kl[0] + jk[1] * kl[1]) + jk[2] * kl[2]) / rjk / rkl;
        sinn = r_sqrt((R)1 - cosn * cosn);
        cotann = cosn / sinn;
      }
      R cost = (m[0] * nn[0] + m[1] * nn[1]) + m[2] * nn[2];
      const R signt = -((m[0] * kl[0] + m[1] * kl[1]) + m[2] * kl[2]);
      if (cost > (R)1.0) cost = (R)1.0;
      else if (cost < (R)-1.0) cost = (R)-1.0;
      R phi = r_acos(cost) * (R)B.r2d;
      if (signt < (R)0) phi = (R)360.0 - phi;
      const int t = tl.x;
      const float4* T = B.tt + B.tt_off[t];
      const R bin = (R)B.tt_bin[t];
      const int k = fint(phi / bin);
      if (k < 0 || k > B.tt_ndat[t]) { atomicOr(err, EB_TORSION); continue; }
      R fijkl, vijkl;
      const float4 r0 = T[k];
      if (phi == (R)360.0) {
        fijkl = (R)r0.y; vijkl = (R)r0.z;
      } else {
        const float4 r1 = T[k + 1];
        const R alpha = (phi - (R)r0.x) / bin;
        fijkl = (R)r0.y * ((R)1.0 - alpha) + alpha * (R)r1.y;
        vijkl = (R)r0.z * ((R)1.0 - alpha) + alpha * (R)r1.z;
      }
      acc[6 + tl.y - 1] += (double)vijkl;
      R f1[3], f4[3], f12[3], a[3];
      for (int c = 0; c < 3; ++c) {
        f1[c] = -(fijkl * m[c] / sinm / rij);
        f4[c] = fijkl * nn[c] / sinn / rkl;
        f12[c] = fijkl * (cotanm * m[c] + cotann * nn[c]) / rjk;
      }
      addf<A>(B.fb, e.x, f1, err);
      addf<A>(B.fb, e.w, f4, err);
      for (int c = 0; c < 3; ++c) a[c] = -f1[c];
      addf<A>(B.fb, e.y, a, err);
      addf<A>(B.fb, e.y, f12, err);
      for (int c = 0; c < 3; ++c) a[c] = -f4[c];
      addf<A>(B.fb, e.z, a, err);
      for (int c = 0; c < 3; ++c) a[c] = -f12[c];
      addf<A>(B.fb, e.z, a, err);
    } else {  // ------------------------------------------ out of plane
      const int q = u - B.nb - B.na - B.nt;
      const int4 e = B.oops[q];
      const int2 tl = B.oops_t[q];
      R ri[3], rj[3], rk[3], rl[3], ij[3], jk[3], kl[3];
      pos(e.x, ri); pos(e.y, rj); pos(e.z, rk); pos(e.w, rl);
      for (int c = 0; c < 3; ++c) { ij[c] = ri[c] - rj[c]; jk[c] = rk[c] - rj[c]; kl[c] = rk[c] - rl[c]; }
      const R rij = r_sqrt((ij[0] * ij[0] + ij[1] * ij[1]) + ij[2] * ij[2]);
      const R rjk = r_sqrt((jk[0] * jk[0] + jk[1] * jk[1]) + jk[2] * jk[2]);
      const R rkl = r_sqrt((kl[0] * kl[0] + kl[1] * kl[1]) + kl[2] * kl[2]);
      R m[3], nn[3], mn[3];
      m[0] = ij[1] * jk[2] - ij[2] * jk[1];
      m[1] = -ij[0] * jk[2] + ij[2] * jk[0];
      m[2] = ij[0] * jk[1] - ij[1] * jk[0];
      const R rm = r_sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
      for (int c = 0; c < 3; ++c) m[c] = m[c] / rm;
      const R cm = ((ij[0] * jk[0] + ij[1] * jk[1]) + ij[2] * jk[2]) / rij / rjk;
      const R sm = r_sqrt((R)1 - cm * cm);
      const R ctm = cm / sm;
      nn[0] = jk[1] * kl[2] - jk[2] * kl[1];
      nn[1] = -jk[0] * kl[2] + jk[2] * kl[0];
      nn[2] = jk[0] * kl[1] - jk[1] * kl[0];
      const R rn = r_sqrt((nn[0] * nn[0] + nn[1] * nn[1]) + nn[2] * nn[2]);
      for (int c = 0; c < 3; ++c) nn[c] = nn[c] / rn;
      const R cn = ((jk[0] * kl[0] + jk[1] * kl[1]) + jk[2] * kl[2]) / rjk / rkl;
      const R sn = r_sqrt((R)1 - cn * cn);
      const R ctn = cn / sn;
      R cost = (m[0] * nn[0] + m[1] * nn[1]) + m[2] * nn[2];
      mn[0] = m[1] * nn[2] - m[2] * nn[1];
      mn[1] = -m[0] * nn[2] + m[2] * nn[0];
      mn[2] = m[0] * nn[1] - m[1] * nn[0];
      const R sgn = copysign((R)1.0, (mn[0] * jk[0] + mn[1] * jk[1]) + mn[2] * jk[2]);
      const R eps = (R)1.0e-7f;
      if (cost > (R)1.0 + eps || cost < -((R)1.0 + eps)) { atomicOr(err, EB_OOP); continue; }
      if (cost > (R)1.0) cost = (R)1.0;
      else if (cost < (R)-1.0) cost = (R)-1.0;
      R phi = r_acos(cost);
      phi = sgn * phi;
      phi = phi * (R)B.r2d;
      const R phit = (R)180.0 + phi;
      const int t = tl.x;
      const float4* T = B.to + B.to_off[t];
      const R bin = (R)B.to_bin[t];
      int k = fint(r_round(phit / bin));
      if (k < 0 || k > B.to_ndat[t]) { atomicOr(err, EB_OOP); continue; }
      R alpha = r_abs(r_abs(phi) - r_abs((R)T[k].x)) / bin;
      if (alpha > (R)1.0) {
        k = k + 1;
        alpha = r_abs(r_abs(phi) - r_abs((R)T[k].x)) / bin;
      }
      const float4 r0 = T[k], r1 = T[k + 1];
      const R fijkl = (R)r0.y * ((R)1.0 - alpha) + alpha * (R)r1.y;
      const R vijkl = (R)r0.z * ((R)1.0 - alpha) + alpha * (R)r1.z;
      acc[9 + tl.y - 1] += (double)vijkl;
      R f1[3], f4[3], f12[3], a[3];
      for (int c = 0; c < 3; ++c) {
        f1[c] = fijkl * m[c] / sm / rij;
        f4[c] = -(fijkl * nn[c] / sn / rkl);
        f12[c] = fijkl * (ctm * m[c] + ctn * nn[c]) / rjk;
      }
      addf<A>(B.fb, e.x, f1, err);
      addf<A>(B.fb, e.w, f4, err);
      for (int c = 0; c < 3; ++c) a[c] = -f1[c];
      addf<A>(B.fb, e.y, a, err);
      addf<A>(B.fb, e.y, f12, err);
      for (int c = 0; c < 3; ++c) a[c] = -f4[c];
      addf<A>(B.fb, e.z, a, err);
      for (int c = 0; c < 3; ++c) a[c] = -f12[c];
      addf<A>(B.fb, e.z, a, err);
    }
  }
  if (overext) atomicAdd(&sc->bond_overext, overext);
  double out[12];
  block_sum<12>(acc, red, out);
  if (threadIdx.x == 0)
    for (int k = 0; k < 12; ++k) B.part[k * B.part_stride + bk.b] = out[k];
}

// ------------------------------------------------------------ integration
template <typename R>
struct MoveArgs {
  Scalars* sc;
  int natoms;
  double* S;  // (3,NATOMS) unwrapped, FP64 state
  double* V;  // (3,NATOMS)
  typename Prec<R>::acc_t* fnb;
  typename Prec<R>::acc_t* fb;
  const int* tbits;         // label in bits 16.. (1 atom, 2 bead)
  const double* mass;       // per particle
  const double* invmass;    // per particle
  double dt;
  int update;               // 0: bonded virial only (force stage without MOVE)
  double* part;             // 18 per block
  int part_stride;
};

// MOVE.F90:32-88 (leap-frog with Berendsen factors per class) and the
// bonded virial sum of NEW_FORCE.F90:73-80, which uses the positions before
// the update.  Partials: PTK(6) atoms, PTK(6) beads, bonded virial(6).  The
// bonded forces are folded into the nonbonded array (fnb becomes the total
// force FXYZ of the step) and cleared for the next step.
template <typename R, bool B>
__global__ void __launch_bounds__(256) k_move(__grid_constant__ const MoveArgs<R> M0, const MoveArgs<R>* const* tab,
                                              const BlockMap bm) {
  using P = Prec<R>;
  pdl_wait();
  pdl_trigger();
  const Blk bk = blk<B>(bm);
  const MoveArgs<R>& M = B ? *tab[bk.sys] : M0;
  Scalars* sc = M.sc;
  __shared__ double red[18 * 8];
  double acc[18];
#pragma unroll
  for (int k = 0; k < 18; ++k) acc[k] = 0.0;
  const double lam0 = sc->lam[0], lam1 = sc->lam[1];
  const int nrun = sc->skip ? 0 : M.natoms;
  for (int i = bk.b * blockDim.x + threadIdx.x; i < nrun; i += bk.g * blockDim.x) {
    // every load of the particle is issued before its first store: the
    // arrays may alias as far as the compiler knows, so a store between two
    // loads would make each wait for the one before
    double s[3], v[3], fb[3], f[3];
    typename P::acc_t qb[3], qn[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      s[c] = M.S[3 * (size_t)i + c];
      v[c] = M.V[3 * (size_t)i + c];
      qb[c] = M.fb[3 * (size_t)i + c];
      qn[c] = M.fnb[3 * (size_t)i + c];
    }
    int tb = 0;
    double m = 0.0, im = 0.0;
    if (M.update) { tb = M.tbits[i]; m = M.mass[i]; im = M.invmass[i]; }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      fb[c] = P::get(qb[c]);
      f[c] = P::get(qn[c]) + fb[c];
      M.fnb[3 * (size_t)i + c] = qn[c] + qb[c];
      M.fb[3 * (size_t)i + c] = 0;
    }
    acc[12] += fb[0] * s[0];
    acc[13] += fb[1] * s[1];
    acc[14] += fb[2] * s[2];
    acc[15] += fb[1] * s[0];
    acc[16] += fb[2] * s[0];
    acc[17] += fb[2] * s[1];
    if (!M.update) continue;
    const int cls = (tb >> 16) == 2 ? 1 : 0;
    const double lam = cls ? lam1 : lam0;
    double vt[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double vn = (v[c] + M.dt * f[c] * im) * lam;
      M.V[3 * (size_t)i + c] = vn;
      M.S[3 * (size_t)i + c] = s[c] + M.dt * vn;
      vt[c] = 0.5 * (vn + v[c]);
    }
    const int o = 6 * cls;
    acc[o + 0] += m * vt[0] * vt[0];
    acc[o + 1] += m * vt[1] * vt[1];
    acc[o + 2] += m * vt[2] * vt[2];
    acc[o + 3] += m * vt[0] * vt[1];
    acc[o + 4] += m * vt[0] * vt[2];
    acc[o + 5] += m * vt[1] * vt[2];
  }
  double out[18];
  block_sum<18>(acc, red, out);
  if (threadIdx.x == 0)
    for (int k = 0; k < 18; ++k) M.part[k * M.part_stride + bk.b] = out[k];
}

// Initial kinetic energies (main.F90:179-195).  Partials: EK atoms, EK beads.
__global__ void k_kinetic(int natoms, const double* V, const int* tbits, const double* mass, double* part, int stride) {
  __shared__ double red[2 * 8];
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < natoms; i += gridDim.x * blockDim.x) {
    const double* v = V + 3 * (size_t)i;
    acc[(tbits[i] >> 16) == 2 ? 1 : 0] += mass[i] * ((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
  }
  double out[2];
  block_sum<2>(acc, red, out);
  if (threadIdx.x == 0) { part[blockIdx.x] = out[0]; part[stride + blockIdx.x] = out[1]; }
}

struct MomArgs {
  Scalars* sc;
  int natoms, halt_drift;
  double* V;
  const double* mass;
  const double* invmass;
  double* part;  // 3 per block, nblocks blocks
  int nblocks;
};

// MOMENTUM.f90:14-29 in FP64 on steps that are multiples of HALT_DRIFT
// (NEW_LOOP.F90:108-114): partial sums of m v, then the removal.
template <bool B>
__global__ void k_mom_sum(__grid_constant__ const MomArgs A0, const MomArgs* const* tab, const BlockMap bm) {
  const Blk bk = blk<B>(bm);
  const MomArgs& A = B ? *tab[bk.sys] : A0;
  const Scalars* sc = A.sc;
  if (sc->skip || sc->step % A.halt_drift != 0) return;
  __shared__ double red[3 * 8];
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = bk.b * blockDim.x + threadIdx.x; i < A.natoms; i += bk.g * blockDim.x)
    for (int c = 0; c < 3; ++c) acc[c] += A.V[3 * (size_t)i + c] * A.mass[i];
  double out[3];
  block_sum<3>(acc, red, out);
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) A.part[c * A.nblocks + bk.b] = out[c];
}

template <bool B>
__global__ void k_mom_apply(__grid_constant__ const MomArgs A0, const MomArgs* const* tab, const BlockMap bm) {
  const Blk bk = blk<B>(bm);
  const MomArgs& A = B ? *tab[bk.sys] : A0;
  const Scalars* sc = A.sc;
  if (sc->skip || sc->step % A.halt_drift != 0) return;
  __shared__ double tot[3];
  if (threadIdx.x < 32) {
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
      for (int b = threadIdx.x; b < A.nblocks; b += 32) s += A.part[c * A.nblocks + b];
      s = warp_sum(s);
      if (threadIdx.x == 0) tot[c] = s / (double)A.natoms;
    }
  }
  __syncthreads();
  for (int i = bk.b * blockDim.x + threadIdx.x; i < A.natoms; i += bk.g * blockDim.x)
    for (int c = 0; c < 3; ++c) A.V[3 * (size_t)i + c] -= tot[c] * A.invmass[i];
}

// SCALEBP.f90:37-39: positions scaled with the box on the steps the
// barostat changed it.
template <typename R, bool B>
__global__ void k_scale_positions(__grid_constant__ const MoveArgs<R> M0, const MoveArgs<R>* const* tab,
                                  const BlockMap bm) {
  const Blk bk = blk<B>(bm);
  const MoveArgs<R>& M = B ? *tab[bk.sys] : M0;
  const Scalars* sc = M.sc;
  if (sc->skip) return;
  const double miu = sc->miu;
  if (miu == 1.0) return;
  for (int i = bk.b * blockDim.x + threadIdx.x; i < M.natoms; i += bk.g * blockDim.x)
    for (int c = 0; c < 3; ++c) M.S[3 * (size_t)i + c] *= miu;
}

// ------------------------------------------------------------- reductions
struct FinalArgs {
  Scalars* sc;
  int fixed;                         // nonbonded accumulators in fixed point (FP32 path)
  const double* p_b; int g_b;        // bonded partials (12 x g_b)
  const double* p_mv; int g_mv;      // move partials (18 x g_mv)
  int mts;                           // MTS run
  int move;                          // 1: full step (kinetic part, thermostat, barostat)
  int ensemble;
  double temp_in, fac, pfac, pressure, mktemp, mktemp_atom, mktemp_bead;
  ObsD* ring; int ring_cap;
};

// Sum of g partials by one warp: each lane adds its own in increasing order
// (p[lane], p[lane+32], ...), then the lanes are summed.  Eight loads per lane
// are issued before they are added, so the warp waits for memory once per
// eight rather than once per partial; the order of the additions is the same.
__device__ double wsum(const double* p, int g) {
  double s = 0.0;
  for (int b0 = threadIdx.x & 31; b0 < g; b0 += 8 * 32) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = b0 + 32 * k < g ? p[b0 + 32 * k] : 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (b0 + 32 * k < g) s += v[k];
  }
  return warp_sum(s);
}

// Deterministic reduction of all partials into the observables, the MTS
// auxiliary history (MTS_SAVEAUXS / MTS_LOADAUXS), the thermostat factors of
// the next step and the barostat window (SCALEBP.f90:18-41).  The
// nonbonded accumulators are read and cleared for the next step.
template <bool B>
__global__ void k_finalize(__grid_constant__ const FinalArgs F0, const FinalArgs* const* tab, const BlockMap bm) {
  pdl_wait();
  const Blk bk = blk<B>(bm);
  const FinalArgs& F = B ? *tab[bk.sys] : F0;
  Scalars* sc = F.sc;
  __shared__ double q[64];
  if (sc->skip) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  // q[0..8] atom NB, q[9..17] bead NB, q[18..29] bonded, q[30..47] move
  if (threadIdx.x < 18) {
    unsigned long long* p = &sc->nbacc[threadIdx.x / 9][threadIdx.x % 9];
    const unsigned long long v = *p;
    q[threadIdx.x] = F.fixed ? (double)(long long)v * kEnInv : __longlong_as_double((long long)v);
    *p = 0ull;
  }
  for (int k = 18 + warp; k < 48; k += nw) {
    double v;
    if (k < 30) v = wsum(F.p_b + (size_t)(k - 18) * F.g_b, F.g_b);
    else v = wsum(F.p_mv + (size_t)(k - 30) * F.g_mv, F.g_mv);
    if (lane == 0) q[k] = v;
  }
  __syncthreads();
  if (threadIdx.x) return;
  ObsD& o = sc->obs;
  double bead_v[3], bead_pt[6];
  for (int c = 0; c < 3; ++c) bead_v[c] = q[9 + c];
  for (int c = 0; c < 6; ++c) bead_pt[c] = q[12 + c];
  const int m = sc->mts_m;
  if (F.mts) {
    if (m >= 1 && m <= 3) {
      for (int c = 0; c < 3; ++c) sc->mts_vnb[m - 1][c] = bead_v[c];
      for (int c = 0; c < 5; ++c) sc->mts_pt[c][m - 1] = bead_pt[c];  // PT23 is not saved (MTS_LOOP.f90:193-199)
    } else {
      const double coef = (double)(m - 3) * 0.5;
      for (int c = 0; c < 3; ++c) bead_v[c] = sc->mts_vnb[2][c] + coef * (sc->mts_vnb[2][c] - sc->mts_vnb[0][c]);
      for (int c = 0; c < 6; ++c) bead_pt[c] = sc->mts_pt[c][2] + coef * (sc->mts_pt[c][2] - sc->mts_pt[c][0]);
    }
  }
  for (int c = 0; c < 3; ++c) {
    o.v_nb[c] = q[c] + bead_v[c];
    o.v_bond[c] = q[18 + c];
    o.v_angle[c] = q[21 + c];
    o.v_torsion[c] = q[24 + c];
    o.v_oop[c] = q[27 + c];
  }
  double pt[6];
  for (int c = 0; c < 6; ++c) pt[c] = q[3 + c] + bead_pt[c] + q[42 + c];
  if (F.move) {
    // MOVE.F90:90-115
    for (int c = 0; c < 6; ++c) pt[c] += q[30 + c] + q[36 + c];
    o.ek[0] = 0.5 * (q[30] + q[31] + q[32]);
    o.ek[1] = 0.5 * (q[36] + q[37] + q[38]);
    o.temp = (o.ek[0] + o.ek[1]) * F.mktemp;
    o.temp_atom = o.ek[0] * F.mktemp_atom;
    o.temp_bead = o.ek[1] * F.mktemp_bead;
    sc->temp_atom = o.temp_atom;
    sc->temp_bead = o.temp_bead;
    const double vol = sc->box[0] * sc->box[1] * sc->box[2];
    for (int c = 0; c < 6; ++c) pt[c] /= vol;
    if (F.ensemble == 1 || F.ensemble == 2) {  // MOVE.F90:32-38, for the next step
      sc->lam[0] = sqrt(1.0 + F.fac * ((F.temp_in / o.temp_atom) - 1.0));
      sc->lam[1] = sqrt(1.0 + F.fac * ((F.temp_in / o.temp_bead) - 1.0));
    }
    if (F.ensemble == 2) {  // SCALEBP.f90:18-41
      sc->iavp = sc->iavp + 1;
      if (sc->iavp > 10) sc->iavp -= 10;
      sc->sp[sc->iavp - 1] = (pt[0] + pt[1] + pt[2]) / 3.0;
      if (sc->step % 10 == 0) {
        double avp = 0.0;
        for (int i = 0; i < 10; ++i) avp += sc->sp[i];
        const double p = avp / 10.0;
        const double miu = pow(1.0 + (p - F.pressure) * F.pfac, 1.0 / 3.0);
        sc->miu = miu;
        for (int c = 0; c < 3; ++c) {
          sc->box[c] *= miu;
          sc->boxinv[c] = 1.0 / sc->box[c];
          sc->box2[c] = sc->box[c] / 2.0;
          sc->boxf[c] = (float)sc->box[c];
          sc->boxinvf[c] = 1.0f / sc->boxf[c];
          sc->box2f[c] = sc->boxf[c] / 2.0f;
        }
      }
    }
  }
  sc->done = sc->step >= sc->stop_at;
  for (int c = 0; c < 6; ++c) o.pt[c] = pt[c];
  for (int c = 0; c < 3; ++c) o.box[c] = sc->box[c];
  o.bond_overext = (long long)sc->bond_overext;
  o.cell_clamps = (long long)sc->cell_clamps;
  o.step = sc->step;
  o.status = (int)sc->err;
  if (F.ring) {
    int slot = sc->step - sc->ring_base;
    if (slot >= 0 && slot < F.ring_cap) F.ring[slot] = o;
  }
}

// Step counter, observable ring base and step limit of the next run.
__global__ void k_set_counter(Scalars* sc, int step_before, int ring_base, int last) {
  sc->step = step_before;
  sc->ring_base = ring_base;
  sc->skip = 0;
  sc->stop_at = last;
  sc->done = step_before >= last ? 1 : 0;
}

// Initial temperatures and Berendsen factors (main.F90:174-195).
__global__ void k_init_temps(const double* part, int g, Scalars* sc, double mktemp, double mktemp_atom,
                             double mktemp_bead, double temp_in, double fac, int ensemble) {
  __shared__ double q[2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < 2) {
    double v = wsum(part + (size_t)warp * g, g);
    if (lane == 0) q[warp] = v;
  }
  __syncthreads();
  if (threadIdx.x) return;
  ObsD& o = sc->obs;
  o.ek[0] = 0.5 * q[0];
  o.ek[1] = 0.5 * q[1];
  o.temp = (o.ek[0] + o.ek[1]) * mktemp;
  o.temp_atom = o.ek[0] * mktemp_atom;
  o.temp_bead = o.ek[1] * mktemp_bead;
  sc->temp_atom = o.temp_atom;
  sc->temp_bead = o.temp_bead;
  if (ensemble == 1 || ensemble == 2) {
    sc->lam[0] = sqrt(1.0 + fac * ((temp_in / o.temp_atom) - 1.0));
    sc->lam[1] = sqrt(1.0 + fac * ((temp_in / o.temp_bead) - 1.0));
  } else {
    sc->lam[0] = sc->lam[1] = 1.0;
  }
}

}  // namespace ibg
