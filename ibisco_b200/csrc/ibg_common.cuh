// Shared definitions of the B200 step: precision policies, device scalar
// block, error bits and warp/block reduction helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ibg {

// Error bits raised by kernels; the host maps the lowest set bit to a status.
enum : unsigned {
  EB_LIST_OVERFLOW = 1u << 0,  // a particle reached MAXNAB neighbours
  EB_TORSION = 1u << 1,        // torsion angle outside its table
  EB_OOP = 1u << 2,            // out-of-plane angle outside its table
  EB_FIXED = 1u << 3,          // a force left the fixed-point range
  EB_CELL_GRID = 1u << 4,      // fewer than 3 cells per dimension
  EB_TABLE_RANGE = 1u << 5,    // nonbonded distance beyond its table
  EB_MISSING_TABLE = 1u << 6,  // listed pair without a nonbonded table
  EB_CAPACITY = 1u << 7,       // neighbour-list / cell storage exhausted
  EB_BAD_INDEX = 1u << 8,      // a caller's particle id outside 1..NITEMS
};

// 64-bit fixed-point force accumulation: value * 2^32, two's complement in
// unsigned long long so that atomicAdd wraps like signed addition.  The
// representable range is |F| < 2^31 reduced force units per particle at a
// resolution of 2^-32.
constexpr float kFixScale = 4294967296.0f;        // 2^32
constexpr double kFixInv = 1.0 / 4294967296.0;   // 2^-32
constexpr float kFixMax = 2147483520.0f;          // largest float below 2^31

// Slot-ordered nonbonded force sums, in blocks of 32 slots: a block's 32 x
// sums, then its 32 y sums and its 32 z sums.  A slot's three sums lie 256
// bytes apart (one address and two fixed offsets per particle), and the sums
// of neighbouring slots share sectors.  fs_at(t) is slot t's x sum; its y and
// z sums follow at +32 and +64.
__host__ __device__ __forceinline__ size_t fs_at(int t) { return (size_t)(t >> 5) * 96 + (t & 31); }
__host__ __device__ __forceinline__ size_t fs_len(int n) { return (size_t)((n + 31) >> 5) * 96; }

// Observables in the order of ibg_obs (ek[2] .. pt[6], box[3]).
struct ObsD {
  double ek[2], temp, temp_atom, temp_bead;
  double v_nb[3], v_bond[3], v_angle[3], v_torsion[3], v_oop[3];
  double pt[6];
  double box[3];
  long long bond_overext, cell_clamps;
  int step, status;
};

// Device-resident scalars of one system.
struct Scalars {
  int step;          // current step number
  int rebuild;       // list rebuild this step
  int mts_m;         // MOD(step, 3+NMTS), -1 without MTS
  int ring_base;     // step whose observables go to ring slot 0
  double box[3], boxinv[3], box2[3];  // FP64 box (integration, FP64 path)
  float boxf[3], boxinvf[3], box2f[3];  // REAL*4 box (FP32 path geometry)
  int ncell[2][3];   // cell grid of the atom / bead list
  double lam[2];     // Berendsen factors for atoms / beads (MOVE.F90:32-38)
  double temp_atom, temp_bead;
  double miu;        // SCALEBP factor of this step (1 if none)
  // MTS history (module_MTS.f90): V_NB(label) and PT11..PT13 for m=1..3
  double mts_vnb[3][3];
  double mts_pt[6][3];
  // SCALEBP running window (SCALEBP.f90:18-21)
  int iavp, pad1;
  double sp[10];
  unsigned err;
  int abort;          // a list outgrew its storage: the rest of the run is a no-op
  int skip;           // this step does nothing (aborted run, or the step limit reached)
  int stop_at;        // last step this system runs (batched runs stop each system here)
  int done;           // stop_at reached: set by the last step's k_finalize
  int need_rows[2];   // rows of 32 entries a slice of each list needed
  unsigned work[4];   // dynamic work counters: nonbonded atom/bead, list build atom/bead
  unsigned near_n[2];  // pairs at the cutoff left by the FP32 nonbonded kernel, per list
  int need_near[2];    // pairs at the cutoff a list needed room for (the step is repeated)
  // nonbonded V_NB(1..3) and PT11..PT23 of the atom / bead list: 64-bit fixed
  // point at 2^-24 (FP32 path; order independent) or double (FP64 path)
  unsigned long long nbacc[2][9];
  unsigned long long bond_overext, cell_clamps;
  double mom[3];     // momentum removal (MOMENTUM.f90)
  ObsD obs;          // observables of the last step
};

constexpr double kEnInv = 1.0 / 16777216.0;  // 2^-24, energy/virial fixed point

// Blocks of a batched launch.  Block b of the grid serves system sys_of[b] as
// its local block b - start[s] of start[s+1] - start[s].  A single-system
// launch (B = false) uses the whole grid.
struct BlockMap {
  const int* sys_of;
  const int* start;
};
struct Blk {
  int sys, b, g;
};

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialization may start while the kernel before it in the stream still
// runs; pdl_wait() returns once that kernel has completed and its writes are
// visible (at once when the launch was an ordinary one).  pdl_trigger() lets
// the next kernel's launch begin before this one ends.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
template <bool B>
__device__ __forceinline__ Blk blk(const BlockMap& m) {
  if (!B) return Blk{0, (int)blockIdx.x, (int)gridDim.x};
  const int s = __ldg(m.sys_of + blockIdx.x);
  const int b0 = __ldg(m.start + s);
  return Blk{s, (int)blockIdx.x - b0, __ldg(m.start + s + 1) - b0};
}

// Copy one system's argument block into shared memory (every thread of the
// block takes part; returns after a barrier).  Batched kernels whose bodies
// keep many argument fields live read them from there instead of holding them
// in registers.
template <typename T>
__device__ __forceinline__ void stage_args(T* dst, const T* src) {
  static_assert(sizeof(T) % 4 == 0, "argument blocks are whole words");
  for (int i = threadIdx.x; i < (int)(sizeof(T) / 4); i += blockDim.x) ((int*)dst)[i] = ((const int*)src)[i];
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum of K values per thread; thread 0 of the block gets
// the result in out[].  Needs K*32 doubles of shared memory.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* smem, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
    for (int k = 0; k < K; ++k) smem[warp * K + k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += smem[w * K + k];
      out[k] = s;
    }
  }
  __syncthreads();
}

// Exact block sum of K 64-bit integers per thread; the results are left in
// smem[0..K-1] (needs 32 + 32*K entries of shared memory) for every thread.
template <int K>
__device__ __forceinline__ void block_sum_i64(long long (&v)[K], long long* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
    for (int k = 0; k < K; ++k) smem[32 + warp * K + k] = v[k];
  __syncthreads();
  if (threadIdx.x < K) {
    long long s = 0;
    for (int w = 0; w < nw; ++w) s += smem[32 + w * K + threadIdx.x];
    smem[threadIdx.x] = s;
  }
  __syncthreads();
}

}  // namespace ibg
