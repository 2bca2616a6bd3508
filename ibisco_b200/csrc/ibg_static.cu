// Nonbonded forces of one particle list with no memory allocation.
//
// Some callers cannot allocate device memory when they need the forces: a
// host that already owns every byte of device memory through its own
// allocator (a Fortran or framework memory pool), or a loop that must not
// stall the device (cudaMalloc and cudaFree can synchronise it).  This entry
// point serves them: the caller passes its device arrays in and out, and the
// scratch the computation needs -- the 64-bit fixed-point force sums and the
// per-block energy/virial partial sums -- lives in one file-scope
// __device__ array of fixed size that every GPU loading the library holds
// until the process exits.  The call reads its error word back and waits for
// its stream before it returns.
//
// The computation is NONBONDED_FORCE.F90:45-104 on the reference's own data
// layout (INDEX_LIST, LIST(MAXNAB,N), NNEBS, the nonbonded tables after
// FTABLE), in REAL*4 with the reference's operation order, summed in the same
// fixed point as the context path.  Particle types, table numbers and table
// rows are checked before they index anything: a type outside 1..NTYPE or a
// table number outside 1..NNBTYPE counts as a missing table, a row whose
// successor lies beyond the caller's table column as out of range.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/ibisco_gpu.h"
#include "ibg_common.cuh"

namespace {

constexpr int kStaticBlocks = IBG_STATIC_MAX_BLOCKS;
constexpr long long kStaticForceWords = 3LL * IBG_STATIC_MAX_PARTICLES;
constexpr long long kStaticBytes = kStaticForceWords * 8 + 9LL * kStaticBlocks * 8;

// The scratch: fixed-point forces (3 x MAX particles) followed by the
// per-block partial sums (9 x MAX blocks).  Shared by every call.
static __device__ __align__(256) unsigned char ibg_static_scratch[kStaticBytes];

std::mutex g_mu;
void* g_ptr[64] = {nullptr};

struct StaticArgs {
  int nitems, n, maxnab, ntype, nnbtype, ld_nb;
  const float* rxyz;
  const int* itype;
  const int* type_label;
  const int* index_list;
  const int* list;
  const int* nnebs;
  const int* inbondt;
  const float* rnbond;
  const float* nbond_force;
  const float* nbond_pot;
  const float* binnb;
  const int* ndatnb;
  float box[3], boxinv[3];
  float rcutsq;
  unsigned long long* f;  // scratch: 3 * nitems
  double* part;           // scratch: 9 * gridDim.x
  unsigned* err;          // scratch word after the partials
};

__global__ void k_static_zero(unsigned long long* f, long long nwords, unsigned* err) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nwords; k += (long long)gridDim.x * blockDim.x)
    f[k] = 0ull;
  if (blockIdx.x == 0 && threadIdx.x == 0) *err = 0u;
}

__device__ __forceinline__ long long fixq(float v, unsigned* err) {
  if (!(fabsf(v) < ibg::kFixMax)) {
    atomicOr(err, ibg::EB_FIXED);
    v = (v == v) ? copysignf(ibg::kFixMax, v) : 0.0f;
  }
  return __float2ll_rn(v * ibg::kFixScale);
}

// One thread per list entry A; REAL*4 arithmetic in the reference's order.
__global__ void __launch_bounds__(256) k_static_pairs(StaticArgs a) {
  __shared__ double red[9 * 8];
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) acc[k] = 0.0;
  for (int A = blockIdx.x * blockDim.x + threadIdx.x; A < a.n; A += gridDim.x * blockDim.x) {
    const int i = a.index_list[A] - 1;
    if (i < 0 || i >= a.nitems) { atomicOr(a.err, ibg::EB_BAD_INDEX); continue; }
    const float rx = a.rxyz[3 * i], ry = a.rxyz[3 * i + 1], rz = a.rxyz[3 * i + 2];
    const int ti = a.itype[i];
    const int li = a.type_label[i];
    const bool ti_ok = ti >= 1 && ti <= a.ntype;
    long long f0 = 0, f1 = 0, f2 = 0;
    const int cnt = min(a.nnebs[i], a.maxnab);
    for (int k = 0; k < cnt; ++k) {
      const int j = a.list[(long long)A * a.maxnab + k] - 1;
      if (j < 0 || j >= a.nitems) { atomicOr(a.err, ibg::EB_BAD_INDEX); continue; }
      float d0 = rx - a.rxyz[3 * j], d1 = ry - a.rxyz[3 * j + 1], d2 = rz - a.rxyz[3 * j + 2];
      d0 = __fsub_rn(d0, __fmul_rn(roundf(__fmul_rn(d0, a.boxinv[0])), a.box[0]));
      d1 = __fsub_rn(d1, __fmul_rn(roundf(__fmul_rn(d1, a.boxinv[1])), a.box[1]));
      d2 = __fsub_rn(d2, __fmul_rn(roundf(__fmul_rn(d2, a.boxinv[2])), a.box[2]));
      const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1)), __fmul_rn(d2, d2));
      if (!(r2 < a.rcutsq)) continue;
      const int tj = a.itype[j];
      if (!ti_ok || tj < 1 || tj > a.ntype) { atomicOr(a.err, ibg::EB_MISSING_TABLE); continue; }
      const int tab = a.inbondt[(ti - 1) + a.ntype * (tj - 1)];
      if (tab < 1 || tab > a.nnbtype) { atomicOr(a.err, ibg::EB_MISSING_TABLE); continue; }
      const float r = __fsqrt_rn(r2);
      const float bin = a.binnb[tab - 1];
      const int ni = (int)__fdiv_rn(r, bin);
      if (ni < 0 || ni > a.ndatnb[tab - 1] || ni + 1 >= a.ld_nb) { atomicOr(a.err, ibg::EB_TABLE_RANGE); continue; }
      const long long row = (long long)a.ld_nb * (tab - 1) + ni;
      const float alpha = __fdiv_rn(__fsub_rn(r, a.rnbond[row]), bin);
      const float one_a = __fsub_rn(1.0f, alpha);
      const float fij = __fadd_rn(__fmul_rn(a.nbond_force[row], one_a), __fmul_rn(a.nbond_force[row + 1], alpha));
      const float vij = __fadd_rn(__fmul_rn(a.nbond_pot[row], one_a), __fmul_rn(a.nbond_pot[row + 1], alpha));
      if (li == 1) acc[0] += (double)vij;
      else if (li == 2) {
        const int lj = a.type_label[j];
        if (lj == 2) acc[1] += (double)vij;
        else if (lj == 3) acc[2] += (double)vij;
      } else if (li == 3) acc[2] += (double)vij;
      const float fx = __fmul_rn(fij, d0), fy = __fmul_rn(fij, d1), fz = __fmul_rn(fij, d2);
      const long long qx = fixq(fx, a.err), qy = fixq(fy, a.err), qz = fixq(fz, a.err);
      f0 += qx; f1 += qy; f2 += qz;
      atomicAdd(&a.f[3 * (long long)j + 0], (unsigned long long)(-qx));
      atomicAdd(&a.f[3 * (long long)j + 1], (unsigned long long)(-qy));
      atomicAdd(&a.f[3 * (long long)j + 2], (unsigned long long)(-qz));
      acc[3] += (double)__fmul_rn(fx, d0);
      acc[4] += (double)__fmul_rn(fy, d1);
      acc[5] += (double)__fmul_rn(fz, d2);
      acc[6] += (double)__fmul_rn(fy, d0);
      acc[7] += (double)__fmul_rn(fz, d0);
      acc[8] += (double)__fmul_rn(fz, d1);
    }
    atomicAdd(&a.f[3 * (long long)i + 0], (unsigned long long)f0);
    atomicAdd(&a.f[3 * (long long)i + 1], (unsigned long long)f1);
    atomicAdd(&a.f[3 * (long long)i + 2], (unsigned long long)f2);
  }
  double out[9];
  ibg::block_sum<9>(acc, red, out);
  if (threadIdx.x == 0)
    for (int k = 0; k < 9; ++k) a.part[9 * blockIdx.x + k] = out[k];
}

// Forces to FP64 (3,NITEMS) and the block partials, in block order, to
// V_NB(1..3), PT11, PT22, PT33, PT12, PT13, PT23.
__global__ void k_static_finish(const unsigned long long* f, const double* part, int nblocks, int nitems,
                                double* fxyz, double* sums) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < 3LL * nitems;
       k += (long long)gridDim.x * blockDim.x)
    fxyz[k] = (double)(long long)f[k] * ibg::kFixInv;
  if (blockIdx.x == 0 && threadIdx.x < 9) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += part[9 * b + threadIdx.x];
    sums[threadIdx.x] = s;
  }
}

void msg(char* err, int errlen, const char* text) {
  if (err && errlen > 0) std::snprintf(err, errlen, "%s", text);
}

}  // namespace

extern "C" int ibg_nonbonded_static(int nitems, int n, const float* rxyz, const int* itype, const int* type_label,
                                    const int* index_list, const int* list, int maxnab, const int* nnebs, int ntype,
                                    const int* inbondt, int nnbtype, int ld_nb, const float* rnbond,
                                    const float* nbond_force, const float* nbond_pot, const float* binnb,
                                    const int* ndatnb, const float* box, float rcutsq, double* fxyz, double* sums,
                                    void* stream, char* err, int errlen) {
  if (nitems < 1 || n < 0 || n > nitems || maxnab < 1 || ntype < 1 || nnbtype < 1 || ld_nb < 2 || !rxyz ||
      !itype || !type_label || !index_list || !nnebs ||
      !inbondt || !rnbond || !nbond_force || !nbond_pot || !binnb || !ndatnb || !box || !fxyz || !sums ||
      (n > 0 && !list)) {
    msg(err, errlen, "ibg_nonbonded_static: invalid argument");
    return IBG_E_INVALID;
  }
  if (nitems > IBG_STATIC_MAX_PARTICLES) {
    msg(err, errlen, "ibg_nonbonded_static: more particles than IBG_STATIC_MAX_PARTICLES");
    return IBG_E_CAPACITY;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    msg(err, errlen, "ibg_nonbonded_static: no usable current CUDA device");
    return IBG_E_CUDA;
  }
  void* base = nullptr;
  {
    // First call on this device: resolve the scratch array's device address
    // with the device current (in host code the symbol is only a stand-in).
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ptr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, ibg_static_scratch);
      if (e != cudaSuccess) {
        msg(err, errlen, cudaGetErrorString(e));
        return IBG_E_CUDA;
      }
      g_ptr[dev] = p;
    }
    base = g_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  StaticArgs a;
  a.nitems = nitems; a.n = n; a.maxnab = maxnab; a.ntype = ntype; a.nnbtype = nnbtype; a.ld_nb = ld_nb;
  a.rxyz = rxyz; a.itype = itype; a.type_label = type_label; a.index_list = index_list; a.list = list;
  a.nnebs = nnebs; a.inbondt = inbondt; a.rnbond = rnbond; a.nbond_force = nbond_force; a.nbond_pot = nbond_pot;
  a.binnb = binnb; a.ndatnb = ndatnb; a.rcutsq = rcutsq;
  for (int c = 0; c < 3; ++c) { a.box[c] = box[c]; a.boxinv[c] = 1.0f / box[c]; }
  a.f = (unsigned long long*)base;
  a.part = (double*)((unsigned char*)base + kStaticForceWords * 8);
  a.err = (unsigned*)(a.part + 9LL * kStaticBlocks - 1);  // last partial slot is never a block's
  const int blocks = (int)std::min<long long>(std::max(1, (n + 255) / 256), kStaticBlocks - 1);
  k_static_zero<<<std::max(1, std::min(1024, (3 * nitems + 255) / 256)), 256, 0, st>>>(a.f, 3LL * nitems, a.err);
  k_static_pairs<<<blocks, 256, 0, st>>>(a);
  k_static_finish<<<std::max(1, std::min(1024, (3 * nitems + 255) / 256)), 256, 0, st>>>(a.f, a.part, blocks,
                                                                                          nitems, fxyz, sums);
  unsigned bits = 0;
  cudaError_t e = cudaMemcpyAsync(&bits, a.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    msg(err, errlen, cudaGetErrorString(e));
    return IBG_E_CUDA;
  }
  if (bits & ibg::EB_FIXED) { msg(err, errlen, "force outside the 64-bit fixed-point range"); return IBG_E_FIXED_OVERFLOW; }
  if (bits & ibg::EB_MISSING_TABLE) { msg(err, errlen, "listed pair without a nonbonded table"); return IBG_E_MISSING_TABLE; }
  if (bits & ibg::EB_TABLE_RANGE) { msg(err, errlen, "nonbonded distance beyond its table"); return IBG_E_TABLE_RANGE; }
  if (bits & ibg::EB_BAD_INDEX) { msg(err, errlen, "particle id outside 1..nitems in index_list or list"); return IBG_E_INVALID; }
  msg(err, errlen, "");
  return IBG_OK;
}
