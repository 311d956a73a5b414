// ADE pole pass of the warp-specialised step: the deferred post(n-1) + pre(n) update of every
// pole (openem/kernels/dispersion.cu:68-207), run between the H and the E update, with its
// polarisation currents J left in a pole-indexed array for the E kernel.
//
// One warp per 32-cell segment that holds poles; lane = cell. The list of such segments is
// built once on the device. Each cell's poles are stored contiguously after those of the
// cells before it (seg_ofs + a warp-ballot prefix of the per-cell counts), component by
// component; J of component c of a cell is written at the cell's first pole of component c.
// The arithmetic and the summation order are those of the inline ADE of the other E kernels
// (oem_arith.cuh), so every kernel variant produces the same bits.
#include <algorithm>
#include <cuda_runtime.h>
#include <stdint.h>

#include "oem_arith.cuh"
#include "oem_internal.cuh"

namespace oem {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__global__ void k_list_pole_segments(const uint32_t* seg, int64_t nseg, uint32_t n_total,
                                     int64_t* list, unsigned long long* count) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += stride) {
    const uint32_t end = (s + 1 < nseg) ? seg[s + 1] : n_total;
    if (end > seg[s]) {
      const unsigned long long q = atomicAdd(count, 1ull);
      if (list) list[q] = s;
    }
  }
}

constexpr int kSegPoles = 256;  // pole states of one segment staged per warp

// The pole update of one cell on states held in `st` (shared or global memory), J written to
// the cell's first pole of each component; `en` holds the cell's E^n.
__device__ __forceinline__ void ade_cell_poles(const YeeParams& P, const MatRec& M, float2* st,
                                               uint32_t gp, const float (&en)[3],
                                               const float4* pcoef, const int* pset_ofs) {
  int po = 0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int n = M.np[c];
    if (n == 0) continue;
    const float4* cf = pcoef + pset_ofs[M.pset[c]];
    float acc = 0.f;
    int tt = 0;
    for (; tt + 1 < n; tt += 2) {
      float2 s0 = st[po + tt], s1 = st[po + tt + 1];
      const float d0 = ade_pole(s0, cf[tt], en[c]);
      const float d1 = ade_pole(s1, cf[tt + 1], en[c]);
      st[po + tt] = s0;
      st[po + tt + 1] = s1;
      acc = __fadd_rn(__fadd_rn(acc, d0), d1);
    }
    if (tt < n) {
      float2 s0 = st[po + tt];
      acc = __fadd_rn(acc, ade_pole(s0, cf[tt], en[c]));
      st[po + tt] = s0;
    }
    P.J[gp + (uint32_t)po] = acc;
    po += n;
  }
}

// What a segment needs before its pole states can be read: its pole range, and per lane the
// cell's material and E^n. Loaded one segment ahead of the update.
struct SegLoad {
  int64_t s = -1;
  uint32_t a = 0, b = 0, m = 0;
  float e[3] = {0.f, 0.f, 0.f};
};

__device__ __forceinline__ SegLoad seg_load(const YeeParams& P, int64_t s, int64_t nseg,
                                            int lane) {
  SegLoad L;
  if (s < 0) return L;
  L.s = s;
  const int64_t cell = s * 32 + lane;
  L.a = P.seg_ofs[s];
  L.b = (s + 1 < nseg) ? P.seg_ofs[s + 1] : P.n_pole_total;
  L.m = P.mat16 ? (uint32_t)P.mat16[cell] : P.mat32[cell];
#pragma unroll
  for (int c = 0; c < 3; ++c) L.e[c] = P.f[c][cell];
  return L;
}

// One segment on one warp: its poles (contiguous in memory) are read into shared memory with
// coalesced loads, updated there cell by cell, and written back coalesced; a segment with more
// poles than the buffer holds is updated in place in global memory.
__device__ __forceinline__ void ade_segment(const YeeParams& P, const SegLoad& L, float2* st,
                                            int lane, const MatRec* mats, const float4* pcoef,
                                            const int* pset_ofs) {
  const int n = (int)(L.b - L.a);
  const MatRec& M = mats[L.m];
  const int npc = M.reserved;
  const unsigned lt = (1u << lane) - 1u;
  int pre = 0;
#pragma unroll
  for (int bb = 0; bb < 6; ++bb) pre += __popc(__ballot_sync(kFull, (npc >> bb) & 1) & lt) << bb;
  if (n <= kSegPoles) {
    for (int t = lane; t < n; t += 32) st[t] = P.P[L.a + t];
    __syncwarp();
    if (npc > 0) ade_cell_poles(P, M, st + pre, L.a + (uint32_t)pre, L.e, pcoef, pset_ofs);
    __syncwarp();
    for (int t = lane; t < n; t += 32) P.P[L.a + t] = st[t];
    __syncwarp();
  } else if (npc > 0) {
    ade_cell_poles(P, M, P.P + L.a + pre, L.a + (uint32_t)pre, L.e, pcoef, pset_ofs);
  }
}

// Warps stride over the listed segments (the grid is about one resident wave): while a warp
// updates segment q it has already loaded the pole range, materials and E^n of its next
// segment and the index of the one after, so each segment waits on one dependent load (its
// pole states) instead of three. In the captured step it runs on a graph branch of its own:
// beside the snapshots of the step before (within one run call), or beside the H update.
constexpr int kAdeMats = 64;    // material records staged in shared memory when they fit
constexpr int kAdeCoefs = 256;  // pole coefficient rows staged likewise
constexpr int kAdeSets = 64;

template <bool SMEM>
__global__ void __launch_bounds__(256) k_ade_segments(YeeParams P, const int64_t* segs,
                                                      int64_t nsegs, int64_t nseg, int n_mats) {
  __shared__ float2 buf[8][kSegPoles];
  // SMEM: the material records, pole sets and coefficients fit here, read as shared memory
  __shared__ MatRec smats[SMEM ? kAdeMats : 1];
  __shared__ float4 scoef[SMEM ? kAdeCoefs : 1];
  __shared__ int sofs[SMEM ? kAdeSets + 1 : 1];
  const MatRec* mats = SMEM ? smats : P.mats;
  const float4* pcoef = SMEM ? scoef : P.pcoef;
  const int* pset_ofs = SMEM ? sofs : P.pset_ofs;
  if (SMEM) {
    const uint4* src = reinterpret_cast<const uint4*>(P.mats);
    uint4* dst = reinterpret_cast<uint4*>(smats);
    for (int q = threadIdx.x; q < n_mats * 4; q += blockDim.x) dst[q] = src[q];
    for (int q = threadIdx.x; q < P.n_coef; q += blockDim.x) scoef[q] = P.pcoef[q];
    for (int q = threadIdx.x; q <= P.n_sets; q += blockDim.x) sofs[q] = P.pset_ofs[q];
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int64_t stride = (int64_t)gridDim.x * 8;
  int64_t q = (int64_t)blockIdx.x * 8 + w;
  SegLoad cur = seg_load(P, q < nsegs ? segs[q] : -1, nseg, lane);
  int64_t s2 = q + stride < nsegs ? segs[q + stride] : -1;
  while (cur.s >= 0) {
    const int64_t q3 = q + 2 * stride;
    const int64_t s3 = q3 < nsegs ? segs[q3] : -1;
    const SegLoad nxt = seg_load(P, s2, nseg, lane);
    ade_segment(P, cur, buf[w], lane, mats, pcoef, pset_ofs);
    cur = nxt;
    s2 = s3;
    q += stride;
  }
}

}  // namespace

cudaError_t launch_list_pole_segments(const YeeParams& P, int64_t nseg, int64_t* list,
                                      unsigned long long* count, cudaStream_t s) {
  const int blocks = (int)std::min<int64_t>((nseg + 255) / 256, 148 * 32);
  k_list_pole_segments<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(P.seg_ofs, nseg, P.n_pole_total,
                                                               list, count);
  return cudaGetLastError();
}

cudaError_t launch_ade_segments(const YeeParams& P, const int64_t* segs, int64_t nsegs,
                                int64_t nseg, int max_blocks, int n_mats, cudaStream_t s) {
  if (nsegs <= 0) return cudaSuccess;
  // about one resident wave (5 blocks of 8 warps per SM); each warp strides over the list
  int64_t blocks = std::min<int64_t>((nsegs + 7) / 8, 148 * 5);
  if (max_blocks > 0 && blocks > max_blocks) blocks = max_blocks;
  if (n_mats <= kAdeMats && P.n_coef <= kAdeCoefs && P.n_sets <= kAdeSets)
    k_ade_segments<true><<<(unsigned)blocks, 256, 0, s>>>(P, segs, nsegs, nseg, n_mats);
  else
    k_ade_segments<false><<<(unsigned)blocks, 256, 0, s>>>(P, segs, nsegs, nseg, n_mats);
  return cudaGetLastError();
}

}  // namespace oem
