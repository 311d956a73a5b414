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

__global__ void __launch_bounds__(256) k_ade_segments(YeeParams P, const int64_t* segs,
                                                      int64_t nsegs) {
  const int lane = threadIdx.x & 31;
  const int64_t q = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (q >= nsegs) return;  // warp-uniform
  const int64_t s = segs[q];
  const int64_t cell = s * 32 + lane;
  const uint32_t m = P.mat16 ? (uint32_t)P.mat16[cell] : P.mat32[cell];
  const MatRec& M = P.mats[m];
  const int npc = M.reserved;
  const unsigned lt = (1u << lane) - 1u;
  int pre = 0;
#pragma unroll
  for (int b = 0; b < 6; ++b) pre += __popc(__ballot_sync(kFull, (npc >> b) & 1) & lt) << b;
  if (npc == 0) return;
  const uint32_t gp = P.seg_ofs[s] + (uint32_t)pre;
  int po = 0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int n = M.np[c];
    if (n == 0) continue;
    const float en = P.f[c][cell];
    const float4* cf = P.pcoef + P.pset_ofs[M.pset[c]];
    float acc = 0.f;
    int tt = 0;
    for (; tt + 1 < n; tt += 2) {
      const uint32_t g = gp + (uint32_t)(po + tt);
      float2 s0 = P.P[g], s1 = P.P[g + 1];
      const float d0 = ade_pole(s0, __ldg(cf + tt), en);
      const float d1 = ade_pole(s1, __ldg(cf + tt + 1), en);
      P.P[g] = s0;
      P.P[g + 1] = s1;
      acc = __fadd_rn(__fadd_rn(acc, d0), d1);
    }
    if (tt < n) {
      const uint32_t g = gp + (uint32_t)(po + tt);
      float2 s0 = P.P[g];
      acc = __fadd_rn(acc, ade_pole(s0, __ldg(cf + tt), en));
      P.P[g] = s0;
    }
    P.J[gp + (uint32_t)po] = acc;
    po += n;
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
                                cudaStream_t s) {
  if (nsegs <= 0) return cudaSuccess;
  const int64_t blocks = (nsegs + 7) / 8;
  k_ade_segments<<<(unsigned)blocks, 256, 0, s>>>(P, segs, nsegs);
  return cudaGetLastError();
}

}  // namespace oem
