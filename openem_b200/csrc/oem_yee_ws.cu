// Warp-specialised, fully asynchronous Yee kernels for sm_100a (the default step kernels).
//
// A block owns a 128 (z) x 4 (y) tile and walks a chunk of x planes. Warp 4 is the producer:
// its lane 0 stages everything one plane needs into a 3-deep shared-memory ring -- field tiles
// with cp.async.bulk.tensor (TMA), the CPML psi rows of slab cells and the polarisation
// currents of the plane's dispersive cells with 1D cp.async.bulk copies -- ahead of the four
// consumer warps, one per tile row, four z cells per lane. A stage is published by a "full"
// mbarrier (producer arrival + transaction bytes) and recycled through an "empty" mbarrier
// that each consumer warp arrives on once it is done with it. Consumers issue no synchronous
// global load except for wrapped neighbours (periodic seams) and rows whose currents do not fit
// the stage's window; they write H/E and psi straight back. The ADE pole states are advanced
// by a separate pass (oem_ade.cu) that runs between the two updates and leaves J behind.
//
// Every mbarrier wait is bounded (2^20 polls); a wait that gives up sets *err, stops the
// issuing side and the waiting side, and the producer drains what it issued (again bounded).
//
// The arithmetic per cell is that of the basic kernels (openem/kernels/yee.cu:60-240), pinned
// in oem_arith.cuh, so both produce the same bits.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

#include "oem_internal.cuh"
#include "oem_arith.cuh"

namespace oem {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kTY = 4;
constexpr int kTZ = 128;
constexpr int kBZ = 136;
// Ring depth, blocks per SM and the E kernel's psi / current pool (build-time knobs). Two
// stages let three blocks of each kernel share an SM (<= 136 registers, <= 75 KB of shared
// memory per block): on the 512^3 dispersive grid the E update runs 12% faster than with three
// stages and two blocks, the latency of the shallower ring hidden by the third block.
#ifndef OEM_WS_STAGES
#define OEM_WS_STAGES 2
#endif
#ifndef OEM_WS_MINBLOCKS
#define OEM_WS_MINBLOCKS 3
#endif
#ifndef OEM_WS_EPOOL
#define OEM_WS_EPOOL 2560
#endif
constexpr int kS = OEM_WS_STAGES;
constexpr int kBoxW = 704;                      // floats per 136 x 5 halo-box slot (128-B aligned)
constexpr uint32_t kWideBytes = 5 * kBZ * 4;    // bytes a halo box transfers
constexpr uint32_t kTileBytes = kTY * kTZ * 4;  // bytes a 128 x 4 tile transfers
constexpr int kZMax = 32;                       // z-slab depths staged when <= this and % 4 == 0
constexpr int kSmemMats = 64;
constexpr int kXMax = 64;                       // x planes per block (segment table size)

// H kernel stage (floats)
constexpr int kH_EB = 0;                  // E halo box x3
constexpr int kH_EN = kH_EB + 3 * kBoxW;  // E tile of the x-neighbour plane x3
constexpr int kH_HT = kH_EN + 3 * 512;    // H tile x3
constexpr int kH_PX = kH_HT + 3 * 512;    // psi x-slab rows [2][4][128]
constexpr int kH_PY = kH_PX + 1024;       // psi y-slab rows [2][4][128]
constexpr int kH_PZ = kH_PY + 1024;       // psi z-slab rows [2 slots][2 sides][4 x depth]
constexpr int kHStage = kH_PZ + 512;
// E kernel stage (32-bit words)
constexpr int kE_HB = 0;                  // H halo box x3 (rows j0-1.., cols k0-4..)
constexpr int kE_HP = kE_HB + 3 * kBoxW;  // Hy, Hz tiles of the previous plane
constexpr int kE_ET = kE_HP + 2 * 512;    // E tile x3
constexpr int kE_MT = kE_ET + 3 * 512;    // material tile (uint16 or uint32)
// A per-plane pool: the psi rows the plane needs (x rows 1024 floats, y rows 1024, z rows 512,
// each only when present), then the pole-state window in the rest.
constexpr int kE_POOL = kE_MT + 512;
constexpr int kEPool = OEM_WS_EPOOL;
static_assert(kEPool >= 2560, "the pool must hold the x, y and z psi rows of a plane");
constexpr int kE_PT = kE_POOL + kEPool;   // [2r]: pole start of row r, [2r+1]: window offset,
                                          // [8..10]: psi x/y/z offsets, [11]: window start
constexpr int kEStage = kE_PT + 32;
static_assert((kHStage * 4) % 128 == 0 && (kEStage * 4) % 128 == 0, "stage alignment");
static_assert((kH_EN * 4) % 128 == 0 && (kH_HT * 4) % 128 == 0 && (kH_PX * 4) % 128 == 0 &&
                  (kH_PY * 4) % 128 == 0 && (kH_PZ * 4) % 128 == 0,
              "H slots aligned");
static_assert((kE_HP * 4) % 128 == 0 && (kE_ET * 4) % 128 == 0 && (kE_MT * 4) % 128 == 0 &&
                  (kE_POOL * 4) % 128 == 0 && (kE_PT * 4) % 128 == 0,
              "E slots aligned");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  for (uint32_t it = 0; it < (1u << 20); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  atomicExch(err, 1);
  return false;
}
// A producer's wait for a free stage: gives up after `limit` polls (setting *err), or early once
// another warp of the grid has set *err (read every 4096 polls), so a block whose consumers have
// left does not run out its own bound. Consumers wait with mbar_wait (the extra check in their
// per-plane wait cost the E update 1.5%), and so does a producer's final drain of its own
// copies, which must complete whatever happened elsewhere.
constexpr uint32_t kPolls = 1u << 20;
__device__ __forceinline__ bool mbar_wait_live(uint64_t* bar, uint32_t parity, int* err,
                                               uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 4095u) == 4095u && *reinterpret_cast<volatile int*>(err) != 0) return false;
  }
  atomicExch(err, 1);
  return false;
}
__device__ __forceinline__ void tma3(void* dst, const CUtensorMap* map, uint64_t* bar, int c0,
                                     int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
// 1D bulk copy global -> shared; both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool in_slab(const DevAxis& A, int q) {
  return q < A.lo || q >= A.n - A.hi;
}

// Global address of the psi row (4 consecutive cells at k) of slab array (a, slot).
__device__ __forceinline__ float* psi_addr(const PsiSet& S, int a, int slot, const DevAxis& A,
                                          int i, int j, int k, int ny, int nzp) {
  const int q = (a == 0) ? i : ((a == 1) ? j : k);
  int side, ql, L;
  if (q < A.lo) {
    side = 0; ql = q; L = A.lo;
  } else {
    side = 1; ql = q - (A.n - A.hi); L = A.hi;
  }
  float* base = S.p[a][slot][side];
  int64_t idx;
  if (a == 0) idx = ((int64_t)ql * ny + j) * nzp + k;
  else if (a == 1) idx = ((int64_t)i * L + ql) * nzp + k;
  else idx = ((int64_t)i * ny + j) * L + ql;
  return base + idx;
}

__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }

// Does the tile's z range [k0, k0+128) overlap the z slab of side `side`, with stageable depth?
__device__ __forceinline__ bool zslab_staged(const DevAxis& Z, int side, int k0) {
  const int L = side ? Z.hi : Z.lo;
  if (L <= 0 || L > kZMax || (L & 3)) return false;
  return side ? (k0 + kTZ > Z.n - L && k0 < Z.n) : (k0 < L);
}

// The psi rows a tile stages, fixed for all planes of a block: the y slab rows among its rows
// and the staged z slab sides; only the x slab planes add rows (two per row and slot).
struct PsiTile {
  uint32_t rowb;     // bytes of one staged row (the tile's z extent)
  int nrows;         // rows of the tile inside the grid
  unsigned ymask;    // rows in a y slab
  bool zs0, zs1;     // staged z slab sides
  uint32_t yzbytes;  // bytes of the y and z rows
  uint32_t xbytes;   // bytes of the x rows of a slab plane
};

__device__ __forceinline__ PsiTile psi_tile(const YeeParams& P, int j0, int k0) {
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  PsiTile t;
  t.rowb = (uint32_t)min(kTZ, P.nzp - k0) * 4;
  t.nrows = min(kTY, P.ny - j0);
  t.ymask = 0;
#pragma unroll
  for (int r = 0; r < kTY; ++r) t.ymask |= (unsigned)(r < t.nrows && in_slab(Y, j0 + r)) << r;
  t.zs0 = zslab_staged(Z, 0, k0);
  t.zs1 = zslab_staged(Z, 1, k0);
  t.yzbytes = 2u * t.rowb * (uint32_t)__popc(t.ymask) +
              (t.zs0 ? 2u * (uint32_t)(t.nrows * Z.lo) * 4 : 0u) +
              (t.zs1 ? 2u * (uint32_t)(t.nrows * Z.hi) * 4 : 0u);
  t.xbytes = 2u * t.rowb * (uint32_t)t.nrows;
  return t;
}

// Producer helper: issue the psi rows of plane i (x rows when `xsl`) for one field family into
// a stage: x rows at px, y rows at py ([slot][row][z] each), z slab rows at pz
// ([slot][side][row * depth]).
__device__ __forceinline__ void stage_psi(const PsiTile& T, const PsiSet& S, const YeeParams& P,
                                          float* px, float* py, float* pz, uint64_t* bar, int i,
                                          int j0, int k0, bool xsl) {
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  for (int r = 0; r < T.nrows; ++r) {
    if (xsl)
      for (int s = 0; s < 2; ++s)
        bulk(px + (s * 4 + r) * kTZ, psi_addr(S, 0, s, X, i, j0 + r, k0, P.ny, P.nzp), T.rowb,
             bar);
    if ((T.ymask >> r) & 1u)
      for (int s = 0; s < 2; ++s)
        bulk(py + (s * 4 + r) * kTZ, psi_addr(S, 1, s, Y, i, j0 + r, k0, P.ny, P.nzp), T.rowb,
             bar);
  }
  for (int side = 0; side < 2; ++side) {
    if (!(side ? T.zs1 : T.zs0)) continue;
    const int L = side ? Z.hi : Z.lo;
    const int kk = side ? Z.n - L : 0;
    for (int s = 0; s < 2; ++s)
      bulk(pz + (s * 2 + side) * kTY * kZMax, psi_addr(S, 2, s, Z, i, j0, kk, P.ny, P.nzp),
           (uint32_t)(T.nrows * L) * 4, bar);
  }
}

// ---------------------------------------------------------------------------------------------
// Shared consumer helpers
// ---------------------------------------------------------------------------------------------

// z coefficients of the block's 128 cells in shared memory: [0] 1/dl, [1] wall mask,
// [2] CPML a, [3] CPML b, [4] CPML 1/kappa, [5] neighbour index (as int bits).
constexpr int kZTab = 6 * kTZ;

__device__ __forceinline__ void load_ztab(float* zt, const DevAxis& Z, bool h_side, int k0,
                                          int nzp, int tid, int nthreads) {
  for (int t = tid; t < kZTab; t += nthreads) {
    const int c = t / kTZ;
    const int k = k0 + (t - c * kTZ);
    const int kk = k < nzp ? k : 0;
    float v;
    switch (c) {
      case 0: v = h_side ? Z.idl_p[kk] : Z.idl_d[kk]; break;
      case 1: v = h_side ? Z.mnx[kk] : Z.mpv[kk]; break;
      case 2: v = h_side ? Z.ah[kk] : Z.ae[kk]; break;
      case 3: v = h_side ? Z.bh[kk] : Z.be[kk]; break;
      case 4: v = h_side ? Z.kh[kk] : Z.ke[kk]; break;
      default: v = __int_as_float(h_side ? Z.nxt[kk] : Z.prv[kk]); break;
    }
    zt[t] = v;
  }
}

// J of the three components of one cell: stored at the cell's first pole of each component.
__device__ __forceinline__ void cell_currents(const MatRec& M, const float* jw, int wp,
                                              const float* J, uint32_t gp, float wv[3]) {
  int po = 0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int n = M.np[c];
    if (n > 0) wv[c] = (wp >= 0) ? jw[wp + po] : J[gp + (uint32_t)po];
    po += n;
  }
}

__device__ __forceinline__ void unpack4(const float4 v, float (&a)[4]) {
  a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
}

// z CPML of one lane's four cells (the two z derivatives da, db of the slots 0 and 1): psi
// from the stage when the slab depth is staged, else from global memory, written back to
// global memory. A lane whose four cells all lie in one slab at a 16-byte-aligned offset does
// it with vector loads and stores; other slab lanes cell by cell.
__device__ __forceinline__ void z_cpml(float (&da)[4], float (&db)[4], unsigned zslm,
                                    const float* zrows, const float* zt, const PsiSet& S,
                                    const YeeParams& P, const DevAxis& Z, int i, int j, int kq,
                                    int k0, int w, int lane) {
  const int side = kq < Z.lo ? 0 : 1;
  const int L = side ? Z.hi : Z.lo;
  const int zq = side ? kq - (Z.n - Z.hi) : kq;
  const int64_t base = ((int64_t)i * P.ny + j) * L;
  if (zslm == 0xFu && (L & 3) == 0 && (zq & 3) == 0) {
    float* g0 = S.p[2][0][side] + base + zq;
    float* g1 = S.p[2][1][side] + base + zq;
    float p0[4], p1[4], a[4], b[4], k[4];
    if (zslab_staged(Z, side, k0)) {
      unpack4(lds4(zrows + (0 * 2 + side) * kTY * kZMax + w * L + zq), p0);
      unpack4(lds4(zrows + (1 * 2 + side) * kTY * kZMax + w * L + zq), p1);
    } else {
      unpack4(*reinterpret_cast<const float4*>(g0), p0);
      unpack4(*reinterpret_cast<const float4*>(g1), p1);
    }
    unpack4(lds4(zt + 2 * kTZ + 4 * lane), a);
    unpack4(lds4(zt + 3 * kTZ + 4 * lane), b);
    unpack4(lds4(zt + 4 * kTZ + 4 * lane), k);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      da[e] = cpml_stretch(da[e], p0[e], a[e], b[e], k[e]);
      db[e] = cpml_stretch(db[e], p1[e], a[e], b[e], k[e]);
    }
    *reinterpret_cast<float4*>(g0) = make_float4(p0[0], p0[1], p0[2], p0[3]);
    *reinterpret_cast<float4*>(g1) = make_float4(p1[0], p1[1], p1[2], p1[3]);
    return;
  }
  for (int e = 0; e < 4; ++e) {
    if (!((zslm >> e) & 1u)) continue;
    const int kk = kq + e;
    const int sd = kk < Z.lo ? 0 : 1;
    const int Ls = sd ? Z.hi : Z.lo;
    const int q = sd ? kk - (Z.n - Z.hi) : kk;
    const int zi = 4 * lane + e;
    const bool staged = zslab_staged(Z, sd, k0);
    float* g0 = psi_addr(S, 2, 0, Z, i, j, kk, P.ny, P.nzp);
    float* g1 = psi_addr(S, 2, 1, Z, i, j, kk, P.ny, P.nzp);
    float p0 = staged ? zrows[(0 * 2 + sd) * kTY * kZMax + w * Ls + q] : *g0;
    float p1 = staged ? zrows[(1 * 2 + sd) * kTY * kZMax + w * Ls + q] : *g1;
    const float a = zt[2 * kTZ + zi], b = zt[3 * kTZ + zi], k = zt[4 * kTZ + zi];
    da[e] = cpml_stretch(da[e], p0, a, b, k);
    db[e] = cpml_stretch(db[e], p1, a, b, k);
    *g0 = p0;
    *g1 = p1;
  }
}

// ---------------------------------------------------------------------------------------------
// H half step
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(160, OEM_WS_MINBLOCKS) k_h_ws(const __grid_constant__ TmaMaps maps, YeeParams P,
                                                 int xch, int* err) {
  extern __shared__ __align__(128) float smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kS * kHStage);
  uint64_t* empty = full + kS;
  float* zt = reinterpret_cast<float*>(empty + kS);
  const int lane = threadIdx.x, w = threadIdx.y;
  const int k0 = blockIdx.x * kTZ;
  const int j0 = blockIdx.y * kTY;
  const int ib = blockIdx.z * xch;
  const int ie = min(ib + xch, P.nx);
  const int np = ie - ib;
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  load_ztab(zt, Z, true, k0, P.nzp, w * 32 + lane, 160);
  if (w == 4 && lane == 0) {
    for (int s = 0; s < kS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kTY);
    }
    mbar_fence_init();
  }
  __syncthreads();

  if (w == 4) {  // ------------------------------------------------------------ producer
    if (lane != 0) return;
    int issued = 0;
    bool ok = true;
    // the tile's y and z psi rows are fixed once; per plane only the x slab rows are added
    const PsiTile pt = psi_tile(P, j0, k0);
    for (int q = 0; q < np && ok; ++q) {
      const int slot = q % kS;
      if (q >= kS) ok = mbar_wait_live(&empty[slot], (uint32_t)((q / kS - 1) & 1), err, kPolls);
      if (!ok) break;
      float* st = smem + slot * kHStage;
      const int i = ib + q;
      const bool xsl = in_slab(X, i);
      const int inext = (i + 1 < P.nx) ? i + 1 : X.nxt[P.nx - 1];
      const uint32_t bytes = 3 * kWideBytes + 5 * kTileBytes + pt.yzbytes + (xsl ? pt.xbytes : 0u);
      mbar_expect_tx(&full[slot], bytes);
      for (int c = 0; c < 3; ++c) {
        tma3(st + kH_EB + c * kBoxW, &maps.e_wide[c], &full[slot], k0, j0, i);
        tma3(st + kH_HT + c * 512, &maps.h_tile[c], &full[slot], k0, j0, i);
      }
      // only Ey, Ez of the next plane enter the x derivatives
      tma3(st + kH_EN + 512, &maps.e_tile[1], &full[slot], k0, j0, inext);
      tma3(st + kH_EN + 1024, &maps.e_tile[2], &full[slot], k0, j0, inext);
      stage_psi(pt, P.psih, P, st + kH_PX, st + kH_PY, st + kH_PZ, &full[slot], i, j0, k0, xsl);
      issued = q + 1;
    }
    for (int q = max(0, issued - kS); q < issued; ++q)  // drain (no-op when consumed)
      mbar_wait(&full[q % kS], (uint32_t)((q / kS) & 1), err);
    return;
  }

  // --------------------------------------------------------------------------- consumers
  const int j = j0 + w;
  const bool row_ok = j < P.ny;
  const int jj = row_ok ? j : 0;
  const int jp = Y.nxt[jj];
  const float mj = Y.mnx[jj], idy = Y.idl_p[jj];
  const bool ysl = row_ok && in_slab(Y, j);
  // a neighbour that is not the adjacent index is fetched from global memory, unless its wall
  // mask is 0: then the staged adjacent value (finite: a field or the zero fill) times 0 gives
  // the same difference
  const bool yspecial = row_ok && jp != j + 1 && mj != 0.0f;
  const int kq = k0 + 4 * lane;
  unsigned kvm = 0, zslm = 0, zspm = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = kq + e;
    const bool kv = row_ok && k < P.nz;
    kvm |= (unsigned)kv << e;
    zslm |= (unsigned)(kv && in_slab(Z, k)) << e;
    zspm |= (unsigned)(kv && __float_as_int(zt[5 * kTZ + 4 * lane + e]) != k + 1 &&
                       zt[kTZ + 4 * lane + e] != 0.0f) << e;
  }
  // a plain row: every cell interior in y and z (adjacent neighbours, unit masks, no CPML)
  const bool yplain = row_ok && !ysl && !yspecial && mj == 1.0f;  // uniform over the warp
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const float ch = P.ch;
  const int ro = w * kBZ + 4 * lane;  // this quad in a halo box
  const int to = w * kTZ + 4 * lane;  // this quad in a tile
  for (int t = 0; t < np; ++t) {
    const int slot = t % kS;
    // the plane's axis values do not depend on the stage: their loads are issued before the
    // wait, which hides their latency
    const int i = ib + t;
    const bool xsl = in_slab(X, i);
    const float mi = X.mnx[i], idx_ = X.idl_p[i];
    const bool xfast = !xsl && i + 1 < P.nx && X.nxt[i] == i + 1 && mi == 1.0f;
    bool got = mbar_wait(&full[slot], (uint32_t)((t / kS) & 1), err);
    if (!__all_sync(kFull, got)) break;
    const float* st = smem + slot * kHStage;
    const int64_t row = i * si + (int64_t)j * sj;
    if (kvm) {
      float ex[4], ey[4], ez[4], yex[4], yez[4], ney[4], nez[4], hx[4], hy[4], hz[4];
      float idz[4], mkz[4];
      unpack4(lds4(st + kH_EB + ro), ex);
      unpack4(lds4(st + kH_EB + kBoxW + ro), ey);
      unpack4(lds4(st + kH_EB + 2 * kBoxW + ro), ez);
      if (yspecial) {
        const int64_t oy = i * si + (int64_t)jp * sj + kq;
        unpack4(*reinterpret_cast<const float4*>(P.f[0] + oy), yex);
        unpack4(*reinterpret_cast<const float4*>(P.f[2] + oy), yez);
      } else {
        unpack4(lds4(st + kH_EB + ro + kBZ), yex);
        unpack4(lds4(st + kH_EB + 2 * kBoxW + ro + kBZ), yez);
      }
      unpack4(lds4(st + kH_EN + 512 + to), ney);
      unpack4(lds4(st + kH_EN + 1024 + to), nez);
      unpack4(lds4(st + kH_HT + to), hx);
      unpack4(lds4(st + kH_HT + 512 + to), hy);
      unpack4(lds4(st + kH_HT + 1024 + to), hz);
      unpack4(lds4(zt + 4 * lane), idz);
      unpack4(lds4(zt + kTZ + 4 * lane), mkz);
      const float ex4 = st[kH_EB + ro + 4];
      const float ey4 = st[kH_EB + kBoxW + ro + 4];
      // z derivatives of all four cells, then the z CPML of the slab lanes in one block
      float dyz[4], dxz[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        float zex = (e < 3) ? ex[e + 1] : ex4;
        float zey = (e < 3) ? ey[e + 1] : ey4;
        if ((zspm >> e) & 1u) {
          const int kp = __float_as_int(zt[5 * kTZ + 4 * lane + e]);
          zex = P.f[0][row + kp];
          zey = P.f[1][row + kp];
        }
        dyz[e] = fdiff(zey, mkz[e], ey[e], idz[e]);
        dxz[e] = fdiff(zex, mkz[e], ex[e], idz[e]);
      }
      if (zslm) z_cpml(dyz, dxz, zslm, st + kH_PZ, zt, P.psih, P, Z, i, j, kq, k0, w, lane);
      if (yplain && xfast) {
        // x and y interior: unit masks, no x/y CPML (the same bits as below, n * 1 == n)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float nhx = h_new(hx[e], ch, __fmul_rn(__fsub_rn(yez[e], ez[e]), idy), dyz[e]);
          const float nhy = h_new(hy[e], ch, dxz[e], __fmul_rn(__fsub_rn(nez[e], ez[e]), idx_));
          const float nhz = h_new(hz[e], ch, __fmul_rn(__fsub_rn(ney[e], ey[e]), idx_),
                                  __fmul_rn(__fsub_rn(yex[e], ex[e]), idy));
          const bool kv = (kvm >> e) & 1u;
          hx[e] = kv ? nhx : hx[e];
          hy[e] = kv ? nhy : hy[e];
          hz[e] = kv ? nhz : hz[e];
        }
      } else {
        const float ay = Y.ah[jj], by = Y.bh[jj], ky = Y.kh[jj];
        const float ax_ = X.ah[i], bx_ = X.bh[i], kx_ = X.kh[i];
        // psi of this quad (x: Hy, Hz; y: Hx, Hz)
        float px[2][4], py[2][4];
        if (xsl)
          for (int s = 0; s < 2; ++s) unpack4(lds4(st + kH_PX + (s * 4 + w) * kTZ + 4 * lane), px[s]);
        if (ysl)
          for (int s = 0; s < 2; ++s) unpack4(lds4(st + kH_PY + (s * 4 + w) * kTZ + 4 * lane), py[s]);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float dzy = fdiff(yez[e], mj, ez[e], idy);
          const float dzx = fdiff(nez[e], mi, ez[e], idx_);
          const float dyx = fdiff(ney[e], mi, ey[e], idx_);
          const float dxy = fdiff(yex[e], mj, ex[e], idy);
          float sy0 = dzy, sy1 = dxy, sx0 = dzx, sx1 = dyx;
          if (ysl) {
            sy0 = cpml_stretch(dzy, py[0][e], ay, by, ky);
            sy1 = cpml_stretch(dxy, py[1][e], ay, by, ky);
          }
          if (xsl) {
            sx0 = cpml_stretch(dzx, px[0][e], ax_, bx_, kx_);
            sx1 = cpml_stretch(dyx, px[1][e], ax_, bx_, kx_);
          }
          const bool kv = (kvm >> e) & 1u;
          hx[e] = kv ? h_new(hx[e], ch, sy0, dyz[e]) : hx[e];  // -(dEz/dy - dEy/dz)
          hy[e] = kv ? h_new(hy[e], ch, dxz[e], sx0) : hy[e];  // -(dEx/dz - dEz/dx)
          hz[e] = kv ? h_new(hz[e], ch, sx1, sy1) : hz[e];     // -(dEy/dx - dEx/dy)
        }
        if (xsl)
          for (int s = 0; s < 2; ++s)
            *reinterpret_cast<float4*>(psi_addr(P.psih, 0, s, X, i, j, kq, P.ny, P.nzp)) =
                make_float4(px[s][0], px[s][1], px[s][2], px[s][3]);
        if (ysl)
          for (int s = 0; s < 2; ++s)
            *reinterpret_cast<float4*>(psi_addr(P.psih, 1, s, Y, i, j, kq, P.ny, P.nzp)) =
                make_float4(py[s][0], py[s][1], py[s][2], py[s][3]);
      }
      *reinterpret_cast<float4*>(P.f[3] + row + kq) = make_float4(hx[0], hx[1], hx[2], hx[3]);
      *reinterpret_cast<float4*>(P.f[4] + row + kq) = make_float4(hy[0], hy[1], hy[2], hy[3]);
      *reinterpret_cast<float4*>(P.f[5] + row + kq) = make_float4(hz[0], hz[1], hz[2], hz[3]);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[slot]);
  }
}

// ---------------------------------------------------------------------------------------------
// E full step with the deferred ADE
// ---------------------------------------------------------------------------------------------
// Snapshot rows of the box monitors that hold cells of this quad (plane i, row j, cells kq ..
// kq + 3): the six components at the cells' own Yee positions, E^{n+1} as just computed and
// H^{n+1/2} from the staged halo box (hb: this quad's Hx; Hy, Hz follow at kBoxW strides),
// into ring row step % T (srow: that row of each box, set once per block in shared memory),
// the layout and values of k_snap_boxes. sbm: the boxes whose rows and z range hold cells of this
// quad (fixed per lane), so that a lane with none skips the call.
__device__ __forceinline__ void snap_quad(const SnapBoxes& sb, float* const* srow, unsigned sbm,
                                          int i, int j, int kq, const float* ex, const float* ey,
                                          const float* ez, const float* hb) {
#pragma unroll
  for (int m = 0; m < kMaxSnapBoxes; ++m) {
    const SnapBox& b = sb.b[m];
    if (!((sbm >> m) & 1u) || (unsigned)(i - b.i0) >= (unsigned)b.ni) continue;
    float hx[4], hy[4], hz[4];
    unpack4(lds4(hb), hx);
    unpack4(lds4(hb + kBoxW), hy);
    unpack4(lds4(hb + 2 * kBoxW), hz);
    float* row = srow[m];
    const int64_t base = ((int64_t)(i - b.i0) * b.nj + (j - b.j0)) * b.nk - b.k0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = kq + e;
      if ((unsigned)(k - b.k0) >= (unsigned)b.nk) continue;
      const int64_t o = base + k;
      row[o] = ex[e];
      row[b.cells + o] = ey[e];
      row[2 * b.cells + o] = ez[e];
      row[3 * b.cells + o] = hx[e];
      row[4 * b.cells + o] = hy[e];
      row[5 * b.cells + o] = hz[e];
    }
  }
}

// The E update's producer warp: per plane of the chunk it waits for a free stage and stages the
// H halo box, the Hy/Hz tiles of the previous plane, the E and material tiles (TMA), the plane's
// psi rows and the window of pole currents of its dispersive rows (bulk copies), then drains its
// own copies before it returns. Lane 0 issues; the warp first reads the chunk's pole ranges.
__device__ __forceinline__ void e_producer(const TmaMaps& maps, const YeeParams& P, float* smem,
                                           uint64_t* full, uint64_t* empty, uint32_t* segt,
                                           int* err, int ib, int np, int j0, int k0, int lane) {
  const DevAxis& X = P.ax[0];
  const bool wide = P.mat32 != nullptr;
  // pole ranges of every (plane, row) of the chunk: the first pole of the tile row and the
  // end of its last segment, all fetched at once by the producer warp
  const int64_t nseg = (int64_t)P.nx * P.ny * P.nzp / 32;
  const int nst = min(4, (P.nzp - k0) / 32);
  if (P.has_ade) {
    for (int t = lane; t < np * kTY; t += 32) {
      const int i = ib + t / kTY, j = j0 + t % kTY;
      uint32_t a = 0u, b = 0u;
      if (j < P.ny) {
        const int64_t s0 = (((int64_t)i * P.ny + j) * P.nzp + k0) >> 5;
        a = __ldg(P.seg_ofs + s0);
        b = (s0 + nst < nseg) ? __ldg(P.seg_ofs + s0 + nst) : P.n_pole_total;
      }
      segt[2 * t] = a;
      segt[2 * t + 1] = b;
    }
    __syncwarp();
  }
  if (lane != 0) return;
  int issued = 0;
  bool ok = true;
  const uint32_t mbytes = (uint32_t)(kTY * kTZ * (wide ? 4 : 2));
  // the tile's y and z psi rows are fixed once; per plane only the x slab rows are added.
  // Pool layout per plane: x rows (1024 floats), y rows (1024), z rows (512) where present,
  // then the pole-current window.
  const PsiTile pt = psi_tile(P, j0, k0);
  for (int q = 0; q < np && ok; ++q) {
    const int slot = q % kS;
    const int i = ib + q;
    const bool xsl = in_slab(X, i);
    int offs[3] = {-1, -1, -1};
    int wbase = 0;
    if (xsl) { offs[0] = wbase; wbase += 1024; }
    if (pt.ymask) { offs[1] = wbase; wbase += 1024; }
    if (pt.zs0 || pt.zs1) { offs[2] = wbase; wbase += 512; }
    const int cap = kEPool - wbase;  // pole currents (floats) this plane can stage
    int pstart[kTY], poff[kTY], pcnt[kTY];
    int used = 0;
#pragma unroll
    for (int r = 0; r < kTY; ++r) {
      const uint32_t a = P.has_ade ? segt[2 * (q * kTY + r)] : 0u;
      const uint32_t b = P.has_ade ? segt[2 * (q * kTY + r) + 1] : 0u;
      pstart[r] = (int)a; poff[r] = -2; pcnt[r] = 0;
      if (b <= a) continue;
      const int a16 = (int)(a & ~3u);  // 16-byte aligned start
      const int n4 = (int)(((b - (uint32_t)a16) + 3u) & ~3u);
      if (used + n4 <= cap) {
        poff[r] = used + ((int)a - a16);
        pcnt[r] = n4;
        used += n4;
      } else {
        poff[r] = -1;  // consumers read this row's poles from global memory
      }
    }
    if (q >= kS) ok = mbar_wait_live(&empty[slot], (uint32_t)((q / kS - 1) & 1), err, kPolls);
    if (!ok) break;
    float* st = smem + slot * kEStage;
    int* tab = reinterpret_cast<int*>(st + kE_PT);
    const int iprev = (i > 0) ? i - 1 : X.prv[0];
    uint32_t bytes = 3 * kWideBytes + 5 * kTileBytes + mbytes + pt.yzbytes +
                     (xsl ? pt.xbytes : 0u) + (uint32_t)used * 4;
#pragma unroll
    for (int r = 0; r < kTY; ++r) {
      tab[2 * r] = pstart[r];
      tab[2 * r + 1] = poff[r];
    }
    tab[8] = offs[0];
    tab[9] = offs[1];
    tab[10] = offs[2];
    tab[11] = wbase;
    mbar_expect_tx(&full[slot], bytes);
    for (int c = 0; c < 3; ++c) {
      tma3(st + kE_HB + c * kBoxW, &maps.h_wide[c], &full[slot], k0 - 4, j0 - 1, i);
      tma3(st + kE_ET + c * 512, &maps.e_tile[c], &full[slot], k0, j0, i);
    }
    tma3(st + kE_HP, &maps.h_tile[1], &full[slot], k0, j0, iprev);
    tma3(st + kE_HP + 512, &maps.h_tile[2], &full[slot], k0, j0, iprev);
    tma3(st + kE_MT, &maps.m_tile, &full[slot], k0, j0, i);
    float* pool = st + kE_POOL;
    stage_psi(pt, P.psie, P, pool + offs[0], pool + offs[1], pool + offs[2], &full[slot], i, j0,
              k0, xsl);
#pragma unroll
    for (int r = 0; r < kTY; ++r)
      if (pcnt[r] > 0) {
        const int a16 = pstart[r] & ~3;
        bulk(pool + wbase + (poff[r] - (pstart[r] - a16)), P.J + a16, (uint32_t)pcnt[r] * 4,
             &full[slot]);
      }
    issued = q + 1;
  }
  for (int q = max(0, issued - kS); q < issued; ++q)
    mbar_wait(&full[q % kS], (uint32_t)((q / kS) & 1), err);
}

template <bool SNAP, bool SMATS>
__global__ void __launch_bounds__(160, OEM_WS_MINBLOCKS) k_e_ws(const __grid_constant__ TmaMaps maps, YeeParams P,
                                                 int xch, int n_mats, int* err,
                                                 const __grid_constant__ SnapBoxes sb) {
  extern __shared__ __align__(128) float smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kS * kEStage);
  uint64_t* empty = full + kS;
  float* zt = reinterpret_cast<float*>(empty + kS);
  MatRec* smats = reinterpret_cast<MatRec*>(zt + kZTab);
  uint32_t* segt = reinterpret_cast<uint32_t*>(smats + kSmemMats);  // [plane][row][start, end]
  // a barrier no thread arrives at (the wait-expiry check), after everything else
  uint64_t* never = reinterpret_cast<uint64_t*>(segt + kXMax * kTY * 2);
  float** srow = reinterpret_cast<float**>(never + 1);  // this step's snapshot row of each box
  const int lane = threadIdx.x, w = threadIdx.y;
  const int tid = w * 32 + lane;
  const int k0 = blockIdx.x * kTZ;
  const int j0 = blockIdx.y * kTY;
  const int ib = blockIdx.z * xch;
  const int ie = min(ib + xch, P.nx);
  const int np = ie - ib;
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const bool wide = P.mat32 != nullptr;
  // SMATS: the plan's material records fit in shared memory (n_mats <= kSmemMats), so the
  // per-cell record loads are shared-memory loads the compiler knows as such
  const MatRec* mats = SMATS ? smats : P.mats;
  if (SMATS) {
    const uint4* src = reinterpret_cast<const uint4*>(P.mats);
    uint4* dst = reinterpret_cast<uint4*>(smats);
    for (int q = tid; q < n_mats * 4; q += 160) dst[q] = src[q];
  }
  load_ztab(zt, Z, false, k0, P.nzp, tid, 160);
  if (SNAP && tid < sb.n)
    srow[tid] = sb.b[tid].snap + (int64_t)(*sb.step % sb.b[tid].T) * 6 * sb.b[tid].cells;
  if (w == 4 && lane == 0) {
    for (int s = 0; s < kS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kTY);
    }
    mbar_init(never, 1);
    mbar_fence_init();
  }
  __syncthreads();

  if (w == 4) {  // ------------------------------------------------------------ producer
    e_producer(maps, P, smem, full, empty, segt, err, ib, np, j0, k0, lane);
    return;
  }

  // --------------------------------------------------------------------------- consumers
  const int j = j0 + w;
  const bool row_ok = j < P.ny;
  const int jj = row_ok ? j : 0;
  const int jm = Y.prv[jj];
  const float mj = Y.mpv[jj], idy = Y.idl_d[jj];
  const bool ysl = row_ok && in_slab(Y, j);
  const bool yspecial = row_ok && jm != j - 1 && mj != 0.0f;  // see the H kernel
  const int kq = k0 + 4 * lane;
  unsigned kvm = 0, zslm = 0, zspm = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = kq + e;
    const bool kv = row_ok && k < P.nz;
    kvm |= (unsigned)kv << e;
    zslm |= (unsigned)(kv && in_slab(Z, k)) << e;
    zspm |= (unsigned)(kv && __float_as_int(zt[5 * kTZ + 4 * lane + e]) != k - 1 &&
                       zt[kTZ + 4 * lane + e] != 0.0f) << e;
  }
  const bool yplain = row_ok && !ysl && !yspecial && mj == 1.0f;  // uniform over the warp
  const unsigned lt = (1u << lane) - 1u;
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const float cw = P.cw;
  const int ro = (w + 1) * kBZ + 4 + 4 * lane;  // this quad in the H halo box
  const int to = w * kTZ + 4 * lane;
  unsigned sbm = 0;  // boxes with cells in this lane's row and z range
  if (SNAP) {
#pragma unroll
    for (int m = 0; m < kMaxSnapBoxes; ++m) {
      const SnapBox& b = sb.b[m];
      if (m < sb.n && row_ok && (unsigned)(j - b.j0) < (unsigned)b.nj && kq < b.k0 + b.nk &&
          kq + 4 > b.k0)
        sbm |= 1u << m;
    }
  }
  for (int t = 0; t < np; ++t) {
    const int slot = t % kS;
    // the plane's axis values, loaded before the wait as in the H update
    const int i = ib + t;
    const bool xsl = in_slab(X, i);
    const float mi = X.mpv[i], idx_ = X.idl_d[i];
    bool got = mbar_wait(&full[slot], (uint32_t)((t / kS) & 1), err);
    // the plan's wait-expiry check: wait on a barrier nothing arrives at, with its short bound,
    // so that the expiry path (error word, early exit of every warp, the producer's drain) runs
    if (P.expire_polls > 0 && got) got = mbar_wait_live(never, 0u, err, (uint32_t)P.expire_polls);
    if (!__all_sync(kFull, got)) break;
    const float* st = smem + slot * kEStage;
    const int* tab = reinterpret_cast<const int*>(st + kE_PT);
    const float* pool = st + kE_POOL;
    const float* jw = pool + tab[11];  // pole currents of the plane's rows
    uint32_t mid[4] = {0u, 0u, 0u, 0u};
    if (row_ok) {
      if (wide) {
        const uint4 m = *reinterpret_cast<const uint4*>(reinterpret_cast<const uint32_t*>(st + kE_MT) + to);
        mid[0] = m.x; mid[1] = m.y; mid[2] = m.z; mid[3] = m.w;
      } else {
        const uint2 m = *reinterpret_cast<const uint2*>(reinterpret_cast<const uint16_t*>(st + kE_MT) + to);
        mid[0] = m.x & 0xffffu; mid[1] = m.x >> 16; mid[2] = m.y & 0xffffu; mid[3] = m.y >> 16;
      }
    }
    // a row whose segments hold no poles (window offset -2) skips the pole bookkeeping
    const bool row_poles = P.has_ade && tab[2 * w + 1] != -2;
    int lane_np = 0;
    if (row_poles) {
#pragma unroll
      for (int e = 0; e < 4; ++e) lane_np += mats[mid[e]].reserved;
    }
    // poles of this lane: global index gp, window index wp (-1: read J from global memory)
    uint32_t gp = 0;
    int wp = -1;
    if (row_poles && __any_sync(kFull, lane_np > 0)) {
      int pre = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) pre += __popc(__ballot_sync(kFull, (lane_np >> b) & 1) & lt) << b;
      gp = (uint32_t)tab[2 * w] + (uint32_t)pre;
      if (tab[2 * w + 1] >= 0) wp = tab[2 * w + 1] + pre;
    }
    const int64_t row = i * si + (int64_t)j * sj;
    if (kvm) {
      float ex[4], ey[4], ez[4], hx[4], hy[4], hz[4], yhx[4], yhz[4], phy[4], phz[4];
      float idz[4], mkz[4];
      unpack4(lds4(st + kE_ET + to), ex);
      unpack4(lds4(st + kE_ET + 512 + to), ey);
      unpack4(lds4(st + kE_ET + 1024 + to), ez);
      unpack4(lds4(st + kE_HB + ro), hx);
      unpack4(lds4(st + kE_HB + kBoxW + ro), hy);
      unpack4(lds4(st + kE_HB + 2 * kBoxW + ro), hz);
      if (yspecial) {
        const int64_t oy = i * si + (int64_t)jm * sj + kq;
        unpack4(*reinterpret_cast<const float4*>(P.f[3] + oy), yhx);
        unpack4(*reinterpret_cast<const float4*>(P.f[5] + oy), yhz);
      } else {
        unpack4(lds4(st + kE_HB + ro - kBZ), yhx);
        unpack4(lds4(st + kE_HB + 2 * kBoxW + ro - kBZ), yhz);
      }
      unpack4(lds4(st + kE_HP + to), phy);
      unpack4(lds4(st + kE_HP + 512 + to), phz);
      unpack4(lds4(zt + 4 * lane), idz);
      unpack4(lds4(zt + kTZ + 4 * lane), mkz);
      const float hxm = st[kE_HB + ro - 1];
      const float hym = st[kE_HB + kBoxW + ro - 1];
      // z derivatives of all four cells, then the z CPML of the slab lanes in one block
      float dyz[4], dxz[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        float zhx = (e > 0) ? hx[e - 1] : hxm;
        float zhy = (e > 0) ? hy[e - 1] : hym;
        if ((zspm >> e) & 1u) {
          const int km = __float_as_int(zt[5 * kTZ + 4 * lane + e]);
          zhx = P.f[3][row + km];
          zhy = P.f[4][row + km];
        }
        dyz[e] = bdiff(hy[e], zhy, mkz[e], idz[e]);  // dHy/dz
        dxz[e] = bdiff(hx[e], zhx, mkz[e], idz[e]);  // dHx/dz
      }
      if (zslm) z_cpml(dyz, dxz, zslm, pool + tab[10], zt, P.psie, P, Z, i, j, kq, k0, w, lane);
      // x and y derivatives (CPML on the x/y slab planes and rows)
      float sy0[4], sy1[4], sx0[4], sx1[4];
      if (yplain && !xsl && i > 0 && X.prv[i] == i - 1 && mi == 1.0f) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          sy0[e] = __fmul_rn(__fsub_rn(hz[e], yhz[e]), idy);   // dHz/dy
          sx0[e] = __fmul_rn(__fsub_rn(hz[e], phz[e]), idx_);  // dHz/dx
          sx1[e] = __fmul_rn(__fsub_rn(hy[e], phy[e]), idx_);  // dHy/dx
          sy1[e] = __fmul_rn(__fsub_rn(hx[e], yhx[e]), idy);   // dHx/dy
        }
      } else {
        const float ay = Y.ae[jj], by = Y.be[jj], ky = Y.ke[jj];
        const float ax_ = X.ae[i], bx_ = X.be[i], kx_ = X.ke[i];
        float px[2][4], py[2][4];
        if (xsl)
          for (int s = 0; s < 2; ++s) unpack4(lds4(pool + tab[8] + (s * 4 + w) * kTZ + 4 * lane), px[s]);
        if (ysl)
          for (int s = 0; s < 2; ++s) unpack4(lds4(pool + tab[9] + (s * 4 + w) * kTZ + 4 * lane), py[s]);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          sy0[e] = bdiff(hz[e], yhz[e], mj, idy);
          sx0[e] = bdiff(hz[e], phz[e], mi, idx_);
          sx1[e] = bdiff(hy[e], phy[e], mi, idx_);
          sy1[e] = bdiff(hx[e], yhx[e], mj, idy);
          if (ysl) {
            sy0[e] = cpml_stretch(sy0[e], py[0][e], ay, by, ky);
            sy1[e] = cpml_stretch(sy1[e], py[1][e], ay, by, ky);
          }
          if (xsl) {
            sx0[e] = cpml_stretch(sx0[e], px[0][e], ax_, bx_, kx_);
            sx1[e] = cpml_stretch(sx1[e], px[1][e], ax_, bx_, kx_);
          }
        }
        if (xsl)
          for (int s = 0; s < 2; ++s)
            *reinterpret_cast<float4*>(psi_addr(P.psie, 0, s, X, i, j, kq, P.ny, P.nzp)) =
                make_float4(px[s][0], px[s][1], px[s][2], px[s][3]);
        if (ysl)
          for (int s = 0; s < 2; ++s)
            *reinterpret_cast<float4*>(psi_addr(P.psie, 1, s, Y, i, j, kq, P.ny, P.nzp)) =
                make_float4(py[s][0], py[s][1], py[s][2], py[s][3]);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const MatRec& M = mats[mid[e]];
        const float4 cab = *reinterpret_cast<const float4*>(&M.ca[0]);
        const float2 cb12 = *reinterpret_cast<const float2*>(&M.cb[1]);
        float wv[3] = {0.f, 0.f, 0.f};
        if (lane_np > 0 && M.reserved > 0) {
          cell_currents(M, jw, wp, P.J, gp, wv);
          gp += (uint32_t)M.reserved;
          if (wp >= 0) wp += M.reserved;
        }
        const bool kv = (kvm >> e) & 1u;
        const float nex = e_new(cab.x, ex[e], cab.w, sy0[e], dyz[e], cw, wv[0]);   // dHz/dy - dHy/dz
        const float ney = e_new(cab.y, ey[e], cb12.x, dxz[e], sx0[e], cw, wv[1]);  // dHx/dz - dHz/dx
        const float nez = e_new(cab.z, ez[e], cb12.y, sx1[e], sy1[e], cw, wv[2]);  // dHy/dx - dHx/dy
        ex[e] = kv ? nex : ex[e];
        ey[e] = kv ? ney : ey[e];
        ez[e] = kv ? nez : ez[e];
      }
      *reinterpret_cast<float4*>(P.f[0] + row + kq) = make_float4(ex[0], ex[1], ex[2], ex[3]);
      *reinterpret_cast<float4*>(P.f[1] + row + kq) = make_float4(ey[0], ey[1], ey[2], ey[3]);
      *reinterpret_cast<float4*>(P.f[2] + row + kq) = make_float4(ez[0], ez[1], ez[2], ez[3]);
      if constexpr (SNAP) {
        if (sbm) snap_quad(sb, srow, sbm, i, j, kq, ex, ey, ez, st + kE_HB + ro);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[slot]);
  }
}

// ---------------------------------------------------------------------------------------------
// Fused H + E step over two field banks
// ---------------------------------------------------------------------------------------------
// One pass reads E^n, H^{n-1/2} (and the H-side psi) from the current bank and writes H^{n+1/2},
// E^{n+1} (and the H-side psi) to the other bank, so every field value crosses HBM once each
// way. Per x plane i a block computes H^{n+1/2}(i) on its four rows plus the row below them
// (warp 4, needed by the E update's y difference) and on the cell before its z range (the
// producer warp, ahead of time, for the z difference), keeps the planes i and i-1 of H^{n+1/2}
// in shared memory, and
// then updates E(i) on its four rows. The first plane of a chunk is preceded by an H-only pass
// over the x neighbour plane X.prv[ib] (own rows). The E-side psi is updated in place (cells are
// owned by one block); the H-side psi goes to the other bank because the halo row and cell read
// psi of cells another block owns. The arithmetic is that of the two-kernel path, bit for bit.
//
// Eligible grids: y and z without periodic wrap (the halo row and cell are the adjacent ones);
// no H-side injection (the H update's result is consumed inside the kernel).
constexpr int kFS = 3;
constexpr int kF_EBS = 832;                   // floats per 136 x 6 E box (128-B aligned)
constexpr int kF_T5 = 640;                    // floats per 128 x 5 tile
constexpr int kF_EB = 0;                      // E^n box x3: rows j0-1 .. j0+4, cols k0 .. k0+135
constexpr int kF_EN = kF_EB + 3 * kF_EBS;     // Ey, Ez of plane X.nxt[i]: rows j0-1 .. j0+3
constexpr int kF_HO = kF_EN + 2 * kF_T5;      // H^{n-1/2} x3: rows j0-1 .. j0+3
constexpr int kF_MT = kF_HO + 3 * kF_T5;      // material tile, rows j0 .. j0+3
constexpr int kFStage = kF_MT + 512;
// Hx, Hy of H^{n+1/2} at (rows j0 .. j0+3, k0 - 1) of the main planes, a ring of kF_HRP planes
// [plane % kF_HRP][c][row], filled kF_HB planes at a time by the 32 producer lanes
constexpr int kF_HRP = 16;
constexpr int kF_HB = 8;
constexpr int kF_HR = kF_HRP * 2 * kTY;
static_assert(kF_HB * kTY == 32 && kF_HRP >= kF_HB + kFS + 1, "halo ring covers the batches");
constexpr uint32_t kF_EBBytes = 6 * kBZ * 4;
constexpr uint32_t kF_T5Bytes = 5 * kTZ * 4;
constexpr int kF_HN = 2 * 3 * 5 * kTZ;        // H^{n+1/2} of two planes [parity][comp][row][z]
static_assert((kF_EN * 4) % 128 == 0 && (kF_HO * 4) % 128 == 0 && (kF_MT * 4) % 128 == 0 &&
                  (kFStage * 4) % 128 == 0 && (kF_EBS * 4) % 128 == 0,
              "fused stage slots aligned");

__device__ __forceinline__ float* hn_row(float* hn, int par, int c, int r) {
  return hn + ((par * 3 + c) * 5 + r) * kTZ;
}

// z CPML of the slab cells of one quad with psi read from `in` and, when `commit`, written to
// `out` (cell by cell; slab lanes are few).
__device__ __forceinline__ void zcpml_io(float (&da)[4], float (&db)[4], unsigned zslm,
                                         const float* zt, const PsiSet& in, const PsiSet& out,
                                         bool commit, const YeeParams& P, int i, int j, int kq,
                                         int lane) {
  const DevAxis& Z = P.ax[2];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    if (!((zslm >> e) & 1u)) continue;
    const int kk = kq + e;
    float p0 = *psi_addr(in, 2, 0, Z, i, j, kk, P.ny, P.nzp);
    float p1 = *psi_addr(in, 2, 1, Z, i, j, kk, P.ny, P.nzp);
    const int zi = 4 * lane + e;
    const float a = zt[2 * kTZ + zi], b = zt[3 * kTZ + zi], k = zt[4 * kTZ + zi];
    da[e] = cpml_stretch(da[e], p0, a, b, k);
    db[e] = cpml_stretch(db[e], p1, a, b, k);
    if (commit) {
      *psi_addr(out, 2, 0, Z, i, j, kk, P.ny, P.nzp) = p0;
      *psi_addr(out, 2, 1, Z, i, j, kk, P.ny, P.nzp) = p1;
    }
  }
}

// H^{n+1/2} of one quad of row jrow (box / tile row hr) of plane i from the stage; written to
// the other bank (field and psi) when `commit`.
__device__ __forceinline__ void fused_h_quad(const YeeParams& P, const FieldOut& out,
                                             const float* st, const float* zt, int i, int jrow,
                                             int hr, int k0, int lane, bool commit,
                                             float (&hx)[4], float (&hy)[4], float (&hz)[4]) {
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const int jp = Y.nxt[jrow];
  const float mj = Y.mnx[jrow], idy = Y.idl_p[jrow];
  const bool ysl = in_slab(Y, jrow);
  const bool yspecial = jp != jrow + 1 && mj != 0.0f;
  const int kq = k0 + 4 * lane;
  unsigned kvm = 0, zslm = 0, zspm = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = kq + e;
    const bool kv = k < P.nz;
    kvm |= (unsigned)kv << e;
    zslm |= (unsigned)(kv && in_slab(Z, k)) << e;
    zspm |= (unsigned)(kv && __float_as_int(zt[5 * kTZ + 4 * lane + e]) != k + 1 &&
                       zt[kTZ + 4 * lane + e] != 0.0f) << e;
  }
  const bool yplain = !ysl && !yspecial && mj == 1.0f;
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const int64_t row = i * si + (int64_t)jrow * sj;
  const int ro = hr * kBZ + 4 * lane;
  const int to = hr * kTZ + 4 * lane;
  const float ch = P.ch;
  const bool xsl = in_slab(X, i);
  const float mi = X.mnx[i], idx_ = X.idl_p[i];
  unpack4(lds4(st + kF_HO + to), hx);
  unpack4(lds4(st + kF_HO + kF_T5 + to), hy);
  unpack4(lds4(st + kF_HO + 2 * kF_T5 + to), hz);
  if (!kvm) return;  // the quad lies past nz: no global access (its row may end before it)
  float ex[4], ey[4], ez[4], yex[4], yez[4], ney[4], nez[4], idz[4], mkz[4];
  unpack4(lds4(st + kF_EB + ro), ex);
  unpack4(lds4(st + kF_EB + kF_EBS + ro), ey);
  unpack4(lds4(st + kF_EB + 2 * kF_EBS + ro), ez);
  if (yspecial) {
    const int64_t oy = i * si + (int64_t)jp * sj + kq;
    unpack4(*reinterpret_cast<const float4*>(P.f[0] + oy), yex);
    unpack4(*reinterpret_cast<const float4*>(P.f[2] + oy), yez);
  } else {
    unpack4(lds4(st + kF_EB + ro + kBZ), yex);
    unpack4(lds4(st + kF_EB + 2 * kF_EBS + ro + kBZ), yez);
  }
  unpack4(lds4(st + kF_EN + to), ney);
  unpack4(lds4(st + kF_EN + kF_T5 + to), nez);
  unpack4(lds4(zt + 4 * lane), idz);
  unpack4(lds4(zt + kTZ + 4 * lane), mkz);
  const float ex4 = st[kF_EB + ro + 4];
  const float ey4 = st[kF_EB + kF_EBS + ro + 4];
  float dyz[4], dxz[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    float zex = (e < 3) ? ex[e + 1] : ex4;
    float zey = (e < 3) ? ey[e + 1] : ey4;
    if ((zspm >> e) & 1u) {
      const int kp = __float_as_int(zt[5 * kTZ + 4 * lane + e]);
      zex = P.f[0][row + kp];
      zey = P.f[1][row + kp];
    }
    dyz[e] = fdiff(zey, mkz[e], ey[e], idz[e]);
    dxz[e] = fdiff(zex, mkz[e], ex[e], idz[e]);
  }
  if (zslm) zcpml_io(dyz, dxz, zslm, zt, P.psih, out.psih, commit, P, i, jrow, kq, lane);
  if (yplain && !xsl && i + 1 < P.nx && X.nxt[i] == i + 1 && mi == 1.0f) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float nhx = h_new(hx[e], ch, __fmul_rn(__fsub_rn(yez[e], ez[e]), idy), dyz[e]);
      const float nhy = h_new(hy[e], ch, dxz[e], __fmul_rn(__fsub_rn(nez[e], ez[e]), idx_));
      const float nhz = h_new(hz[e], ch, __fmul_rn(__fsub_rn(ney[e], ey[e]), idx_),
                              __fmul_rn(__fsub_rn(yex[e], ex[e]), idy));
      const bool kv = (kvm >> e) & 1u;
      hx[e] = kv ? nhx : hx[e];
      hy[e] = kv ? nhy : hy[e];
      hz[e] = kv ? nhz : hz[e];
    }
  } else {
    const float ay = Y.ah[jrow], by = Y.bh[jrow], ky = Y.kh[jrow];
    const float ax_ = X.ah[i], bx_ = X.bh[i], kx_ = X.kh[i];
    float px[2][4], py[2][4];
    if (xsl)
      for (int s = 0; s < 2; ++s)
        unpack4(*reinterpret_cast<const float4*>(psi_addr(P.psih, 0, s, X, i, jrow, kq, P.ny, P.nzp)), px[s]);
    if (ysl)
      for (int s = 0; s < 2; ++s)
        unpack4(*reinterpret_cast<const float4*>(psi_addr(P.psih, 1, s, Y, i, jrow, kq, P.ny, P.nzp)), py[s]);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float dzy = fdiff(yez[e], mj, ez[e], idy);
      const float dzx = fdiff(nez[e], mi, ez[e], idx_);
      const float dyx = fdiff(ney[e], mi, ey[e], idx_);
      const float dxy = fdiff(yex[e], mj, ex[e], idy);
      float sy0 = dzy, sy1 = dxy, sx0 = dzx, sx1 = dyx;
      if (ysl) {
        sy0 = cpml_stretch(dzy, py[0][e], ay, by, ky);
        sy1 = cpml_stretch(dxy, py[1][e], ay, by, ky);
      }
      if (xsl) {
        sx0 = cpml_stretch(dzx, px[0][e], ax_, bx_, kx_);
        sx1 = cpml_stretch(dyx, px[1][e], ax_, bx_, kx_);
      }
      const bool kv = (kvm >> e) & 1u;
      hx[e] = kv ? h_new(hx[e], ch, sy0, dyz[e]) : hx[e];
      hy[e] = kv ? h_new(hy[e], ch, dxz[e], sx0) : hy[e];
      hz[e] = kv ? h_new(hz[e], ch, sx1, sy1) : hz[e];
    }
    if (commit && xsl)
      for (int s = 0; s < 2; ++s)
        *reinterpret_cast<float4*>(psi_addr(out.psih, 0, s, X, i, jrow, kq, P.ny, P.nzp)) =
            make_float4(px[s][0], px[s][1], px[s][2], px[s][3]);
    if (commit && ysl)
      for (int s = 0; s < 2; ++s)
        *reinterpret_cast<float4*>(psi_addr(out.psih, 1, s, Y, i, jrow, kq, P.ny, P.nzp)) =
            make_float4(py[s][0], py[s][1], py[s][2], py[s][3]);
  }
  if (commit) {
    *reinterpret_cast<float4*>(out.f[3] + row + kq) = make_float4(hx[0], hx[1], hx[2], hx[3]);
    *reinterpret_cast<float4*>(out.f[4] + row + kq) = make_float4(hy[0], hy[1], hy[2], hy[3]);
    *reinterpret_cast<float4*>(out.f[5] + row + kq) = make_float4(hz[0], hz[1], hz[2], hz[3]);
  }
}

// Hx, Hy of H^{n+1/2} at (i, j, k) from global memory of the current bank (the halo cell before
// a tile's z range); the same operations as the tile path.
__device__ __forceinline__ void fused_h_cell(const YeeParams& P, int i, int j, int k, float* hxo,
                                             float* hyo) {
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const int64_t id = i * si + (int64_t)j * sj + k;
  const int jp = Y.nxt[j], kp = Z.nxt[k], ip = X.nxt[i];
  const float ex = P.f[0][id], ey = P.f[1][id], ez = P.f[2][id];
  const float dzy0 = fdiff(P.f[2][i * si + (int64_t)jp * sj + k], Y.mnx[j], ez, Y.idl_p[j]);
  float dyz = fdiff(P.f[1][i * si + (int64_t)j * sj + kp], Z.mnx[k], ey, Z.idl_p[k]);
  float dxz = fdiff(P.f[0][i * si + (int64_t)j * sj + kp], Z.mnx[k], ex, Z.idl_p[k]);
  const float dzx0 = fdiff(P.f[2][ip * si + (int64_t)j * sj + k], X.mnx[i], ez, X.idl_p[i]);
  float sy0 = dzy0, sx0 = dzx0;
  if (in_slab(Y, j)) {
    float ps = *psi_addr(P.psih, 1, 0, Y, i, j, k, P.ny, P.nzp);
    sy0 = cpml_stretch(dzy0, ps, Y.ah[j], Y.bh[j], Y.kh[j]);
  }
  if (in_slab(Z, k)) {
    float p0 = *psi_addr(P.psih, 2, 0, Z, i, j, k, P.ny, P.nzp);
    float p1 = *psi_addr(P.psih, 2, 1, Z, i, j, k, P.ny, P.nzp);
    dyz = cpml_stretch(dyz, p0, Z.ah[k], Z.bh[k], Z.kh[k]);
    dxz = cpml_stretch(dxz, p1, Z.ah[k], Z.bh[k], Z.kh[k]);
  }
  if (in_slab(X, i)) {
    float ps = *psi_addr(P.psih, 0, 0, X, i, j, k, P.ny, P.nzp);
    sx0 = cpml_stretch(dzx0, ps, X.ah[i], X.bh[i], X.kh[i]);
  }
  *hxo = h_new(P.f[3][id], P.ch, sy0, dyz);
  *hyo = h_new(P.f[4][id], P.ch, dxz, sx0);
}

__global__ void __launch_bounds__(192, 2) k_he_ws(const __grid_constant__ FusedMaps maps,
                                                  YeeParams P, FieldOut out, int xch,
                                                  int n_mats, int* err) {
  extern __shared__ __align__(128) float smem[];
  float* hn = smem + kFS * kFStage;
  float* zth = hn + kF_HN;
  float* zte = zth + kZTab;
  float* hring = zte + kZTab;
  MatRec* smats = reinterpret_cast<MatRec*>(hring + kF_HR);
  uint64_t* full = reinterpret_cast<uint64_t*>(smats + kSmemMats);
  uint64_t* empty = full + kFS;
  const int lane = threadIdx.x, w = threadIdx.y;
  const int tid = w * 32 + lane;
  const int k0 = blockIdx.x * kTZ;
  const int j0 = blockIdx.y * kTY;
  const int ib = blockIdx.z * xch;
  const int ie = min(ib + xch, P.nx);
  const int np = ie - ib;
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const int pp = X.prv[ib];
  const bool pre = pp != ib;  // the E update of plane ib needs H^{n+1/2} of another plane
  const int nst = np + (pre ? 1 : 0);
  const bool wide = P.mat32 != nullptr;
  const MatRec* mats = P.mats;
  if (n_mats <= kSmemMats) {
    const uint4* src = reinterpret_cast<const uint4*>(P.mats);
    uint4* dst = reinterpret_cast<uint4*>(smats);
    for (int q = tid; q < n_mats * 4; q += 192) dst[q] = src[q];
    mats = smats;
  }
  load_ztab(zth, Z, true, k0, P.nzp, tid, 192);
  load_ztab(zte, Z, false, k0, P.nzp, tid, 192);
  if (w == 5 && lane == 0) {
    for (int s = 0; s < kFS; ++s) {
      // lane 0's arrival with the transaction bytes, and one per producer lane after its
      // halo-ring writes
      mbar_init(&full[s], 1 + 32);
      mbar_init(&empty[s], kTY + 1);
    }
    mbar_fence_init();
  }
  __syncthreads();

  if (w == 5) {  // ------------------------------------------------------------ producer
    // lane 0 issues the stage's copies; at every kF_HB-th main plane the 32 lanes compute the
    // halo cells (row j0 + lane % 4, k0 - 1) of the next kF_HB main planes (plane lane / 4) from
    // global memory at once, so their dependent loads overlap instead of serialising per plane
    int issued = 0;
    bool ok = true;
    const uint32_t mbytes = (uint32_t)(kTY * kTZ * (wide ? 4 : 2));
    for (int q = 0; q < nst && ok; ++q) {
      const int slot = q % kFS;
      if (q >= kFS) ok = mbar_wait_live(&empty[slot], (uint32_t)((q / kFS - 1) & 1), err, kPolls);
      if (!__all_sync(kFull, ok)) break;
      float* st = smem + slot * kFStage;
      const bool main = !(pre && q == 0);
      const int i = main ? ib + q - (pre ? 1 : 0) : pp;
      if (lane == 0) {
        const int inext = X.nxt[i];
        mbar_expect_tx(&full[slot], 3 * kF_EBBytes + 5 * kF_T5Bytes + mbytes);
        for (int c = 0; c < 3; ++c) {
          tma3(st + kF_EB + c * kF_EBS, &maps.e6[c], &full[slot], k0, j0 - 1, i);
          tma3(st + kF_HO + c * kF_T5, &maps.h5[c], &full[slot], k0, j0 - 1, i);
        }
        tma3(st + kF_EN, &maps.e5[0], &full[slot], k0, j0 - 1, inext);
        tma3(st + kF_EN + kF_T5, &maps.e5[1], &full[slot], k0, j0 - 1, inext);
        tma3(st + kF_MT, &maps.m, &full[slot], k0, j0, i);
      }
      const int qm = q - (pre ? 1 : 0);  // main plane index
      if (main && k0 > 0 && qm % kF_HB == 0) {
        const int pm = qm + lane / kTY, r = lane % kTY;
        if (pm < np && j0 + r < P.ny) {
          float a, b;
          fused_h_cell(P, ib + pm, j0 + r, k0 - 1, &a, &b);
          float* hr = hring + (pm % kF_HRP) * 2 * kTY;
          hr[r] = a;
          hr[kTY + r] = b;
        }
      }
      mbar_arrive(&full[slot]);
      issued = q + 1;
    }
    if (lane == 0)
      for (int q = max(0, issued - kFS); q < issued; ++q)  // drain (no-op when consumed)
        mbar_wait(&full[q % kFS], (uint32_t)((q / kFS) & 1), err);
    return;
  }

  // ------------------------------------------------------------------- consumers (warps 0-4)
  // warps 0..3 own rows j0 + w (box row w + 1); warp 4 is the row below (box row 0) and the
  // cell before k0. Every consumer passes every named barrier, also after a failed wait.
  const bool owner = w < kTY;
  const int hr = owner ? w + 1 : 0;
  const int jrow = j0 - 1 + hr;
  const bool row_ok = jrow >= 0 && jrow < P.ny;
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const float cw = P.cw;
  const unsigned lt = (1u << lane) - 1u;
  bool alive = true;
  for (int t = 0; t < nst; ++t) {
    const int slot = t % kFS;
    if (alive) alive = mbar_wait_live(&full[slot], (uint32_t)((t / kFS) & 1), err, kPolls);
    alive = __all_sync(kFull, alive);
    const float* st = smem + slot * kFStage;
    const bool main = !(pre && t == 0);
    const int i = main ? (ib + t - (pre ? 1 : 0)) : pp;
    const int par = t & 1;
    // ---- H^{n+1/2}(i): owners on their rows (committed on main planes), warp 4 below them
    if (alive && row_ok && (owner || main)) {
      float hx[4], hy[4], hz[4];
      fused_h_quad(P, out, st, zth, i, jrow, hr, k0, lane, owner && main, hx, hy, hz);
      *reinterpret_cast<float4*>(hn_row(hn, par, 0, hr) + 4 * lane) = make_float4(hx[0], hx[1], hx[2], hx[3]);
      *reinterpret_cast<float4*>(hn_row(hn, par, 1, hr) + 4 * lane) = make_float4(hy[0], hy[1], hy[2], hy[3]);
      *reinterpret_cast<float4*>(hn_row(hn, par, 2, hr) + 4 * lane) = make_float4(hz[0], hz[1], hz[2], hz[3]);
    }
    __syncwarp();
    if (!owner && lane == 0) mbar_arrive(&empty[slot]);
    asm volatile("bar.sync 1, 160;" ::: "memory");
    // ---- E^{n+1}(i) on the owned rows
    if (owner) {
      if (alive && main && row_ok) {
        const int j = jrow;
        const int jm = Y.prv[j];
        const float mj = Y.mpv[j], idy = Y.idl_d[j];
        const bool ysl = in_slab(Y, j);
        const int hrm = (jm == j) ? hr : hr - 1;
        const int xpar = (X.prv[i] == i) ? par : (par ^ 1);
        const int kq = k0 + 4 * lane;
        unsigned kvm = 0, zslm = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = kq + e;
          const bool kv = k < P.nz;
          kvm |= (unsigned)kv << e;
          zslm |= (unsigned)(kv && in_slab(Z, k)) << e;
        }
        const int to = w * kTZ + 4 * lane;
        uint32_t mid[4] = {0u, 0u, 0u, 0u};
        if (wide) {
          const uint4 m = *reinterpret_cast<const uint4*>(reinterpret_cast<const uint32_t*>(st + kF_MT) + to);
          mid[0] = m.x; mid[1] = m.y; mid[2] = m.z; mid[3] = m.w;
        } else {
          const uint2 m = *reinterpret_cast<const uint2*>(reinterpret_cast<const uint16_t*>(st + kF_MT) + to);
          mid[0] = m.x & 0xffffu; mid[1] = m.x >> 16; mid[2] = m.y & 0xffffu; mid[3] = m.y >> 16;
        }
        int lane_np = 0;
        if (P.has_ade) {
#pragma unroll
          for (int e = 0; e < 4; ++e) lane_np += mats[mid[e]].reserved;
        }
        uint32_t gp = 0;
        if (P.has_ade && __any_sync(kFull, lane_np > 0)) {
          int pre_n = 0;
#pragma unroll
          for (int bb = 0; bb < 8; ++bb)
            pre_n += __popc(__ballot_sync(kFull, (lane_np >> bb) & 1) & lt) << bb;
          gp = P.seg_ofs[(((int64_t)i * P.ny + j) * P.nzp + k0) >> 5] + (uint32_t)pre_n;
        }
        const bool xsl = in_slab(X, i);
        const float mi = X.mpv[i], idx_ = X.idl_d[i];
        const int64_t row = i * si + (int64_t)j * sj;
        const int ro = hr * kBZ + 4 * lane;
        if (kvm) {
        float ex[4], ey[4], ez[4], hx[4], hy[4], hz[4], yhx[4], yhz[4], phy[4], phz[4];
        float idz[4], mkz[4];
        unpack4(lds4(st + kF_EB + ro), ex);
        unpack4(lds4(st + kF_EB + kF_EBS + ro), ey);
        unpack4(lds4(st + kF_EB + 2 * kF_EBS + ro), ez);
        unpack4(lds4(hn_row(hn, par, 0, hr) + 4 * lane), hx);
        unpack4(lds4(hn_row(hn, par, 1, hr) + 4 * lane), hy);
        unpack4(lds4(hn_row(hn, par, 2, hr) + 4 * lane), hz);
        unpack4(lds4(hn_row(hn, par, 0, hrm) + 4 * lane), yhx);
        unpack4(lds4(hn_row(hn, par, 2, hrm) + 4 * lane), yhz);
        unpack4(lds4(hn_row(hn, xpar, 1, hr) + 4 * lane), phy);
        unpack4(lds4(hn_row(hn, xpar, 2, hr) + 4 * lane), phz);
        unpack4(lds4(zte + 4 * lane), idz);
        unpack4(lds4(zte + kTZ + 4 * lane), mkz);
        float hxm, hym;
        if (lane > 0) {
          hxm = hn_row(hn, par, 0, hr)[4 * lane - 1];
          hym = hn_row(hn, par, 1, hr)[4 * lane - 1];
        } else if (k0 > 0) {
          const float* hr = hring + ((t - (pre ? 1 : 0)) % kF_HRP) * 2 * kTY;
          hxm = hr[w];
          hym = hr[kTY + w];
        } else {  // k = 0: the clamped neighbour is the cell itself
          hxm = hx[0];
          hym = hy[0];
        }
        float dyz[4], dxz[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float zhx = (e > 0) ? hx[e - 1] : hxm;
          const float zhy = (e > 0) ? hy[e - 1] : hym;
          dyz[e] = bdiff(hy[e], zhy, mkz[e], idz[e]);
          dxz[e] = bdiff(hx[e], zhx, mkz[e], idz[e]);
        }
        if (zslm) zcpml_io(dyz, dxz, zslm, zte, P.psie, P.psie, true, P, i, j, kq, lane);
        float sy0[4], sy1[4], sx0[4], sx1[4];
        const bool yplain = !ysl && jm == j - 1 && mj == 1.0f;
        if (yplain && !xsl && i > 0 && X.prv[i] == i - 1 && mi == 1.0f) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            sy0[e] = __fmul_rn(__fsub_rn(hz[e], yhz[e]), idy);
            sx0[e] = __fmul_rn(__fsub_rn(hz[e], phz[e]), idx_);
            sx1[e] = __fmul_rn(__fsub_rn(hy[e], phy[e]), idx_);
            sy1[e] = __fmul_rn(__fsub_rn(hx[e], yhx[e]), idy);
          }
        } else {
          const float ay = Y.ae[j], by = Y.be[j], ky = Y.ke[j];
          const float ax_ = X.ae[i], bx_ = X.be[i], kx_ = X.ke[i];
          float px[2][4], py[2][4];
          if (xsl)
            for (int s = 0; s < 2; ++s)
              unpack4(*reinterpret_cast<const float4*>(psi_addr(P.psie, 0, s, X, i, j, kq, P.ny, P.nzp)), px[s]);
          if (ysl)
            for (int s = 0; s < 2; ++s)
              unpack4(*reinterpret_cast<const float4*>(psi_addr(P.psie, 1, s, Y, i, j, kq, P.ny, P.nzp)), py[s]);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            sy0[e] = bdiff(hz[e], yhz[e], mj, idy);
            sx0[e] = bdiff(hz[e], phz[e], mi, idx_);
            sx1[e] = bdiff(hy[e], phy[e], mi, idx_);
            sy1[e] = bdiff(hx[e], yhx[e], mj, idy);
            if (ysl) {
              sy0[e] = cpml_stretch(sy0[e], py[0][e], ay, by, ky);
              sy1[e] = cpml_stretch(sy1[e], py[1][e], ay, by, ky);
            }
            if (xsl) {
              sx0[e] = cpml_stretch(sx0[e], px[0][e], ax_, bx_, kx_);
              sx1[e] = cpml_stretch(sx1[e], px[1][e], ax_, bx_, kx_);
            }
          }
          if (xsl)
            for (int s = 0; s < 2; ++s)
              *reinterpret_cast<float4*>(psi_addr(P.psie, 0, s, X, i, j, kq, P.ny, P.nzp)) =
                  make_float4(px[s][0], px[s][1], px[s][2], px[s][3]);
          if (ysl)
            for (int s = 0; s < 2; ++s)
              *reinterpret_cast<float4*>(psi_addr(P.psie, 1, s, Y, i, j, kq, P.ny, P.nzp)) =
                  make_float4(py[s][0], py[s][1], py[s][2], py[s][3]);
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const MatRec& M = mats[mid[e]];
          const float4 cab = *reinterpret_cast<const float4*>(&M.ca[0]);
          const float2 cb12 = *reinterpret_cast<const float2*>(&M.cb[1]);
          float wv[3] = {0.f, 0.f, 0.f};
          if (lane_np > 0 && M.reserved > 0) {
            cell_currents(M, nullptr, -1, P.J, gp, wv);
            gp += (uint32_t)M.reserved;
          }
          const bool kv = (kvm >> e) & 1u;
          const float nex = e_new(cab.x, ex[e], cab.w, sy0[e], dyz[e], cw, wv[0]);
          const float ney = e_new(cab.y, ey[e], cb12.x, dxz[e], sx0[e], cw, wv[1]);
          const float nez = e_new(cab.z, ez[e], cb12.y, sx1[e], sy1[e], cw, wv[2]);
          ex[e] = kv ? nex : ex[e];
          ey[e] = kv ? ney : ey[e];
          ez[e] = kv ? nez : ez[e];
        }
        *reinterpret_cast<float4*>(out.f[0] + row + kq) = make_float4(ex[0], ex[1], ex[2], ex[3]);
        *reinterpret_cast<float4*>(out.f[1] + row + kq) = make_float4(ey[0], ey[1], ey[2], ey[3]);
        *reinterpret_cast<float4*>(out.f[2] + row + kq) = make_float4(ez[0], ez[1], ez[2], ez[3]);
        }  // kvm
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[slot]);
    }
  }
}

}  // namespace

size_t ws_h_smem() { return (size_t)kS * kHStage * 4 + 2 * kS * sizeof(uint64_t) + kZTab * 4; }
size_t ws_e_smem() {
  return (size_t)kS * kEStage * 4 + (2 * kS + 1) * sizeof(uint64_t) + kZTab * 4 +
         kSmemMats * sizeof(MatRec) + kXMax * kTY * 2 * sizeof(uint32_t) +
         kMaxSnapBoxes * sizeof(float*);
}

int ws_max_xchunk() { return kXMax; }

size_t he_smem() {
  return (size_t)kFS * kFStage * 4 + (size_t)(kF_HN + 2 * kZTab + kF_HR) * 4 +
         kSmemMats * sizeof(MatRec) + 2 * kFS * sizeof(uint64_t);
}

// x planes per block. A block streams its planes one after another (about 2 us each) after
// filling its ring (about six planes' worth), so a grid too small to fill the resident block
// slots even at 8-plane chunks gets as many chunks as there are slots (down to 2 planes per
// block: every block runs at once and the step lasts one short chunk). Larger grids take the
// chunk length whose block count fills the last wave best, less a cost for short chunks.
int ws_xchunk(const YeeParams& P) {
  const int64_t tiles = (int64_t)((P.nzp + kTZ - 1) / kTZ) * ((P.ny + kTY - 1) / kTY);
  const double slots = 148.0 * OEM_WS_MINBLOCKS;
  const int hi = std::min(kXMax, P.nx);
  if ((double)(tiles * ((P.nx + 7) / 8)) <= slots) {
    const int64_t chunks = std::max<int64_t>(1, (int64_t)slots / tiles);
    const int xch = (int)((P.nx + chunks - 1) / chunks);
    return std::min(hi, std::max(std::min(2, hi), xch));
  }
  int best = hi;
  double best_score = -1e30;
  for (int xch = std::min(8, hi); xch <= hi; ++xch) {
    const int64_t chunks = (P.nx + xch - 1) / xch;
    const double waves = (double)(tiles * chunks) / slots;
    const double fill = waves / std::ceil(waves);
    const double score = fill - 2.0 / xch;
    if (score > best_score + 1e-12) {
      best_score = score;
      best = xch;
    }
  }
  return best;
}

// Several blocks of each kernel share an SM; the largest shared-memory carveout makes room.
cudaError_t ws_setup_kernels() {
  cudaError_t e = cudaFuncSetAttribute(k_h_ws, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ws_h_smem());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_h_ws, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
  for (auto* k : {k_e_ws<false, false>, k_e_ws<true, false>, k_e_ws<false, true>,
                  k_e_ws<true, true>}) {
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ws_e_smem());
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxShared);
  }
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_he_ws, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)he_smem());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_he_ws, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
  return e;
}

cudaError_t launch_update_h_ws(const TmaMaps& maps, const YeeParams& P, int xch, int* err,
                               cudaStream_t s) {
  dim3 b(32, kTY + 1, 1), g((P.nzp + kTZ - 1) / kTZ, (P.ny + kTY - 1) / kTY, (P.nx + xch - 1) / xch);
  k_h_ws<<<g, b, ws_h_smem(), s>>>(maps, P, xch, err);
  return cudaGetLastError();
}

cudaError_t launch_update_e_ws(const TmaMaps& maps, const YeeParams& P, int xch, int n_mats,
                               int* err, cudaStream_t s, const SnapBoxes* sb) {
  dim3 b(32, kTY + 1, 1), g((P.nzp + kTZ - 1) / kTZ, (P.ny + kTY - 1) / kTY, (P.nx + xch - 1) / xch);
  if (sb && sb->n > 0)
    (n_mats <= kSmemMats ? k_e_ws<true, true> : k_e_ws<true, false>)<<<g, b, ws_e_smem(), s>>>(
        maps, P, xch, n_mats, err, *sb);
  else
    (n_mats <= kSmemMats ? k_e_ws<false, true> : k_e_ws<false, false>)<<<g, b, ws_e_smem(), s>>>(
        maps, P, xch, n_mats, err, SnapBoxes{});
  return cudaGetLastError();
}

cudaError_t launch_update_he_fused(const FusedMaps& maps, const YeeParams& P, const FieldOut& out,
                                   int xch, int n_mats, int* err, cudaStream_t s) {
  dim3 b(32, kTY + 2, 1), g((P.nzp + kTZ - 1) / kTZ, (P.ny + kTY - 1) / kTY, (P.nx + xch - 1) / xch);
  k_he_ws<<<g, b, he_smem(), s>>>(maps, P, out, xch, n_mats, err);
  return cudaGetLastError();
}

}  // namespace oem
