// TMA-pipelined Yee kernels for sm_100a (the default step kernels).
//
// Block tile: 128 z cells x 4 y rows (one warp per row, four z cells per lane), streaming along
// x over a chunk of planes. Each plane's field tiles are brought into a 4-stage shared-memory
// ring by cp.async.bulk.tensor (issued by one thread, completion tracked by an mbarrier per
// stage), so three planes are in flight per block while one is computed; the x neighbour is
// the adjacent stage, the y and z neighbours are the halo row / columns of the loaded box.
// Every field value is read from HBM once per kernel (halo rows and columns are L2 hits).
// Boundary cells whose neighbour is not the adjacent index (periodic wrap, PMC, symmetry
// walls) read that neighbour directly from global memory, per the axis tables.
//
// Every mbarrier wait is bounded: after ~2^20 polls the kernel records an error in *err,
// drains its outstanding copies (again bounded) and returns, and the host reports
// OEM_ERR_TIMEOUT instead of hanging the device.
//
// The arithmetic per cell is that of the basic kernels (openem/kernels/yee.cu:60-240,
// dispersion.cu:168-207).
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "oem_internal.cuh"
#include "oem_arith.cuh"

namespace oem {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kTY = 4;        // owned rows per block
constexpr int kTZ = 128;      // owned z cells per block
constexpr int kBZ = 136;      // z extent of the halo boxes (16-byte aligned start)
constexpr int kS = 4;         // pipeline stages
constexpr int kSmemMats = 128;  // material records staged in shared memory when n <= this

// Every TMA destination starts on a 128-byte boundary: the (kTY+1) x kBZ halo box (2720 B) is
// given a 704-float (2816 B) slot.
constexpr int kBoxW = (((kTY + 1) * kBZ + 31) / 32) * 32;   // floats per halo-box slot
constexpr uint32_t kWideBytes = (kTY + 1) * kBZ * 4;         // bytes a halo box transfers
constexpr uint32_t kTileBytes = kTY * kTZ * 4;               // bytes a field tile transfers
// H kernel stage: E halo boxes (rows j0.., cols k0..) then H tiles.
constexpr int kHE = 3 * kBoxW;
constexpr int kHH = 3 * kTY * kTZ;
constexpr int kHStage = kHE + kHH;  // floats
// E kernel stage: H halo boxes (rows j0-1.., cols k0-4..), E tiles, material tile.
constexpr int kEH = 3 * kBoxW;
constexpr int kEE = 3 * kTY * kTZ;
constexpr int kEM = kTY * kTZ;      // material indices, up to 4 bytes each
constexpr int kEStage = kEH + kEE + kEM;  // 32-bit words
static_assert((kHStage * 4) % 128 == 0 && (kEStage * 4) % 128 == 0, "stage alignment");
static_assert((kBoxW * 4) % 128 == 0 && (kTY * kTZ * 4) % 128 == 0, "slot alignment");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; false (and *err set) if the phase did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  for (uint32_t it = 0; it < (1u << 20); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  atomicExch(err, 1);
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ float* psi_slab(const PsiSet& S, int a, int slot, const DevAxis& A,
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

__device__ __forceinline__ float stretch_slab(float d, float* psi, float a, float b, float ik) {
  const float p = b * (*psi) + a * d;
  *psi = p;
  return ik * d + p;
}

// psi of one quad (four consecutive z cells) of an x- or y-slab array, held in registers
// between one 128-bit load and one 128-bit store.
struct Psi4 {
  float* ptr = nullptr;
  float v[4] = {0.f, 0.f, 0.f, 0.f};
  __device__ __forceinline__ void load(float* p) {
    ptr = p;
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  }
  __device__ __forceinline__ void store() const {
    if (ptr) *reinterpret_cast<float4*>(ptr) = make_float4(v[0], v[1], v[2], v[3]);
  }
};

__device__ __forceinline__ float stretch_reg(float d, float& psi, float a, float b, float ik) {
  const float p = b * psi + a * d;
  psi = p;
  return ik * d + p;
}

__device__ __forceinline__ bool in_slab(const DevAxis& A, int q) {
  return q < A.lo || q >= A.n - A.hi;
}

__device__ __forceinline__ float4 lds4(const float* p) {
  return *reinterpret_cast<const float4*>(p);
}

__device__ __forceinline__ float comp4(const float4& v, int e) {
  return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

// ---------------------------------------------------------------------------------------------
// H half step
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_h_tma(const __grid_constant__ TmaMaps maps, YeeParams P,
                                               int xch, int* err) {
  extern __shared__ __align__(128) float smem[];
  float* st = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kS * kHStage);
  const int lane = threadIdx.x, w = threadIdx.y;
  const int tid = w * 32 + lane;
  const int k0 = blockIdx.x * kTZ;
  const int j0 = blockIdx.y * kTY;
  const int ib = blockIdx.z * xch;
  const int ie = min(ib + xch, P.nx);
  const int nseq = ie - ib + 1;  // planes ib..ie; the last one is only the x neighbour
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  if (tid == 0) {
    for (int s = 0; s < kS; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int issued = 0;     // sequences issued (thread 0)
  int confirmed = 0;  // sequences whose copies this thread has seen complete
  auto issue = [&](int q) {
    issued = q + 1;
    float* base = st + (q % kS) * kHStage;
    uint64_t* bar = &bars[q % kS];
    int p = ib + q;
    if (p >= P.nx) p = X.nxt[P.nx - 1];
    const bool need_h = q < nseq - 1;
    mbar_expect_tx(bar, 3 * kWideBytes + (need_h ? 3 * kTileBytes : 0u));
    for (int c = 0; c < 3; ++c) tma_load_3d(base + c * kBoxW, &maps.e_wide[c], bar, k0, j0, p);
    if (need_h)
      for (int c = 0; c < 3; ++c) tma_load_3d(base + kHE + c * kTY * kTZ, &maps.h_tile[c], bar, k0, j0, p);
  };
  if (tid == 0)
    for (int q = 0; q < kS && q < nseq; ++q) issue(q);

  const int j = j0 + w;
  const bool row_ok = j < P.ny;
  const int jj = row_ok ? j : 0;
  const int jp = Y.nxt[jj];
  const float mj = Y.mnx[jj], idy = Y.idl_p[jj];
  const float ay = Y.ah[jj], by = Y.bh[jj], ky = Y.kh[jj];
  const bool ysl = row_ok && in_slab(Y, j);
  const bool yspecial = row_ok && jp != j + 1;
  const int kq = k0 + 4 * lane;
  bool kv[4], zsl[4], zspecial[4];
  int kpz[4];
  float idz[4], mkz[4], az[4], bz[4], kz[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = kq + e;
    kv[e] = row_ok && k < P.nz;
    const int kk = k < P.nzp ? k : 0;
    kpz[e] = Z.nxt[kk];
    mkz[e] = Z.mnx[kk];
    idz[e] = Z.idl_p[kk];
    az[e] = Z.ah[kk]; bz[e] = Z.bh[kk]; kz[e] = Z.kh[kk];
    zsl[e] = kv[e] && in_slab(Z, k);
    zspecial[e] = kv[e] && kpz[e] != k + 1;
  }
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const float ch = P.ch;
  bool ok = true;
  for (int t = 0; t < nseq - 1; ++t) {
    const int i = ib + t;
    if (ok) ok = mbar_wait(&bars[t % kS], (uint32_t)((t / kS) & 1), err);
    if (ok) ok = mbar_wait(&bars[(t + 1) % kS], (uint32_t)(((t + 1) / kS) & 1), err);
    if (ok) confirmed = t + 2;
    if (ok && kv[0] | kv[1] | kv[2] | kv[3]) {
      const float* cur = st + (t % kS) * kHStage;
      const float* nxt = st + ((t + 1) % kS) * kHStage;
      const float mi = X.mnx[i], idx_ = X.idl_p[i];
      const float ax_ = X.ah[i], bx_ = X.bh[i], kx_ = X.kh[i];
      const bool xsl = in_slab(X, i);
      const int64_t row = i * si + (int64_t)j * sj;
      const int ro = w * kBZ + 4 * lane;          // own row in the E box
      const float4 ex = lds4(cur + 0 * kBoxW + ro);
      const float4 ey = lds4(cur + 1 * kBoxW + ro);
      const float4 ez = lds4(cur + 2 * kBoxW + ro);
      const float ex4 = cur[0 * kBoxW + ro + 4];
      const float ey4 = cur[1 * kBoxW + ro + 4];
      float4 yex = lds4(cur + 0 * kBoxW + ro + kBZ);
      float4 yez = lds4(cur + 2 * kBoxW + ro + kBZ);
      if (yspecial) {
        const int64_t oy = i * si + (int64_t)jp * sj + kq;
        yex = *reinterpret_cast<const float4*>(P.f[0] + oy);
        yez = *reinterpret_cast<const float4*>(P.f[2] + oy);
      }
      const float4 nex = lds4(nxt + 0 * kBoxW + ro);
      const float4 ney = lds4(nxt + 1 * kBoxW + ro);
      const float4 nez = lds4(nxt + 2 * kBoxW + ro);
      (void)nex;
      const int ho = w * kTZ + 4 * lane;
      float4 h4[3];
      h4[0] = lds4(cur + kHE + 0 * kTY * kTZ + ho);
      h4[1] = lds4(cur + kHE + 1 * kTY * kTZ + ho);
      h4[2] = lds4(cur + kHE + 2 * kTY * kTZ + ho);
      float hx[4] = {h4[0].x, h4[0].y, h4[0].z, h4[0].w};
      float hy[4] = {h4[1].x, h4[1].y, h4[1].z, h4[1].w};
      float hz[4] = {h4[2].x, h4[2].y, h4[2].z, h4[2].w};
      Psi4 px0, px1, py0, py1;  // x-slab Hy, Hz; y-slab Hx, Hz
      if (xsl) {
        px0.load(psi_slab(P.psih, 0, 0, X, i, j, kq, P.ny, P.nzp));
        px1.load(psi_slab(P.psih, 0, 1, X, i, j, kq, P.ny, P.nzp));
      }
      if (ysl) {
        py0.load(psi_slab(P.psih, 1, 0, Y, i, j, kq, P.ny, P.nzp));
        py1.load(psi_slab(P.psih, 1, 1, Y, i, j, kq, P.ny, P.nzp));
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (!kv[e]) continue;
        const int k = kq + e;
        const float exe = comp4(ex, e), eye = comp4(ey, e), eze = comp4(ez, e);
        float zex = (e < 3) ? comp4(ex, e + 1) : ex4;
        float zey = (e < 3) ? comp4(ey, e + 1) : ey4;
        if (zspecial[e]) {
          zex = P.f[0][row + kpz[e]];
          zey = P.f[1][row + kpz[e]];
        }
        {  // Hx: -(dEz/dy - dEy/dz)
          const float dzy = (comp4(yez, e) * mj - eze) * idy;
          const float dyz = (zey * mkz[e] - eye) * idz[e];
          const float sy = ysl ? stretch_reg(dzy, py0.v[e], ay, by, ky) : dzy;
          const float sz = zsl[e] ? stretch_slab(dyz, psi_slab(P.psih, 2, 0, Z, i, j, k, P.ny, P.nzp), az[e], bz[e], kz[e]) : dyz;
          hx[e] -= ch * (sy - sz);
        }
        {  // Hy: -(dEx/dz - dEz/dx)
          const float dxz = (zex * mkz[e] - exe) * idz[e];
          const float dzx = (comp4(nez, e) * mi - eze) * idx_;
          const float sz = zsl[e] ? stretch_slab(dxz, psi_slab(P.psih, 2, 1, Z, i, j, k, P.ny, P.nzp), az[e], bz[e], kz[e]) : dxz;
          const float sx = xsl ? stretch_reg(dzx, px0.v[e], ax_, bx_, kx_) : dzx;
          hy[e] -= ch * (sz - sx);
        }
        {  // Hz: -(dEy/dx - dEx/dy)
          const float dyx = (comp4(ney, e) * mi - eye) * idx_;
          const float dxy = (comp4(yex, e) * mj - exe) * idy;
          const float sx = xsl ? stretch_reg(dyx, px1.v[e], ax_, bx_, kx_) : dyx;
          const float sy = ysl ? stretch_reg(dxy, py1.v[e], ay, by, ky) : dxy;
          hz[e] -= ch * (sx - sy);
        }
      }
      px0.store(); px1.store(); py0.store(); py1.store();
      *reinterpret_cast<float4*>(P.f[3] + row + kq) = make_float4(hx[0], hx[1], hx[2], hx[3]);
      *reinterpret_cast<float4*>(P.f[4] + row + kq) = make_float4(hy[0], hy[1], hy[2], hy[3]);
      *reinterpret_cast<float4*>(P.f[5] + row + kq) = make_float4(hz[0], hz[1], hz[2], hz[3]);
    }
    __syncthreads();
    if (tid == 0 && ok && t + kS < nseq) issue(t + kS);
  }
  if (!ok && tid == 0) {
    // drain: wait (bounded) for the copies still in flight so none lands after exit
    for (int q = confirmed; q < issued; ++q) {
      mbar_wait(&bars[q % kS], (uint32_t)((q / kS) & 1), err);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// E full step with the deferred ADE
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float ade_cell(const YeeParams& P, int set, int np, uint32_t poff,
                                          float en) {
  float w = 0.0f;
  const float4* cf = P.pcoef + P.pset_ofs[set];
  for (int t = 0; t < np; ++t) {
    const float4 c = __ldg(cf + t);
    float2 st = P.P[poff + t];
    w = __fadd_rn(w, ade_pole(st, c, en));
    P.P[poff + t] = st;
  }
  return w;
}

__global__ void __launch_bounds__(128) k_e_tma(const __grid_constant__ TmaMaps maps, YeeParams P,
                                               int xch, int n_mats, int* err) {
  extern __shared__ __align__(128) float smem[];
  float* st = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kS * kEStage);
  MatRec* smats = reinterpret_cast<MatRec*>(bars + kS);
  const int lane = threadIdx.x, w = threadIdx.y;
  const int tid = w * 32 + lane;
  const int k0 = blockIdx.x * kTZ;
  const int j0 = blockIdx.y * kTY;
  const int ib = blockIdx.z * xch;
  const int ie = min(ib + xch, P.nx);
  const int nseq = ie - ib + 1;  // planes ib-1..ie-1; the first one only provides H
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const bool wide = P.mat32 != nullptr;
  const MatRec* mats = P.mats;
  if (n_mats <= kSmemMats) {
    const uint4* src = reinterpret_cast<const uint4*>(P.mats);
    uint4* dst = reinterpret_cast<uint4*>(smats);
    for (int q = tid; q < n_mats * 4; q += 128) dst[q] = src[q];
    mats = smats;
  }
  if (tid == 0) {
    for (int s = 0; s < kS; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int issued = 0;
  int confirmed = 0;
  auto issue = [&](int q) {
    issued = q + 1;
    float* base = st + (q % kS) * kEStage;
    uint64_t* bar = &bars[q % kS];
    int p = ib - 1 + q;
    if (p < 0) p = X.prv[0];
    const bool full = q > 0;
    const uint32_t mbytes = (uint32_t)(kEM * (wide ? 4 : 2));
    mbar_expect_tx(bar, 3 * kWideBytes + (full ? 3 * kTileBytes + mbytes : 0u));
    for (int c = 0; c < 3; ++c)
      tma_load_3d(base + c * kBoxW, &maps.h_wide[c], bar, k0 - 4, j0 - 1, p);
    if (full) {
      for (int c = 0; c < 3; ++c) tma_load_3d(base + kEH + c * kTY * kTZ, &maps.e_tile[c], bar, k0, j0, p);
      tma_load_3d(base + kEH + kEE, &maps.m_tile, bar, k0, j0, p);
    }
  };
  if (tid == 0)
    for (int q = 0; q < kS && q < nseq; ++q) issue(q);

  const int j = j0 + w;
  const bool row_ok = j < P.ny;
  const int jj = row_ok ? j : 0;
  const int jm = Y.prv[jj];
  const float mj = Y.mpv[jj], idy = Y.idl_d[jj];
  const float ay = Y.ae[jj], by = Y.be[jj], ky = Y.ke[jj];
  const bool ysl = row_ok && in_slab(Y, j);
  const bool yspecial = row_ok && jm != j - 1;
  const int kq = k0 + 4 * lane;
  bool kv[4], zsl[4], zspecial[4];
  int kmz[4];
  float idz[4], mkz[4], az[4], bz[4], kz[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = kq + e;
    kv[e] = row_ok && k < P.nz;
    const int kk = k < P.nzp ? k : 0;
    kmz[e] = Z.prv[kk];
    mkz[e] = Z.mpv[kk];
    idz[e] = Z.idl_d[kk];
    az[e] = Z.ae[kk]; bz[e] = Z.be[kk]; kz[e] = Z.ke[kk];
    zsl[e] = kv[e] && in_slab(Z, k);
    zspecial[e] = kv[e] && kmz[e] != k - 1;
  }
  const unsigned lt = (1u << lane) - 1u;
  const unsigned grp = 0xffu << (lane & ~7);
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const float cw = P.cw;
  bool ok = true;
  for (int t = 1; t < nseq; ++t) {
    const int i = ib + t - 1;
    if (ok) ok = mbar_wait(&bars[(t - 1) % kS], (uint32_t)(((t - 1) / kS) & 1), err);
    if (ok) ok = mbar_wait(&bars[t % kS], (uint32_t)((t / kS) & 1), err);
    if (ok) confirmed = t + 1;
    const float* prv = st + ((t - 1) % kS) * kEStage;
    const float* cur = st + (t % kS) * kEStage;
    // material ids (all lanes, for the ballots)
    uint32_t mid[4] = {0u, 0u, 0u, 0u};
    if (ok && row_ok) {
      const int mo = w * kTZ + 4 * lane;
      if (wide) {
        const uint4 m = *reinterpret_cast<const uint4*>(reinterpret_cast<const uint32_t*>(cur + kEH + kEE) + mo);
        mid[0] = m.x; mid[1] = m.y; mid[2] = m.z; mid[3] = m.w;
      } else {
        const uint2 m = *reinterpret_cast<const uint2*>(reinterpret_cast<const uint16_t*>(cur + kEH + kEE) + mo);
        mid[0] = m.x & 0xffffu; mid[1] = m.x >> 16; mid[2] = m.y & 0xffffu; mid[3] = m.y >> 16;
      }
    }
    int npc[4];
    int lane_np = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      npc[e] = P.has_ade ? mats[mid[e]].reserved : 0;
      lane_np += npc[e];
    }
    const int64_t row = i * si + (int64_t)j * sj;
    uint32_t poff = 0;
    // only warps that hold dispersive cells read the segment offset (a dependent global load)
    if (P.has_ade && __any_sync(kFull, lane_np > 0)) {
      int pre = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b)
        pre += __popc(__ballot_sync(kFull, (lane_np >> b) & 1) & lt & grp) << b;
      if (lane_np > 0) poff = P.seg_ofs[(row + kq) >> 5] + (uint32_t)pre;
    }
    if (ok && (kv[0] | kv[1] | kv[2] | kv[3])) {
      const float mi = X.mpv[i], idx_ = X.idl_d[i];
      const float ax_ = X.ae[i], bx_ = X.be[i], kx_ = X.ke[i];
      const bool xsl = in_slab(X, i);
      const int ro = (w + 1) * kBZ + 4 + 4 * lane;  // own row/cols in the H box
      const float4 hx = lds4(cur + 0 * kBoxW + ro);
      const float4 hy = lds4(cur + 1 * kBoxW + ro);
      const float4 hz = lds4(cur + 2 * kBoxW + ro);
      const float hxm = cur[0 * kBoxW + ro - 1];
      const float hym = cur[1 * kBoxW + ro - 1];
      float4 yhx = lds4(cur + 0 * kBoxW + ro - kBZ);
      float4 yhz = lds4(cur + 2 * kBoxW + ro - kBZ);
      if (yspecial) {
        const int64_t oy = i * si + (int64_t)jm * sj + kq;
        yhx = *reinterpret_cast<const float4*>(P.f[3] + oy);
        yhz = *reinterpret_cast<const float4*>(P.f[5] + oy);
      }
      const float4 phy = lds4(prv + 1 * kBoxW + ro);
      const float4 phz = lds4(prv + 2 * kBoxW + ro);
      const int eo = kEH + w * kTZ + 4 * lane;
      const float4 e4x = lds4(cur + eo);
      const float4 e4y = lds4(cur + eo + kTY * kTZ);
      const float4 e4z = lds4(cur + eo + 2 * kTY * kTZ);
      float ex[4] = {e4x.x, e4x.y, e4x.z, e4x.w};
      float ey[4] = {e4y.x, e4y.y, e4y.z, e4y.w};
      float ez[4] = {e4z.x, e4z.y, e4z.z, e4z.w};
      Psi4 px0, px1, py0, py1;  // x-slab Ey, Ez; y-slab Ex, Ez
      if (xsl) {
        px0.load(psi_slab(P.psie, 0, 0, X, i, j, kq, P.ny, P.nzp));
        px1.load(psi_slab(P.psie, 0, 1, X, i, j, kq, P.ny, P.nzp));
      }
      if (ysl) {
        py0.load(psi_slab(P.psie, 1, 0, Y, i, j, kq, P.ny, P.nzp));
        py1.load(psi_slab(P.psie, 1, 1, Y, i, j, kq, P.ny, P.nzp));
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (!kv[e]) continue;
        const int k = kq + e;
        const MatRec& M = mats[mid[e]];
        const float4 cab = *reinterpret_cast<const float4*>(&M.ca[0]);
        const float2 cb12 = *reinterpret_cast<const float2*>(&M.cb[1]);
        const int np = npc[e];
        const float hxe = comp4(hx, e), hye = comp4(hy, e), hze = comp4(hz, e);
        float zhx = (e > 0) ? comp4(hx, e - 1) : hxm;
        float zhy = (e > 0) ? comp4(hy, e - 1) : hym;
        if (zspecial[e]) {
          zhx = P.f[3][row + kmz[e]];
          zhy = P.f[4][row + kmz[e]];
        }
        {  // Ex: dHz/dy - dHy/dz
          const float en = ex[e];
          const float wv = (np > 0 && M.np[0] > 0) ? ade_cell(P, M.pset[0], M.np[0], poff, en) : 0.0f;
          const float dzy = (hze - comp4(yhz, e) * mj) * idy;
          const float dyz = (hye - zhy * mkz[e]) * idz[e];
          const float sy = ysl ? stretch_reg(dzy, py0.v[e], ay, by, ky) : dzy;
          const float sz = zsl[e] ? stretch_slab(dyz, psi_slab(P.psie, 2, 0, Z, i, j, k, P.ny, P.nzp), az[e], bz[e], kz[e]) : dyz;
          ex[e] = e_new(cab.x, en, cab.w, sy, sz, cw, wv);
        }
        {  // Ey: dHx/dz - dHz/dx
          const float en = ey[e];
          const float wv = (np > 0 && M.np[1] > 0)
                               ? ade_cell(P, M.pset[1], M.np[1], poff + M.np[0], en) : 0.0f;
          const float dxz = (hxe - zhx * mkz[e]) * idz[e];
          const float dzx = (hze - comp4(phz, e) * mi) * idx_;
          const float sz = zsl[e] ? stretch_slab(dxz, psi_slab(P.psie, 2, 1, Z, i, j, k, P.ny, P.nzp), az[e], bz[e], kz[e]) : dxz;
          const float sx = xsl ? stretch_reg(dzx, px0.v[e], ax_, bx_, kx_) : dzx;
          ey[e] = e_new(cab.y, en, cb12.x, sz, sx, cw, wv);
        }
        {  // Ez: dHy/dx - dHx/dy
          const float en = ez[e];
          const float wv = (np > 0 && M.np[2] > 0)
                               ? ade_cell(P, M.pset[2], M.np[2], poff + M.np[0] + M.np[1], en) : 0.0f;
          const float dyx = (hye - comp4(phy, e) * mi) * idx_;
          const float dxy = (hxe - comp4(yhx, e) * mj) * idy;
          const float sx = xsl ? stretch_reg(dyx, px1.v[e], ax_, bx_, kx_) : dyx;
          const float sy = ysl ? stretch_reg(dxy, py1.v[e], ay, by, ky) : dxy;
          ez[e] = e_new(cab.z, en, cb12.y, sx, sy, cw, wv);
        }
        poff += (uint32_t)np;
      }
      px0.store(); px1.store(); py0.store(); py1.store();
      *reinterpret_cast<float4*>(P.f[0] + row + kq) = make_float4(ex[0], ex[1], ex[2], ex[3]);
      *reinterpret_cast<float4*>(P.f[1] + row + kq) = make_float4(ey[0], ey[1], ey[2], ey[3]);
      *reinterpret_cast<float4*>(P.f[2] + row + kq) = make_float4(ez[0], ez[1], ez[2], ez[3]);
    }
    __syncthreads();
    // stage t-1 is no longer needed: refill it with sequence t-1+kS
    if (tid == 0 && ok && t - 1 + kS < nseq) issue(t - 1 + kS);
  }
  if (!ok && tid == 0) {
    for (int q = confirmed; q < issued; ++q) {
      mbar_wait(&bars[q % kS], (uint32_t)((q / kS) & 1), err);
    }
  }
}

}  // namespace

size_t tma_h_smem() { return (size_t)kS * kHStage * 4 + kS * sizeof(uint64_t); }
size_t tma_e_smem() {
  return (size_t)kS * kEStage * 4 + kS * sizeof(uint64_t) + kSmemMats * sizeof(MatRec);
}

int tma_xchunk(const YeeParams& P) {
  const int64_t tiles = (int64_t)((P.nzp + kTZ - 1) / kTZ) * ((P.ny + kTY - 1) / kTY);
  const int64_t want = 148LL * 3 * 6;  // ~6 waves of 3 resident blocks per SM
  int64_t chunks = (want + tiles - 1) / tiles;
  int xch = (int)((P.nx + chunks - 1) / chunks);
  if (xch < 8) xch = 8;
  if (xch > 64) xch = 64;
  if (xch > P.nx) xch = P.nx;
  return xch;
}

cudaError_t tma_setup_kernels() {
  cudaError_t e = cudaFuncSetAttribute(k_h_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)tma_h_smem());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_e_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)tma_e_smem());
}

cudaError_t launch_update_h_tma(const TmaMaps& maps, const YeeParams& P, int xch, int* err,
                                cudaStream_t s) {
  dim3 b(32, kTY, 1), g((P.nzp + kTZ - 1) / kTZ, (P.ny + kTY - 1) / kTY, (P.nx + xch - 1) / xch);
  k_h_tma<<<g, b, tma_h_smem(), s>>>(maps, P, xch, err);
  return cudaGetLastError();
}

cudaError_t launch_update_e_tma(const TmaMaps& maps, const YeeParams& P, int xch, int n_mats,
                                int* err, cudaStream_t s) {
  dim3 b(32, kTY, 1), g((P.nzp + kTZ - 1) / kTZ, (P.ny + kTY - 1) / kTY, (P.nx + xch - 1) / xch);
  k_e_tma<<<g, b, tma_e_smem(), s>>>(maps, P, xch, n_mats, err);
  return cudaGetLastError();
}

}  // namespace oem
