// Streaming Yee kernels for sm_100a (the default step kernels).
//
// Thread mapping: a warp covers 128 consecutive z cells of one (i, j) row, four per lane, read
// and written as one 128-bit access per field component; a block is 4 warps = 4 rows in y; a
// thread walks a chunk of x planes. Along x the neighbour plane is carried in registers from
// one iteration to the next, so every field value is read from memory once per kernel; along z
// the neighbour comes from the adjacent lane by a warp shuffle; along y it is a 128-bit load of
// the adjacent row (served by L1/L2, since that row is the neighbouring warp's own). Axis
// tables are loaded once per thread (y, z) or once per plane (x, warp-uniform).
//
// The arithmetic per cell is that of the basic kernels in oem_kernels.cu, which follow
// openem/kernels/yee.cu:60-240 and dispersion.cu:168-207.
#include <cuda_runtime.h>
#include <stdint.h>

#include "oem_internal.cuh"
#include "oem_arith.cuh"

namespace oem {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kTY = 4;  // rows (warps) per block

struct F4 {
  float v[4];
};

__device__ __forceinline__ F4 ld4(const float* p) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  F4 r;
  r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
  return r;
}

__device__ __forceinline__ void st4(float* p, const F4& a) {
  *reinterpret_cast<float4*>(p) = make_float4(a.v[0], a.v[1], a.v[2], a.v[3]);
}

__device__ __forceinline__ F4 zero4() {
  F4 r;
  r.v[0] = r.v[1] = r.v[2] = r.v[3] = 0.f;
  return r;
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

// CPML recursion on a slab cell (openem/kernels/yee.cu:60-74).
__device__ __forceinline__ float stretch_slab(float d, float* psi, float a, float b, float ik) {
  const float p = b * (*psi) + a * d;
  *psi = p;
  return ik * d + p;
}

__device__ __forceinline__ bool in_slab(const DevAxis& A, int q) {
  return q < A.lo || q >= A.n - A.hi;
}

// ---------------------------------------------------------------------------------------------
// H half step
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_h_stream(YeeParams P, int xch) {
  const int lane = threadIdx.x;
  const int j = blockIdx.y * kTY + threadIdx.y;
  if (j >= P.ny) return;  // warp-uniform
  const int k0 = (blockIdx.x * 32 + lane) * 4;
  const bool act = k0 < P.nzp;
  const int ib = blockIdx.z * xch;
  const int ie = min(ib + xch, P.nx);
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const float* Ex = P.f[0];
  const float* Ey = P.f[1];
  const float* Ez = P.f[2];
  const float ch = P.ch;

  const int jp = Y.nxt[j];
  const float mj = Y.mnx[j], idy = Y.idl_p[j];
  const float ay = Y.ah[j], by = Y.bh[j], ky = Y.kh[j];
  const bool ysl = in_slab(Y, j);

  bool kv[4], zsl[4];
  int kpz[4];
  float idz[4], mkz[4], az[4], bz[4], kz[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = act ? k0 + e : 0;
    kv[e] = act && (k0 + e) < P.nz;
    kpz[e] = Z.nxt[k];
    mkz[e] = Z.mnx[k];
    idz[e] = Z.idl_p[k];
    az[e] = Z.ah[k]; bz[e] = Z.bh[k]; kz[e] = Z.kh[k];
    zsl[e] = kv[e] && in_slab(Z, k0 + e);
  }

  F4 ex = zero4(), ey = zero4(), ez = zero4();
  if (act) {
    const int64_t o = ib * si + j * sj + k0;
    ex = ld4(Ex + o); ey = ld4(Ey + o); ez = ld4(Ez + o);
  }
  for (int i = ib; i < ie; ++i) {
    const int64_t row = i * si + j * sj;
    const int ip = X.nxt[i];
    const float mi = X.mnx[i], idx_ = X.idl_p[i];
    const float ax_ = X.ah[i], bx_ = X.bh[i], kx_ = X.kh[i];
    const bool xsl = in_slab(X, i);
    F4 nex = zero4(), ney = zero4(), nez = zero4(), yex = zero4(), yez = zero4();
    F4 hx = zero4(), hy = zero4(), hz = zero4();
    if (act) {
      const int64_t on = ip * si + j * sj + k0;
      nex = ld4(Ex + on); ney = ld4(Ey + on); nez = ld4(Ez + on);
      const int64_t oy = i * si + jp * sj + k0;
      yex = ld4(Ex + oy); yez = ld4(Ez + oy);
      hx = ld4(P.f[3] + row + k0); hy = ld4(P.f[4] + row + k0); hz = ld4(P.f[5] + row + k0);
    }
    // z-forward neighbours of Ex and Ey
    float zex[4], zey[4];
    const float sx0 = __shfl_down_sync(kFull, ex.v[0], 1);
    const float sy0 = __shfl_down_sync(kFull, ey.v[0], 1);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      zex[e] = (e < 3) ? ex.v[e + 1] : sx0;
      zey[e] = (e < 3) ? ey.v[e + 1] : sy0;
      if (kv[e] && (kpz[e] != k0 + e + 1 || (e == 3 && lane == 31))) {
        zex[e] = Ex[row + kpz[e]];
        zey[e] = Ey[row + kpz[e]];
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (!kv[e]) continue;
      const int k = k0 + e;
      {  // Hx: -(dEz/dy - dEy/dz)
        const float dzy = (yez.v[e] * mj - ez.v[e]) * idy;
        const float dyz = (zey[e] * mkz[e] - ey.v[e]) * idz[e];
        const float sy = ysl ? stretch_slab(dzy, psi_slab(P.psih, 1, 0, Y, i, j, k, P.ny, P.nzp), ay, by, ky) : dzy;
        const float sz = zsl[e] ? stretch_slab(dyz, psi_slab(P.psih, 2, 0, Z, i, j, k, P.ny, P.nzp), az[e], bz[e], kz[e]) : dyz;
        hx.v[e] -= ch * (sy - sz);
      }
      {  // Hy: -(dEx/dz - dEz/dx)
        const float dxz = (zex[e] * mkz[e] - ex.v[e]) * idz[e];
        const float dzx = (nez.v[e] * mi - ez.v[e]) * idx_;
        const float sz = zsl[e] ? stretch_slab(dxz, psi_slab(P.psih, 2, 1, Z, i, j, k, P.ny, P.nzp), az[e], bz[e], kz[e]) : dxz;
        const float sx = xsl ? stretch_slab(dzx, psi_slab(P.psih, 0, 0, X, i, j, k, P.ny, P.nzp), ax_, bx_, kx_) : dzx;
        hy.v[e] -= ch * (sz - sx);
      }
      {  // Hz: -(dEy/dx - dEx/dy)
        const float dyx = (ney.v[e] * mi - ey.v[e]) * idx_;
        const float dxy = (yex.v[e] * mj - ex.v[e]) * idy;
        const float sx = xsl ? stretch_slab(dyx, psi_slab(P.psih, 0, 1, X, i, j, k, P.ny, P.nzp), ax_, bx_, kx_) : dyx;
        const float sy = ysl ? stretch_slab(dxy, psi_slab(P.psih, 1, 1, Y, i, j, k, P.ny, P.nzp), ay, by, ky) : dxy;
        hz.v[e] -= ch * (sx - sy);
      }
    }
    if (act) {
      st4(P.f[3] + row + k0, hx); st4(P.f[4] + row + k0, hy); st4(P.f[5] + row + k0, hz);
    }
    if (i + 1 < ie) {
      if (ip == i + 1) {
        ex = nex; ey = ney; ez = nez;
      } else if (act) {
        const int64_t o = (i + 1) * si + j * sj + k0;
        ex = ld4(Ex + o); ey = ld4(Ey + o); ez = ld4(Ez + o);
      }
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

__global__ void __launch_bounds__(128) k_e_stream(YeeParams P, int xch, int smem_mats) {
  extern __shared__ MatRec s_mats[];
  const MatRec* mats = P.mats;
  if (smem_mats) {
    const int nm = smem_mats;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const uint4* src = reinterpret_cast<const uint4*>(P.mats);
    uint4* dst = reinterpret_cast<uint4*>(s_mats);
    for (int q = tid; q < nm * 4; q += 32 * kTY) dst[q] = src[q];
    __syncthreads();
    mats = s_mats;
  }
  const int lane = threadIdx.x;
  const int j = blockIdx.y * kTY + threadIdx.y;
  if (j >= P.ny) return;  // warp-uniform (after the block-wide staging)
  const int k0 = (blockIdx.x * 32 + lane) * 4;
  const bool act = k0 < P.nzp;
  const int ib = blockIdx.z * xch;
  const int ie = min(ib + xch, P.nx);
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const float* Hx = P.f[3];
  const float* Hy = P.f[4];
  const float* Hz = P.f[5];
  const float cw = P.cw;

  const int jm = Y.prv[j];
  const float mj = Y.mpv[j], idy = Y.idl_d[j];
  const float ay = Y.ae[j], by = Y.be[j], ky = Y.ke[j];
  const bool ysl = in_slab(Y, j);

  bool kv[4], zsl[4];
  int kmz[4];
  float idz[4], mkz[4], az[4], bz[4], kz[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = act ? k0 + e : 0;
    kv[e] = act && (k0 + e) < P.nz;
    kmz[e] = Z.prv[k];
    mkz[e] = Z.mpv[k];
    idz[e] = Z.idl_d[k];
    az[e] = Z.ae[k]; bz[e] = Z.be[k]; kz[e] = Z.ke[k];
    zsl[e] = kv[e] && in_slab(Z, k0 + e);
  }
  const unsigned lt = (1u << lane) - 1u;
  const unsigned grp = 0xffu << (lane & ~7);

  F4 phx = zero4(), phy = zero4(), phz = zero4();  // H of the previous plane
  int prev_i = -2;
  for (int i = ib; i < ie; ++i) {
    const int64_t row = i * si + j * sj;
    const int im = X.prv[i];
    const float mi = X.mpv[i], idx_ = X.idl_d[i];
    const float ax_ = X.ae[i], bx_ = X.be[i], kx_ = X.ke[i];
    const bool xsl = in_slab(X, i);
    F4 hx = zero4(), hy = zero4(), hz = zero4(), yhx = zero4(), yhz = zero4();
    F4 ex = zero4(), ey = zero4(), ez = zero4();
    uint32_t mid[4] = {0u, 0u, 0u, 0u};
    if (act) {
      hx = ld4(Hx + row + k0); hy = ld4(Hy + row + k0); hz = ld4(Hz + row + k0);
      const int64_t oy = i * si + jm * sj + k0;
      yhx = ld4(Hx + oy); yhz = ld4(Hz + oy);
      if (!(im == i - 1 && prev_i == i - 1)) {
        const int64_t op = im * si + j * sj + k0;
        phy = ld4(Hy + op); phz = ld4(Hz + op);
      }
      ex = ld4(P.f[0] + row + k0); ey = ld4(P.f[1] + row + k0); ez = ld4(P.f[2] + row + k0);
      if (P.mat16) {
        const uint2 m = *reinterpret_cast<const uint2*>(P.mat16 + row + k0);
        mid[0] = m.x & 0xffffu; mid[1] = m.x >> 16; mid[2] = m.y & 0xffffu; mid[3] = m.y >> 16;
      } else {
        const uint4 m = *reinterpret_cast<const uint4*>(P.mat32 + row + k0);
        mid[0] = m.x; mid[1] = m.y; mid[2] = m.z; mid[3] = m.w;
      }
    }
    // ADE: first pole of each element
    int npc[4];
    int lane_np = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      npc[e] = P.has_ade ? mats[mid[e]].reserved : 0;
      lane_np += npc[e];
    }
    uint32_t poff0 = 0;
    if (P.has_ade) {
      int pre = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b)
        pre += __popc(__ballot_sync(kFull, (lane_np >> b) & 1) & lt & grp) << b;
      if (act) poff0 = P.seg_ofs[(row + k0) >> 5] + (uint32_t)pre;
    }
    // z-backward neighbours of Hx and Hy
    float zhx[4], zhy[4];
    const float sx3 = __shfl_up_sync(kFull, hx.v[3], 1);
    const float sy3 = __shfl_up_sync(kFull, hy.v[3], 1);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      zhx[e] = (e > 0) ? hx.v[e - 1] : sx3;
      zhy[e] = (e > 0) ? hy.v[e - 1] : sy3;
      if (kv[e] && (kmz[e] != k0 + e - 1 || (e == 0 && lane == 0))) {
        zhx[e] = Hx[row + kmz[e]];
        zhy[e] = Hy[row + kmz[e]];
      }
    }
    uint32_t poff = poff0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (!kv[e]) continue;
      const int k = k0 + e;
      const MatRec& M = mats[mid[e]];
      const float4 cab = *reinterpret_cast<const float4*>(&M.ca[0]);  // ca0 ca1 ca2 cb0
      const float2 cb12 = *reinterpret_cast<const float2*>(&M.cb[1]);
      const int np = npc[e];
      {  // Ex: dHz/dy - dHy/dz
        const float en = ex.v[e];
        const float w = (np > 0 && M.np[0] > 0) ? ade_cell(P, M.pset[0], M.np[0], poff, en) : 0.0f;
        const float dzy = (hz.v[e] - yhz.v[e] * mj) * idy;
        const float dyz = (hy.v[e] - zhy[e] * mkz[e]) * idz[e];
        const float sy = ysl ? stretch_slab(dzy, psi_slab(P.psie, 1, 0, Y, i, j, k, P.ny, P.nzp), ay, by, ky) : dzy;
        const float sz = zsl[e] ? stretch_slab(dyz, psi_slab(P.psie, 2, 0, Z, i, j, k, P.ny, P.nzp), az[e], bz[e], kz[e]) : dyz;
        ex.v[e] = e_new(cab.x, en, cab.w, sy, sz, cw, w);
      }
      {  // Ey: dHx/dz - dHz/dx
        const float en = ey.v[e];
        const float w = (np > 0 && M.np[1] > 0)
                            ? ade_cell(P, M.pset[1], M.np[1], poff + M.np[0], en) : 0.0f;
        const float dxz = (hx.v[e] - zhx[e] * mkz[e]) * idz[e];
        const float dzx = (hz.v[e] - phz.v[e] * mi) * idx_;
        const float sz = zsl[e] ? stretch_slab(dxz, psi_slab(P.psie, 2, 1, Z, i, j, k, P.ny, P.nzp), az[e], bz[e], kz[e]) : dxz;
        const float sx = xsl ? stretch_slab(dzx, psi_slab(P.psie, 0, 0, X, i, j, k, P.ny, P.nzp), ax_, bx_, kx_) : dzx;
        ey.v[e] = e_new(cab.y, en, cb12.x, sz, sx, cw, w);
      }
      {  // Ez: dHy/dx - dHx/dy
        const float en = ez.v[e];
        const float w = (np > 0 && M.np[2] > 0)
                            ? ade_cell(P, M.pset[2], M.np[2], poff + M.np[0] + M.np[1], en) : 0.0f;
        const float dyx = (hy.v[e] - phy.v[e] * mi) * idx_;
        const float dxy = (hx.v[e] - yhx.v[e] * mj) * idy;
        const float sx = xsl ? stretch_slab(dyx, psi_slab(P.psie, 0, 1, X, i, j, k, P.ny, P.nzp), ax_, bx_, kx_) : dyx;
        const float sy = ysl ? stretch_slab(dxy, psi_slab(P.psie, 1, 1, Y, i, j, k, P.ny, P.nzp), ay, by, ky) : dxy;
        ez.v[e] = e_new(cab.z, en, cb12.y, sx, sy, cw, w);
      }
      poff += (uint32_t)np;
    }
    if (act) {
      st4(P.f[0] + row + k0, ex); st4(P.f[1] + row + k0, ey); st4(P.f[2] + row + k0, ez);
    }
    phy = hy;
    phz = hz;
    prev_i = i;
  }
}

}  // namespace

int stream_xchunk(const YeeParams& P) {
  // enough blocks for ~8 waves of 148 SMs x 12 resident blocks, planes per thread in [4, 32]
  const int64_t tiles = (int64_t)((P.nzp + 127) / 128) * ((P.ny + kTY - 1) / kTY);
  int64_t want = 148LL * 12 * 8;
  int64_t chunks = (want + tiles - 1) / tiles;
  int xch = (int)((P.nx + chunks - 1) / chunks);
  if (xch < 4) xch = 4;
  if (xch > 32) xch = 32;
  if (xch > P.nx) xch = P.nx;
  return xch;
}

cudaError_t launch_update_h_stream(const YeeParams& P, int xch, cudaStream_t s) {
  dim3 b(32, kTY, 1), g((P.nzp + 127) / 128, (P.ny + kTY - 1) / kTY, (P.nx + xch - 1) / xch);
  k_h_stream<<<g, b, 0, s>>>(P, xch);
  return cudaGetLastError();
}

cudaError_t launch_update_e_stream(const YeeParams& P, int xch, int n_mats, cudaStream_t s) {
  dim3 b(32, kTY, 1), g((P.nzp + 127) / 128, (P.ny + kTY - 1) / kTY, (P.nx + xch - 1) / xch);
  const int smem = (n_mats <= 512) ? n_mats : 0;
  k_e_stream<<<g, b, (size_t)smem * sizeof(MatRec), s>>>(P, xch, smem);
  return cudaGetLastError();
}

}  // namespace oem
