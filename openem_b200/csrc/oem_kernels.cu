// Step-loop kernels of the sm_100a engine: Yee H and E updates (CPML psi in the boundary slabs,
// conductivity and PEC folded into per-material coefficients, ADE pole update inlined into the
// E update), plane-wave and point-dipole injection, field time sampling, batched DFT snapshot
// and flush, early-termination reductions.
//
// The update equations are those of OpenEM (openem/kernels/yee.cu:60-240,
// dispersion.cu:168-207, source_dft.cu:39-206, 273-319, 440-779); the data layout and the
// way cells find their coefficients and pole states are this engine's:
//   * fields are (nx, ny, nzp) with nzp a multiple of 32, so one warp covers one 32-cell z
//     segment of one row;
//   * one material index per cell selects a 64-byte tuple (ca, cb, eps, pole set) x 3;
//   * psi exists only inside the CPML slabs; elsewhere the stretched derivative is the plain
//     derivative (identity coefficients);
//   * ADE pole states are packed in cell order; a cell finds its first pole from the offset of
//     its 32-cell segment plus a warp-ballot prefix sum of the pole counts of the lanes before
//     it, so no per-entry index arrays are read.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "oem_internal.cuh"
#include "oem_arith.cuh"

namespace oem {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float* psi_at(const PsiSet& S, int a, int slot, const DevAxis& A,
                                        int i, int j, int k, int ny, int nzp) {
  const int q = (a == 0) ? i : ((a == 1) ? j : k);
  int side, ql, L;
  if (q < A.lo) {
    side = 0; ql = q; L = A.lo;
  } else if (q >= A.n - A.hi) {
    side = 1; ql = q - (A.n - A.hi); L = A.hi;
  } else {
    return nullptr;
  }
  float* base = S.p[a][slot][side];
  int64_t idx;
  if (a == 0) idx = ((int64_t)ql * ny + j) * nzp + k;
  else if (a == 1) idx = ((int64_t)i * L + ql) * nzp + k;
  else idx = ((int64_t)i * ny + j) * L + ql;
  return base + idx;
}

// CPML recursion (openem/kernels/yee.cu:60-74): psi = b psi + a d; return d/kappa + psi.
// Outside the slabs the coefficients are the identity and psi is identically zero.
__device__ __forceinline__ float stretch(float d, float* psi, float a, float b, float ik) {
  if (psi == nullptr) return d;
  return cpml_stretch(d, *psi, a, b, ik);
}

__device__ __forceinline__ uint32_t mat_id(const YeeParams& P, int64_t id) {
  return P.mat16 ? (uint32_t)P.mat16[id] : P.mat32[id];
}

// Deferred ADE of one component: post(n-1) with E^n, then pre(n) with E^n; returns
// w = sum 2 Re(dP) (openem/kernels/dispersion.cu:168-207, bitwise the same sequence).
__device__ __forceinline__ float ade(const YeeParams& P, int set, int np, uint32_t poff,
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

// H half step, one thread per cell (openem/kernels/yee.cu:76-137).
__global__ void __launch_bounds__(128) k_update_h(YeeParams P) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= P.nz || j >= P.ny) return;
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const int64_t id = i * si + j * sj + k;
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const int ip = X.nxt[i], jp = Y.nxt[j], kp = Z.nxt[k];
  const float mi = X.mnx[i], mj = Y.mnx[j], mk = Z.mnx[k];
  const float* Ex = P.f[0];
  const float* Ey = P.f[1];
  const float* Ez = P.f[2];
  const float ex = Ex[id], ey = Ey[id], ez = Ez[id];
  const int64_t idi = ip * si + j * sj + k;
  const int64_t idj = i * si + jp * sj + k;
  const int64_t idk = i * si + j * sj + kp;
  const float ch = P.ch;
  {  // Hx: mu0 dHx/dt = -(dEz/dy - dEy/dz)
    const float dzy = fdiff(Ez[idj], mj, ez, Y.idl_p[j]);
    const float dyz = fdiff(Ey[idk], mk, ey, Z.idl_p[k]);
    const float sy = stretch(dzy, psi_at(P.psih, 1, 0, Y, i, j, k, P.ny, P.nzp), Y.ah[j], Y.bh[j], Y.kh[j]);
    const float sz = stretch(dyz, psi_at(P.psih, 2, 0, Z, i, j, k, P.ny, P.nzp), Z.ah[k], Z.bh[k], Z.kh[k]);
    P.f[3][id] = h_new(P.f[3][id], ch, sy, sz);
  }
  {  // Hy: mu0 dHy/dt = -(dEx/dz - dEz/dx)
    const float dxz = fdiff(Ex[idk], mk, ex, Z.idl_p[k]);
    const float dzx = fdiff(Ez[idi], mi, ez, X.idl_p[i]);
    const float sz = stretch(dxz, psi_at(P.psih, 2, 1, Z, i, j, k, P.ny, P.nzp), Z.ah[k], Z.bh[k], Z.kh[k]);
    const float sx = stretch(dzx, psi_at(P.psih, 0, 0, X, i, j, k, P.ny, P.nzp), X.ah[i], X.bh[i], X.kh[i]);
    P.f[4][id] = h_new(P.f[4][id], ch, sz, sx);
  }
  {  // Hz: mu0 dHz/dt = -(dEy/dx - dEx/dy)
    const float dyx = fdiff(Ey[idi], mi, ey, X.idl_p[i]);
    const float dxy = fdiff(Ex[idj], mj, ex, Y.idl_p[j]);
    const float sx = stretch(dyx, psi_at(P.psih, 0, 1, X, i, j, k, P.ny, P.nzp), X.ah[i], X.bh[i], X.kh[i]);
    const float sy = stretch(dxy, psi_at(P.psih, 1, 1, Y, i, j, k, P.ny, P.nzp), Y.ah[j], Y.bh[j], Y.kh[j]);
    P.f[5][id] = h_new(P.f[5][id], ch, sx, sy);
  }
}

// E full step with the ADE inlined, one thread per cell (openem/kernels/yee.cu:154-240 and
// dispersion.cu:168-207). Block (32, 4): each warp is one aligned 32-cell z segment.
__global__ void __launch_bounds__(128) k_update_e(YeeParams P) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (j >= P.ny) return;  // warp-uniform: a warp lies in one row
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const int64_t id = i * si + j * sj + k;
  const MatRec& M = P.mats[mat_id(P, id)];
  uint32_t poff = 0;
  if (P.has_ade) {
    const int npc = M.np[0] + M.np[1] + M.np[2];
    const unsigned lt = (1u << (threadIdx.x & 31)) - 1u;
    int pre = 0;
#pragma unroll
    for (int b = 0; b < 6; ++b) pre += __popc(__ballot_sync(kFull, (npc >> b) & 1) & lt) << b;
    poff = P.seg_ofs[id >> 5] + (uint32_t)pre;
  }
  if (k >= P.nz) return;
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const int im = X.prv[i], jm = Y.prv[j], km = Z.prv[k];
  const float mi = X.mpv[i], mj = Y.mpv[j], mk = Z.mpv[k];
  const float* Hx = P.f[3];
  const float* Hy = P.f[4];
  const float* Hz = P.f[5];
  const float hx = Hx[id], hy = Hy[id], hz = Hz[id];
  const int64_t idi = im * si + j * sj + k;
  const int64_t idj = i * si + jm * sj + k;
  const int64_t idk = i * si + j * sj + km;
  const float cw = P.cw;
  {  // Ex: eps dEx/dt = dHz/dy - dHy/dz
    const float en = P.f[0][id];
    const float w = (M.np[0] > 0) ? ade(P, M.pset[0], M.np[0], poff, en) : 0.0f;
    const float dzy = bdiff(hz, Hz[idj], mj, Y.idl_d[j]);
    const float dyz = bdiff(hy, Hy[idk], mk, Z.idl_d[k]);
    const float sy = stretch(dzy, psi_at(P.psie, 1, 0, Y, i, j, k, P.ny, P.nzp), Y.ae[j], Y.be[j], Y.ke[j]);
    const float sz = stretch(dyz, psi_at(P.psie, 2, 0, Z, i, j, k, P.ny, P.nzp), Z.ae[k], Z.be[k], Z.ke[k]);
    P.f[0][id] = e_new(M.ca[0], en, M.cb[0], sy, sz, cw, w);
  }
  {  // Ey: eps dEy/dt = dHx/dz - dHz/dx
    const float en = P.f[1][id];
    const float w = (M.np[1] > 0) ? ade(P, M.pset[1], M.np[1], poff + M.np[0], en) : 0.0f;
    const float dxz = bdiff(hx, Hx[idk], mk, Z.idl_d[k]);
    const float dzx = bdiff(hz, Hz[idi], mi, X.idl_d[i]);
    const float sz = stretch(dxz, psi_at(P.psie, 2, 1, Z, i, j, k, P.ny, P.nzp), Z.ae[k], Z.be[k], Z.ke[k]);
    const float sx = stretch(dzx, psi_at(P.psie, 0, 0, X, i, j, k, P.ny, P.nzp), X.ae[i], X.be[i], X.ke[i]);
    P.f[1][id] = e_new(M.ca[1], en, M.cb[1], sz, sx, cw, w);
  }
  {  // Ez: eps dEz/dt = dHy/dx - dHx/dy
    const float en = P.f[2][id];
    const float w = (M.np[2] > 0)
                        ? ade(P, M.pset[2], M.np[2], poff + M.np[0] + M.np[1], en) : 0.0f;
    const float dyx = bdiff(hy, Hy[idi], mi, X.idl_d[i]);
    const float dxy = bdiff(hx, Hx[idj], mj, Y.idl_d[j]);
    const float sx = stretch(dyx, psi_at(P.psie, 0, 1, X, i, j, k, P.ny, P.nzp), X.ae[i], X.be[i], X.ke[i]);
    const float sy = stretch(dxy, psi_at(P.psie, 1, 1, Y, i, j, k, P.ny, P.nzp), Y.ae[j], Y.be[j], Y.ke[j]);
    P.f[2][id] = e_new(M.ca[2], en, M.cb[2], sx, sy, cw, w);
  }
}

// One-face TF/SF plane wave, H side (openem/kernels/source_dft.cu:40-55).
__global__ void k_plane_h(YeeParams P, PlaneSrc s, const int* step) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  const int n = *step;
  if (i >= P.nx || j >= P.ny || n < 0 || n >= s.ntab) return;
  const float inc = (float)s.d_ex[n];
  float* H = P.f[s.pol == 0 ? 4 : 3];
  H[((int64_t)i * P.ny + j) * P.nzp + s.kh] += s.coef_h * inc;
}

// One-face TF/SF plane wave, E side (openem/kernels/source_dft.cu:58-73).
__global__ void k_plane_e(YeeParams P, PlaneSrc s, const int* step) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  const int n = *step;
  if (i >= P.nx || j >= P.ny || n < 0 || n >= s.ntab) return;
  const int64_t id = ((int64_t)i * P.ny + j) * P.nzp + s.ks;
  const float inc = (float)s.d_hy[n];
  const float cb = P.mats[mat_id(P, id)].cb[s.pol];
  P.f[s.pol][id] += cb * s.coef_e * inc;
}

// Point dipoles, one thread per distinct (component, cell); its stencil points are added in a
// fixed order, so the result is deterministic (openem/kernels/source_dft.cu:147-206 uses
// atomicAdd instead).
__global__ void k_dipoles(YeeParams P, DipoleSet d, const int* step, SnapBoxes sb) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *step;
  if (t >= d.n_targets || n < 0 || n >= d.nsteps1) return;
  const int c = d.d_tcomp[t];
  const int64_t id = d.d_target[t];
  float* F = P.f[d.magnetic ? 3 + c : c];
  const float cc = d.magnetic ? P.ch : P.mats[mat_id(P, id)].cb[c];
  float v = F[id];
  for (int q = d.d_ofs[t]; q < d.d_ofs[t + 1]; ++q) {
    const float a = (float)d.d_amp[(int64_t)d.d_src[q] * d.nsteps1 + n];
    v += -cc * d.d_coef[q] * a;
  }
  F[id] = v;
  // E dipoles after an E update that wrote the box snapshots itself: the target's row in each
  // box that holds it takes the injected value, as a snapshot taken after this kernel would
  for (int m = 0; m < sb.n; ++m) {
    const SnapBox& b = sb.b[m];
    const int k = (int)(id % P.nzp);
    const int j = (int)((id / P.nzp) % P.ny);
    const int i = (int)(id / ((int64_t)P.nzp * P.ny));
    if ((unsigned)(i - b.i0) >= (unsigned)b.ni || (unsigned)(j - b.j0) >= (unsigned)b.nj ||
        (unsigned)(k - b.k0) >= (unsigned)b.nk)
      continue;
    const int64_t o = ((int64_t)(i - b.i0) * b.nj + (j - b.j0)) * b.nk + (k - b.k0);
    b.snap[(int64_t)(n % b.T) * 6 * b.cells + (int64_t)c * b.cells + o] = v;
  }
  if (d.d_amp_im) {  // complex plan: the imaginary part of the amplitude drives the im field
    float* Fi = P.fi[d.magnetic ? 3 + c : c];
    float w = Fi[id];
    for (int q = d.d_ofs[t]; q < d.d_ofs[t + 1]; ++q) {
      const float a = (float)d.d_amp_im[(int64_t)d.d_src[q] * d.nsteps1 + n];
      w += -cc * d.d_coef[q] * a;
    }
    Fi[id] = w;
  }
}

// Absorber decay of one slab and one field family (openem/kernels/absorber.cu:20-70): the
// bounding box spans the whole grid except nlay layers along the axis; (j, k) flattened with k
// innermost, i on blockIdx.y. E: the normal component sits at the half cell; H: the tangential
// ones. Complex plans decay both parts.
__global__ void k_absorb(YeeParams P, Absorber a, int is_e, int bj, int bk) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = blockIdx.y;
  if (tid >= bj * bk) return;
  const int jj = tid / bk;
  const int kk = tid - jj * bk;
  const int i = a.axis == 0 ? a.g0 + ii : ii;
  const int j = a.axis == 1 ? a.g0 + jj : jj;
  const int k = a.axis == 2 ? a.g0 + kk : kk;
  const int l = a.axis == 0 ? ii : (a.axis == 1 ? jj : kk);
  const int64_t id = ((int64_t)i * P.ny + j) * P.nzp + k;
  const float di = a.d_int[l], dh = a.d_half[l];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const bool half = is_e ? (c == a.axis) : (c != a.axis);
    const float d = half ? dh : di;
    const int q = is_e ? c : 3 + c;
    P.f[q][id] = __fmul_rn(P.f[q][id], d);
    if (P.cplx) P.fi[q][id] = __fmul_rn(P.fi[q][id], d);
  }
}

// Field time monitor, one shot of the two-shot H average (openem/kernels/source_dft.cu:282-319).
__global__ void k_time_sample(YeeParams P, TimeMon m, const int* step, int add) {
  const int m_ref = (*step + 1) - add;
  const int soff = m_ref - m.beg;
  if (soff < 0 || m_ref >= m.end || soff % m.iv) return;
  const int slot = soff / m.iv;
  if (slot >= m.nslots) return;
  const int cc = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y * blockDim.y + threadIdx.y;
  const int a = blockIdx.z;
  if (a >= m.ni || b >= m.nj || cc >= m.nk) return;
  const int64_t id = ((int64_t)(m.i0 + a) * P.ny + (m.j0 + b)) * P.nzp + (m.k0 + cc);
  const int64_t cells = (int64_t)m.ni * m.nj * m.nk;
  const int64_t off = ((int64_t)a * m.nj + b) * m.nk + cc;
  for (int q = 0; q < m.nc; ++q) {
    const int comp = m.comps[q];
    const float w = comp < 3 ? (add ? 0.0f : 1.0f) : 0.5f;
    if (w == 0.0f) continue;
    const int64_t o = ((int64_t)q * m.nslots + slot) * cells + off;
    const float v = w * P.f[comp][id];
    m.d_buf[o] = add ? m.d_buf[o] + v : v;
    if (m.d_buf_i) {
      const float vi = w * P.fi[comp][id];
      m.d_buf_i[o] = add ? m.d_buf_i[o] + vi : vi;
    }
  }
}

// DFT snapshot of a flux plane: (E_t1, E_t2, colocated H_t1, colocated H_t2) into ring row
// step % T (openem/kernels/source_dft.cu:532-564 stores six raw values; the colocation
// average (H[k] + H[k-1]) / 2 is taken here in the same fp32 arithmetic).
__global__ void k_snap_plane(YeeParams P, Monitor m, const int* step) {
  const int p2 = blockIdx.x * blockDim.x + threadIdx.x;
  const int p1 = blockIdx.y * blockDim.y + threadIdx.y;
  if (p1 >= m.n1 || p2 >= m.n2) return;
  const int t1 = (m.axis == 0) ? 1 : 0;
  const int t2 = (m.axis == 2) ? 1 : 2;
  int c[3];
  c[m.axis] = m.km; c[t1] = p1; c[t2] = p2;
  const int64_t id = ((int64_t)c[0] * P.ny + c[1]) * P.nzp + c[2];
  c[m.axis] = m.km - 1;
  const int64_t idm = ((int64_t)c[0] * P.ny + c[1]) * P.nzp + c[2];
  const int64_t off = (int64_t)p1 * m.n2 + p2;
  float* row = m.d_snap + (int64_t)((*step) % m.T) * (m.cplx ? 8 : 4) * m.cells;
  // loads first (see k_snap_boxes)
  const float e1 = P.f[t1][id], e2 = P.f[t2][id];
  const float h1 = P.f[3 + t1][id], h1m = P.f[3 + t1][idm];
  const float h2 = P.f[3 + t2][id], h2m = P.f[3 + t2][idm];
  if (m.cplx) {
    const float e1i = P.fi[t1][id], e2i = P.fi[t2][id];
    const float h1i = P.fi[3 + t1][id], h1mi = P.fi[3 + t1][idm];
    const float h2i = P.fi[3 + t2][id], h2mi = P.fi[3 + t2][idm];
    row[4 * m.cells + off] = e1i;
    row[5 * m.cells + off] = e2i;
    row[6 * m.cells + off] = 0.5f * (h1i + h1mi);
    row[7 * m.cells + off] = 0.5f * (h2i + h2mi);
  }
  row[off] = e1;
  row[m.cells + off] = e2;
  row[2 * m.cells + off] = 0.5f * (h1 + h1m);
  row[3 * m.cells + off] = 0.5f * (h2 + h2m);
}

// DFT snapshot of box monitors (openem/kernels/source_dft.cu:453-478): the six components at
// their Yee positions into ring row step % T, every box of the plan in one launch: block ranges
// per box (blk0), cb blocks of 256 points per plane of a box, so that the boxes' reads overlap (a thin box across rows reads 8
// bytes of every 64 it fetches and is latency-bound; the others stream beside it).
__global__ void __launch_bounds__(256) k_snap_boxes(YeeParams P,
                                                    const __grid_constant__ BoxSnapSet S,
                                                    const int* step) {
  int q = 0;
  while (q + 1 < S.n && blockIdx.x >= S.blk0[q + 1]) ++q;
  const Monitor& m = S.m[q];
  const uint32_t bl = blockIdx.x - S.blk0[q];
  const uint32_t a = bl / S.cb[q];  // plane of the box
  const uint32_t t = (bl - a * S.cb[q]) * 256u + threadIdx.x;
  const uint32_t njk = (uint32_t)m.nj * (uint32_t)m.nk;
  if (t >= njk) return;
  const uint32_t b = t / (uint32_t)m.nk;
  const uint32_t cc = t - b * (uint32_t)m.nk;
  float* row = m.d_snap + (int64_t)((*step) % m.T) * (m.cplx ? 12 : 6) * m.cells;
  const int64_t id = ((int64_t)(m.i0 + (int)a) * P.ny + (m.j0 + (int)b)) * P.nzp + (m.k0 + (int)cc);
  const int64_t o = (int64_t)a * njk + t;
  // every load before the first store: the compiler cannot move a load above a store to a
  // pointer that may alias it, and a thin box's reads are latency-bound
  float v[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) v[c] = P.f[c][id];
  if (m.cplx) {
    float vi[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) vi[c] = P.fi[c][id];
#pragma unroll
    for (int c = 0; c < 6; ++c) row[(6 + c) * m.cells + o] = vi[c];
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) row[c * m.cells + o] = v[c];
}

// Batched DFT flush (openem/kernels/source_dft.cu:440-530 real fields,
// openem/kernels/bloch.cu:389-481 complex fields): at a batch boundary, or when forced, fold the
// not-yet-folded snapshot rows into the float64 accumulators. Per (component, point, frequency)
// the rows are summed in step order into an fp32 partial, which is then added to the float64
// accumulator once; a complex ring holds NC real rows then NC imaginary rows per step and the
// product is (u_re + i u_im)(cos + i sin). done[0] holds the last step already folded.
//
// One thread per (component, point), points fastest: it holds the batch's (at most 32)
// snapshot values of its entry in registers, so the ring is read from memory once, and walks
// every frequency; the phase rows of the batch are staged in shared memory a chunk of
// frequencies at a time (the same float4 for every thread of a warp). Each accumulator is read
// and written once per flush, coalesced over the points. A grid of a few blocks per SM strides
// over tiles of 128 entries, so that the launch of a step without a batch boundary costs little.
constexpr int kFlushF = 16;  // frequencies per staged phase chunk
constexpr int kFlushG = 4;   // frequencies whose sums a thread forms together
static_assert(kFlushF % kFlushG == 0, "whole groups per chunk");
template <int NC, bool CPLX>
__global__ void __launch_bounds__(128, 4) k_flush(Monitor m, const int* step, int forced) {
  const int s_now = forced ? (*step - 1) : *step;
  if (!forced && ((s_now + 1) % m.T) != 0) return;
  // the ring holds the last T <= 32 steps: older unfolded rows (steps run without monitors)
  // are gone and are not folded
  const int s_lo = max(*m.d_done + 1, s_now - m.T + 1);
  if (s_lo > s_now) return;
  const int ns = s_now - s_lo + 1;  // rows to fold, 1..T
  constexpr int NE = NC / 2;        // E components come first
  // the phase rows of the chunk, split by field family: [0] (cos, sin) at the E times, [1] at
  // the H times, so that a thread reads the pair of its component with one load
  __shared__ float2 sph[2][32][kFlushF];
  const int64_t cells = m.cells;
  const int64_t items = (int64_t)NC * cells;
  for (int64_t base = (int64_t)blockIdx.x * 128; base < items; base += (int64_t)gridDim.x * 128) {
    const int64_t it = base + threadIdx.x;
    const bool act = it < items;
    const int c = act ? (int)(it / cells) : 0;
    const int64_t pt = act ? it - (int64_t)c * cells : 0;
    const bool isE = c < NE;
    float vr[32], vi[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) {
      vr[q] = 0.f;
      vi[q] = 0.f;
      if (act && q < ns) {
        const int s = s_lo + q;
        const float* row = m.d_snap + (int64_t)(s % m.T) * (CPLX ? 2 : 1) * NC * cells;
        vr[q] = row[(int64_t)c * cells + pt];
        if (CPLX) vi[q] = row[(int64_t)(NC + c) * cells + pt];
      }
    }
    for (int f0 = 0; f0 < m.nf; f0 += kFlushF) {
      const int nfc = min(kFlushF, m.nf - f0);
      __syncthreads();  // the previous chunk's rows are no longer read
      for (int e = threadIdx.x; e < ns * kFlushF; e += 128) {
        const int q = e / kFlushF, ff = e - q * kFlushF;
        if (ff < nfc) {
          const float4 ph = __ldg(reinterpret_cast<const float4*>(m.d_phase) +
                                  ((int64_t)(s_lo + q) * m.nf + f0 + ff));
          sph[0][q][ff] = make_float2(ph.x, ph.y);
          sph[1][q][ff] = make_float2(ph.z, ph.w);
        }
      }
      __syncthreads();
      // groups of kFlushG frequencies: the group's accumulators are loaded before its partial
      // sums are formed, so their DRAM latency overlaps the arithmetic, and the group's
      // independent sums interleave
      for (int g = 0; g < nfc; g += kFlushG) {
        const int ng = min(kFlushG, nfc - g);
        double accR[kFlushG], accI[kFlushG];
#pragma unroll
        for (int u = 0; u < kFlushG; ++u) {
          accR[u] = 0.0;
          accI[u] = 0.0;
          if (act && u < ng) {
            const int64_t o = ((int64_t)c * m.nf + f0 + g + u) * cells + pt;
            accR[u] = m.d_re[o];
            accI[u] = m.d_im[o];
          }
        }
        float aR[kFlushG], aI[kFlushG];
#pragma unroll
        for (int u = 0; u < kFlushG; ++u) {
          aR[u] = 0.f;
          aI[u] = 0.f;
        }
        const float2 (*fam)[kFlushF] = sph[isE ? 0 : 1];
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          if (q < ns) {
#pragma unroll
            for (int u = 0; u < kFlushG; ++u) {
              const float2 ph = fam[q][g + u];
              const float co = ph.x, si = ph.y;
              if (CPLX) {
                aR[u] = fmaf(-vi[q], si, fmaf(vr[q], co, aR[u]));
                aI[u] = fmaf(vi[q], co, fmaf(vr[q], si, aI[u]));
              } else {
                aR[u] = fmaf(vr[q], co, aR[u]);
                aI[u] = fmaf(vr[q], si, aI[u]);
              }
            }
          }
        }
#pragma unroll
        for (int u = 0; u < kFlushG; ++u) {
          if (act && u < ng) {
            const int64_t o = ((int64_t)c * m.nf + f0 + g + u) * cells + pt;
            m.d_re[o] = accR[u] + (double)aR[u];
            m.d_im[o] = accI[u] + (double)aI[u];
          }
        }
      }
    }
  }
  // the last block to finish records the folded step: every block read done[0] at its start
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(m.d_count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    if (s_now > *m.d_done) *m.d_done = s_now;
    *m.d_count = 0u;
  }
}

__global__ void k_step_advance(int* step) {
  if (blockIdx.x == 0 && threadIdx.x == 0) ++*step;
}

// Float64 volume-weighted sums for early termination (openem/solver.py:107-121, 160-203),
// one partial per block: [sum V|E|^2, sum V eps |E|^2, sum V |H|^2]. V is the Yee dual volume
// of the E component of the same index (openem/grid.py:350-366); OpenEM weights Hx, Hy, Hz with
// those same three volumes (openem/solver.py:176), and so does this sum.
__global__ void __launch_bounds__(256) k_energy(YeeParams P, const double* dxp, const double* dxd,
                                                const double* dyp, const double* dyd,
                                                const double* dzp, const double* dzd,
                                                double* part) {
  __shared__ double sh[3][256];
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t % P.nz);
    const int64_t r = t / P.nz;
    const int j = (int)(r % P.ny);
    const int i = (int)(r / P.ny);
    const int64_t id = ((int64_t)i * P.ny + j) * P.nzp + k;
    const MatRec& M = P.mats[mat_id(P, id)];
    const double vex = dxp[i] * dyd[j] * dzd[k];
    const double vey = dxd[i] * dyp[j] * dzd[k];
    const double vez = dxd[i] * dyd[j] * dzp[k];
    const double ex = P.f[0][id], ey = P.f[1][id], ez = P.f[2][id];
    const double hx = P.f[3][id], hy = P.f[4][id], hz = P.f[5][id];
    double ax2 = ex * ex, ay2 = ey * ey, az2 = ez * ez;
    double bx2 = hx * hx, by2 = hy * hy, bz2 = hz * hz;
    if (P.cplx) {  // |u|^2 of complex fields
      const double exi = P.fi[0][id], eyi = P.fi[1][id], ezi = P.fi[2][id];
      const double hxi = P.fi[3][id], hyi = P.fi[4][id], hzi = P.fi[5][id];
      ax2 += exi * exi; ay2 += eyi * eyi; az2 += ezi * ezi;
      bx2 += hxi * hxi; by2 += hyi * hyi; bz2 += hzi * hzi;
    }
    const double e0 = vex * ax2, e1 = vey * ay2, e2 = vez * az2;
    s0 += e0 + e1 + e2;
    s1 += e0 * M.eps[0] + e1 * M.eps[1] + e2 * M.eps[2];
    s2 += vex * bx2 + vey * by2 + vez * bz2;  // H weighted like E (openem/solver.py:176)
  }
  sh[0][threadIdx.x] = s0;
  sh[1][threadIdx.x] = s1;
  sh[2][threadIdx.x] = s2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
      sh[2][threadIdx.x] += sh[2][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x + 0] = sh[0][0];
    part[3 * blockIdx.x + 1] = sh[1][0];
    part[3 * blockIdx.x + 2] = sh[2][0];
  }
}

// Copy an unpadded (nx, ny, nz) material index into the padded (nx, ny, nzp) layout, shifted by
// one (0 is the padding material); flags indices >= n_mat.
template <class Tin, class Tout>
__global__ void k_pad_index(const Tin* in, Tout* out, int ny, int nz, int nzp, int64_t total,
                            uint32_t n_mat, unsigned* bad) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t % nzp);
    const int64_t r = t / nzp;
    Tout v = 0;
    if (k < nz) {
      const uint32_t m = (uint32_t)in[r * nz + k];
      if (m >= n_mat) {
        atomicOr(bad, 1u);
      } else {
        v = (Tout)(m + 1);
      }
    }
    out[t] = v;
  }
}

}  // namespace

cudaError_t launch_pad_index(const void* in, int in_bytes, uint16_t* out16, uint32_t* out32,
                             int nx, int ny, int nz, int nzp, uint32_t n_mat, unsigned* bad,
                             cudaStream_t s) {
  const int64_t total = (int64_t)nx * ny * nzp;
  const int nb = (int)std::min<int64_t>((total + 255) / 256, 148 * 64);
  if (in_bytes == 2) {
    const uint16_t* a = static_cast<const uint16_t*>(in);
    if (out16) k_pad_index<<<nb, 256, 0, s>>>(a, out16, ny, nz, nzp, total, n_mat, bad);
    else k_pad_index<<<nb, 256, 0, s>>>(a, out32, ny, nz, nzp, total, n_mat, bad);
  } else {
    const uint32_t* a = static_cast<const uint32_t*>(in);
    if (out16) k_pad_index<<<nb, 256, 0, s>>>(a, out16, ny, nz, nzp, total, n_mat, bad);
    else k_pad_index<<<nb, 256, 0, s>>>(a, out32, ny, nz, nzp, total, n_mat, bad);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------------------------

cudaError_t launch_update_h(const YeeParams& P, cudaStream_t s) {
  dim3 b(32, 4, 1), g(P.nzp / 32, (P.ny + 3) / 4, P.nx);
  k_update_h<<<g, b, 0, s>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_update_e(const YeeParams& P, cudaStream_t s) {
  dim3 b(32, 4, 1), g(P.nzp / 32, (P.ny + 3) / 4, P.nx);
  k_update_e<<<g, b, 0, s>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_plane_h(const YeeParams& P, const PlaneSrc& src, const int* step,
                           cudaStream_t s) {
  dim3 b(32, 8, 1), g((P.ny + 31) / 32, (P.nx + 7) / 8, 1);
  k_plane_h<<<g, b, 0, s>>>(P, src, step);
  return cudaGetLastError();
}

cudaError_t launch_plane_e(const YeeParams& P, const PlaneSrc& src, const int* step,
                           cudaStream_t s) {
  dim3 b(32, 8, 1), g((P.ny + 31) / 32, (P.nx + 7) / 8, 1);
  k_plane_e<<<g, b, 0, s>>>(P, src, step);
  return cudaGetLastError();
}

cudaError_t launch_dipoles(const YeeParams& P, const DipoleSet& d, const int* step,
                           cudaStream_t s, const SnapBoxes* sb) {
  if (d.n_targets == 0) return cudaSuccess;
  SnapBoxes none{};
  const SnapBoxes& b = (sb && !d.magnetic && !d.d_amp_im) ? *sb : none;
  k_dipoles<<<(d.n_targets + 63) / 64, 64, 0, s>>>(P, d, step, b);
  return cudaGetLastError();
}

cudaError_t launch_time_sample(const YeeParams& P, const TimeMon& m, const int* step, int add,
                               cudaStream_t s) {
  dim3 b(32, 4, 1), g((m.nk + 31) / 32, (m.nj + 3) / 4, m.ni);
  k_time_sample<<<g, b, 0, s>>>(P, m, step, add);
  return cudaGetLastError();
}

cudaError_t launch_absorb(const YeeParams& P, const Absorber& a, int is_e, cudaStream_t s) {
  const int box[3] = {a.axis == 0 ? a.nlay : P.nx, a.axis == 1 ? a.nlay : P.ny,
                      a.axis == 2 ? a.nlay : P.nz};
  const int64_t njk = (int64_t)box[1] * box[2];
  dim3 g((unsigned)((njk + 255) / 256), (unsigned)box[0], 1);
  k_absorb<<<g, 256, 0, s>>>(P, a, is_e, box[1], box[2]);
  return cudaGetLastError();
}

// Time-modulated coefficients of step n (openem/kernels/modulation.cu:40-79): eps at t_n and
// t_n+1 from the per-entry phase (cos phi, sin phi) and the step's (cos, sin) of omega t, the
// D-form ca / cb written into the cell's own material record before the E update reads it.
__global__ void k_modulate(YeeParams P, Modulation m, const int* step) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *step;
  if (e >= m.n || n < 0 || n >= m.ntab) return;
  const float4 cs = m.cs[n];
  const float a = m.amp[e], cp = m.cph[e], sp = m.sph[e], es = m.eps[e];
  const float e0 = __fadd_rn(es, __fmul_rn(a, __fadd_rn(__fmul_rn(cs.x, cp), __fmul_rn(cs.y, sp))));
  const float e1 = __fadd_rn(es, __fmul_rn(a, __fadd_rn(__fmul_rn(cs.z, cp), __fmul_rn(cs.w, sp))));
  const float sd = m.sd[e];
  const float den = __fadd_rn(__fadd_rn(e1, sd), m.gg[e]);
  const int64_t id = m.cell[e];
  MatRec& M = m.mats[mat_id(P, id)];
  const int c = m.comp[e];
  M.ca[c] = __fdiv_rn(__fsub_rn(e0, sd), den);
  M.cb[c] = __fdiv_rn(m.dte, den);
}

cudaError_t launch_modulate(const YeeParams& P, const Modulation& m, const int* step,
                            cudaStream_t s) {
  if (m.n <= 0) return cudaSuccess;
  k_modulate<<<(m.n + 127) / 128, 128, 0, s>>>(P, m, step);
  return cudaGetLastError();
}

// Instantaneous colocated flux (openem/readout.py:20-73 with the geometry of
// openem/flux.py:146-164, 534-578): one thread per (plane, sample); the second shot of step
// m = n (kept E^n with H^{n+1/2}) and the first shot of m = n + 1 (E^{n+1} with H^{n+1/2}, E kept)
// each reduce to one block partial; k_flux_time_fold sums the partials in block order.
__device__ __forceinline__ bool ft_slot(const FluxTimeMon& m, int mref, int* slot) {
  const int off = mref - m.beg;
  if (off < 0 || mref >= m.end || off % m.iv) return false;
  *slot = off / m.iv;
  return *slot < m.slots;
}

__device__ __forceinline__ double ft_field(const YeeParams& P, const float* F, int ax, int kn,
                                           int q1, int q2, int t1, int t2) {
  int c[3];
  c[ax] = kn; c[t1] = q1; c[t2] = q2;
  return (double)F[((int64_t)c[0] * P.ny + c[1]) * P.nzp + c[2]];
}

__global__ void __launch_bounds__(256) k_flux_time(YeeParams P, FluxTimeMon m, const int* step) {
  const int n = *step;
  int slot1, slot0;
  const bool s1 = ft_slot(m, n, &slot1), s0 = ft_slot(m, n + 1, &slot0);
  if (!s1 && !s0) return;  // uniform over the grid
  const int t1 = m.axis == 0 ? 1 : 0, t2 = m.axis == 2 ? 1 : 2;
  const int64_t per = (int64_t)m.n1 * m.n2, total = per * m.nplanes;
  double c1 = 0.0, c0 = 0.0;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(q / per);
    const int64_t r = q - p * per;
    const int u = (int)(r / m.n2), v = (int)(r - (int64_t)u * m.n2);
    const int kh = m.kh[p];
    const double h0 = m.wh[p][0], h1 = m.wh[p][1];
    const float* Ht1 = P.f[3 + t1];
    const float* Ht2 = P.f[3 + t2];
    // H_t2 along t1 (cells lo1 / hi1 at edge e2), H_t1 along t2 (cells lo2 / hi2 at edge e1)
    auto hnorm = [&](const float* H, int q1, int q2) {
      return h0 * ft_field(P, H, m.axis, kh, q1, q2, t1, t2) +
             h1 * ft_field(P, H, m.axis, kh + 1, q1, q2, t1, t2);
    };
    const double hv = m.wlo1[m.n1 + u] * hnorm(Ht2, m.lo1[u], m.e2[v]) +
                      m.whi1[u] * hnorm(Ht2, m.hi1[u], m.e2[v]);
    const double hu = m.wlo2[m.n2 + v] * hnorm(Ht1, m.e1[u], m.lo2[v]) +
                      m.whi2[v] * hnorm(Ht1, m.e1[u], m.hi2[v]);
    const double wd = 0.5 * m.w[p] * m.dS[r];
    double* keep = m.ekeep + ((int64_t)p * 2) * per + r;
    if (s1) c1 += wd * (keep[0] * hv - keep[per] * hu);
    if (s0) {
      const int ke = m.ke[p];
      const double eu = m.wlo1[u] * ft_field(P, P.f[t1], m.axis, ke, m.lo1[u], m.e2[v], t1, t2) +
                        m.whi1[u] * ft_field(P, P.f[t1], m.axis, ke, m.hi1[u], m.e2[v], t1, t2);
      const double ev = m.wlo2[v] * ft_field(P, P.f[t2], m.axis, ke, m.e1[u], m.lo2[v], t1, t2) +
                        m.whi2[v] * ft_field(P, P.f[t2], m.axis, ke, m.e1[u], m.hi2[v], t1, t2);
      keep[0] = eu;
      keep[per] = ev;
      c0 += wd * (eu * hv - ev * hu);
    }
  }
  // block reduction in a fixed order
  __shared__ double red[2][8];
  for (int o = 16; o > 0; o >>= 1) {
    c1 += __shfl_down_sync(0xffffffffu, c1, o);
    c0 += __shfl_down_sync(0xffffffffu, c0, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { red[0][w] = c1; red[1][w] = c0; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += red[0][k]; b += red[1][k]; }
    m.part[2 * blockIdx.x] = a;
    m.part[2 * blockIdx.x + 1] = b;
  }
}

__global__ void k_flux_time_fold(FluxTimeMon m, const int* step) {
  const int n = *step;
  int slot1, slot0;
  const bool s1 = ft_slot(m, n, &slot1), s0 = ft_slot(m, n + 1, &slot0);
  if (threadIdx.x != 0 || (!s1 && !s0)) return;
  double a = 0.0, b = 0.0;
  for (int k = 0; k < m.nblocks; ++k) { a += m.part[2 * k]; b += m.part[2 * k + 1]; }
  if (s1) m.buf[slot1] += a;  // the second shot completes slot m = n
  if (s0) m.buf[slot0] = b;   // the first shot opens slot m = n + 1
}

cudaError_t launch_flux_time(const YeeParams& P, const FluxTimeMon& m, const int* step,
                             cudaStream_t s) {
  k_flux_time<<<m.nblocks, 256, 0, s>>>(P, m, step);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_flux_time_fold<<<1, 32, 0, s>>>(m, step);
  return cudaGetLastError();
}

// TFSF box face corrections (openem/kernels/tfsf.cu:31-86): one thread per point of a group of
// faces that touch disjoint cells; the table row of the step interpolated at the point's column.
__global__ void k_tfsf(YeeParams P, const oem_tfsf_face* faces, const int64_t* ofs, int nfaces,
                       int64_t total, const double* tab, int rows, int row_n, const int* step,
                       int is_e) {
  const int n = *step;
  if (n < 0 || n >= rows) return;
  const double* row = tab + (int64_t)n * row_n;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int f = 0;
    while (f + 1 < nfaces && t >= ofs[f + 1]) ++f;
    const oem_tfsf_face& F = faces[f];
    const int64_t r = t - ofs[f];
    const int p = (int)(r / F.nq), q = (int)(r - (int64_t)p * F.nq);
    const double pos = F.c0 + F.cp * (double)p + F.cq * (double)q;
    int i0 = (int)floor(pos);
    double w = pos - (double)i0;
    if (i0 < 0) { i0 = 0; w = 0.0; }
    else if (i0 >= row_n - 1) { i0 = row_n - 1; w = 0.0; }
    const int i1 = i0 + 1 < row_n ? i0 + 1 : i0;
    const float val = (float)(row[i0] + w * (row[i1] - row[i0]));
    const int64_t id = F.base + (int64_t)p * F.sp + (int64_t)q * F.sq;
    float* Fd = P.f[F.comp];
    if (is_e) {
      const float cb = P.mats[mat_id(P, id)].cb[F.comp];
      Fd[id] = __fadd_rn(Fd[id], __fmul_rn(__fmul_rn(cb, F.coef), val));
    } else {
      Fd[id] = __fadd_rn(Fd[id], __fmul_rn(F.coef, val));
    }
  }
}

cudaError_t launch_tfsf(const YeeParams& P, const Tfsf& t, int is_e, const int* step,
                        cudaStream_t s) {
  const auto& groups = is_e ? t.e_groups : t.h_groups;
  const auto& points = is_e ? t.e_points : t.h_points;
  const oem_tfsf_face* faces = is_e ? t.e_faces : t.h_faces;
  const int64_t* ofs = is_e ? t.e_ofs : t.h_ofs;
  for (size_t g = 0; g < groups.size(); ++g) {
    const int64_t total = points[g];
    if (total <= 0) continue;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
    const int first = groups[g].first;
    k_tfsf<<<blocks, 256, 0, s>>>(P, faces + first, ofs + first + (int64_t)g, groups[g].second,
                                  total, is_e ? t.hy_tab : t.ex_tab, is_e ? t.hy_rows : t.ex_rows,
                                  is_e ? t.hy_n : t.ex_n, step, is_e);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Fully anisotropic cells (openem/kernels/tensor.cu:49-135): out = wbase base + M_row <F>,
// the other two components averaged over the 4 neighbours {cell, +1 along a} x {cell, -1 along
// b} with the boundary masks. First pass: rhs = M1 <E^n> (before the E update); second pass:
// enew = rhs + M2 <c>, c the curl the passthrough cells hold after the E-side injection.
__global__ void k_tensor_dot(YeeParams P, TensorSet t, int second) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= t.n) return;
  const int a = t.comp[e];
  const int64_t id = t.cell[e];
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const int c0[3] = {(int)(id / si), (int)((id / sj) % P.ny), (int)(id % sj)};
  const float* m = (second ? t.m2 : t.m1) + 3 * (int64_t)e;
  float acc = second ? t.rhs[e] : 0.0f;
  acc = __fadd_rn(acc, __fmul_rn(m[a], P.f[a][id]));
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    const DevAxis& A = P.ax[a];
    const DevAxis& B = P.ax[b];
    int ca[3] = {c0[0], c0[1], c0[2]};
    ca[a] = A.nxt[c0[a]];
    int cb[3] = {c0[0], c0[1], c0[2]};
    cb[b] = B.prv[c0[b]];
    int cab[3] = {ca[0], ca[1], ca[2]};
    cab[b] = cb[b];
    const float wa = A.mnx[c0[a]], wb = B.mpv[c0[b]];
    const float* F = P.f[b];
    auto at = [&](const int* c) { return F[c[0] * si + c[1] * sj + c[2]]; };
    float sum = __fadd_rn(at(c0), __fmul_rn(wa, at(ca)));
    sum = __fadd_rn(sum, __fmul_rn(wb, at(cb)));
    sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(wa, wb), at(cab)));
    acc = __fadd_rn(acc, __fmul_rn(m[b], __fmul_rn(0.25f, sum)));
  }
  (second ? t.enew : t.rhs)[e] = acc;
}

// Write E^{n+1} of the entries (times the PEC-wall factor of the other two axes).
__global__ void k_tensor_scatter(YeeParams P, TensorSet t) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= t.n) return;
  P.f[t.comp[e]][t.cell[e]] = __fmul_rn(t.enew[e], t.pec[e]);
}

cudaError_t launch_tensor_pre(const YeeParams& P, const TensorSet& t, cudaStream_t s) {
  if (t.n <= 0) return cudaSuccess;
  k_tensor_dot<<<(t.n + 127) / 128, 128, 0, s>>>(P, t, 0);
  return cudaGetLastError();
}

cudaError_t launch_tensor_post(const YeeParams& P, const TensorSet& t, cudaStream_t s) {
  if (t.n <= 0) return cudaSuccess;
  k_tensor_dot<<<(t.n + 127) / 128, 128, 0, s>>>(P, t, 1);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_tensor_scatter<<<(t.n + 127) / 128, 128, 0, s>>>(P, t);
  return cudaGetLastError();
}

// Slanted-interface cells, first pass (openem/kernels/dispersion_mix.cu:41-85): both pole
// branches advance to the half step, the arithmetic one driven by E^n, the harmonic one by
// d_h^n; SP = sum 2 Re(P_half), SQ = sum Re(Q_half).
__global__ void k_mix_pre(YeeParams P, MixSet m) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n) return;
  const float en = P.f[m.comp[e]][m.cell[e]];
  const float dh = m.dh[e];
  float s = 0.0f;
  for (int t = m.p_ofs[e]; t < m.p_ofs[e + 1]; ++t) {
    const float4 c = m.pc[t];
    float2 p = m.P[t];
    const float dr = __fadd_rn(__fsub_rn(__fmul_rn(c.x, p.x), __fmul_rn(c.y, p.y)),
                               __fmul_rn(c.z, en));
    const float di = __fadd_rn(__fadd_rn(__fmul_rn(c.x, p.y), __fmul_rn(c.y, p.x)),
                               __fmul_rn(c.w, en));
    p.x = __fadd_rn(p.x, dr);
    p.y = __fadd_rn(p.y, di);
    m.P[t] = p;
    s = __fadd_rn(s, __fmul_rn(2.0f, p.x));
  }
  m.sp[e] = s;
  s = 0.0f;
  for (int t = m.q_ofs[e]; t < m.q_ofs[e + 1]; ++t) {
    const float4 c = m.qc[t];
    float2 q = m.Q[t];
    const float dr = __fadd_rn(__fsub_rn(__fmul_rn(c.x, q.x), __fmul_rn(c.y, q.y)),
                               __fmul_rn(c.z, dh));
    const float di = __fadd_rn(__fadd_rn(__fmul_rn(c.x, q.y), __fmul_rn(c.y, q.x)),
                               __fmul_rn(c.w, dh));
    q.x = __fadd_rn(q.x, dr);
    q.y = __fadd_rn(q.y, di);
    m.Q[t] = q;
    s = __fadd_rn(s, q.x);
  }
  m.sq[e] = s;
}

// Second pass (openem/kernels/dispersion_mix.cu:87-135): the E array holds the pass-through
// value (stretched curl, minus J, plus the E-side sources); d_tot advances by dt/eps0 times it,
// the scalar equation gives d_h^{n+1} = (d_tot - k1 SQ - (1 - beta) SP) / (k1 k2 + beta),
// E^{n+1} = k2 d_h + SQ, and both branches take their step-(n+1) terms.
__global__ void k_mix_post(YeeParams P, MixSet m) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n) return;
  float* F = P.f[m.comp[e]];
  const int64_t id = m.cell[e];
  const float dt_new = __fadd_rn(m.dtot[e], __fmul_rn(m.dte, F[id]));
  m.dtot[e] = dt_new;
  const float4 k = m.k[e];
  const float dh = __fmul_rn(
      __fsub_rn(__fsub_rn(dt_new, __fmul_rn(k.x, m.sq[e])), __fmul_rn(k.z, m.sp[e])), k.w);
  m.dh[e] = dh;
  const float en = __fadd_rn(__fmul_rn(k.y, dh), m.sq[e]);
  for (int t = m.p_ofs[e]; t < m.p_ofs[e + 1]; ++t) {
    const float4 c = m.pc[t];
    float2 p = m.P[t];
    p.x = __fadd_rn(p.x, __fmul_rn(c.z, en));
    p.y = __fadd_rn(p.y, __fmul_rn(c.w, en));
    m.P[t] = p;
  }
  for (int t = m.q_ofs[e]; t < m.q_ofs[e + 1]; ++t) {
    const float4 c = m.qc[t];
    float2 q = m.Q[t];
    q.x = __fadd_rn(q.x, __fmul_rn(c.z, dh));
    q.y = __fadd_rn(q.y, __fmul_rn(c.w, dh));
    m.Q[t] = q;
  }
  F[id] = en;
}

cudaError_t launch_mix_pre(const YeeParams& P, const MixSet& m, cudaStream_t s) {
  if (m.n <= 0) return cudaSuccess;
  k_mix_pre<<<(m.n + 127) / 128, 128, 0, s>>>(P, m);
  return cudaGetLastError();
}

cudaError_t launch_mix_post(const YeeParams& P, const MixSet& m, cudaStream_t s) {
  if (m.n <= 0) return cudaSuccess;
  k_mix_post<<<(m.n + 127) / 128, 128, 0, s>>>(P, m);
  return cudaGetLastError();
}

cudaError_t launch_snapshot(const YeeParams& P, const Monitor& m, const int* step,
                            cudaStream_t s) {
  if (m.kind != 0) return cudaErrorInvalidValue;  // boxes: launch_snapshot_boxes
  dim3 b(32, 4, 1), g((m.n2 + 31) / 32, (m.n1 + 3) / 4, 1);
  k_snap_plane<<<g, b, 0, s>>>(P, m, step);
  return cudaGetLastError();
}

cudaError_t launch_snapshot_boxes(const YeeParams& P, const Monitor* const* boxes, int n,
                                  const int* step, cudaStream_t s) {
  for (int g0 = 0; g0 < n; g0 += kMaxBoxSnap) {
    BoxSnapSet S;
    S.n = std::min(kMaxBoxSnap, n - g0);
    int64_t total = 0;
    for (int q = 0; q < S.n; ++q) {
      const Monitor& m = *boxes[g0 + q];
      const int64_t njk = (int64_t)m.nj * m.nk;
      if (njk >= (1LL << 31)) return cudaErrorInvalidValue;  // one box plane per 32-bit index
      S.m[q] = m;
      S.cb[q] = (uint32_t)((njk + 255) / 256);
      S.blk0[q] = (uint32_t)total;
      total += (int64_t)m.ni * S.cb[q];
      if (total >= (1LL << 31)) return cudaErrorInvalidValue;
    }
    S.blk0[S.n] = (uint32_t)total;
    k_snap_boxes<<<(unsigned)total, 256, 0, s>>>(P, S, step);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_flush(const Monitor& m, const int* step, int forced, cudaStream_t s) {
  const int64_t nb = std::min<int64_t>(((int64_t)m.ncomp * m.cells + 127) / 128, 148 * 4);
  if (m.T > 32) return cudaErrorInvalidValue;  // a thread holds at most 32 rows
  if (m.cplx) {
    if (m.ncomp == 4)
      k_flush<4, true><<<(unsigned)nb, 128, 0, s>>>(m, step, forced);
    else
      k_flush<6, true><<<(unsigned)nb, 128, 0, s>>>(m, step, forced);
  } else if (m.ncomp == 4) {
    k_flush<4, false><<<(unsigned)nb, 128, 0, s>>>(m, step, forced);
  } else {
    k_flush<6, false><<<(unsigned)nb, 128, 0, s>>>(m, step, forced);
  }
  return cudaGetLastError();
}

// (re, im) pairs of n values side by side: the layout of a host complex128 array. Values with
// a non-finite part are counted into *bad (one atomic per warp that saw any), so the host need
// not scan the readout for them.
__global__ void k_interleave(const double* __restrict__ re, const double* __restrict__ im,
                             double2* __restrict__ out, int64_t n, unsigned long long* bad) {
  unsigned cnt = 0;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const double a = re[q], b = im[q];
    cnt += (isfinite(a) && isfinite(b)) ? 0u : 1u;
    out[q] = make_double2(a, b);
  }
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  if (cnt && (threadIdx.x & 31) == 0) atomicAdd(bad, (unsigned long long)cnt);
}

cudaError_t launch_interleave(const double* re, const double* im, double2* out, int64_t n,
                              unsigned long long* bad, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int64_t nb = std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_interleave<<<(unsigned)nb, 256, 0, s>>>(re, im, out, n, bad);
  return cudaGetLastError();
}

cudaError_t launch_step_advance(int* step, cudaStream_t s) {
  k_step_advance<<<1, 32, 0, s>>>(step);
  return cudaGetLastError();
}

int energy_block_count(const YeeParams& P) {
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  int64_t nb = (n + 255) / 256;
  if (nb > kEnergyMaxBlocks) nb = kEnergyMaxBlocks;
  return (int)(nb < 1 ? 1 : nb);
}

cudaError_t launch_energy(const YeeParams& P, double* const dl[3][2], double* part, int nblocks,
                          cudaStream_t s) {
  k_energy<<<nblocks, 256, 0, s>>>(P, dl[0][0], dl[0][1], dl[1][0], dl[1][1], dl[2][0],
                                   dl[2][1], part);
  return cudaGetLastError();
}

}  // namespace oem
