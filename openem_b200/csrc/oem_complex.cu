// Complex-field (Bloch) Yee updates and the mode-source injection of both paths.
//
// A complex plan carries every field and CPML psi as a real and an imaginary float32 array. The
// spacings, CPML coefficients and material coefficients are real, so the update of each part is
// the real update; the complex phase enters only through the neighbour masks, which are
// exp(+-i 2 pi k) at the periodic seam of a Bloch axis (openem/kernels/bloch.cu:1-221). The
// masked neighbour is formed as (n_re m_re - n_im m_im, n_re m_im + n_im m_re) with
// round-to-nearest intrinsics: with m_im = 0 that is n m exactly, so at k = 0 each part follows
// the real path bit for bit.
//
// One thread per cell (block 32 x 4 over (k, j), one grid z slice per x plane).
#include <cuda_runtime.h>
#include <stdint.h>

#include "oem_arith.cuh"
#include "oem_internal.cuh"

namespace oem {

namespace {

__device__ __forceinline__ float* psi_ptr(const PsiSet& S, int a, int slot, const DevAxis& A,
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

// CPML of both parts (the coefficients are real): psi_re / psi_im at the same slab position.
__device__ __forceinline__ void stretch_c(float& dr, float& di, float* pr, float* pi, float a,
                                          float b, float ik) {
  if (pr == nullptr) return;
  dr = cpml_stretch(dr, *pr, a, b, ik);
  di = cpml_stretch(di, *pi, a, b, ik);
}

// masked neighbour n * m
__device__ __forceinline__ void cmask(float nr, float ni, float mr, float mi, float& outr,
                                      float& outi) {
  outr = __fsub_rn(__fmul_rn(nr, mr), __fmul_rn(ni, mi));
  outi = __fadd_rn(__fmul_rn(nr, mi), __fmul_rn(ni, mr));
}

__device__ __forceinline__ uint32_t mat_of(const YeeParams& P, int64_t id) {
  return P.mat16 ? (uint32_t)P.mat16[id] : P.mat32[id];
}

// H half step (openem/kernels/bloch.cu:38-126)
__global__ void __launch_bounds__(128) k_update_h_c(YeeParams P) {
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
  const float mir = X.mnx[i], mii = X.mnx_i[i];
  const float mjr = Y.mnx[j], mji = Y.mnx_i[j];
  const float mkr = Z.mnx[k], mki = Z.mnx_i[k];
  const int64_t idi = ip * si + j * sj + k;
  const int64_t idj = i * si + jp * sj + k;
  const int64_t idk = i * si + j * sj + kp;
  const float ch = P.ch;
  const float *Er[3] = {P.f[0], P.f[1], P.f[2]}, *Ei[3] = {P.fi[0], P.fi[1], P.fi[2]};
  // forward differences of (component c along axis a with neighbour index nb, mask m)
  auto fd = [&](int c, int64_t nb, float mr, float mi, float idl, float& dr, float& di) {
    float nr, ni;
    cmask(Er[c][nb], Ei[c][nb], mr, mi, nr, ni);
    dr = __fmul_rn(__fsub_rn(nr, Er[c][id]), idl);
    di = __fmul_rn(__fsub_rn(ni, Ei[c][id]), idl);
  };
  {  // Hx: -(dEz/dy - dEy/dz)
    float syr, syi, szr, szi;
    fd(2, idj, mjr, mji, Y.idl_p[j], syr, syi);
    fd(1, idk, mkr, mki, Z.idl_p[k], szr, szi);
    stretch_c(syr, syi, psi_ptr(P.psih, 1, 0, Y, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psih_i, 1, 0, Y, i, j, k, P.ny, P.nzp), Y.ah[j], Y.bh[j], Y.kh[j]);
    stretch_c(szr, szi, psi_ptr(P.psih, 2, 0, Z, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psih_i, 2, 0, Z, i, j, k, P.ny, P.nzp), Z.ah[k], Z.bh[k], Z.kh[k]);
    P.f[3][id] = h_new(P.f[3][id], ch, syr, szr);
    P.fi[3][id] = h_new(P.fi[3][id], ch, syi, szi);
  }
  {  // Hy: -(dEx/dz - dEz/dx)
    float szr, szi, sxr, sxi;
    fd(0, idk, mkr, mki, Z.idl_p[k], szr, szi);
    fd(2, idi, mir, mii, X.idl_p[i], sxr, sxi);
    stretch_c(szr, szi, psi_ptr(P.psih, 2, 1, Z, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psih_i, 2, 1, Z, i, j, k, P.ny, P.nzp), Z.ah[k], Z.bh[k], Z.kh[k]);
    stretch_c(sxr, sxi, psi_ptr(P.psih, 0, 0, X, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psih_i, 0, 0, X, i, j, k, P.ny, P.nzp), X.ah[i], X.bh[i], X.kh[i]);
    P.f[4][id] = h_new(P.f[4][id], ch, szr, sxr);
    P.fi[4][id] = h_new(P.fi[4][id], ch, szi, sxi);
  }
  {  // Hz: -(dEy/dx - dEx/dy)
    float sxr, sxi, syr, syi;
    fd(1, idi, mir, mii, X.idl_p[i], sxr, sxi);
    fd(0, idj, mjr, mji, Y.idl_p[j], syr, syi);
    stretch_c(sxr, sxi, psi_ptr(P.psih, 0, 1, X, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psih_i, 0, 1, X, i, j, k, P.ny, P.nzp), X.ah[i], X.bh[i], X.kh[i]);
    stretch_c(syr, syi, psi_ptr(P.psih, 1, 1, Y, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psih_i, 1, 1, Y, i, j, k, P.ny, P.nzp), Y.ah[j], Y.bh[j], Y.kh[j]);
    P.f[5][id] = h_new(P.f[5][id], ch, sxr, syr);
    P.fi[5][id] = h_new(P.fi[5][id], ch, sxi, syi);
  }
}

// E full step of the lossless, non-dispersive complex subset (openem/kernels/bloch.cu:128-221)
__global__ void __launch_bounds__(128) k_update_e_c(YeeParams P) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= P.nz || j >= P.ny) return;
  const int64_t sj = P.nzp, si = (int64_t)P.ny * P.nzp;
  const int64_t id = i * si + j * sj + k;
  const DevAxis& X = P.ax[0];
  const DevAxis& Y = P.ax[1];
  const DevAxis& Z = P.ax[2];
  const int im = X.prv[i], jm = Y.prv[j], km = Z.prv[k];
  const float mir = X.mpv[i], mii = X.mpv_i[i];
  const float mjr = Y.mpv[j], mji = Y.mpv_i[j];
  const float mkr = Z.mpv[k], mki = Z.mpv_i[k];
  const int64_t idi = im * si + j * sj + k;
  const int64_t idj = i * si + jm * sj + k;
  const int64_t idk = i * si + j * sj + km;
  const MatRec& M = P.mats[mat_of(P, id)];
  const float cw = P.cw;
  const float *Hr[3] = {P.f[3], P.f[4], P.f[5]}, *Hi[3] = {P.fi[3], P.fi[4], P.fi[5]};
  auto bd = [&](int c, int64_t nb, float mr, float mi, float idl, float& dr, float& di) {
    float nr, ni;
    cmask(Hr[c][nb], Hi[c][nb], mr, mi, nr, ni);
    dr = __fmul_rn(__fsub_rn(Hr[c][id], nr), idl);
    di = __fmul_rn(__fsub_rn(Hi[c][id], ni), idl);
  };
  {  // Ex: dHz/dy - dHy/dz
    float syr, syi, szr, szi;
    bd(2, idj, mjr, mji, Y.idl_d[j], syr, syi);
    bd(1, idk, mkr, mki, Z.idl_d[k], szr, szi);
    stretch_c(syr, syi, psi_ptr(P.psie, 1, 0, Y, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psie_i, 1, 0, Y, i, j, k, P.ny, P.nzp), Y.ae[j], Y.be[j], Y.ke[j]);
    stretch_c(szr, szi, psi_ptr(P.psie, 2, 0, Z, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psie_i, 2, 0, Z, i, j, k, P.ny, P.nzp), Z.ae[k], Z.be[k], Z.ke[k]);
    P.f[0][id] = e_new(M.ca[0], P.f[0][id], M.cb[0], syr, szr, cw, 0.f);
    P.fi[0][id] = e_new(M.ca[0], P.fi[0][id], M.cb[0], syi, szi, cw, 0.f);
  }
  {  // Ey: dHx/dz - dHz/dx
    float szr, szi, sxr, sxi;
    bd(0, idk, mkr, mki, Z.idl_d[k], szr, szi);
    bd(2, idi, mir, mii, X.idl_d[i], sxr, sxi);
    stretch_c(szr, szi, psi_ptr(P.psie, 2, 1, Z, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psie_i, 2, 1, Z, i, j, k, P.ny, P.nzp), Z.ae[k], Z.be[k], Z.ke[k]);
    stretch_c(sxr, sxi, psi_ptr(P.psie, 0, 0, X, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psie_i, 0, 0, X, i, j, k, P.ny, P.nzp), X.ae[i], X.be[i], X.ke[i]);
    P.f[1][id] = e_new(M.ca[1], P.f[1][id], M.cb[1], szr, sxr, cw, 0.f);
    P.fi[1][id] = e_new(M.ca[1], P.fi[1][id], M.cb[1], szi, sxi, cw, 0.f);
  }
  {  // Ez: dHy/dx - dHx/dy
    float sxr, sxi, syr, syi;
    bd(1, idi, mir, mii, X.idl_d[i], sxr, sxi);
    bd(0, idj, mjr, mji, Y.idl_d[j], syr, syi);
    stretch_c(sxr, sxi, psi_ptr(P.psie, 0, 1, X, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psie_i, 0, 1, X, i, j, k, P.ny, P.nzp), X.ae[i], X.be[i], X.ke[i]);
    stretch_c(syr, syi, psi_ptr(P.psie, 1, 1, Y, i, j, k, P.ny, P.nzp),
              psi_ptr(P.psie_i, 1, 1, Y, i, j, k, P.ny, P.nzp), Y.ae[j], Y.be[j], Y.ke[j]);
    P.f[2][id] = e_new(M.ca[2], P.f[2][id], M.cb[2], sxr, syr, cw, 0.f);
    P.fi[2][id] = e_new(M.ca[2], P.fi[2][id], M.cb[2], sxi, syi, cw, 0.f);
  }
}

// Bloch seam terms of the split complex update. Away from a Bloch seam the real and the
// imaginary parts follow the real update with the same (real) coefficients, so the
// warp-specialised real kernels update each part with the real part m_re of the neighbour
// masks. At a seam face the complex product n m adds -n_im m_im to the real part and
// +n_re m_im to the imaginary part of a forward difference (the negatives for a backward one);
// these kernels add those terms, times the update's coefficient, to the components whose
// derivative along the seam axis they enter (a Bloch axis carries no CPML, so the derivative
// enters unstretched). Per axis a, the (updated component, differentiated component, sign of
// the coefficient) pairs follow the curl of k_update_h_c / k_update_e_c.
__device__ __forceinline__ int64_t seam_cell(const YeeParams& P, int a, int q, int t, int* c) {
  const int u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;
  const int nv = v == 1 ? P.ny : P.nz;
  c[a] = q;
  c[u] = t / nv;
  c[v] = t - c[u] * nv;
  return ((int64_t)c[0] * P.ny + c[1]) * P.nzp + c[2];
}

__global__ void k_seam_h(YeeParams P, int a, int q) {
  const int u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;
  const int nu = u == 0 ? P.nx : P.ny, nv = v == 1 ? P.ny : P.nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nu * nv) return;
  int c[3];
  const int64_t id = seam_cell(P, a, q, t, c);
  const DevAxis& A = P.ax[a];
  c[a] = A.nxt[q];
  const int64_t nb = ((int64_t)c[0] * P.ny + c[1]) * P.nzp + c[2];
  const float mi = A.mnx_i[q], idl = A.idl_p[q];
  // (H component, E component, sign of ch)
  const int tab[3][2][3] = {{{4, 2, 1}, {5, 1, -1}}, {{3, 2, -1}, {5, 0, 1}}, {{3, 1, 1}, {4, 0, -1}}};
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int h = tab[a][r][0], e = tab[a][r][1];
    const float g = tab[a][r][2] > 0 ? P.ch : -P.ch;
    const float ddr = __fmul_rn(__fmul_rn(-P.fi[e][nb], mi), idl);
    const float ddi = __fmul_rn(__fmul_rn(P.f[e][nb], mi), idl);
    P.f[h][id] = __fmaf_rn(g, ddr, P.f[h][id]);
    P.fi[h][id] = __fmaf_rn(g, ddi, P.fi[h][id]);
  }
}

__global__ void k_seam_e(YeeParams P, int a, int q) {
  const int u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;
  const int nu = u == 0 ? P.nx : P.ny, nv = v == 1 ? P.ny : P.nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nu * nv) return;
  int c[3];
  const int64_t id = seam_cell(P, a, q, t, c);
  const DevAxis& A = P.ax[a];
  c[a] = A.prv[q];
  const int64_t nb = ((int64_t)c[0] * P.ny + c[1]) * P.nzp + c[2];
  const float mi = A.mpv_i[q], idl = A.idl_d[q];
  const MatRec& M = P.mats[mat_of(P, id)];
  // (E component, H component, sign of cb)
  const int tab[3][2][3] = {{{1, 5, -1}, {2, 4, 1}}, {{0, 5, 1}, {2, 3, -1}}, {{0, 4, -1}, {1, 3, 1}}};
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int e = tab[a][r][0], h = tab[a][r][1];
    const float g = tab[a][r][2] > 0 ? M.cb[e] : -M.cb[e];
    const float ddr = __fmul_rn(__fmul_rn(P.fi[h][nb], mi), idl);
    const float ddi = __fmul_rn(__fmul_rn(-P.f[h][nb], mi), idl);
    P.f[e][id] = __fmaf_rn(g, ddr, P.f[e][id]);
    P.fi[e][id] = __fmaf_rn(g, ddi, P.fi[e][id]);
  }
}

// Padded index of plane cell (o1, o2) of a mode plane along `axis` (tangential pair in cyclic
// order: axis 0 -> (y, z), 1 -> (z, x), 2 -> (x, y)).
__device__ __forceinline__ int64_t plane_cell(const YeeParams& P, int axis, int kp, int o1,
                                              int o2) {
  if (axis == 0) return ((int64_t)kp * P.ny + o1) * P.nzp + o2;
  if (axis == 1) return ((int64_t)o2 * P.ny + kp) * P.nzp + o1;
  return ((int64_t)o1 * P.ny + o2) * P.nzp + kp;
}

// Mode source, H side (openem/kernels/source_dft.cu:84-105, bloch.cu:326-350): the E profiles
// times amp(n dt). H_t1 += c_h1 * (E_t2 amp), H_t2 += c_h2 * (E_t1 amp); the real path adds the
// real part, a complex plan both parts. Terms (base profile, broadband corrections) are added
// in order.
__global__ void k_mode_h(YeeParams P, ModeSrc m, const int* step) {
  const int o2 = blockIdx.x * blockDim.x + threadIdx.x;
  const int o1 = blockIdx.y * blockDim.y + threadIdx.y;
  const int n = *step;
  if (o1 >= m.n1 || o2 >= m.n2 || n < 0 || n >= m.ntab) return;
  const int t1 = (m.axis + 1) % 3, t2 = (m.axis + 2) % 3;
  const int64_t id = plane_cell(P, m.axis, m.kh, o1, o2);
  const int64_t plane = (int64_t)m.n1 * m.n2;
  const int64_t o = (int64_t)o1 * m.n2 + o2;
  float h1r = P.f[3 + t1][id], h2r = P.f[3 + t2][id];
  float h1i = P.cplx ? P.fi[3 + t1][id] : 0.f, h2i = P.cplx ? P.fi[3 + t2][id] : 0.f;
  for (int q = 0; q < m.nterms; ++q) {
    const float* pr = m.d_prof + (int64_t)q * 8 * plane;
    const float e1r = pr[o], e1i = pr[plane + o], e2r = pr[2 * plane + o], e2i = pr[3 * plane + o];
    const float ar = (float)m.d_amp_e[2 * ((int64_t)q * m.ntab + n)];
    const float ai = (float)m.d_amp_e[2 * ((int64_t)q * m.ntab + n) + 1];
    h1r = __fadd_rn(h1r, __fmul_rn(m.ch1, __fsub_rn(__fmul_rn(e2r, ar), __fmul_rn(e2i, ai))));
    h2r = __fadd_rn(h2r, __fmul_rn(m.ch2, __fsub_rn(__fmul_rn(e1r, ar), __fmul_rn(e1i, ai))));
    if (P.cplx) {
      h1i = __fadd_rn(h1i, __fmul_rn(m.ch1, __fadd_rn(__fmul_rn(e2r, ai), __fmul_rn(e2i, ar))));
      h2i = __fadd_rn(h2i, __fmul_rn(m.ch2, __fadd_rn(__fmul_rn(e1r, ai), __fmul_rn(e1i, ar))));
    }
  }
  P.f[3 + t1][id] = h1r;
  P.f[3 + t2][id] = h2r;
  if (P.cplx) {
    P.fi[3 + t1][id] = h1i;
    P.fi[3 + t2][id] = h2i;
  }
}

// Mode source, E side (openem/kernels/source_dft.cu:108-128, bloch.cu:352-384): the H
// profiles times amp((n + 1/2) dt), scaled by the cell's cb.
__global__ void k_mode_e(YeeParams P, ModeSrc m, const int* step) {
  const int o2 = blockIdx.x * blockDim.x + threadIdx.x;
  const int o1 = blockIdx.y * blockDim.y + threadIdx.y;
  const int n = *step;
  if (o1 >= m.n1 || o2 >= m.n2 || n < 0 || n >= m.ntab) return;
  const int t1 = (m.axis + 1) % 3, t2 = (m.axis + 2) % 3;
  const int64_t id = plane_cell(P, m.axis, m.ks, o1, o2);
  const int64_t plane = (int64_t)m.n1 * m.n2;
  const int64_t o = (int64_t)o1 * m.n2 + o2;
  const MatRec& M = P.mats[mat_of(P, id)];
  const float c1 = __fmul_rn(M.cb[t1], m.ce1), c2 = __fmul_rn(M.cb[t2], m.ce2);
  float e1r = P.f[t1][id], e2r = P.f[t2][id];
  float e1i = P.cplx ? P.fi[t1][id] : 0.f, e2i = P.cplx ? P.fi[t2][id] : 0.f;
  for (int q = 0; q < m.nterms; ++q) {
    const float* pr = m.d_prof + (int64_t)q * 8 * plane + 4 * plane;
    const float h1r = pr[o], h1i = pr[plane + o], h2r = pr[2 * plane + o], h2i = pr[3 * plane + o];
    const float ar = (float)m.d_amp_h[2 * ((int64_t)q * m.ntab + n)];
    const float ai = (float)m.d_amp_h[2 * ((int64_t)q * m.ntab + n) + 1];
    e1r = __fadd_rn(e1r, __fmul_rn(c1, __fsub_rn(__fmul_rn(h2r, ar), __fmul_rn(h2i, ai))));
    e2r = __fadd_rn(e2r, __fmul_rn(c2, __fsub_rn(__fmul_rn(h1r, ar), __fmul_rn(h1i, ai))));
    if (P.cplx) {
      e1i = __fadd_rn(e1i, __fmul_rn(c1, __fadd_rn(__fmul_rn(h2r, ai), __fmul_rn(h2i, ar))));
      e2i = __fadd_rn(e2i, __fmul_rn(c2, __fadd_rn(__fmul_rn(h1r, ai), __fmul_rn(h1i, ar))));
    }
  }
  P.f[t1][id] = e1r;
  P.f[t2][id] = e2r;
  if (P.cplx) {
    P.fi[t1][id] = e1i;
    P.fi[t2][id] = e2i;
  }
}

}  // namespace

cudaError_t launch_seam_h(const YeeParams& P, const SeamFace& f, cudaStream_t s) {
  const int a = f.axis;
  const int64_t n = (int64_t)(a == 0 ? P.ny : P.nx) * (a == 2 ? P.ny : P.nz);
  if (n <= 0 || n >= (1LL << 31)) return cudaErrorInvalidValue;
  k_seam_h<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, a, f.q);
  return cudaGetLastError();
}

cudaError_t launch_seam_e(const YeeParams& P, const SeamFace& f, cudaStream_t s) {
  const int a = f.axis;
  const int64_t n = (int64_t)(a == 0 ? P.ny : P.nx) * (a == 2 ? P.ny : P.nz);
  if (n <= 0 || n >= (1LL << 31)) return cudaErrorInvalidValue;
  k_seam_e<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, a, f.q);
  return cudaGetLastError();
}

cudaError_t launch_update_h_c(const YeeParams& P, cudaStream_t s) {
  dim3 b(32, 4, 1), g((P.nzp + 31) / 32, (P.ny + 3) / 4, P.nx);
  k_update_h_c<<<g, b, 0, s>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_update_e_c(const YeeParams& P, cudaStream_t s) {
  dim3 b(32, 4, 1), g((P.nzp + 31) / 32, (P.ny + 3) / 4, P.nx);
  k_update_e_c<<<g, b, 0, s>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_mode_h(const YeeParams& P, const ModeSrc& m, const int* step, cudaStream_t s) {
  dim3 b(32, 4, 1), g((m.n2 + 31) / 32, (m.n1 + 3) / 4, 1);
  k_mode_h<<<g, b, 0, s>>>(P, m, step);
  return cudaGetLastError();
}

cudaError_t launch_mode_e(const YeeParams& P, const ModeSrc& m, const int* step, cudaStream_t s) {
  dim3 b(32, 4, 1), g((m.n2 + 31) / 32, (m.n1 + 3) / 4, 1);
  k_mode_e<<<g, b, 0, s>>>(P, m, step);
  return cudaGetLastError();
}

}  // namespace oem
