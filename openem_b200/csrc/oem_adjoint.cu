// Discrete adjoint of the real-field step: the transpose of the forward update, run backward in
// time, for an objective that is a weighted sum of flux-plane powers at monitor frequencies.
//
// Forward step n (the kernels of oem_kernels.cu / oem_yee_ws.cu, same arithmetic):
//   H^{n+1/2} = H^{n-1/2} - ch (S_a - S_b),   S = d / kappa + psi',  psi' = b psi + a d,
//                                             d = (E[nxt] m - E) / dl        (forward differences)
//   E^{n+1}   = ca E^n + cb (S_a - S_b) [+ sources, all proportional to cb],
//                                             d = (H - H[prv] m) / dl        (backward differences)
// is linear in (E, H, psi). Its transpose, applied from step N-1 down to 0 to the adjoint
// state (lambda_E, lambda_H, lambda_psi):
//   1. objective sources of step n: lambda_E += dJ/dE^{n+1}, lambda_H += dJ/dH^{n+1/2};
//   2. reverse E update: gradient terms, S_bar = +-cb lambda_E, psi: psi_bar = lambda_psi +
//      S_bar, d_bar = S_bar / kappa + a psi_bar, lambda_psi <- b psi_bar; lambda_E <- ca lambda_E;
//      lambda_H gathers the transposed backward differences of d_bar;
//   3. reverse H update: S_bar = -+ch lambda_H, same psi rule; lambda_E gathers the transposed
//      forward differences; lambda_H passes through.
// Gradients: with T^n = (E^{n+1} - ca E^n) / cb (the curl term including every cb-proportional
// source), dJ/dca = sum_n lambda_E^{n+1} E^n and dJ/dcb = sum_n lambda_E^{n+1} T^n per
// component and cell, accumulated in float64.
//
// Dispersive cells. The pole pass of step n (oem_arith.cuh ade_pole, per pole of a component)
//   p = s + B E^n,  d = (A - 1) p + B E^n,  s' = p + d,  J = sum 2 Re(d)
// feeds E^{n+1} = ... - cb cw J. Its transpose, with the adjoint pole state lambda_s (complex,
// zero after the last step since the states are no output) and lambda_J = -cb cw lambda_E^{n+1}:
//   lambda_d = lambda_s + 2 lambda_J (real part),  lambda_p = lambda_s + conj(A - 1) lambda_d,
//   lambda_E^n += Re(conj(B) (lambda_d + lambda_p)),  lambda_s <- lambda_p.
//
// The transposed differences are gathers (one thread per cell): a cell receives its own term
// and the terms of the cells whose neighbour it is; at a clamped wall or a PMC / symmetry plane a
// cell can be its own neighbour, so the inverse neighbour relation is checked explicitly.
//
// Two launches per reverse step: k_adj_ka gathers lambda_E from the previous H-side d_bar (the
// transposed H update of step n + 1) and then runs the E part of step n; k_adj_kb gathers
// lambda_H from the E-side d_bar and runs the H part. Gradients are kept for the cells of one
// box (the design region) only, from E^n and E^{n+1} of that box.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "oem_internal.cuh"

namespace oem {

namespace {

__device__ __forceinline__ int64_t psi_index(const DevAxis& A, int a, int i, int j, int k,
                                             int ny, int nzp, int* side) {
  const int q = (a == 0) ? i : ((a == 1) ? j : k);
  int ql, L;
  if (q < A.lo) {
    *side = 0; ql = q; L = A.lo;
  } else if (q >= A.n - A.hi) {
    *side = 1; ql = q - (A.n - A.hi); L = A.hi;
  } else {
    return -1;
  }
  if (a == 0) return ((int64_t)ql * ny + j) * nzp + k;
  if (a == 1) return ((int64_t)i * L + ql) * nzp + k;
  return ((int64_t)i * ny + j) * L + ql;
}

// adjoint of S = d / kappa + (b psi + a d) for one slab array (or S = d outside the slabs)
__device__ __forceinline__ float dbar_of(float sbar, const PsiSet& LP, int a, int slot,
                                         const DevAxis& A, const float* ca, const float* cb,
                                         const float* ck, int q, int i, int j, int k, int ny,
                                         int nzp) {
  int side = 0;
  const int64_t pi = psi_index(A, a, i, j, k, ny, nzp, &side);
  if (pi < 0) return sbar;
  float* lp = LP.p[a][slot][side] + pi;
  const float pbar = *lp + sbar;
  *lp = cb[q] * pbar;
  return ck[q] * sbar + ca[q] * pbar;
}

__device__ __forceinline__ uint32_t mat_of(const YeeParams& P, int64_t id) {
  return P.mat16 ? (uint32_t)P.mat16[id] : P.mat32[id];
}

// objective sources of step n on one flux plane: coef (4, nf, n1, n2, 2) per term (E_t1, E_t2,
// H_t1, H_t2 colocated) the weights of (cos, sin) of the forward phase table row n
__global__ void k_adj_src(YeeParams P, AdjFlux af, AdjState S, int n) {
  const int o2 = blockIdx.x * blockDim.x + threadIdx.x;
  const int o1 = blockIdx.y * blockDim.y + threadIdx.y;
  if (o1 >= af.n1 || o2 >= af.n2) return;
  const int t1 = (af.axis == 0) ? 1 : 0;
  const int t2 = (af.axis == 2) ? 1 : 2;
  int c[3];
  c[af.axis] = af.km; c[t1] = o1; c[t2] = o2;
  const int64_t id = ((int64_t)c[0] * P.ny + c[1]) * P.nzp + c[2];
  c[af.axis] = af.km - 1;
  const int64_t idm = ((int64_t)c[0] * P.ny + c[1]) * P.nzp + c[2];
  const int64_t plane = (int64_t)af.n1 * af.n2;
  const int64_t p = (int64_t)o1 * af.n2 + o2;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (int f = 0; f < af.nf; ++f) {
    const float* ph = af.phase + ((int64_t)n * af.nf + f) * 4;
    for (int t = 0; t < 4; ++t) {
      const double* w = af.coef + (((int64_t)t * af.nf + f) * plane + p) * 2;
      const double co = t < 2 ? ph[0] : ph[2], si = t < 2 ? ph[1] : ph[3];
      a[t] += co * w[0] + si * w[1];
    }
  }
  S.lam[t1][id] += (float)a[0];
  S.lam[t2][id] += (float)a[1];
  S.lam[3 + t1][id] += (float)(0.5 * a[2]);
  S.lam[3 + t1][idm] += (float)(0.5 * a[2]);
  S.lam[3 + t2][id] += (float)(0.5 * a[3]);
  S.lam[3 + t2][idm] += (float)(0.5 * a[3]);
}

// index of cell (i, j, k) moved to q along axis a
__device__ __forceinline__ int64_t moved(const YeeParams& P, int a, int i, int j, int k, int q) {
  if (a == 0) i = q;
  else if (a == 1) j = q;
  else k = q;
  return ((int64_t)i * P.ny + j) * P.nzp + k;
}

// The cells q' of an axis that can name q as a neighbour: q - 1, q, q + 1 and, on a periodic
// axis, the wrap partner (prv / nxt of q); each listed once.
__device__ __forceinline__ int neighbour_candidates(const DevAxis& A, int q, int* c) {
  int n = 0;
  const int raw[5] = {q - 1, q, q + 1, A.prv[q], A.nxt[q]};
#pragma unroll
  for (int t = 0; t < 5; ++t) {
    const int v = raw[t];
    if (v < 0 || v >= A.n) continue;
    bool seen = false;
    for (int u = 0; u < n; ++u) seen |= (c[u] == v);
    if (!seen) c[n++] = v;
  }
  return n;
}

// transposed backward difference along axis a of term array db into lambda at (i, j, k):
// own idl d_bar, minus m idl d_bar of every cell c' with prv(c') = this cell
__device__ __forceinline__ float gather_bwd(const YeeParams& P, const float* db, int a, int i,
                                            int j, int k) {
  const DevAxis& A = P.ax[a];
  const int q = a == 0 ? i : (a == 1 ? j : k);
  float v = A.idl_d[q] * db[moved(P, a, i, j, k, q)];
  // away from both ends the neighbour tables are q -+ 1 (wraps and clamps sit at the ends):
  // exactly one cell, q + 1, names q as its backward neighbour
  if (q > 0 && q < A.n - 1) {
    v -= A.mpv[q + 1] * A.idl_d[q + 1] * db[moved(P, a, i, j, k, q + 1)];
    return v;
  }
  int cand[5];
  const int nc = neighbour_candidates(A, q, cand);
  for (int t = 0; t < nc; ++t) {
    const int qq = cand[t];
    if (A.prv[qq] != q) continue;
    v -= A.mpv[qq] * A.idl_d[qq] * db[moved(P, a, i, j, k, qq)];
  }
  return v;
}

// transposed forward difference along axis a: minus own idl d_bar, plus m idl d_bar of every
// cell c' with nxt(c') = this cell
__device__ __forceinline__ float gather_fwd(const YeeParams& P, const float* db, int a, int i,
                                            int j, int k) {
  const DevAxis& A = P.ax[a];
  const int q = a == 0 ? i : (a == 1 ? j : k);
  float v = -A.idl_p[q] * db[moved(P, a, i, j, k, q)];
  // away from both ends exactly one cell, q - 1, names q as its forward neighbour
  if (q > 0 && q < A.n - 1) {
    v += A.mnx[q - 1] * A.idl_p[q - 1] * db[moved(P, a, i, j, k, q - 1)];
    return v;
  }
  int cand[5];
  const int nc = neighbour_candidates(A, q, cand);
  for (int t = 0; t < nc; ++t) {
    const int qq = cand[t];
    if (A.nxt[qq] != q) continue;
    v += A.mnx[qq] * A.idl_p[qq] * db[moved(P, a, i, j, k, qq)];
  }
  return v;
}

// reverse step n, E side: lambda_E += transposed forward differences of the H-side d_bar (the
// H update of step n + 1), then the gradient terms (box cells), the adjoint psi, the six E-side
// d_bar and lambda_E <- ca lambda_E
__global__ void __launch_bounds__(128) k_adj_ka(YeeParams P, AdjState S, const float* en_box,
                                                const float* en1_box) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (j >= P.ny) return;  // warp-uniform: a warp is one aligned 32-cell z segment of a row
  const int64_t id = ((int64_t)i * P.ny + j) * P.nzp + k;
  // first pole of this cell: the segment's offset plus the poles of the lanes before it (the
  // padding cells past nz hold the pole-free material 0)
  uint32_t poff = 0;
  if (S.lps) {
    const MatRec& Mp = P.mats[mat_of(P, id)];
    const int npc = Mp.np[0] + Mp.np[1] + Mp.np[2];
    const unsigned lt = (1u << (threadIdx.x & 31)) - 1u;
    int pre = 0;
#pragma unroll
    for (int b = 0; b < 6; ++b) pre += __popc(__ballot_sync(0xffffffffu, (npc >> b) & 1) & lt) << b;
    poff = P.seg_ofs[id >> 5] + (uint32_t)pre;
  }
  if (k >= P.nz) return;
  // Ez: Hx y-term (0), Hy x-term (3); Ey: Hx z-term (1), Hz x-term (4); Ex: Hy z-term (2),
  // Hz y-term (5)
  float lam[3];
  lam[2] = S.lam[2][id] + (gather_fwd(P, S.dbarh[0], 1, i, j, k) + gather_fwd(P, S.dbarh[3], 0, i, j, k));
  lam[1] = S.lam[1][id] + (gather_fwd(P, S.dbarh[1], 2, i, j, k) + gather_fwd(P, S.dbarh[4], 0, i, j, k));
  lam[0] = S.lam[0][id] + (gather_fwd(P, S.dbarh[2], 2, i, j, k) + gather_fwd(P, S.dbarh[5], 1, i, j, k));
  const MatRec& M = P.mats[mat_of(P, id)];
  const int bi = i - S.box[0], bj = j - S.box[1], bk = k - S.box[2];
  const bool inbox = bi >= 0 && bi < S.box[3] && bj >= 0 && bj < S.box[4] && bk >= 0 &&
                     bk < S.box[5];
  const int64_t nb = (int64_t)S.box[3] * S.box[4] * S.box[5];
  const int64_t t = inbox ? ((int64_t)bi * S.box[4] + bj) * S.box[5] + bk : 0;
  // (axis a, psi slot) of the S_a and S_b terms of each component, d_bar index 2c and 2c+1
  const int ax_a[3] = {1, 2, 0}, ax_b[3] = {2, 0, 1};
  const int sl_a[3] = {0, 1, 1}, sl_b[3] = {0, 0, 1};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float ca = M.ca[c], cb = M.cb[c];
    if (inbox && lam[c] != 0.f) {
      const double e0 = en_box[c * nb + t], e1v = en1_box[c * nb + t];
      S.gca[c][t] += (double)lam[c] * e0;
      if (cb != 0.f) S.gcb[c][t] += (double)lam[c] * (e1v - (double)ca * e0) / (double)cb;
    }
    const float sa = cb * lam[c], sb = -cb * lam[c];
    const int aa = ax_a[c], ab = ax_b[c];
    const DevAxis& Aa = P.ax[aa];
    const DevAxis& Ab = P.ax[ab];
    const int qa = aa == 0 ? i : (aa == 1 ? j : k);
    const int qb = ab == 0 ? i : (ab == 1 ? j : k);
    S.dbare[2 * c][id] = dbar_of(sa, S.lpsie, aa, sl_a[c], Aa, Aa.ae, Aa.be, Aa.ke, qa, i, j, k,
                                 P.ny, P.nzp);
    S.dbare[2 * c + 1][id] = dbar_of(sb, S.lpsie, ab, sl_b[c], Ab, Ab.ae, Ab.be, Ab.ke, qb, i,
                                     j, k, P.ny, P.nzp);
    float lam_n = ca * lam[c];
    if (S.lps && M.np[c] > 0) {  // the transposed pole pass of this component
      const float lj = -cb * P.cw * lam[c];
      const float4* cf = P.pcoef + P.pset_ofs[M.pset[c]];
      for (int t = 0; t < M.np[c]; ++t) {
        const float4 q = cf[t];  // (Re(A-1), Im(A-1), Re B, Im B)
        float2& ls = S.lps[poff + t];
        const float ldr = ls.x + 2.0f * lj, ldi = ls.y;
        const float lpr = ls.x + (q.x * ldr + q.y * ldi);
        const float lpi = ls.y + (q.x * ldi - q.y * ldr);
        lam_n += q.z * (ldr + lpr) + q.w * (ldi + lpi);
        ls = make_float2(lpr, lpi);
      }
    }
    if (S.lps) poff += (uint32_t)M.np[c];
    S.lam[c][id] = lam_n;
  }
}

// reverse step n, H side: lambda_H += transposed backward differences of the E-side d_bar, then
// the adjoint psi and the six H-side d_bar (lambda_H passes through)
__global__ void __launch_bounds__(128) k_adj_kb(YeeParams P, AdjState S) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= P.nz || j >= P.ny) return;
  const int64_t id = ((int64_t)i * P.ny + j) * P.nzp + k;
  // Hz: Ex y-term (0), Ey x-term (3); Hy: Ex z-term (1), Ez x-term (4); Hx: Ey z-term (2),
  // Ez y-term (5)
  float lam[3];
  lam[2] = S.lam[5][id] + (gather_bwd(P, S.dbare[0], 1, i, j, k) + gather_bwd(P, S.dbare[3], 0, i, j, k));
  lam[1] = S.lam[4][id] + (gather_bwd(P, S.dbare[1], 2, i, j, k) + gather_bwd(P, S.dbare[4], 0, i, j, k));
  lam[0] = S.lam[3][id] + (gather_bwd(P, S.dbare[2], 2, i, j, k) + gather_bwd(P, S.dbare[5], 1, i, j, k));
  const int ax_a[3] = {1, 2, 0}, ax_b[3] = {2, 0, 1};
  const int sl_a[3] = {0, 1, 1}, sl_b[3] = {0, 0, 1};
#pragma unroll
  for (int h = 0; h < 3; ++h) {
    S.lam[3 + h][id] = lam[h];
    const float sa = -P.ch * lam[h], sb = P.ch * lam[h];
    const int aa = ax_a[h], ab = ax_b[h];
    const DevAxis& Aa = P.ax[aa];
    const DevAxis& Ab = P.ax[ab];
    const int qa = aa == 0 ? i : (aa == 1 ? j : k);
    const int qb = ab == 0 ? i : (ab == 1 ? j : k);
    S.dbarh[2 * h][id] = dbar_of(sa, S.lpsih, aa, sl_a[h], Aa, Aa.ah, Aa.bh, Aa.kh, qa, i, j, k,
                                 P.ny, P.nzp);
    S.dbarh[2 * h + 1][id] = dbar_of(sb, S.lpsih, ab, sl_b[h], Ab, Ab.ah, Ab.bh, Ab.kh, qb, i,
                                     j, k, P.ny, P.nzp);
  }
}

// E of the box cells into a (3, box) buffer (the step's E for the gradient terms)
__global__ void k_adj_snap(YeeParams P, AdjState S, float* dst) {
  const int64_t nb = (int64_t)S.box[3] * S.box[4] * S.box[5];
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nb;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int bk = (int)(t % S.box[5]);
    const int64_t r = t / S.box[5];
    const int bj = (int)(r % S.box[4]), bi = (int)(r / S.box[4]);
    const int64_t id = ((int64_t)(S.box[0] + bi) * P.ny + (S.box[1] + bj)) * P.nzp + (S.box[2] + bk);
    dst[t] = P.f[0][id];
    dst[nb + t] = P.f[1][id];
    dst[2 * nb + t] = P.f[2][id];
  }
}

}  // namespace

cudaError_t launch_adj_src(const YeeParams& P, const AdjFlux& a, const AdjState& S, int n,
                           cudaStream_t s) {
  dim3 b(32, 4, 1), g((a.n2 + 31) / 32, (a.n1 + 3) / 4, 1);
  k_adj_src<<<g, b, 0, s>>>(P, a, S, n);
  return cudaGetLastError();
}

cudaError_t launch_adj_step(const YeeParams& P, const AdjState& S, const float* en_box,
                            const float* en1_box, cudaStream_t s) {
  dim3 b(32, 4, 1), g((P.nzp + 31) / 32, (P.ny + 3) / 4, P.nx);
  k_adj_ka<<<g, b, 0, s>>>(P, S, en_box, en1_box);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_adj_kb<<<g, b, 0, s>>>(P, S);
  return cudaGetLastError();
}

// E of the gradient box after the step the counter names (row step + 1 of the history), inside
// the step graph of the forward run.
__global__ void k_hist_snap(YeeParams P, int b0, int b1, int b2, int n0, int n1, int n2,
                            float* hist, const int* step, int64_t n_total) {
  const int64_t row = (int64_t)(*step) + 1;
  if (row > n_total) return;
  const int64_t nb = (int64_t)n0 * n1 * n2;
  float* dst = hist + row * 3 * nb;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nb;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = t / ((int64_t)n1 * n2), r = t - a * n1 * n2;
    const int64_t b = r / n2, c = r - b * n2;
    const int64_t id = ((b0 + a) * P.ny + (b1 + b)) * P.nzp + (b2 + c);
#pragma unroll
    for (int q = 0; q < 3; ++q) dst[q * nb + t] = P.f[q][id];
  }
}

cudaError_t launch_hist_snap(const YeeParams& P, const int* box, float* hist, const int* step,
                             int64_t n_total, cudaStream_t s) {
  const int64_t nb = (int64_t)box[3] * box[4] * box[5];
  const int blocks = (int)std::min<int64_t>((nb + 255) / 256, 148 * 8);
  k_hist_snap<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(P, box[0], box[1], box[2], box[3], box[4],
                                                      box[5], hist, step, n_total);
  return cudaGetLastError();
}

cudaError_t launch_adj_snap(const YeeParams& P, const AdjState& S, float* dst, cudaStream_t s) {
  const int64_t nb = (int64_t)S.box[3] * S.box[4] * S.box[5];
  const int blocks = (int)std::min<int64_t>((nb + 255) / 256, 148 * 8);
  k_adj_snap<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(P, S, dst);
  return cudaGetLastError();
}

}  // namespace oem
