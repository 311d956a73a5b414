// Per-cell arithmetic of the Yee and ADE updates, shared by every kernel variant.
//
// Each operation is written with explicit round-to-nearest intrinsics, so that the result does
// not depend on how the compiler would contract a multiply and an add in a given kernel: the
// one-thread-per-cell kernels and the pipelined kernels produce the same bits, and a wall
// mask of 1 (an interior cell) can be dropped without changing them, since n * 1 == n exactly.
#pragma once

#include <cuda_runtime.h>

namespace oem {

// Forward difference for the H update: (n * m - c) / dl (openem/kernels/yee.cu:76-137).
__device__ __forceinline__ float fdiff(float n, float m, float c, float idl) {
  return __fmul_rn(__fsub_rn(__fmul_rn(n, m), c), idl);
}
// Backward difference for the E update: (c - n * m) / dl (openem/kernels/yee.cu:154-240).
__device__ __forceinline__ float bdiff(float c, float n, float m, float idl) {
  return __fmul_rn(__fsub_rn(c, __fmul_rn(n, m)), idl);
}
// CPML recursion (openem/kernels/yee.cu:60-74): psi = b psi + a d; return d / kappa + psi.
__device__ __forceinline__ float cpml_stretch(float d, float& psi, float a, float b, float ik) {
  const float p = __fmaf_rn(b, psi, __fmul_rn(a, d));
  psi = p;
  return __fmaf_rn(ik, d, p);
}
// H^{n+1/2} = H^{n-1/2} - (dt / mu0) (sa - sb).
__device__ __forceinline__ float h_new(float h, float ch, float sa, float sb) {
  return __fmaf_rn(-ch, __fsub_rn(sa, sb), h);
}

// One ADE pole of one E component. Trapezoid pole-residue update
// (openem/kernels/dispersion.cu:168-207), deferred so that the post-update of step n-1 and the
// pre-update of step n run together with E^n:
//   p  = s + B E^n           (post-update of the previous step)
//   d  = (A - 1) p + B E^n   (pre-update increment)
//   s' = p + d,  contribution 2 Re(d) to the polarisation current
// with c = (Re(A-1), Im(A-1), Re(B), Im(B)).
__device__ __forceinline__ float ade_pole(float2& s, const float4 c, const float en) {
  const float ben_r = __fmul_rn(c.z, en);
  const float ben_i = __fmul_rn(c.w, en);
  const float pr = __fadd_rn(s.x, ben_r);
  const float pi = __fadd_rn(s.y, ben_i);
  const float dr = __fmaf_rn(c.x, pr, __fmaf_rn(-c.y, pi, ben_r));
  const float di = __fmaf_rn(c.x, pi, __fmaf_rn(c.y, pr, ben_i));
  s.x = __fadd_rn(pr, dr);
  s.y = __fadd_rn(pi, di);
  return __fmul_rn(2.0f, dr);
}

// E^{n+1} = ca E^n + cb (sa - sb - cw J) for one component (openem/kernels/yee.cu:154-240).
__device__ __forceinline__ float e_new(float ca, float en, float cb, float sa, float sb, float cw,
                                       float j) {
  return __fmaf_rn(ca, en, __fmul_rn(cb, __fsub_rn(__fsub_rn(sa, sb), __fmul_rn(cw, j))));
}

}  // namespace oem
