// C ABI of the engine (include/oem_b200.h): plan lifecycle, table upload, CUDA-graph stepping,
// readout. The host side of OpenEM's step loop (openem/solver.py:403-511, _time_loop
// :1165-1213) is split here into "build once" (oem_plan_finalize) and "step many"
// (oem_plan_run); the float64 coefficient math stays in the Python host.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "oem_internal.cuh"

namespace oem {

static thread_local std::string g_last_error;

// Host side of the phasor readout, one per device per process: two pinned halves of a staging
// buffer. The DMA of chunk q fills one half while host threads copy chunk q - 1 out of the other
// into the caller's (pageable) array, so the copy-out runs near the link rate instead of
// through the driver's single-threaded pageable staging. Readouts on one device take turns.
struct ReadStage {
  std::mutex mu;
  char* half[2] = {nullptr, nullptr};
  size_t bytes = 0;  // of each half
  cudaEvent_t ev[2] = {nullptr, nullptr};
};
static std::mutex g_stage_mu;
static std::map<int, ReadStage*> g_stages;

static ReadStage* read_stage(int device) {
  std::lock_guard<std::mutex> g(g_stage_mu);
  ReadStage*& r = g_stages[device];
  if (!r) r = new ReadStage();
  return r;
}

// Grow the stage to halves of at least cbytes; false when no pinned memory could be had (the
// stage is then empty). The caller holds rs->mu and has made the device current.
static bool grow_stage(ReadStage* rs, size_t cbytes) {
  if (rs->bytes >= cbytes) return true;
  for (int b = 0; b < 2; ++b) {
    if (rs->half[b]) cudaFreeHost(rs->half[b]);
    rs->half[b] = nullptr;
    if (!rs->ev[b]) cudaEventCreateWithFlags(&rs->ev[b], cudaEventDisableTiming);
  }
  rs->bytes = 0;
  if (cudaHostAlloc((void**)&rs->half[0], cbytes, cudaHostAllocDefault) == cudaSuccess &&
      cudaHostAlloc((void**)&rs->half[1], cbytes, cudaHostAllocDefault) == cudaSuccess &&
      rs->ev[0] && rs->ev[1]) {
    rs->bytes = cbytes;
    return true;
  }
  cudaGetLastError();
  for (int b = 0; b < 2; ++b) {
    if (rs->half[b]) cudaFreeHost(rs->half[b]);
    rs->half[b] = nullptr;
  }
  return false;
}

// Ask for transparent huge pages on the page-aligned interior of a large output range before
// its first touch: a fresh 1.2 GB readout array otherwise takes 300k page faults. A hint only
// (no effect where huge pages are disabled).
static void advise_huge_pages(void* p, size_t n) {
  const uintptr_t a = ((uintptr_t)p + 4095) & ~(uintptr_t)4095;
  const uintptr_t b = ((uintptr_t)p + n) & ~(uintptr_t)4095;
  if (b > a + ((uintptr_t)4 << 20)) madvise((void*)a, b - a, MADV_HUGEPAGE);
}

// Copy n bytes with up to 16 host threads (pieces of at least 4 MB).
static void par_memcpy(char* dst, const char* src, size_t n) {
  const size_t kMin = (size_t)4 << 20;
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = (int)std::min<size_t>(std::min<size_t>(16, hw), std::max<size_t>(1, n / kMin));
  if (nt == 1) {
    memcpy(dst, src, n);
    return;
  }
  const size_t per = (n + nt - 1) / nt;
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) {
    const size_t a = t * per, b = std::min(n, a + per);
    if (a < b) th.emplace_back([=] { memcpy(dst + a, src + a, b - a); });
  }
  memcpy(dst, src, std::min(n, per));
  for (std::thread& x : th) x.join();
}

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_error(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  cudaGetLastError();  // clear a sticky launch error so the next call sees its own status
  return set_error(OEM_ERR_CUDA, m);
}

static int check_plan(oem_plan* p, bool want_final) {
  if (!p) return set_error(OEM_ERR_INVALID, "null plan");
  if (want_final && !p->finalized) return set_error(OEM_ERR_STATE, "plan is not finalized");
  if (!want_final && p->finalized)
    return set_error(OEM_ERR_STATE, "plan is already finalized; tables can no longer change");
  return OEM_OK;
}

static int use_device(oem_plan* p) {
  OEM_CUDA(cudaSetDevice(p->device));
  return OEM_OK;
}

static int64_t padded_index(const oem_plan* p, int i, int j, int k) {
  return ((int64_t)i * p->ny + j) * p->nzp + k;
}

// Upload one axis (z tables padded to nzp with values that keep padding threads in range).
static int upload_axis(oem_plan* p, int a) {
  const AxisHost& h = p->axh[a];
  const int n = (a == 0) ? p->nx : (a == 1) ? p->ny : p->nz;
  const int np = (a == 2) ? p->nzp : n;
  auto pad_f = [&](const std::vector<double>& v, size_t off, double fill) {
    std::vector<float> o(np, (float)fill);
    for (int q = 0; q < n; ++q) o[q] = (float)v[off + q];
    return o;
  };
  auto pad_i = [&](const std::vector<int>& v, int fill) {
    std::vector<int> o(np, fill);
    for (int q = 0; q < n; ++q) o[q] = v[q];
    return o;
  };
  DevAxis& D = p->yp.ax[a];
  float* d;
  int* di;
  int rc;
#define UPF(field, vec, off, fill)                                        \
  {                                                                       \
    std::vector<float> t_ = pad_f(vec, off, fill);                        \
    if ((rc = dupload(p, &d, t_.data(), t_.size()))) return rc;           \
    D.field = d;                                                          \
  }
  UPF(idl_p, h.idl_p, 0, 1.0);
  UPF(idl_d, h.idl_d, 0, 1.0);
  UPF(mnx, h.mnx, 0, 0.0);
  UPF(mpv, h.mpv, 0, 0.0);
  if (p->is_complex) {
    const std::vector<double> zero(n, 0.0);
    UPF(mnx_i, (h.mnx_i.empty() ? zero : h.mnx_i), 0, 0.0);
    UPF(mpv_i, (h.mpv_i.empty() ? zero : h.mpv_i), 0, 0.0);
  }
  UPF(ae, h.pml_e, 0, 0.0);
  UPF(be, h.pml_e, n, 1.0);
  UPF(ke, h.pml_e, 2 * (size_t)n, 1.0);
  UPF(ah, h.pml_h, 0, 0.0);
  UPF(bh, h.pml_h, n, 1.0);
  UPF(kh, h.pml_h, 2 * (size_t)n, 1.0);
#undef UPF
  {
    std::vector<int> t = pad_i(h.nxt, n - 1);
    if ((rc = dupload(p, &di, t.data(), t.size()))) return rc;
    D.nxt = di;
  }
  {
    std::vector<int> t = pad_i(h.prv, n - 1);
    if ((rc = dupload(p, &di, t.data(), t.size()))) return rc;
    D.prv = di;
  }
  D.n = n;
  D.lo = h.lo;
  D.hi = h.hi;
  // float64 primal / dual spacings for the energy sums
  std::vector<double> dlp(n), dld(n);
  for (int q = 0; q < n; ++q) {
    dlp[q] = 1.0 / h.idl_p[q];
    dld[q] = 1.0 / h.idl_d[q];
  }
  if ((rc = dupload(p, &p->d_dl[a][0], dlp.data(), (size_t)n))) return rc;
  if ((rc = dupload(p, &p->d_dl[a][1], dld.data(), (size_t)n))) return rc;
  return OEM_OK;
}

static int alloc_psi(oem_plan* p) {
  int rc;
  for (int a = 0; a < 3; ++a) {
    const AxisHost& h = p->axh[a];
    for (int side = 0; side < 2; ++side) {
      const int L = side == 0 ? h.lo : h.hi;
      size_t cnt = 0;
      if (L > 0) {
        if (a == 0) cnt = (size_t)L * p->ny * p->nzp;
        else if (a == 1) cnt = (size_t)p->nx * L * p->nzp;
        else cnt = (size_t)p->nx * p->ny * L;
      }
      for (int slot = 0; slot < 2; ++slot) {
        float* ph = nullptr;
        float* pe = nullptr;
        float* phi = nullptr;
        float* pei = nullptr;
        if (cnt) {
          if ((rc = dalloc(p, &ph, cnt))) return rc;
          if ((rc = dalloc(p, &pe, cnt))) return rc;
          if (p->is_complex) {
            if ((rc = dalloc(p, &phi, cnt))) return rc;
            if ((rc = dalloc(p, &pei, cnt))) return rc;
          }
        }
        p->yp.psih.p[a][slot][side] = ph;
        p->yp.psie.p[a][slot][side] = pe;
        p->yp.psih_i.p[a][slot][side] = phi;
        p->yp.psie_i.p[a][slot][side] = pei;
      }
    }
  }
  return OEM_OK;
}

// The imaginary part of a complex plan seen as a real plan: its field and psi arrays in place
// of the real ones (the real kernels read only f, psih and psie).
static YeeParams imag_part(const YeeParams& P) {
  YeeParams Q = P;
  for (int c = 0; c < 6; ++c) {
    Q.f[c] = P.fi[c];
    Q.fi[c] = P.f[c];
  }
  Q.psih = P.psih_i;
  Q.psie = P.psie_i;
  Q.psih_i = P.psih;
  Q.psie_i = P.psie;
  return Q;
}

static cudaError_t run_h(oem_plan* p, cudaStream_t s) {
  if (p->is_complex && p->cplx_ws) {
    cudaError_t e = launch_update_h_ws(p->tma, p->yp, p->xch, p->d_err, s);
    if (e == cudaSuccess) e = launch_update_h_ws(p->tma_i, imag_part(p->yp), p->xch, p->d_err, s);
    for (const SeamFace& f : p->seam_h)
      if (e == cudaSuccess) e = launch_seam_h(p->yp, f, s);
    return e;
  }
  if (p->is_complex) return launch_update_h_c(p->yp, s);
  if (p->basic_kernels == 1) return launch_update_h(p->yp, s);
  if (p->basic_kernels == 2) return launch_update_h_stream(p->yp, p->xch, s);
  if (p->basic_kernels == 3) return launch_update_h_ws(p->tma, p->yp, p->xch, p->d_err, s);
  return launch_update_h_tma(p->tma, p->yp, p->xch, p->d_err, s);
}

static cudaError_t run_e(oem_plan* p, cudaStream_t s, const SnapBoxes* sb = nullptr) {
  if (p->is_complex && p->cplx_ws) {
    const int nm = (int)p->mats.size();
    cudaError_t e = launch_update_e_ws(p->tma, p->yp, p->xch, nm, p->d_err, s);
    if (e == cudaSuccess)
      e = launch_update_e_ws(p->tma_i, imag_part(p->yp), p->xch, nm, p->d_err, s);
    for (const SeamFace& f : p->seam_e)
      if (e == cudaSuccess) e = launch_seam_e(p->yp, f, s);
    return e;
  }
  if (p->is_complex) return launch_update_e_c(p->yp, s);
  if (p->basic_kernels == 1) return launch_update_e(p->yp, s);
  if (p->basic_kernels == 2) return launch_update_e_stream(p->yp, p->xch, (int)p->mats.size(), s);
  if (p->basic_kernels == 3) {
    if (p->yp.has_ade) {
      cudaError_t e = launch_ade_segments(p->yp, p->d_ade_segs, p->n_ade_segs,
                                          (int64_t)p->nx * p->ny * p->nzp / 32, 0, (int)p->mats.size(), s);
      if (e != cudaSuccess) return e;
    }
    return launch_update_e_ws(p->tma, p->yp, p->xch, (int)p->mats.size(), p->d_err, s, sb);
  }
  return launch_update_e_tma(p->tma, p->yp, p->xch, (int)p->mats.size(), p->d_err, s);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  }
  return fn;
}

// 3D tensor map over one padded (nx, ny, nzp) array, box (bz, by, 1), zero fill out of bounds.
static int encode_map(oem_plan* p, CUtensorMap* m, const void* base, bool u16, bool u32, int bz,
                      int by) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return set_error(OEM_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t es = u16 ? 2 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)p->nzp, (cuuint64_t)p->ny, (cuuint64_t)p->nx};
  cuuint64_t strides[2] = {(cuuint64_t)p->nzp * es, (cuuint64_t)p->ny * p->nzp * es};
  cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUtensorMapDataType dt = u16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                     : (u32 ? CU_TENSOR_MAP_DATA_TYPE_UINT32
                                            : CU_TENSOR_MAP_DATA_TYPE_FLOAT32);
  CUresult r = fn(m, dt, 3, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(OEM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return OEM_OK;
}

int make_tma_maps_of(oem_plan* p, TmaMaps& m, const YeeParams& P) {
  int rc;
  for (int c = 0; c < 3; ++c) {
    if ((rc = encode_map(p, &m.e_wide[c], P.f[c], false, false, 136, 5))) return rc;
    if ((rc = encode_map(p, &m.e_tile[c], P.f[c], false, false, 128, 4))) return rc;
    if ((rc = encode_map(p, &m.h_wide[c], P.f[3 + c], false, false, 136, 5))) return rc;
    if ((rc = encode_map(p, &m.h_tile[c], P.f[3 + c], false, false, 128, 4))) return rc;
  }
  if (P.mat16) return encode_map(p, &m.m_tile, P.mat16, true, false, 128, 4);
  return encode_map(p, &m.m_tile, P.mat32, false, true, 128, 4);
}

int make_tma_maps(oem_plan* p) { return make_tma_maps_of(p, p->tma, p->yp); }


// Tensor maps of the fused kernel reading bank b.
static int make_fused_maps(oem_plan* p, int b) {
  int rc;
  FusedMaps& m = p->fmaps[b];
  for (int c = 0; c < 3; ++c) {
    if ((rc = encode_map(p, &m.e6[c], p->bank_f[b][c], false, false, 136, 6))) return rc;
    if ((rc = encode_map(p, &m.h5[c], p->bank_f[b][3 + c], false, false, 128, 5))) return rc;
  }
  for (int c = 0; c < 2; ++c)
    if ((rc = encode_map(p, &m.e5[c], p->bank_f[b][1 + c], false, false, 128, 5))) return rc;
  const YeeParams& P = p->yp;
  if (P.mat16) return encode_map(p, &m.m, P.mat16, true, false, 128, 4);
  return encode_map(p, &m.m, P.mat32, false, true, 128, 4);
}

// The fused step applies when the warp-specialised kernels run on a real plan whose y and z axes
// do not wrap and nothing is injected on the H side.
static bool fused_eligible(oem_plan* p) {
  if (!p->want_fused || p->basic_kernels != 3 || p->is_complex) return false;
  if (!p->planes.empty() || !p->modesrcs.empty() || !p->tfsfs.empty() || !p->absorbers.empty())
    return false;
  for (const DipoleSet& d : p->dipoles)
    if (d.magnetic) return false;
  for (int a = 1; a < 3; ++a) {
    const AxisHost& h = p->axh[a];
    const int n = (int)h.prv.size();
    if (n < 1 || h.prv[0] != 0) return false;  // periodic wrap at the low end
    for (int q = 1; q < n; ++q)
      if (h.prv[q] != q - 1) return false;
  }
  const AxisHost& x = p->axh[0];
  for (int q = 1; q < (int)x.prv.size(); ++q)
    if (x.prv[q] != q - 1) return false;
  return true;
}

// Non-zero when a kernel's bounded wait gave up since the last check.
static int check_device_error(oem_plan* p) {
  int h = 0;
  OEM_CUDA(cudaMemcpy(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    cudaMemset(p->d_err, 0, sizeof(int));
    return set_error(OEM_ERR_TIMEOUT,
                     "a device pipeline wait exceeded its bound; the results of this run are "
                     "invalid");
  }
  return OEM_OK;
}

// One time step (openem/solver.py:1145-1162).
static int enqueue_e_side(oem_plan* p, cudaStream_t s, bool monitors, bool ade_next = false);

// The box monitors whose snapshots the E update of this step writes, or null: only on a step
// that records monitors.
static const SnapBoxes* snap_boxes(const oem_plan* p, bool monitors) {
  return (monitors && p->snapk.n > 0) ? &p->snapk : nullptr;
}

// The current field bank becomes b: every kernel enqueued afterwards (sources, monitors,
// readouts) reads and writes that bank.
static void set_bank(oem_plan* p, int b) {
  p->bank = b;
  for (int c = 0; c < 6; ++c) p->yp.f[c] = p->bank_f[b][c];
  p->yp.psih = p->bank_psih[b];
}

static int launch_ade(oem_plan* p, cudaStream_t s, int max_blocks = 0) {
  cudaError_t e = launch_ade_segments(p->yp, p->d_ade_segs, p->n_ade_segs,
                                      (int64_t)p->nx * p->ny * p->nzp / 32, max_blocks,
                                      (int)p->mats.size(), s);
  return e == cudaSuccess ? OEM_OK : cuda_error(e, "ade");
}

// One step. ade_here: the step runs its own pole pass (beside the H update when the plan has a
// side stream); otherwise the previous step ran it (ade_next there). ade_next: the pole pass of
// the following step runs on the side stream once this step's E-side sources are in.
static int enqueue_step(oem_plan* p, cudaStream_t s, bool monitors = true, bool ade_here = true,
                        bool ade_next = false) {
  const YeeParams& P = p->yp;
  cudaError_t e;
  if (p->fused) {
    for (const MixSet& x : p->mixes)
      if ((e = launch_mix_pre(P, x, s)) != cudaSuccess) return cuda_error(e, "mix_pre");
    for (const Modulation& m : p->mods)
      if ((e = launch_modulate(P, m, p->d_step, s)) != cudaSuccess) return cuda_error(e, "modulate");
    for (const TensorSet& t : p->tensors)
      if ((e = launch_tensor_pre(P, t, s)) != cudaSuccess) return cuda_error(e, "tensor_pre");
    if (P.has_ade && (e = launch_ade_segments(P, p->d_ade_segs, p->n_ade_segs,
                                              (int64_t)p->nx * p->ny * p->nzp / 32, 0, (int)p->mats.size(), s)) !=
                         cudaSuccess)
      return cuda_error(e, "ade");
    const int nb = p->bank ^ 1;
    FieldOut out;
    for (int c = 0; c < 6; ++c) out.f[c] = p->bank_f[nb][c];
    out.psih = p->bank_psih[nb];
    if ((e = launch_update_he_fused(p->fmaps[p->bank], P, out, p->xch, (int)p->mats.size(),
                                    p->d_err, s)) != cudaSuccess)
      return cuda_error(e, "update_he");
    set_bank(p, nb);
    return enqueue_e_side(p, s, monitors);
  }
  // the pole pass depends on E^n only: when the step runs its own (ade_here) it goes on a
  // branch beside the H update and joins before the E update
  const bool fork = p->side_stream != nullptr;
  for (const MixSet& x : p->mixes)
    if ((e = launch_mix_pre(P, x, s)) != cudaSuccess) return cuda_error(e, "mix_pre");
  for (const Modulation& m : p->mods)
    if ((e = launch_modulate(P, m, p->d_step, s)) != cudaSuccess) return cuda_error(e, "modulate");
  for (const TensorSet& t : p->tensors)
    if ((e = launch_tensor_pre(P, t, s)) != cudaSuccess) return cuda_error(e, "tensor_pre");
  if (fork && ade_here) {
    OEM_CUDA(cudaEventRecord(p->ev_fork, s));
    OEM_CUDA(cudaStreamWaitEvent(p->side_stream, p->ev_fork, 0));
    int rc = launch_ade(p, p->side_stream);
    if (rc) return rc;
    OEM_CUDA(cudaEventRecord(p->ev_join, p->side_stream));
  }
  if ((e = run_h(p, s)) != cudaSuccess) return cuda_error(e, "update_h");
  for (const DipoleSet& d : p->dipoles)
    if (d.magnetic && (e = launch_dipoles(P, d, p->d_step, s)) != cudaSuccess)
      return cuda_error(e, "dipoles_h");
  for (const PlaneSrc& src : p->planes)
    if ((e = launch_plane_h(P, src, p->d_step, s)) != cudaSuccess)
      return cuda_error(e, "plane_h");
  for (const Tfsf& t : p->tfsfs)
    if ((e = launch_tfsf(P, t, 0, p->d_step, s)) != cudaSuccess) return cuda_error(e, "tfsf_h");
  for (const ModeSrc& m : p->modesrcs)
    if ((e = launch_mode_h(P, m, p->d_step, s)) != cudaSuccess) return cuda_error(e, "mode_h");
  for (const Absorber& a : p->absorbers)
    if ((e = launch_absorb(P, a, 0, s)) != cudaSuccess) return cuda_error(e, "absorb_h");
  const SnapBoxes* sb = snap_boxes(p, monitors);
  if (fork) {
    if (ade_here) OEM_CUDA(cudaStreamWaitEvent(s, p->ev_join, 0));
    e = launch_update_e_ws(p->tma, P, p->xch, (int)p->mats.size(), p->d_err, s, sb);
  } else {
    e = run_e(p, s, sb);
  }
  if (e != cudaSuccess) return cuda_error(e, "update_e");
  return enqueue_e_side(p, s, monitors, fork && ade_next);
}

// After the E update: E-side injection, absorber, time / flux-time samples, DFT snapshots and
// flushes, the step counter. ade_next: the next step's pole pass (it reads E^{n+1} with every
// E-side source in) runs on the side stream beside the monitors and joins at the end.
static int enqueue_e_side(oem_plan* p, cudaStream_t s, bool monitors, bool ade_next) {
  const YeeParams& P = p->yp;
  cudaError_t e;
  for (const PlaneSrc& src : p->planes)
    if ((e = launch_plane_e(P, src, p->d_step, s)) != cudaSuccess)
      return cuda_error(e, "plane_e");
  for (const Tfsf& t : p->tfsfs)
    if ((e = launch_tfsf(P, t, 1, p->d_step, s)) != cudaSuccess) return cuda_error(e, "tfsf_e");
  for (const ModeSrc& m : p->modesrcs)
    if ((e = launch_mode_e(P, m, p->d_step, s)) != cudaSuccess) return cuda_error(e, "mode_e");
  const SnapBoxes* sb = snap_boxes(p, monitors);
  for (const DipoleSet& d : p->dipoles)
    if (!d.magnetic && (e = launch_dipoles(P, d, p->d_step, s, sb)) != cudaSuccess)
      return cuda_error(e, "dipoles_e");
  for (const MixSet& x : p->mixes)
    if ((e = launch_mix_post(P, x, s)) != cudaSuccess) return cuda_error(e, "mix_post");
  for (const TensorSet& t : p->tensors)
    if ((e = launch_tensor_post(P, t, s)) != cudaSuccess) return cuda_error(e, "tensor_post");
  for (const Absorber& a : p->absorbers)
    if ((e = launch_absorb(P, a, 1, s)) != cudaSuccess) return cuda_error(e, "absorb_e");
  if (ade_next) {
    OEM_CUDA(cudaEventRecord(p->ev_fork, s));
    OEM_CUDA(cudaStreamWaitEvent(p->side_stream, p->ev_fork, 0));
    // four blocks per SM instead of five: the snapshot blocks find room beside them
    int rc = launch_ade(p, p->side_stream, 148 * 4);
    if (rc) return rc;
    OEM_CUDA(cudaEventRecord(p->ev_join, p->side_stream));
  }
  for (const TimeMon& m : p->tmons) {
    if (!monitors) break;
    if ((e = launch_time_sample(P, m, p->d_step, 1, s)) != cudaSuccess)
      return cuda_error(e, "time_sample");
    if ((e = launch_time_sample(P, m, p->d_step, 0, s)) != cudaSuccess)
      return cuda_error(e, "time_sample");
  }
  for (const FluxTimeMon& m : p->ftmons) {
    if (!monitors) break;
    if ((e = launch_flux_time(P, m, p->d_step, s)) != cudaSuccess) return cuda_error(e, "flux_time");
  }
  if (monitors) {
    // plane monitors one launch each, every box monitor in one launch (box rows are already
    // written by the E update and the E dipoles when sb is set), then the flushes
    const Monitor* boxes[64];
    int nb = 0;
    for (const Monitor& m : p->mons) {
      if (m.kind != 1) {
        if ((e = launch_snapshot(P, m, p->d_step, s)) != cudaSuccess)
          return cuda_error(e, "snapshot");
      } else if (!sb) {
        boxes[nb++] = &m;
        if (nb == 64) {
          if ((e = launch_snapshot_boxes(P, boxes, nb, p->d_step, s)) != cudaSuccess)
            return cuda_error(e, "snapshot");
          nb = 0;
        }
      }
    }
    if (nb && (e = launch_snapshot_boxes(P, boxes, nb, p->d_step, s)) != cudaSuccess)
      return cuda_error(e, "snapshot");
    for (const Monitor& m : p->mons)
      if ((e = launch_flush(m, p->d_step, 0, s)) != cudaSuccess) return cuda_error(e, "flush");
  }
  if (p->hist && (e = launch_hist_snap(P, p->gbox, p->hist, p->d_step, p->n_total, s)) !=
                     cudaSuccess)
    return cuda_error(e, "gradient box history");
  if ((e = launch_step_advance(p->d_step, s)) != cudaSuccess) return cuda_error(e, "step");
  if (ade_next) OEM_CUDA(cudaStreamWaitEvent(s, p->ev_join, 0));
  return OEM_OK;
}

// ---- checkpoints: the six fields and every CPML psi array, copied device to device ----
static void state_arrays(oem_plan* p, std::vector<std::pair<float*, size_t>>& v) {
  const size_t ncp = (size_t)p->nx * p->ny * p->nzp;
  for (int c = 0; c < 6; ++c) v.push_back({p->yp.f[c], ncp});
  for (int a = 0; a < 3; ++a) {
    const AxisHost& h = p->axh[a];
    for (int side = 0; side < 2; ++side) {
      const int L = side == 0 ? h.lo : h.hi;
      if (L <= 0) continue;
      size_t cnt = a == 0 ? (size_t)L * p->ny * p->nzp
                          : (a == 1 ? (size_t)p->nx * L * p->nzp : (size_t)p->nx * p->ny * L);
      for (int slot = 0; slot < 2; ++slot) {
        v.push_back({p->yp.psih.p[a][slot][side], cnt});
        v.push_back({p->yp.psie.p[a][slot][side], cnt});
      }
    }
  }
  // ADE pole states (a segment recomputed from a checkpoint needs them; the pole currents are
  // recomputed from them)
  if (p->yp.P && p->n_pole_total > 0)
    v.push_back({reinterpret_cast<float*>(p->yp.P), 2 * (size_t)p->n_pole_total});
}

static int save_state(oem_plan* p, int slot, cudaStream_t s) {
  if (slot < 0 || slot >= (int)p->ckpt.size()) return OEM_OK;  // past the planned step count
  std::vector<std::pair<float*, size_t>> v;
  state_arrays(p, v);
  float* dst = p->ckpt[slot];
  for (auto& a : v) {
    OEM_CUDA(cudaMemcpyAsync(dst, a.first, a.second * sizeof(float), cudaMemcpyDeviceToDevice, s));
    dst += a.second;
  }
  p->ckpt_step[slot] = p->steps;
  return OEM_OK;
}

static int load_state(oem_plan* p, int slot, cudaStream_t s) {
  std::vector<std::pair<float*, size_t>> v;
  state_arrays(p, v);
  const float* src = p->ckpt[slot];
  for (auto& a : v) {
    OEM_CUDA(cudaMemcpyAsync(a.first, src, a.second * sizeof(float), cudaMemcpyDeviceToDevice, s));
    src += a.second;
  }
  const int n = (int)p->ckpt_step[slot];
  OEM_CUDA(cudaMemcpyAsync(p->d_step, &n, sizeof(int), cudaMemcpyHostToDevice, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  return OEM_OK;
}

// mode 0: nsteps self-contained steps (the first runs its own pole pass; with ade_ahead each
// later one has it run by the step before); 1: one step whose pole pass ran before it and
// which runs the next one's (graph_mid); 2: one step whose pole pass ran before it (graph_last).
static int capture(oem_plan* p, int nsteps, cudaGraphExec_t* out, int mode = 0) {
  cudaGraph_t g = nullptr;
  const int bank0 = p->bank;
  OEM_CUDA(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal));
  int rc = OEM_OK;
  for (int q = 0; q < nsteps && rc == OEM_OK; ++q) {
    const bool here = mode == 0 && (q == 0 || !p->ade_ahead);
    const bool next = mode == 1 || (mode == 0 && p->ade_ahead && q + 1 < nsteps);
    rc = enqueue_step(p, p->cap_stream, true, here, next);
  }
  if (p->fused) set_bank(p, bank0);  // capturing ran nothing: the fields are still in bank0
  cudaError_t e = cudaStreamEndCapture(p->cap_stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
  if (nsteps == 1 && mode == 0) {
    // the kernels one step launches: the kernel nodes of the one-step graph
    size_t nn = 0;
    e = cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (e == cudaSuccess && nn) e = cudaGraphGetNodes(g, nodes.data(), &nn);
    int kernels = 0;
    for (size_t q = 0; q < nn && e == cudaSuccess; ++q) {
      cudaGraphNodeType t;
      e = cudaGraphNodeGetType(nodes[q], &t);
      kernels += (e == cudaSuccess && t == cudaGraphNodeTypeKernel) ? 1 : 0;
    }
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return cuda_error(e, "cudaGraphGetNodes");
    }
    p->step_kernels = kernels;
  }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
  return OEM_OK;
}

}  // namespace oem

using namespace oem;

extern "C" {

int oem_version(void) { return 100; }

const char* oem_last_error(void) { return g_last_error.c_str(); }

int oem_plan_create(int device, int nx, int ny, int nz, double ch, double cw, oem_plan** out) {
  if (!out) return set_error(OEM_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1)
    return set_error(OEM_ERR_INVALID, "grid dimensions must be positive");
  const int64_t nzp = ((int64_t)nz + 31) / 32 * 32;
  if ((int64_t)nx * ny * nzp > ((int64_t)1 << 40))
    return set_error(OEM_ERR_INVALID, "grid too large");
  if ((int64_t)nx * ny * nzp / 32 > 0xffffffffLL)
    return set_error(OEM_ERR_INVALID, "grid too large for 32-bit segment offsets");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceCount");
  if (device < 0 || device >= ndev)
    return set_error(OEM_ERR_INVALID, "device " + std::to_string(device) + " out of range");
  oem_plan* p = new oem_plan();
  p->device = device;
  p->nx = nx;
  p->ny = ny;
  p->nz = nz;
  p->nzp = (int)nzp;
  p->ch = ch;
  p->cw = cw;
  const char* kind = getenv("OEM_B200_KERNELS");
  // warp-specialised TMA kernels unless asked otherwise; below ~1.5M cells the one-thread-per-
  // cell kernels finish a step sooner (a pipelined block needs several planes to fill its ring)
  p->basic_kernels = (double)nx * ny * nz < 1.5e6 ? 1 : 3;
  if (kind && strcmp(kind, "basic") == 0) p->basic_kernels = 1;
  if (kind && strcmp(kind, "stream") == 0) p->basic_kernels = 2;
  if (kind && (strcmp(kind, "ws") == 0 || strcmp(kind, "fused") == 0)) p->basic_kernels = 3;
  if (kind && strcmp(kind, "tma") == 0) p->basic_kernels = 0;
  // the fused H + E step (two field banks) only when asked for: it is exact but latency-bound
  // and slower than the two pipelined kernels on the grids measured so far
  p->want_fused = kind && strcmp(kind, "fused") == 0;
  if (const char* fz = getenv("OEM_B200_FUSED")) p->want_fused = p->want_fused && strcmp(fz, "0") != 0;
  *out = p;
  return OEM_OK;
}

int oem_plan_destroy(oem_plan* p) {
  if (!p) return OEM_OK;
  if (p->stage_thread.joinable()) p->stage_thread.join();
  cudaSetDevice(p->device);
  for (int b = 0; b < 2; ++b) {
    if (p->graph_many[b]) cudaGraphExecDestroy(p->graph_many[b]);
    if (p->graph_one[b]) cudaGraphExecDestroy(p->graph_one[b]);
  }
  if (p->graph_mid) cudaGraphExecDestroy(p->graph_mid);
  if (p->graph_last) cudaGraphExecDestroy(p->graph_last);
  if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
  if (p->side_stream) cudaStreamDestroy(p->side_stream);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  for (void* a : p->allocs) cudaFree(a);
  delete p;
  return OEM_OK;
}

int oem_plan_set_axis(oem_plan* p, int axis, const double* idl_p, const double* idl_d,
                      const int32_t* nxt, const int32_t* prv, const double* mnx,
                      const double* mpv, const double* pml_e, const double* pml_h, int slab_lo,
                      int slab_hi) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (axis < 0 || axis > 2) return set_error(OEM_ERR_INVALID, "axis must be 0, 1 or 2");
  if (!idl_p || !idl_d || !nxt || !prv || !mnx || !mpv || !pml_e || !pml_h)
    return set_error(OEM_ERR_INVALID, "null axis table");
  const int n = axis == 0 ? p->nx : axis == 1 ? p->ny : p->nz;
  if (slab_lo < 0 || slab_hi < 0 || slab_lo + slab_hi > n)
    return set_error(OEM_ERR_INVALID, "psi slabs overlap or exceed the axis");
  AxisHost& h = p->axh[axis];
  h.idl_p.assign(idl_p, idl_p + n);
  h.idl_d.assign(idl_d, idl_d + n);
  h.nxt.assign(nxt, nxt + n);
  h.prv.assign(prv, prv + n);
  h.mnx.assign(mnx, mnx + n);
  h.mpv.assign(mpv, mpv + n);
  h.pml_e.assign(pml_e, pml_e + 3 * (size_t)n);
  h.pml_h.assign(pml_h, pml_h + 3 * (size_t)n);
  for (int q = 0; q < n; ++q) {
    if (h.nxt[q] < 0 || h.nxt[q] >= n || h.prv[q] < 0 || h.prv[q] >= n)
      return set_error(OEM_ERR_INVALID, "neighbour index out of range on axis " +
                                            std::to_string(axis));
    if (!(h.idl_p[q] > 0.0) || !(h.idl_d[q] > 0.0))
      return set_error(OEM_ERR_INVALID, "spacings must be positive");
    const bool in_slab = q < slab_lo || q >= n - slab_hi;
    if (!in_slab) {
      for (const std::vector<double>* v : {&h.pml_e, &h.pml_h}) {
        if ((*v)[q] != 0.0 || (*v)[n + q] != 1.0 || (*v)[2 * (size_t)n + q] != 1.0)
          return set_error(OEM_ERR_INVALID,
                           "CPML coefficients are not the identity outside the psi slabs on "
                           "axis " + std::to_string(axis) + " at index " + std::to_string(q));
      }
    }
  }
  h.lo = slab_lo;
  h.hi = slab_hi;
  h.set = true;
  return OEM_OK;
}

int oem_plan_set_materials(oem_plan* p, int n_mat, const uint32_t* table, int index_bytes,
                           const void* index) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (n_mat < 1 || !table || !index) return set_error(OEM_ERR_INVALID, "empty material table");
  if (index_bytes != 2 && index_bytes != 4)
    return set_error(OEM_ERR_INVALID, "index_bytes must be 2 or 4");
  if (index_bytes == 2 && n_mat > 65535)
    return set_error(OEM_ERR_INVALID, "more than 65535 materials need a 4-byte index");
  p->mats.resize((size_t)n_mat + 1);
  MatRec& v = p->mats[0];  // material 0: padding cells (E held at zero)
  for (int c = 0; c < 3; ++c) {
    v.ca[c] = 0.f; v.cb[c] = 0.f; v.eps[c] = 1.f; v.pset[c] = -1; v.np[c] = 0;
  }
  v.reserved = 0;
  memcpy(&p->mats[1], table, sizeof(MatRec) * (size_t)n_mat);
  for (int m = 1; m <= n_mat; ++m)
    p->mats[m].reserved = p->mats[m].np[0] + p->mats[m].np[1] + p->mats[m].np[2];
  for (int m = 1; m <= n_mat; ++m)
    for (int c = 0; c < 3; ++c) {
      const MatRec& r = p->mats[m];
      if (r.pset[c] < 0 && r.np[c] != 0)
        return set_error(OEM_ERR_INVALID, "non-dispersive material with a pole count");
      if (r.np[c] < 0 || r.np[c] > 15)
        return set_error(OEM_ERR_INVALID, "pole count per component must be 0..15");
    }
  const size_t ncell = (size_t)p->nx * p->ny * p->nz;
  p->index_bytes = index_bytes;
  p->mat_index.resize(ncell * index_bytes);
  memcpy(p->mat_index.data(), index, ncell * index_bytes);
  // range check
  if (index_bytes == 2) {
    const uint16_t* q = reinterpret_cast<const uint16_t*>(p->mat_index.data());
    for (size_t t = 0; t < ncell; ++t)
      if (q[t] >= n_mat) return set_error(OEM_ERR_INVALID, "material index out of range");
  } else {
    const uint32_t* q = reinterpret_cast<const uint32_t*>(p->mat_index.data());
    for (size_t t = 0; t < ncell; ++t)
      if (q[t] >= (uint32_t)n_mat) return set_error(OEM_ERR_INVALID, "material index out of range");
  }
  return OEM_OK;
}

int oem_plan_set_pole_sets(oem_plan* p, int n_sets, const int32_t* set_ofs, const float* coef,
                           const uint32_t* seg_ofs, int64_t n_seg, int64_t n_pole_total) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (n_sets < 1 || !set_ofs || !coef || !seg_ofs)
    return set_error(OEM_ERR_INVALID, "empty pole-set table");
  const int64_t want_seg = (int64_t)p->nx * p->ny * p->nzp / 32;
  if (n_seg != want_seg)
    return set_error(OEM_ERR_INVALID, "seg_ofs must hold one entry per 32-cell segment (" +
                                          std::to_string(want_seg) + ")");
  if (n_pole_total < 0 || n_pole_total > 0xffffffffLL)
    return set_error(OEM_ERR_INVALID, "pole count out of range");
  p->pset_ofs.assign(set_ofs, set_ofs + n_sets + 1);
  if (p->pset_ofs[0] != 0) return set_error(OEM_ERR_INVALID, "set_ofs[0] must be 0");
  for (int s = 0; s < n_sets; ++s)
    if (p->pset_ofs[s + 1] < p->pset_ofs[s]) return set_error(OEM_ERR_INVALID, "set_ofs not monotone");
  p->pcoef.assign(coef, coef + 4 * (size_t)p->pset_ofs[n_sets]);
  p->seg_ofs.assign(seg_ofs, seg_ofs + n_seg);
  p->n_pole_total = n_pole_total;
  return OEM_OK;
}

// Material table from the host, per-cell index already on the device (unpadded C order).
int oem_plan_set_materials_device(oem_plan* p, int n_mat, const uint32_t* table, int index_bytes,
                                  const void* d_index) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (n_mat < 1 || !table || !d_index) return set_error(OEM_ERR_INVALID, "empty material table");
  if (index_bytes != 2 && index_bytes != 4)
    return set_error(OEM_ERR_INVALID, "index_bytes must be 2 or 4");
  if (index_bytes == 2 && n_mat > 65535)
    return set_error(OEM_ERR_INVALID, "more than 65535 materials need a 4-byte index");
  if ((rc = use_device(p))) return rc;
  p->mats.resize((size_t)n_mat + 1);
  MatRec& v = p->mats[0];
  for (int c = 0; c < 3; ++c) {
    v.ca[c] = 0.f; v.cb[c] = 0.f; v.eps[c] = 1.f; v.pset[c] = -1; v.np[c] = 0;
  }
  v.reserved = 0;
  memcpy(&p->mats[1], table, sizeof(MatRec) * (size_t)n_mat);
  for (int m = 1; m <= n_mat; ++m) {
    MatRec& r = p->mats[m];
    for (int c = 0; c < 3; ++c) {
      if (r.pset[c] < 0 && r.np[c] != 0)
        return set_error(OEM_ERR_INVALID, "non-dispersive material with a pole count");
      if (r.np[c] < 0 || r.np[c] > 15)
        return set_error(OEM_ERR_INVALID, "pole count per component must be 0..15");
    }
    r.reserved = r.np[0] + r.np[1] + r.np[2];
  }
  p->index_bytes = index_bytes;
  const bool wide = index_bytes == 4 || (size_t)n_mat + 1 > 65535;
  const size_t ncp = (size_t)p->nx * p->ny * p->nzp;
  unsigned* bad = nullptr;
  if ((rc = dalloc(p, &bad, 1))) return rc;
  cudaError_t e;
  if (wide) {
    if ((rc = dalloc(p, &p->dev_mat32, ncp, false))) return rc;
    e = launch_pad_index(d_index, index_bytes, nullptr, p->dev_mat32, p->nx, p->ny, p->nz, p->nzp,
                         (uint32_t)n_mat, bad, 0);
  } else {
    if ((rc = dalloc(p, &p->dev_mat16, ncp, false))) return rc;
    e = launch_pad_index(d_index, index_bytes, p->dev_mat16, nullptr, p->nx, p->ny, p->nz, p->nzp,
                         (uint32_t)n_mat, bad, 0);
  }
  if (e != cudaSuccess) return cuda_error(e, "pad_index");
  unsigned hbad = 0;
  OEM_CUDA(cudaMemcpy(&hbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (hbad) return set_error(OEM_ERR_INVALID, "material index out of range");
  p->dev_index = true;
  return OEM_OK;
}

// Pole sets from the host, segment offsets already on the device.
int oem_plan_set_pole_sets_device(oem_plan* p, int n_sets, const int32_t* set_ofs,
                                  const float* coef, const uint32_t* d_seg_ofs, int64_t n_seg,
                                  int64_t n_pole_total) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (n_sets < 1 || !set_ofs || !coef || !d_seg_ofs)
    return set_error(OEM_ERR_INVALID, "empty pole-set table");
  const int64_t want_seg = (int64_t)p->nx * p->ny * p->nzp / 32;
  if (n_seg != want_seg)
    return set_error(OEM_ERR_INVALID, "seg_ofs must hold one entry per 32-cell segment (" +
                                          std::to_string(want_seg) + ")");
  if (n_pole_total < 0 || n_pole_total > 0xffffffffLL)
    return set_error(OEM_ERR_INVALID, "pole count out of range");
  if ((rc = use_device(p))) return rc;
  p->pset_ofs.assign(set_ofs, set_ofs + n_sets + 1);
  if (p->pset_ofs[0] != 0) return set_error(OEM_ERR_INVALID, "set_ofs[0] must be 0");
  for (int s = 0; s < n_sets; ++s)
    if (p->pset_ofs[s + 1] < p->pset_ofs[s]) return set_error(OEM_ERR_INVALID, "set_ofs not monotone");
  p->pcoef.assign(coef, coef + 4 * (size_t)p->pset_ofs[n_sets]);
  if ((rc = dalloc(p, &p->dev_seg, (size_t)n_seg, false))) return rc;
  OEM_CUDA(cudaMemcpy(p->dev_seg, d_seg_ofs, (size_t)n_seg * sizeof(uint32_t),
                      cudaMemcpyDeviceToDevice));
  p->seg_ofs.clear();
  p->n_pole_total = n_pole_total;
  return OEM_OK;
}

int oem_plan_add_plane_source(oem_plan* p, int pol, int kh, int ks, double coef_h, double coef_e,
                              int64_t n_tab, const double* ex_tab, const double* hy_tab) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (pol != 0 && pol != 1) return set_error(OEM_ERR_UNSUPPORTED, "plane wave polarisation must be Ex or Ey");
  if (kh < 0 || kh >= p->nz || ks < 0 || ks >= p->nz)
    return set_error(OEM_ERR_INVALID, "plane-wave injection planes out of range");
  if (n_tab < 1 || !ex_tab || !hy_tab) return set_error(OEM_ERR_INVALID, "empty incident table");
  if ((rc = use_device(p))) return rc;
  PlaneSrc s;
  s.pol = pol;
  s.kh = kh;
  s.ks = ks;
  s.coef_h = (float)coef_h;
  s.coef_e = (float)coef_e;
  s.ntab = n_tab;
  if ((rc = dupload(p, &s.d_ex, ex_tab, (size_t)n_tab))) return rc;
  if ((rc = dupload(p, &s.d_hy, hy_tab, (size_t)n_tab))) return rc;
  p->planes.push_back(s);
  return OEM_OK;
}

static int add_dipoles_impl(oem_plan* p, int magnetic, int n_pts, const int32_t* ijk,
                            const int32_t* comp, const float* coef, const int32_t* src, int n_src,
                            int64_t nsteps1, const double* amp, const double* amp_im) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (n_pts < 1 || n_src < 1 || nsteps1 < 1 || !ijk || !comp || !coef || !src || !amp)
    return set_error(OEM_ERR_INVALID, "empty dipole table");
  if ((rc = use_device(p))) return rc;
  // Group points by (component, cell), keeping their input order inside a group.
  std::map<std::pair<int64_t, int>, std::vector<int>> groups;
  std::vector<std::pair<int64_t, int>> order;
  for (int q = 0; q < n_pts; ++q) {
    const int i = ijk[3 * q], j = ijk[3 * q + 1], k = ijk[3 * q + 2];
    if (i < 0 || i >= p->nx || j < 0 || j >= p->ny || k < 0 || k >= p->nz)
      return set_error(OEM_ERR_INVALID, "dipole stencil point outside the grid");
    if (comp[q] < 0 || comp[q] > 2) return set_error(OEM_ERR_INVALID, "dipole component out of range");
    if (src[q] < 0 || src[q] >= n_src) return set_error(OEM_ERR_INVALID, "dipole source index out of range");
    auto key = std::make_pair(padded_index(p, i, j, k), (int)comp[q]);
    auto it = groups.find(key);
    if (it == groups.end()) {
      order.push_back(key);
      groups[key] = {q};
    } else {
      it->second.push_back(q);
    }
  }
  std::vector<int64_t> tgt;
  std::vector<int> tcomp, ofs(1, 0), psrc;
  std::vector<float> pcoef;
  for (const auto& key : order) {
    tgt.push_back(key.first);
    tcomp.push_back(key.second);
    for (int q : groups[key]) {
      pcoef.push_back(coef[q]);
      psrc.push_back(src[q]);
    }
    ofs.push_back((int)pcoef.size());
  }
  DipoleSet d;
  d.magnetic = magnetic ? 1 : 0;
  d.n_targets = (int)tgt.size();
  d.nsteps1 = nsteps1;
  d.n_src = n_src;
  if ((rc = dupload(p, &d.d_target, tgt.data(), tgt.size()))) return rc;
  if ((rc = dupload(p, &d.d_tcomp, tcomp.data(), tcomp.size()))) return rc;
  if ((rc = dupload(p, &d.d_ofs, ofs.data(), ofs.size()))) return rc;
  if ((rc = dupload(p, &d.d_coef, pcoef.data(), pcoef.size()))) return rc;
  if ((rc = dupload(p, &d.d_src, psrc.data(), psrc.size()))) return rc;
  if ((rc = dupload(p, &d.d_amp, amp, (size_t)n_src * nsteps1))) return rc;
  if (amp_im && (rc = dupload(p, &d.d_amp_im, amp_im, (size_t)n_src * nsteps1))) return rc;
  p->dipoles.push_back(d);
  return OEM_OK;
}

int oem_plan_add_dipoles(oem_plan* p, int magnetic, int n_pts, const int32_t* ijk,
                         const int32_t* comp, const float* coef, const int32_t* src, int n_src,
                         int64_t nsteps1, const double* amp) {
  if (p && p->is_complex)
    return set_error(OEM_ERR_STATE, "a complex plan takes complex dipole amplitudes");
  return add_dipoles_impl(p, magnetic, n_pts, ijk, comp, coef, src, n_src, nsteps1, amp,
                          nullptr);
}

int oem_plan_add_dipoles_complex(oem_plan* p, int magnetic, int n_pts, const int32_t* ijk,
                                 const int32_t* comp, const float* coef, const int32_t* src,
                                 int n_src, int64_t nsteps1, const double* amp_re,
                                 const double* amp_im) {
  if (!p || !p->is_complex)
    return set_error(OEM_ERR_STATE, "complex dipole amplitudes need a complex plan");
  if (!amp_im) return set_error(OEM_ERR_INVALID, "null imaginary amplitude table");
  return add_dipoles_impl(p, magnetic, n_pts, ijk, comp, coef, src, n_src, nsteps1, amp_re,
                          amp_im);
}

int oem_plan_set_xchunk(oem_plan* p, int xch) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (xch < 0 || xch > 4096) return set_error(OEM_ERR_INVALID, "x chunk must be 0..4096");
  p->xch_user = xch;
  return OEM_OK;
}

int oem_plan_set_wait_expiry_check(oem_plan* p, int polls) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (polls < 0 || polls > (1 << 20))
    return set_error(OEM_ERR_INVALID, "polls must be 0..2^20");
  p->yp.expire_polls = polls;
  return OEM_OK;
}

int oem_plan_set_gradient_box(oem_plan* p, const int* box) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (!box || box[3] < 1 || box[4] < 1 || box[5] < 1 || box[0] < 0 || box[1] < 0 ||
      box[2] < 0 || box[0] + box[3] > p->nx || box[1] + box[4] > p->ny || box[2] + box[5] > p->nz)
    return set_error(OEM_ERR_INVALID, "gradient box outside the grid");
  for (int q = 0; q < 6; ++q) p->gbox[q] = box[q];
  p->gbox_set = true;
  return OEM_OK;
}

int oem_plan_enable_checkpoints(oem_plan* p, int k) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (k < 1) return set_error(OEM_ERR_INVALID, "checkpoint interval must be >= 1");
  p->ckpt_k = k;
  return OEM_OK;
}

int oem_plan_adjoint_flux(oem_plan* p, int mon_id, const double* weights, const double* dA1,
                          const double* dA2, double* g_ca, double* g_cb, void* stream) {
  if (!p) return set_error(OEM_ERR_INVALID, "null plan");
  const int box[6] = {0, 0, 0, p->nx, p->ny, p->nz};
  return oem_plan_adjoint_flux_box(p, mon_id, weights, dA1, dA2, box, g_ca, g_cb, stream);
}

int oem_plan_adjoint_flux_box(oem_plan* p, int mon_id, const double* weights, const double* dA1,
                              const double* dA2, const int* box, double* g_ca, double* g_cb,
                              void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (!box || box[3] < 1 || box[4] < 1 || box[5] < 1 || box[0] < 0 || box[1] < 0 ||
      box[2] < 0 || box[0] + box[3] > p->nx || box[1] + box[4] > p->ny || box[2] + box[5] > p->nz)
    return set_error(OEM_ERR_INVALID, "gradient box outside the grid");
  if (p->ckpt_k < 1) return set_error(OEM_ERR_STATE, "checkpoints were not enabled");
  if (p->steps != p->n_total) return set_error(OEM_ERR_STATE, "run the whole forward pass first");
  if (mon_id < 0 || mon_id >= (int)p->mons.size() || p->mons[mon_id].kind != 0)
    return set_error(OEM_ERR_INVALID, "not a flux monitor id");
  if (p->mons[mon_id].n_total < p->n_total)
    return set_error(OEM_ERR_INVALID, "the monitor's phase table is shorter than the run");
  if (!weights || !dA1 || !dA2 || !g_ca || !g_cb) return set_error(OEM_ERR_INVALID, "null argument");
  if (p->is_complex || !p->absorbers.empty() || !p->mixes.empty() || !p->tensors.empty() ||
      !p->mods.empty())
    return set_error(OEM_ERR_UNSUPPORTED,
                     "the adjoint covers real plans without absorbers, mixed or tensor media or "
                     "time modulation");
  for (int64_t q = 0; q < (int64_t)p->ckpt.size(); ++q)
    if (p->ckpt_step[q] != q * p->ckpt_k) return set_error(OEM_ERR_STATE, "missing checkpoint");
  if ((rc = use_device(p))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Monitor& m = p->mons[mon_id];
  if ((rc = oem_plan_flush(p, stream))) return rc;
  const int64_t plane = m.cells, nf = m.nf;
  std::vector<double> re((size_t)4 * nf * plane), im(re.size());
  OEM_CUDA(cudaMemcpy(re.data(), m.d_re, re.size() * sizeof(double), cudaMemcpyDeviceToHost));
  OEM_CUDA(cudaMemcpy(im.data(), m.d_im, im.size() * sizeof(double), cudaMemcpyDeviceToHost));
  // objective J = sum_f w_f 1/2 sum_p [Re(E1 H2*) dA1 - Re(E2 H1*) dA2] (transverse axes
  // ascending): per term the weights of (cos, sin) of the phase table
  std::vector<double> coef((size_t)4 * nf * plane * 2);
  auto at = [&](int c, int64_t f, int64_t q) { return ((size_t)c * nf + f) * plane + q; };
  for (int64_t f = 0; f < nf; ++f)
    for (int o1 = 0; o1 < m.n1; ++o1)
      for (int o2 = 0; o2 < m.n2; ++o2) {
        const int64_t q = (int64_t)o1 * m.n2 + o2;
        const double a1 = dA1[q], a2 = dA2[q];
        const double w = 0.5 * weights[f];
        const double e1r = re[at(0, f, q)], e1i = im[at(0, f, q)];
        const double e2r = re[at(1, f, q)], e2i = im[at(1, f, q)];
        const double h1r = re[at(2, f, q)], h1i = im[at(2, f, q)];
        const double h2r = re[at(3, f, q)], h2i = im[at(3, f, q)];
        const double v[4][2] = {{w * a1 * h2r, w * a1 * h2i}, {-w * a2 * h1r, -w * a2 * h1i},
                                {-w * a2 * e2r, -w * a2 * e2i}, {w * a1 * e1r, w * a1 * e1i}};
        for (int c = 0; c < 4; ++c) {
          coef[2 * at(c, f, q)] = v[c][0];
          coef[2 * at(c, f, q) + 1] = v[c][1];
        }
      }
  // adjoint buffers for this call
  std::vector<void*> tmp;
  auto alloc = [&](auto** ptr, size_t count) -> int {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(**ptr));
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_error(OEM_ERR_NOMEM, "adjoint buffers do not fit in device memory");
    }
    tmp.push_back(q);
    OEM_CUDA(cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(**ptr), s));
    *ptr = static_cast<std::remove_reference_t<decltype(*ptr)>>(q);
    return OEM_OK;
  };
  auto release = [&]() { cudaStreamSynchronize(s); for (void* q : tmp) cudaFree(q); };
  const size_t ncp = (size_t)p->nx * p->ny * p->nzp;
  const int K = p->ckpt_k;
  AdjState S{};
  AdjFlux af{};
  double* dcoef = nullptr;
  float* seg = nullptr;
  for (int q = 0; q < 6; ++q) S.box[q] = box[q];
  const size_t nb = (size_t)box[3] * box[4] * box[5];
  rc = OEM_OK;
  for (int c = 0; c < 6 && !rc; ++c) rc = alloc(&S.lam[c], ncp);
  for (int c = 0; c < 6 && !rc; ++c) rc = alloc(&S.dbare[c], ncp);
  for (int c = 0; c < 6 && !rc; ++c) rc = alloc(&S.dbarh[c], ncp);
  for (int c = 0; c < 3 && !rc; ++c) rc = alloc(&S.gca[c], nb);
  for (int c = 0; c < 3 && !rc; ++c) rc = alloc(&S.gcb[c], nb);
  if (!rc && p->yp.has_ade) rc = alloc(&S.lps, (size_t)std::max<int64_t>(p->n_pole_total, 1));
  for (int a = 0; a < 3 && !rc; ++a)
    for (int side = 0; side < 2 && !rc; ++side) {
      const int L = side == 0 ? p->axh[a].lo : p->axh[a].hi;
      if (L <= 0) continue;
      size_t cnt = a == 0 ? (size_t)L * p->ny * p->nzp
                          : (a == 1 ? (size_t)p->nx * L * p->nzp : (size_t)p->nx * p->ny * L);
      for (int slot = 0; slot < 2 && !rc; ++slot) {
        rc = alloc(&S.lpsih.p[a][slot][side], cnt);
        if (!rc) rc = alloc(&S.lpsie.p[a][slot][side], cnt);
      }
    }
  // E of the box at every step: recorded during the forward run when this box was declared
  // before it, else recomputed segment by segment from the checkpoints
  bool use_hist = p->hist != nullptr;
  for (int q = 0; q < 6; ++q) use_hist = use_hist && p->gbox[q] == box[q];
  if (!rc) rc = alloc(&dcoef, coef.size());
  if (!rc && !use_hist) rc = alloc(&seg, (size_t)(K + 1) * 3 * nb);
  if (rc) {
    release();
    return rc;
  }
  OEM_CUDA(cudaMemcpyAsync(dcoef, coef.data(), coef.size() * sizeof(double),
                           cudaMemcpyHostToDevice, s));
  af.axis = m.axis; af.km = m.km; af.n1 = m.n1; af.n2 = m.n2; af.nf = (int)nf;
  af.phase = m.d_phase;
  af.coef = dcoef;
  const int64_t N = p->n_total;
  const int64_t nseg = (N + K - 1) / K;
  const YeeParams& P = p->yp;
  cudaError_t e = cudaSuccess;
  for (int64_t sg = nseg - 1; sg >= 0 && !rc; --sg) {
    const int64_t n0 = sg * K, n1 = std::min<int64_t>(N, n0 + K);
    if (!use_hist) {
      // recompute the segment from its checkpoint, keeping E of the box at every step
      if ((rc = load_state(p, (int)sg, s))) break;
      for (int64_t t = 0; t <= n1 - n0 && !rc; ++t) {
        if (t > 0) rc = enqueue_step(p, s, false);
        if (!rc && (e = launch_adj_snap(P, S, seg + (size_t)t * 3 * nb, s)) != cudaSuccess)
          rc = cuda_error(e, "segment copy");
      }
    }
    for (int64_t n = n1 - 1; n >= n0 && !rc; --n) {
      const float* en = use_hist ? p->hist + (size_t)n * 3 * nb : seg + (size_t)(n - n0) * 3 * nb;
      const float* en1 =
          use_hist ? p->hist + (size_t)(n + 1) * 3 * nb : seg + (size_t)(n - n0 + 1) * 3 * nb;
      if ((e = launch_adj_src(P, af, S, (int)n, s)) != cudaSuccess) rc = cuda_error(e, "adj_src");
      if (!rc && (e = launch_adj_step(P, S, en, en1, s)) != cudaSuccess)
        rc = cuda_error(e, "adj_step");
    }
  }
  if (!rc)
    for (int c = 0; c < 3 && !rc; ++c)
      if ((e = cudaMemcpyAsync(g_ca + (size_t)c * nb, S.gca[c], nb * sizeof(double),
                               cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
          (e = cudaMemcpyAsync(g_cb + (size_t)c * nb, S.gcb[c], nb * sizeof(double),
                               cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        rc = cuda_error(e, "gradient readout");
  release();
  return rc;
}

int oem_plan_add_absorber(oem_plan* p, int axis, int g0, int nlay, const double* decay_int,
                          const double* decay_half) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (axis < 0 || axis > 2) return set_error(OEM_ERR_INVALID, "absorber axis must be 0, 1 or 2");
  const int n = axis == 0 ? p->nx : axis == 1 ? p->ny : p->nz;
  if (nlay < 1 || g0 < 0 || g0 + nlay > n)
    return set_error(OEM_ERR_INVALID, "absorber layers outside the axis");
  if (!decay_int || !decay_half) return set_error(OEM_ERR_INVALID, "null decay profile");
  for (int l = 0; l < nlay; ++l)
    if (!(decay_int[l] > 0.0 && decay_int[l] <= 1.0) || !(decay_half[l] > 0.0 && decay_half[l] <= 1.0))
      return set_error(OEM_ERR_INVALID, "absorber decay factors must lie in (0, 1]");
  if ((rc = use_device(p))) return rc;
  Absorber a;
  a.axis = axis; a.g0 = g0; a.nlay = nlay;
  std::vector<float> di(decay_int, decay_int + nlay), dh(decay_half, decay_half + nlay);
  if ((rc = dupload(p, &a.d_int, di.data(), di.size()))) return rc;
  if ((rc = dupload(p, &a.d_half, dh.data(), dh.size()))) return rc;
  p->absorbers.push_back(a);
  return OEM_OK;
}

int oem_plan_add_modulation(oem_plan* p, int n_entry, const int* comp, const int64_t* cell,
                            const float* amp, const float* cph, const float* sph,
                            const float* eps_s, const float* sd, const float* gg, int ntab,
                            const float* cs_tab, double dte) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (n_entry < 1 || ntab < 1) return set_error(OEM_ERR_INVALID, "empty modulation");
  if (!comp || !cell || !amp || !cph || !sph || !eps_s || !sd || !gg || !cs_tab)
    return set_error(OEM_ERR_INVALID, "null modulation table");
  if (p->is_complex) return set_error(OEM_ERR_UNSUPPORTED, "time modulation on a complex plan");
  const int64_t ncell = (int64_t)p->nx * p->ny * p->nz;
  std::vector<uint8_t> seen((size_t)3 * ncell, 0);
  for (int e = 0; e < n_entry; ++e) {
    if (comp[e] < 0 || comp[e] > 2 || cell[e] < 0 || cell[e] >= ncell)
      return set_error(OEM_ERR_INVALID, "modulation entry outside the grid");
    uint8_t& f = seen[(size_t)comp[e] * ncell + cell[e]];
    if (f) return set_error(OEM_ERR_INVALID, "duplicate (comp, cell) modulation entry");
    f = 1;
    if (!(eps_s[e] - std::fabs(amp[e]) > 0.f))
      return set_error(OEM_ERR_INVALID, "eps_s - |amp| must stay positive");
  }
  if ((rc = use_device(p))) return rc;
  Modulation m;
  m.n = n_entry;
  m.ntab = ntab;
  m.dte = (float)dte;
  std::vector<int64_t> padded(n_entry);
  for (int e = 0; e < n_entry; ++e) {
    const int64_t r = cell[e] / p->nz, k = cell[e] % p->nz;
    padded[e] = r * p->nzp + k;
  }
  if ((rc = dupload(p, &m.comp, comp, n_entry))) return rc;
  if ((rc = dupload(p, &m.cell, padded.data(), n_entry))) return rc;
  if ((rc = dupload(p, &m.amp, amp, n_entry))) return rc;
  if ((rc = dupload(p, &m.cph, cph, n_entry))) return rc;
  if ((rc = dupload(p, &m.sph, sph, n_entry))) return rc;
  if ((rc = dupload(p, &m.eps, eps_s, n_entry))) return rc;
  if ((rc = dupload(p, &m.sd, sd, n_entry))) return rc;
  if ((rc = dupload(p, &m.gg, gg, n_entry))) return rc;
  if ((rc = dupload(p, &m.cs, reinterpret_cast<const float4*>(cs_tab), (size_t)ntab))) return rc;
  p->mods.push_back(m);
  p->mod_cells.emplace_back(cell, cell + n_entry);
  return OEM_OK;
}

int oem_plan_set_axis_phase(oem_plan* p, int axis, const double* mnx_im, const double* mpv_im) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (axis < 0 || axis > 2) return set_error(OEM_ERR_INVALID, "axis must be 0, 1 or 2");
  if (!mnx_im || !mpv_im) return set_error(OEM_ERR_INVALID, "null mask table");
  if (!p->axh[axis].set) return set_error(OEM_ERR_STATE, "set the axis tables first");
  if (!p->dipoles.empty() || !p->mons.empty() || !p->tmons.empty() || !p->planes.empty())
    return set_error(OEM_ERR_STATE, "mark the plan complex before adding sources and monitors");
  const int n = axis == 0 ? p->nx : axis == 1 ? p->ny : p->nz;
  p->axh[axis].mnx_i.assign(mnx_im, mnx_im + n);
  p->axh[axis].mpv_i.assign(mpv_im, mpv_im + n);
  p->is_complex = true;
  return OEM_OK;
}

int oem_plan_add_mode_source(oem_plan* p, int axis, int kh, int ks, int n1, int n2,
                             double coef_h1, double coef_h2, double coef_e1, double coef_e2,
                             int n_terms, const float* profiles, int64_t ntab,
                             const double* amp_e, const double* amp_h) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (axis < 0 || axis > 2) return set_error(OEM_ERR_INVALID, "mode axis must be 0, 1 or 2");
  const int dims[3] = {p->nx, p->ny, p->nz};
  const int t1 = (axis + 1) % 3, t2 = (axis + 2) % 3;
  if (n1 != dims[t1] || n2 != dims[t2])
    return set_error(OEM_ERR_INVALID, "mode profile must cover the whole plane (n_t1, n_t2)");
  if (kh < 0 || kh >= dims[axis] || ks < 0 || ks >= dims[axis])
    return set_error(OEM_ERR_INVALID, "mode injection plane outside the grid");
  if (n_terms < 1 || ntab < 1 || !profiles || !amp_e || !amp_h)
    return set_error(OEM_ERR_INVALID, "empty mode source");
  if ((rc = use_device(p))) return rc;
  ModeSrc m;
  m.axis = axis; m.kh = kh; m.ks = ks; m.n1 = n1; m.n2 = n2; m.nterms = n_terms;
  m.ch1 = (float)coef_h1; m.ch2 = (float)coef_h2; m.ce1 = (float)coef_e1; m.ce2 = (float)coef_e2;
  m.ntab = ntab;
  const size_t plane = (size_t)n1 * n2;
  if ((rc = dupload(p, &m.d_prof, profiles, (size_t)n_terms * 8 * plane))) return rc;
  if ((rc = dupload(p, &m.d_amp_e, amp_e, (size_t)n_terms * ntab * 2))) return rc;
  if ((rc = dupload(p, &m.d_amp_h, amp_h, (size_t)n_terms * ntab * 2))) return rc;
  p->modesrcs.push_back(m);
  return OEM_OK;
}

static int add_monitor_common(oem_plan* p, Monitor& m, int nf, int64_t n_total, const float* phase,
                              int batch, int* id) {
  int rc;
  if (nf < 1 || n_total < 1 || !phase || !id) return set_error(OEM_ERR_INVALID, "empty monitor");
  if (batch < 1 || batch > 32) return set_error(OEM_ERR_INVALID, "batch must be 1..32");
  if ((rc = use_device(p))) return rc;
  m.nf = nf;
  m.T = batch;
  m.n_total = n_total;
  if ((rc = dupload(p, &m.d_phase, phase, (size_t)n_total * nf * 4))) return rc;
  m.cplx = p->is_complex ? 1 : 0;
  if ((rc = dalloc(p, &m.d_snap, (size_t)m.T * m.ncomp * (m.cplx ? 2 : 1) * m.cells))) return rc;
  if ((rc = dalloc(p, &m.d_re, (size_t)m.ncomp * nf * m.cells))) return rc;
  if ((rc = dalloc(p, &m.d_im, (size_t)m.ncomp * nf * m.cells))) return rc;
  int minus1 = -1;
  if ((rc = dupload(p, &m.d_done, &minus1, 1))) return rc;
  if ((rc = dalloc(p, &m.d_count, 1))) return rc;
  *id = (int)p->mons.size();
  p->mons.push_back(m);
  return OEM_OK;
}

int oem_plan_add_flux_monitor(oem_plan* p, int axis, int km, int nf, int64_t n_total,
                              const float* phase, int batch, int* id) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (axis < 0 || axis > 2) return set_error(OEM_ERR_INVALID, "monitor axis must be 0..2");
  const int dims[3] = {p->nx, p->ny, p->nz};
  if (km < 1 || km >= dims[axis])
    return set_error(OEM_ERR_INVALID, "flux plane index must be in [1, n) of its normal axis");
  Monitor m;
  m.kind = 0;
  m.axis = axis;
  m.km = km;
  const int t1 = axis == 0 ? 1 : 0, t2 = axis == 2 ? 1 : 2;
  m.n1 = dims[t1];
  m.n2 = dims[t2];
  m.ncomp = 4;
  m.cells = (int64_t)m.n1 * m.n2;
  return add_monitor_common(p, m, nf, n_total, phase, batch, id);
}

int oem_plan_add_box_monitor(oem_plan* p, int i0, int j0, int k0, int ni, int nj, int nk, int nf,
                             int64_t n_total, const float* phase, int batch, int* id) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (ni < 1 || nj < 1 || nk < 1 || i0 < 0 || j0 < 0 || k0 < 0 || i0 + ni > p->nx ||
      j0 + nj > p->ny || k0 + nk > p->nz)
    return set_error(OEM_ERR_INVALID, "field monitor box outside the grid");
  Monitor m;
  m.kind = 1;
  m.i0 = i0; m.j0 = j0; m.k0 = k0;
  m.ni = ni; m.nj = nj; m.nk = nk;
  m.ncomp = 6;
  m.cells = (int64_t)ni * nj * nk;
  return add_monitor_common(p, m, nf, n_total, phase, batch, id);
}

int oem_plan_add_time_monitor(oem_plan* p, int nc, const int32_t* comps, int i0, int j0, int k0,
                              int ni, int nj, int nk, int beg, int end, int iv, int nslots,
                              int* id) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (nc < 1 || nc > 6 || !comps || !id) return set_error(OEM_ERR_INVALID, "bad component list");
  if (ni < 1 || nj < 1 || nk < 1 || i0 < 0 || j0 < 0 || k0 < 0 || i0 + ni > p->nx ||
      j0 + nj > p->ny || k0 + nk > p->nz)
    return set_error(OEM_ERR_INVALID, "time monitor box outside the grid");
  if (iv < 1 || nslots < 0) return set_error(OEM_ERR_INVALID, "bad sampling interval");
  if ((rc = use_device(p))) return rc;
  TimeMon m;
  m.nc = nc;
  for (int q = 0; q < nc; ++q) {
    if (comps[q] < 0 || comps[q] > 5) return set_error(OEM_ERR_INVALID, "component out of range");
    m.comps[q] = comps[q];
  }
  m.i0 = i0; m.j0 = j0; m.k0 = k0; m.ni = ni; m.nj = nj; m.nk = nk;
  m.beg = beg; m.end = end; m.iv = iv; m.nslots = nslots;
  if ((rc = dalloc(p, &m.d_buf, (size_t)nc * std::max(nslots, 1) * ni * nj * nk))) return rc;
  if (p->is_complex &&
      (rc = dalloc(p, &m.d_buf_i, (size_t)nc * std::max(nslots, 1) * ni * nj * nk)))
    return rc;
  *id = (int)p->tmons.size();
  p->tmons.push_back(m);
  return OEM_OK;
}

int oem_plan_add_flux_time_monitor(oem_plan* p, int axis, int nplanes, const double* w,
                                   const int* ke, const int* kh, const double* wh, int n1,
                                   const int* e1, const int* lo1, const int* hi1,
                                   const double* wlo1, const double* whi1, int n2, const int* e2,
                                   const int* lo2, const int* hi2, const double* wlo2,
                                   const double* whi2, const double* dS, int beg, int end, int iv,
                                   int nslots, int* id) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (p->is_complex) return set_error(OEM_ERR_UNSUPPORTED, "flux time monitors on a complex plan");
  if (axis < 0 || axis > 2) return set_error(OEM_ERR_INVALID, "monitor axis must be 0..2");
  if (nplanes < 1 || nplanes > 2 || n1 < 1 || n2 < 1 || iv < 1 || nslots < 0 || !id)
    return set_error(OEM_ERR_INVALID, "bad flux time monitor shape");
  if (!w || !ke || !kh || !wh || !e1 || !lo1 || !hi1 || !wlo1 || !whi1 || !e2 || !lo2 || !hi2 ||
      !wlo2 || !whi2 || !dS)
    return set_error(OEM_ERR_INVALID, "null flux time table");
  const int dims[3] = {p->nx, p->ny, p->nz};
  const int t1 = axis == 0 ? 1 : 0, t2 = axis == 2 ? 1 : 2;
  for (int q = 0; q < nplanes; ++q)
    if (ke[q] < 0 || ke[q] >= dims[axis] || kh[q] < 0 || kh[q] + 1 >= dims[axis])
      return set_error(OEM_ERR_INVALID, "flux time plane outside the grid");
  auto inside = [](const int* a, int n, int lim) {
    for (int q = 0; q < n; ++q)
      if (a[q] < 0 || a[q] >= lim) return false;
    return true;
  };
  if (!inside(e1, n1, dims[t1]) || !inside(lo1, n1, dims[t1]) || !inside(hi1, n1, dims[t1]) ||
      !inside(e2, n2, dims[t2]) || !inside(lo2, n2, dims[t2]) || !inside(hi2, n2, dims[t2]))
    return set_error(OEM_ERR_INVALID, "flux time sample outside the grid");
  if ((rc = use_device(p))) return rc;
  FluxTimeMon m;
  m.axis = axis;
  m.nplanes = nplanes;
  for (int q = 0; q < nplanes; ++q) {
    m.w[q] = w[q];
    m.ke[q] = ke[q];
    m.kh[q] = kh[q];
    m.wh[q][0] = wh[2 * q];
    m.wh[q][1] = wh[2 * q + 1];
  }
  m.n1 = n1; m.n2 = n2;
  m.beg = beg; m.end = end; m.iv = iv; m.slots = nslots;
  const int64_t samples = (int64_t)nplanes * n1 * n2;
  m.nblocks = (int)std::max<int64_t>(1, std::min<int64_t>((samples + 255) / 256, 148 * 4));
  if ((rc = dupload(p, &m.e1, e1, n1)) || (rc = dupload(p, &m.lo1, lo1, n1)) ||
      (rc = dupload(p, &m.hi1, hi1, n1)) || (rc = dupload(p, &m.wlo1, wlo1, 2 * (size_t)n1)) ||
      (rc = dupload(p, &m.whi1, whi1, n1)) || (rc = dupload(p, &m.e2, e2, n2)) ||
      (rc = dupload(p, &m.lo2, lo2, n2)) || (rc = dupload(p, &m.hi2, hi2, n2)) ||
      (rc = dupload(p, &m.wlo2, wlo2, 2 * (size_t)n2)) || (rc = dupload(p, &m.whi2, whi2, n2)) ||
      (rc = dupload(p, &m.dS, dS, (size_t)n1 * n2)))
    return rc;
  if ((rc = dalloc(p, &m.ekeep, (size_t)samples * 2)) ||
      (rc = dalloc(p, &m.part, (size_t)m.nblocks * 2)) ||
      (rc = dalloc(p, &m.buf, (size_t)std::max(nslots, 1))))
    return rc;
  *id = (int)p->ftmons.size();
  p->ftmons.push_back(m);
  return OEM_OK;
}

int oem_plan_read_flux_time(oem_plan* p, int id, double* out, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (id < 0 || id >= (int)p->ftmons.size() || !out)
    return set_error(OEM_ERR_INVALID, "flux time monitor id out of range");
  if ((rc = use_device(p))) return rc;
  const FluxTimeMon& m = p->ftmons[id];
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (m.slots)
    OEM_CUDA(cudaMemcpyAsync(out, m.buf, (size_t)m.slots * sizeof(double), cudaMemcpyDeviceToHost, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  return check_device_error(p);
}

static int tfsf_side(oem_plan* p, int n, const oem_tfsf_face* faces, oem_tfsf_face** dfaces,
                     int64_t** dofs, std::vector<std::pair<int, int>>& groups,
                     std::vector<int64_t>& points) {
  int rc;
  const int64_t ncp = (int64_t)p->nx * p->ny * p->nzp;
  std::vector<int64_t> ofs;
  for (int f = 0; f < n; ++f) {
    const oem_tfsf_face& F = faces[f];
    if (F.comp < 0 || F.comp > 5 || F.np < 0 || F.nq < 0)
      return set_error(OEM_ERR_INVALID, "bad TFSF face");
    if (F.np > 0 && F.nq > 0) {
      const int64_t last = F.base + (int64_t)(F.np - 1) * F.sp + (int64_t)(F.nq - 1) * F.sq;
      if (F.base < 0 || last < 0 || F.base >= ncp || last >= ncp)
        return set_error(OEM_ERR_INVALID, "TFSF face outside the grid");
    }
    if (f > 0 && F.group < faces[f - 1].group)
      return set_error(OEM_ERR_INVALID, "TFSF faces must be ordered by group");
    if (f == 0 || F.group != faces[f - 1].group) {
      groups.push_back({f, 0});
      points.push_back(0);
      ofs.push_back(0);
    }
    groups.back().second += 1;
    points.back() += (int64_t)F.np * F.nq;
    ofs.push_back(points.back());
  }
  if (n == 0) return OEM_OK;
  if ((rc = dupload(p, dfaces, faces, (size_t)n))) return rc;
  if ((rc = dupload(p, dofs, ofs.data(), ofs.size()))) return rc;
  return OEM_OK;
}

int oem_plan_add_tfsf(oem_plan* p, int n_e, const oem_tfsf_face* e_faces, int n_h,
                      const oem_tfsf_face* h_faces, int ex_rows, int ex_n, const double* ex_tab,
                      int hy_rows, int hy_n, const double* hy_tab) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (p->is_complex) return set_error(OEM_ERR_UNSUPPORTED, "TFSF boxes on a complex plan");
  if (n_e < 0 || n_h < 0 || (n_e && !e_faces) || (n_h && !h_faces) || !ex_tab || !hy_tab ||
      ex_rows < 1 || ex_n < 1 || hy_rows < 1 || hy_n < 1)
    return set_error(OEM_ERR_INVALID, "bad TFSF tables");
  if ((rc = use_device(p))) return rc;
  Tfsf t;
  if ((rc = tfsf_side(p, n_e, e_faces, &t.e_faces, &t.e_ofs, t.e_groups, t.e_points))) return rc;
  if ((rc = tfsf_side(p, n_h, h_faces, &t.h_faces, &t.h_ofs, t.h_groups, t.h_points))) return rc;
  t.ex_rows = ex_rows; t.ex_n = ex_n; t.hy_rows = hy_rows; t.hy_n = hy_n;
  if ((rc = dupload(p, &t.ex_tab, ex_tab, (size_t)ex_rows * ex_n))) return rc;
  if ((rc = dupload(p, &t.hy_tab, hy_tab, (size_t)hy_rows * hy_n))) return rc;
  p->tfsfs.push_back(std::move(t));
  return OEM_OK;
}

int oem_plan_add_tensor(oem_plan* p, int n_entry, const int* comp, const int64_t* cell,
                        const float* m1, const float* m2, const float* pec) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (p->is_complex) return set_error(OEM_ERR_UNSUPPORTED, "tensor media on a complex plan");
  if (n_entry < 1 || !comp || !cell || !m1 || !m2 || !pec)
    return set_error(OEM_ERR_INVALID, "empty tensor table");
  const int64_t ncell = (int64_t)p->nx * p->ny * p->nz;
  std::vector<int64_t> padded(n_entry);
  for (int e = 0; e < n_entry; ++e) {
    if (comp[e] < 0 || comp[e] > 2 || cell[e] < 0 || cell[e] >= ncell)
      return set_error(OEM_ERR_INVALID, "tensor entry outside the grid");
    padded[e] = cell[e] / p->nz * p->nzp + cell[e] % p->nz;
  }
  if ((rc = use_device(p))) return rc;
  TensorSet t;
  t.n = n_entry;
  if ((rc = dupload(p, &t.comp, comp, n_entry)) || (rc = dupload(p, &t.cell, padded.data(), n_entry)) ||
      (rc = dupload(p, &t.m1, m1, 3 * (size_t)n_entry)) ||
      (rc = dupload(p, &t.m2, m2, 3 * (size_t)n_entry)) || (rc = dupload(p, &t.pec, pec, n_entry)) ||
      (rc = dalloc(p, &t.rhs, n_entry)) || (rc = dalloc(p, &t.enew, n_entry)))
    return rc;
  p->tensors.push_back(t);
  return OEM_OK;
}

int oem_plan_add_dispersion_mix(oem_plan* p, int n_entry, const int* comp, const int64_t* cell,
                                const int* p_ofs, const float* p_coef, int n_p, const int* q_ofs,
                                const float* q_coef, int n_q, const float* k, double dte) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  if (p->is_complex) return set_error(OEM_ERR_UNSUPPORTED, "mixed dispersion on a complex plan");
  if (n_entry < 1 || !comp || !cell || !p_ofs || !q_ofs || !k || n_p < 0 || n_q < 0 ||
      (n_p > 0 && !p_coef) || (n_q > 0 && !q_coef))
    return set_error(OEM_ERR_INVALID, "empty mixed-dispersion table");
  if (!(dte > 0.0)) return set_error(OEM_ERR_INVALID, "dt / eps0 must be positive");
  const int64_t ncell = (int64_t)p->nx * p->ny * p->nz;
  std::vector<int64_t> padded(n_entry);
  for (int e = 0; e < n_entry; ++e) {
    if (comp[e] < 0 || comp[e] > 2 || cell[e] < 0 || cell[e] >= ncell)
      return set_error(OEM_ERR_INVALID, "mixed-dispersion entry outside the grid");
    padded[e] = cell[e] / p->nz * p->nzp + cell[e] % p->nz;
  }
  for (const int* ofs : {p_ofs, q_ofs}) {
    const int last = ofs == p_ofs ? n_p : n_q;
    if (ofs[0] != 0 || ofs[n_entry] != last)
      return set_error(OEM_ERR_INVALID, "pole offsets do not span the pole table");
    for (int e = 0; e < n_entry; ++e)
      if (ofs[e + 1] < ofs[e]) return set_error(OEM_ERR_INVALID, "pole offsets not monotonic");
  }
  if ((rc = use_device(p))) return rc;
  MixSet m;
  m.n = n_entry;
  m.dte = (float)dte;
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4* pc = n_p ? reinterpret_cast<const float4*>(p_coef) : &zero4;
  const float4* qc = n_q ? reinterpret_cast<const float4*>(q_coef) : &zero4;
  if ((rc = dupload(p, &m.comp, comp, n_entry)) ||
      (rc = dupload(p, &m.cell, padded.data(), n_entry)) ||
      (rc = dupload(p, &m.p_ofs, p_ofs, (size_t)n_entry + 1)) ||
      (rc = dupload(p, &m.q_ofs, q_ofs, (size_t)n_entry + 1)) ||
      (rc = dupload(p, &m.pc, pc, std::max(n_p, 1))) ||
      (rc = dupload(p, &m.qc, qc, std::max(n_q, 1))) ||
      (rc = dupload(p, &m.k, reinterpret_cast<const float4*>(k), n_entry)) ||
      (rc = dalloc(p, &m.P, std::max(n_p, 1))) || (rc = dalloc(p, &m.Q, std::max(n_q, 1))) ||
      (rc = dalloc(p, &m.sp, n_entry)) || (rc = dalloc(p, &m.sq, n_entry)) ||
      (rc = dalloc(p, &m.dtot, n_entry)) || (rc = dalloc(p, &m.dh, n_entry)))
    return rc;
  p->mixes.push_back(m);
  return OEM_OK;
}

// Box snapshots written by the warp-specialised E update (k_e_ws<true>) instead of k_snap_boxes,
// when OEM_B200_SNAP=update asks for it: a real plan on those kernels whose only E-side work
// after the update is E dipoles (they rewrite the rows of their targets), with one to
// kMaxSnapBoxes box monitors. Exact, but slower on the 512^3 workload (the E update 1.228 against
// 1.085 ms, the step 2.255 against 2.207 ms): the one lane per warp that holds a z-normal box's
// cells delays its warp's release of every stage, in half the blocks.
static void plan_snap_boxes(oem_plan* p) {
  p->snapk = SnapBoxes{};
  const char* ev = getenv("OEM_B200_SNAP");
  if (!ev || strcmp(ev, "update") != 0) return;
  if (p->is_complex || p->fused || p->basic_kernels != 3) return;
  if (!p->planes.empty() || !p->tfsfs.empty() || !p->modesrcs.empty() || !p->mixes.empty() ||
      !p->tensors.empty() || !p->absorbers.empty())
    return;
  int nb = 0;
  for (const Monitor& m : p->mons) nb += m.kind == 1;
  if (nb == 0 || nb > kMaxSnapBoxes) return;
  for (const Monitor& m : p->mons) {
    if (m.kind != 1) continue;
    SnapBox& b = p->snapk.b[p->snapk.n++];
    b.i0 = m.i0; b.ni = m.ni; b.j0 = m.j0; b.nj = m.nj; b.k0 = m.k0; b.nk = m.nk;
    b.T = m.T;
    b.cells = m.cells;
    b.snap = m.d_snap;
  }
  p->snapk.step = p->d_step;
}

int oem_plan_finalize(oem_plan* p, int64_t n_total) {
  int rc = check_plan(p, false);
  if (rc) return rc;
  for (int a = 0; a < 3; ++a)
    if (!p->axh[a].set) return set_error(OEM_ERR_STATE, "axis " + std::to_string(a) + " not set");
  if (p->mats.empty()) return set_error(OEM_ERR_STATE, "materials not set");
  if (n_total < 0) return set_error(OEM_ERR_INVALID, "negative step count");
  for (const PlaneSrc& s : p->planes)
    if (s.ntab < n_total) return set_error(OEM_ERR_INVALID, "plane-wave table shorter than the run");
  for (const DipoleSet& d : p->dipoles)
    if (d.nsteps1 < n_total) return set_error(OEM_ERR_INVALID, "dipole table shorter than the run");
  for (const ModeSrc& m : p->modesrcs)
    if (m.ntab < n_total) return set_error(OEM_ERR_INVALID, "mode amplitude table shorter than the run");
  if (p->is_complex && (p->n_pole_total > 0 || !p->pset_ofs.empty()))
    return set_error(OEM_ERR_UNSUPPORTED, "dispersive media on a complex (Bloch) plan");
  for (const Monitor& m : p->mons)
    if (m.n_total < n_total) return set_error(OEM_ERR_INVALID, "phase table shorter than the run");
  for (const Modulation& m : p->mods)
    if (m.ntab < n_total) return set_error(OEM_ERR_INVALID, "modulation table shorter than the run");
  for (const Tfsf& t : p->tfsfs)
    if (t.ex_rows < n_total + 1 || t.hy_rows < n_total)
      return set_error(OEM_ERR_INVALID, "TFSF incident table shorter than the run");
  if (!p->mods.empty() && !p->dev_index) {
    // every modulated cell owns its material record: the kernel rewrites it in place
    std::vector<int64_t> owner(p->mats.size(), -1);
    auto idx_of = [&](int64_t c) -> int64_t {
      return p->index_bytes == 2 ? reinterpret_cast<const uint16_t*>(p->mat_index.data())[c]
                                 : reinterpret_cast<const uint32_t*>(p->mat_index.data())[c];
    };
    for (const auto& cells : p->mod_cells)
      for (int64_t c : cells) {
        int64_t& o = owner[(size_t)idx_of(c) + 1];
        if (o >= 0 && o != c)
          return set_error(OEM_ERR_INVALID, "two modulated cells share a material record");
        o = c;
      }
    const int64_t ncell = (int64_t)p->nx * p->ny * p->nz;
    for (int64_t c = 0; c < ncell; ++c) {
      const int64_t o = owner[(size_t)idx_of(c) + 1];
      if (o >= 0 && o != c)
        return set_error(OEM_ERR_INVALID, "a modulated cell shares its material record");
    }
  }
  p->mod_cells.clear();
  if ((rc = use_device(p))) return rc;
  p->n_total = n_total;
  YeeParams& P = p->yp;
  P.nx = p->nx; P.ny = p->ny; P.nz = p->nz; P.nzp = p->nzp;
  P.ch = (float)p->ch;
  P.cw = (float)p->cw;
  const size_t ncp = (size_t)p->nx * p->ny * p->nzp;
  for (int c = 0; c < 6; ++c)
    if ((rc = dalloc(p, &P.f[c], ncp))) return rc;
  if (p->is_complex) {
    for (int c = 0; c < 6; ++c)
      if ((rc = dalloc(p, &P.fi[c], ncp))) return rc;
    P.cplx = 1;
    // Large grids split the update: the warp-specialised real kernels on each part, then the
    // seam faces (cells whose neighbour mask has an imaginary part) add the terms of the
    // complex product. Needs the seam axes free of CPML slabs (their derivative enters
    // unstretched) and at most a few seam faces; otherwise the complex one-thread-per-cell
    // kernels.
    p->seam_h.clear();
    p->seam_e.clear();
    bool split = p->basic_kernels == 3;
    for (int a = 0; a < 3 && split; ++a) {
      const AxisHost& h = p->axh[a];
      const int n = a == 0 ? p->nx : a == 1 ? p->ny : p->nz;
      bool any = false;
      for (int q = 0; q < n; ++q) {
        if (!h.mnx_i.empty() && h.mnx_i[q] != 0.0) { p->seam_h.push_back({a, q}); any = true; }
        if (!h.mpv_i.empty() && h.mpv_i[q] != 0.0) { p->seam_e.push_back({a, q}); any = true; }
      }
      if (any && (h.lo > 0 || h.hi > 0)) split = false;
    }
    if (p->seam_h.size() + p->seam_e.size() > 12) split = false;
    p->cplx_ws = split;
    p->basic_kernels = split ? 3 : 1;
  }
  for (int a = 0; a < 3; ++a)
    if ((rc = upload_axis(p, a))) return rc;
  if ((rc = alloc_psi(p))) return rc;
  // materials: table with the padding material at 0, padded index shifted by one
  MatRec* dm;
  if ((rc = dupload(p, &dm, p->mats.data(), p->mats.size()))) return rc;
  P.mats = dm;
  for (Modulation& m : p->mods) m.mats = dm;
  const bool wide = p->index_bytes == 4 || p->mats.size() > 65535;
  if (p->dev_index) {
    P.mat16 = p->dev_mat16;
    P.mat32 = p->dev_mat32;
  } else {
    const size_t row = (size_t)p->nz;
    if (!wide) {
      std::vector<uint16_t> idx(ncp, 0);
      const uint16_t* src = reinterpret_cast<const uint16_t*>(p->mat_index.data());
      for (size_t r = 0; r < (size_t)p->nx * p->ny; ++r)
        for (size_t k = 0; k < row; ++k) idx[r * p->nzp + k] = (uint16_t)(src[r * row + k] + 1);
      uint16_t* d;
      if ((rc = dupload(p, &d, idx.data(), ncp))) return rc;
      P.mat16 = d;
      P.mat32 = nullptr;
    } else {
      std::vector<uint32_t> idx(ncp, 0);
      for (size_t r = 0; r < (size_t)p->nx * p->ny; ++r)
        for (size_t k = 0; k < row; ++k) {
          const size_t t = r * row + k;
          uint32_t v;
          if (p->index_bytes == 2) v = reinterpret_cast<const uint16_t*>(p->mat_index.data())[t];
          else v = reinterpret_cast<const uint32_t*>(p->mat_index.data())[t];
          idx[r * p->nzp + k] = v + 1;
        }
      uint32_t* d;
      if ((rc = dupload(p, &d, idx.data(), ncp))) return rc;
      P.mat32 = d;
      P.mat16 = nullptr;
    }
    std::vector<uint8_t>().swap(p->mat_index);
  }
  // ADE
  bool any_pole = false;
  for (const MatRec& m : p->mats)
    for (int c = 0; c < 3; ++c) any_pole |= m.np[c] > 0;
  P.has_ade = 0;
  if (any_pole) {
    if (p->pset_ofs.empty()) return set_error(OEM_ERR_STATE, "dispersive materials without pole sets");
    const int nsets = (int)p->pset_ofs.size() - 1;
    for (const MatRec& m : p->mats)
      for (int c = 0; c < 3; ++c)
        if (m.np[c] > 0 && (m.pset[c] >= nsets ||
                            p->pset_ofs[m.pset[c] + 1] - p->pset_ofs[m.pset[c]] != m.np[c]))
          return set_error(OEM_ERR_INVALID, "material pole count disagrees with its pole set");
    float4* dc;
    int* dofs;
    uint32_t* dseg;
    float2* dP;
    if ((rc = dupload(p, &dc, reinterpret_cast<const float4*>(p->pcoef.data()), p->pcoef.size() / 4))) return rc;
    if ((rc = dupload(p, &dofs, p->pset_ofs.data(), p->pset_ofs.size()))) return rc;
    if (p->dev_seg) {
      dseg = p->dev_seg;
    } else if ((rc = dupload(p, &dseg, p->seg_ofs.data(), p->seg_ofs.size()))) {
      return rc;
    }
    // four float2 of slack: bulk copies of a row's poles are widened to 16-byte boundaries
    if ((rc = dalloc(p, &dP, (size_t)std::max<int64_t>(p->n_pole_total, 1) + 4))) return rc;
    P.pcoef = dc;
    P.pset_ofs = dofs;
    P.seg_ofs = dseg;
    P.P = dP;
    P.n_pole_total = (uint32_t)p->n_pole_total;
    P.n_coef = (int)(p->pcoef.size() / 4);
    P.n_sets = (int)p->pset_ofs.size() - 1;
    if (p->basic_kernels == 3) {
      // separate pole pass: pole-indexed currents (four floats of slack for 16-byte-aligned
      // bulk reads) and the list of segments that hold poles
      if ((rc = dalloc(p, &P.J, (size_t)std::max<int64_t>(p->n_pole_total, 1) + 4))) return rc;
      const int64_t nseg = (int64_t)p->nx * p->ny * p->nzp / 32;
      unsigned long long* dcount = nullptr;
      if ((rc = dalloc(p, &dcount, 1))) return rc;
      OEM_CUDA(launch_list_pole_segments(P, nseg, nullptr, dcount, 0));
      unsigned long long h = 0;
      OEM_CUDA(cudaMemcpy(&h, dcount, sizeof(h), cudaMemcpyDeviceToHost));
      p->n_ade_segs = (int64_t)h;
      if ((rc = dalloc(p, &p->d_ade_segs, (size_t)std::max<int64_t>(p->n_ade_segs, 1)))) return rc;
      OEM_CUDA(cudaMemset(dcount, 0, sizeof(h)));
      OEM_CUDA(launch_list_pole_segments(P, nseg, p->d_ade_segs, dcount, 0));
      OEM_CUDA(cudaStreamSynchronize(0));
    }
    P.has_ade = 1;
  }
  if (p->ckpt_k > 0) {  // fields, psi and pole states of every K-th step
    std::vector<std::pair<float*, size_t>> v;
    state_arrays(p, v);
    p->ckpt_floats = 0;
    for (auto& a : v) p->ckpt_floats += a.second;
    const int64_t nslot = (n_total + p->ckpt_k - 1) / p->ckpt_k;
    p->ckpt.assign((size_t)std::max<int64_t>(nslot, 1), nullptr);
    p->ckpt_step.assign(p->ckpt.size(), -1);
    for (float*& b : p->ckpt)
      if ((rc = dalloc(p, &b, p->ckpt_floats, false))) return rc;
  }
  if ((rc = dalloc(p, &p->d_step, 1))) return rc;
  if (p->gbox_set && p->ckpt_k > 0 && !p->is_complex) {
    // the box history replaces the reverse pass's forward recompute when it fits: at most
    // 8 GB and a quarter of the free memory
    const char* hv = getenv("OEM_B200_ADJ_HISTORY");
    const size_t nbx = (size_t)p->gbox[3] * p->gbox[4] * p->gbox[5];
    const size_t bytes = ((size_t)n_total + 1) * 3 * nbx * sizeof(float);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); free_b = 0; }
    if (!(hv && strcmp(hv, "0") == 0) && bytes <= ((size_t)8 << 30) && bytes <= free_b / 4)
      if ((rc = dalloc(p, &p->hist, ((size_t)n_total + 1) * 3 * nbx))) return rc;
  }
  if ((rc = dalloc(p, &p->d_err, 1))) return rc;
  p->xch = p->basic_kernels == 2 ? stream_xchunk(P)
                                  : (p->basic_kernels == 3 ? ws_xchunk(P) : tma_xchunk(P));
  if (p->basic_kernels == 0 || p->basic_kernels == 3) {
    // grids the tensor-map encoder refuses run on the register-streaming kernels
    if (make_tma_maps(p) != OEM_OK ||
        (p->cplx_ws && make_tma_maps_of(p, p->tma_i, imag_part(P)) != OEM_OK)) {
      if (p->is_complex) {
        p->cplx_ws = false;
        p->basic_kernels = 1;
        p->xch = tma_xchunk(P);
      } else {
        p->basic_kernels = 2;
        p->xch = stream_xchunk(P);
      }
    } else {
      cudaError_t e = p->basic_kernels == 3 ? ws_setup_kernels() : tma_setup_kernels();
      if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute");
    }
  }
  if (p->xch_user > 0) p->xch = p->xch_user;
  if (const char* xs = getenv("OEM_B200_XCHUNK")) p->xch = std::max(1, atoi(xs));
  if (p->basic_kernels == 3) p->xch = std::min(p->xch, ws_max_xchunk());
  if (fused_eligible(p)) {
    // the second field bank and H-side psi the fused step writes into
    for (int c = 0; c < 6; ++c) {
      p->bank_f[0][c] = P.f[c];
      if ((rc = dalloc(p, &p->bank_f[1][c], ncp))) return rc;
    }
    p->bank_psih[0] = P.psih;
    for (int a = 0; a < 3; ++a)
      for (int side = 0; side < 2; ++side) {
        const int L = side == 0 ? p->axh[a].lo : p->axh[a].hi;
        if (L <= 0) continue;
        const size_t cnt = a == 0 ? (size_t)L * p->ny * p->nzp
                                  : (a == 1 ? (size_t)p->nx * L * p->nzp
                                            : (size_t)p->nx * p->ny * L);
        for (int slot = 0; slot < 2; ++slot)
          if ((rc = dalloc(p, &p->bank_psih[1].p[a][slot][side], cnt))) return rc;
      }
    if ((rc = make_fused_maps(p, 0)) || (rc = make_fused_maps(p, 1))) return rc;
    p->fused = true;
    set_bank(p, 0);
  }
  plan_snap_boxes(p);
  p->energy_blocks = energy_block_count(P);
  if ((rc = dalloc(p, &p->d_energy_part, 3 * (size_t)p->energy_blocks))) return rc;
  // capture: G steps per graph for small grids (launch overhead), 1 for large ones
  OEM_CUDA(cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking));
  if (p->basic_kernels == 3 && !p->fused && P.has_ade && p->n_ade_segs > 0) {
    OEM_CUDA(cudaStreamCreateWithFlags(&p->side_stream, cudaStreamNonBlocking));
    OEM_CUDA(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
    OEM_CUDA(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));
  }
  const double cells = (double)ncp;
  int G = (int)std::min(32.0, std::max(1.0, 4.0e6 / cells));
  p->graph_steps = G;
  {
    // the pole pass runs a step ahead only where nothing of the step before the E update
    // (modulation, the mixed-form and tensor pre-passes) changes what it reads
    const char* ade = getenv("OEM_B200_ADE");
    p->ade_ahead = p->side_stream != nullptr && p->mods.empty() && p->mixes.empty() &&
                   p->tensors.empty() && !(ade && strcmp(ade, "inline") == 0);
  }
  for (int b = 0; b < (p->fused ? 2 : 1); ++b) {
    if (p->fused) set_bank(p, b);
    if ((rc = capture(p, 1, &p->graph_one[b]))) return rc;
    if (G > 1 && (rc = capture(p, G, &p->graph_many[b]))) return rc;
  }
  if (p->ade_ahead) {
    if ((rc = capture(p, 1, &p->graph_mid, 1))) return rc;
    if ((rc = capture(p, 1, &p->graph_last, 2))) return rc;
  }
  if (p->fused) set_bank(p, 0);
  // setup work runs on the legacy default stream; waiting for it alone leaves other plans'
  // (non-blocking) streams running, which a server with several plans in flight relies on
  OEM_CUDA(cudaStreamSynchronize(0));
  p->finalized = true;
  {
    // the pinned readout stage of a plan whose largest phasor readout takes 16 MB or more is
    // grown on a host thread now (page locking of up to 128 MB takes tens of milliseconds,
    // hidden behind the steps); the first readout joins it
    int64_t most = 0;
    for (const Monitor& q : p->mons) most = std::max(most, (int64_t)q.ncomp * q.nf * q.cells);
    const size_t cbytes = (size_t)std::min(most, (int64_t)1 << 22) * sizeof(double2);
    if ((size_t)most * sizeof(double2) >= ((size_t)16 << 20)) {
      ReadStage* rs = read_stage(p->device);
      const int dev = p->device;
      p->stage_thread = std::thread([rs, dev, cbytes] {
        std::lock_guard<std::mutex> g(rs->mu);
        if (rs->bytes >= cbytes || cudaSetDevice(dev) != cudaSuccess) return;
        grow_stage(rs, cbytes);
      });
    }
  }
  return OEM_OK;
}

int oem_plan_run(oem_plan* p, int64_t nsteps, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (nsteps < 0) return set_error(OEM_ERR_INVALID, "negative step count");
  if (p->steps + nsteps > p->n_total)
    return set_error(OEM_ERR_INVALID, "asked to run past the nominal step count " +
                                          std::to_string(p->n_total) + " (tables end there)");
  if ((rc = use_device(p))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int64_t left = nsteps;
  if (p->timing && p->ckpt_k > 0)
    return set_error(OEM_ERR_STATE, "timing mode does not save adjoint checkpoints");
  if (p->timing) {
    // Direct launches with CUDA events around the two update kernels; events come from a pool
    // sized for this call and are read once at the end, so the stream never waits on the host.
    const int64_t n = nsteps;
    std::vector<cudaEvent_t> ev((size_t)n * 6);
    for (auto& evq : ev) OEM_CUDA(cudaEventCreate(&evq));
    for (int64_t q = 0; q < n; ++q) {
      cudaEvent_t* E = &ev[(size_t)q * 6];
      cudaError_t e;
      if (p->fused) {
        // E[0] ade E[5] fused E[1] ... E[4]: the pole pass and the fused kernel timed apart
        OEM_CUDA(cudaEventRecord(E[0], s));
        for (const MixSet& x : p->mixes)
          if ((e = launch_mix_pre(p->yp, x, s)) != cudaSuccess) return cuda_error(e, "mix_pre");
        for (const Modulation& m : p->mods)
          if ((e = launch_modulate(p->yp, m, p->d_step, s)) != cudaSuccess)
            return cuda_error(e, "modulate");
        for (const TensorSet& t : p->tensors)
          if ((e = launch_tensor_pre(p->yp, t, s)) != cudaSuccess) return cuda_error(e, "tensor_pre");
        if (p->yp.has_ade &&
            (e = launch_ade_segments(p->yp, p->d_ade_segs, p->n_ade_segs,
                                     (int64_t)p->nx * p->ny * p->nzp / 32, 0, (int)p->mats.size(), s)) != cudaSuccess)
          return cuda_error(e, "ade");
        OEM_CUDA(cudaEventRecord(E[5], s));
        const int nb = p->bank ^ 1;
        FieldOut out;
        for (int c = 0; c < 6; ++c) out.f[c] = p->bank_f[nb][c];
        out.psih = p->bank_psih[nb];
        if ((e = launch_update_he_fused(p->fmaps[p->bank], p->yp, out, p->xch,
                                        (int)p->mats.size(), p->d_err, s)) != cudaSuccess)
          return cuda_error(e, "update_he");
        OEM_CUDA(cudaEventRecord(E[1], s));
        set_bank(p, nb);
        if ((rc = enqueue_e_side(p, s, true))) return rc;
        OEM_CUDA(cudaEventRecord(E[4], s));
        continue;
      }
      for (const MixSet& x : p->mixes)
        if ((e = launch_mix_pre(p->yp, x, s)) != cudaSuccess) return cuda_error(e, "mix_pre");
      for (const Modulation& m : p->mods)
        if ((e = launch_modulate(p->yp, m, p->d_step, s)) != cudaSuccess)
          return cuda_error(e, "modulate");
      for (const TensorSet& t : p->tensors)
        if ((e = launch_tensor_pre(p->yp, t, s)) != cudaSuccess) return cuda_error(e, "tensor_pre");
      OEM_CUDA(cudaEventRecord(E[0], s));
      e = run_h(p, s);
      if (e != cudaSuccess) return cuda_error(e, "update_h");
      OEM_CUDA(cudaEventRecord(E[1], s));
      for (const DipoleSet& d : p->dipoles)
        if (d.magnetic && (e = launch_dipoles(p->yp, d, p->d_step, s)) != cudaSuccess)
          return cuda_error(e, "dipoles_h");
      for (const PlaneSrc& src : p->planes)
        if ((e = launch_plane_h(p->yp, src, p->d_step, s)) != cudaSuccess) return cuda_error(e, "plane_h");
      for (const Tfsf& t : p->tfsfs)
        if ((e = launch_tfsf(p->yp, t, 0, p->d_step, s)) != cudaSuccess) return cuda_error(e, "tfsf_h");
      for (const ModeSrc& m : p->modesrcs)
        if ((e = launch_mode_h(p->yp, m, p->d_step, s)) != cudaSuccess) return cuda_error(e, "mode_h");
      for (const Absorber& a : p->absorbers)
        if ((e = launch_absorb(p->yp, a, 0, s)) != cudaSuccess) return cuda_error(e, "absorb_h");
      OEM_CUDA(cudaEventRecord(E[2], s));
      const bool split = p->basic_kernels == 3 && p->yp.has_ade;
      if (split) {
        // the pole pass and the E kernel timed apart
        if ((e = launch_ade_segments(p->yp, p->d_ade_segs, p->n_ade_segs,
                                     (int64_t)p->nx * p->ny * p->nzp / 32, 0, (int)p->mats.size(), s)) != cudaSuccess)
          return cuda_error(e, "ade");
        OEM_CUDA(cudaEventRecord(E[5], s));
        e = launch_update_e_ws(p->tma, p->yp, p->xch, (int)p->mats.size(), p->d_err, s,
                               snap_boxes(p, true));
      } else {
        e = run_e(p, s, snap_boxes(p, true));
      }
      if (e != cudaSuccess) return cuda_error(e, "update_e");
      OEM_CUDA(cudaEventRecord(E[3], s));
      if ((rc = enqueue_e_side(p, s, true))) return rc;
      OEM_CUDA(cudaEventRecord(E[4], s));
    }
    if (n > 0) OEM_CUDA(cudaEventSynchronize(ev[(size_t)n * 6 - 2]));
    auto add = [&](const char* nm, double ms) {
      for (TimingRec& r : p->trecs)
        if (r.name == nm) { r.count++; r.ms += ms; return; }
      TimingRec r; r.name = nm; r.count = 1; r.ms = ms; p->trecs.push_back(r);
    };
    for (int64_t q = 0; q < n; ++q) {
      cudaEvent_t* E = &ev[(size_t)q * 6];
      float t_h = 0.f, t_e = 0.f, t_all = 0.f, t_ade = 0.f;
      if (p->fused) {
        float t_he = 0.f;
        OEM_CUDA(cudaEventElapsedTime(&t_ade, E[0], E[5]));
        OEM_CUDA(cudaEventElapsedTime(&t_he, E[5], E[1]));
        OEM_CUDA(cudaEventElapsedTime(&t_all, E[0], E[4]));
        if (p->yp.has_ade) add("ade", t_ade);
        add("update_he", t_he);
        add("step", t_all);
        continue;
      }
      OEM_CUDA(cudaEventElapsedTime(&t_h, E[0], E[1]));
      OEM_CUDA(cudaEventElapsedTime(&t_all, E[0], E[4]));
      if (p->basic_kernels == 3 && p->yp.has_ade) {
        OEM_CUDA(cudaEventElapsedTime(&t_ade, E[2], E[5]));
        OEM_CUDA(cudaEventElapsedTime(&t_e, E[5], E[3]));
        add("ade", t_ade);
      } else {
        OEM_CUDA(cudaEventElapsedTime(&t_e, E[2], E[3]));
      }
      add("update_h", t_h);
      add("update_e", t_e);
      add("step", t_all);
    }
    for (auto& evq : ev) cudaEventDestroy(evq);
    p->steps += n;
    return OEM_OK;
  }
  while (left > 0) {
    // with checkpoints, every K-step segment starts from a saved state
    int64_t chunk = left;
    if (p->ckpt_k > 0) {
      if (p->steps % p->ckpt_k == 0 && (rc = save_state(p, (int)(p->steps / p->ckpt_k), s)))
        return rc;
      chunk = std::min<int64_t>(left, p->ckpt_k - p->steps % p->ckpt_k);
    }
    int64_t c = chunk;
    while (c >= p->graph_steps && p->graph_steps > 1) {
      OEM_CUDA(cudaGraphLaunch(p->graph_many[p->bank], s));
      if (p->fused && (p->graph_steps & 1)) set_bank(p, p->bank ^ 1);
      c -= p->graph_steps;
    }
    if (p->ade_ahead && c >= 2) {
      // this step's pole pass, then each step runs the next one's beside its monitors; the
      // last step of the run runs none, so the pole states end at the run's last step
      if ((rc = launch_ade(p, s))) return rc;
      for (; c > 1; --c) OEM_CUDA(cudaGraphLaunch(p->graph_mid, s));
      OEM_CUDA(cudaGraphLaunch(p->graph_last, s));
      --c;
    }
    while (c > 0) {
      OEM_CUDA(cudaGraphLaunch(p->graph_one[p->bank], s));
      if (p->fused) set_bank(p, p->bank ^ 1);
      --c;
    }
    p->steps += chunk;
    left -= chunk;
  }
  return OEM_OK;
}

int oem_plan_flush(oem_plan* p, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if ((rc = use_device(p))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (const Monitor& m : p->mons) {
    cudaError_t e = launch_flush(m, p->d_step, 1, s);
    if (e != cudaSuccess) return cuda_error(e, "flush");
  }
  return OEM_OK;
}

int oem_plan_launches_per_step(oem_plan* p, int* n) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (!n) return set_error(OEM_ERR_INVALID, "null output");
  // counted from the kernel nodes of the captured one-step graph
  *n = p->step_kernels;
  return OEM_OK;
}

int oem_plan_box_snapshots_in_update(oem_plan* p, int* n) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (!n) return set_error(OEM_ERR_INVALID, "null output");
  *n = p->snapk.n;
  return OEM_OK;
}

int oem_plan_pole_pass_ahead(oem_plan* p, int* on) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (!on) return set_error(OEM_ERR_INVALID, "null output");
  *on = p->ade_ahead ? 1 : 0;
  return OEM_OK;
}

int oem_plan_status(oem_plan* p, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if ((rc = use_device(p))) return rc;
  OEM_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  return check_device_error(p);
}

int oem_plan_steps(oem_plan* p, int64_t* steps) {
  if (!p || !steps) return set_error(OEM_ERR_INVALID, "null argument");
  *steps = p->steps;
  return OEM_OK;
}

int oem_plan_read_monitor(oem_plan* p, int id, double* re, double* im, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (id < 0 || id >= (int)p->mons.size()) return set_error(OEM_ERR_INVALID, "monitor id out of range");
  if ((rc = use_device(p))) return rc;
  const Monitor& m = p->mons[id];
  const size_t n = (size_t)m.ncomp * m.nf * m.cells;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  OEM_CUDA(cudaMemcpyAsync(re, m.d_re, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  OEM_CUDA(cudaMemcpyAsync(im, m.d_im, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  return check_device_error(p);
}

int oem_plan_read_monitor_interleaved(oem_plan* p, int id, double* out, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (id < 0 || id >= (int)p->mons.size()) return set_error(OEM_ERR_INVALID, "monitor id out of range");
  if (!out) return set_error(OEM_ERR_INVALID, "null output");
  if ((rc = use_device(p))) return rc;
  const Monitor& m = p->mons[id];
  const int64_t n = (int64_t)m.ncomp * m.nf * m.cells;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // interleaved on the device in chunks through two buffers of at most 4M values (64 MB) the
  // plan keeps after its first readout, each chunk copied out while the next is formed
  if (!p->rd_scratch[0]) {  // sized for the plan's largest monitor, up to 4M values
    int64_t most = 1;
    for (const Monitor& q : p->mons) most = std::max(most, (int64_t)q.ncomp * q.nf * q.cells);
    p->rd_chunk = std::min(most, (int64_t)1 << 22);
    for (int b = 0; b < 2; ++b)
      if ((rc = dalloc(p, &p->rd_scratch[b], (size_t)p->rd_chunk, false))) return rc;
    if ((rc = dalloc(p, &p->d_rd_bad, 1))) return rc;
  }
  const int64_t kChunk = p->rd_chunk;
  cudaError_t e = cudaMemsetAsync(p->d_rd_bad, 0, sizeof(unsigned long long), s);
  const size_t cbytes = (size_t)kChunk * sizeof(double2);
  // readouts of 16 MB and more go through the pinned halves (their copy-out threads also take
  // the page faults of a fresh output array in parallel)
  ReadStage* rs = (size_t)n * sizeof(double2) >= ((size_t)16 << 20) ? read_stage(p->device)
                                                                      : nullptr;
  std::unique_lock<std::mutex> lk;
  if (rs) {
    if (p->stage_thread.joinable()) p->stage_thread.join();  // started at finalize
    lk = std::unique_lock<std::mutex>(rs->mu);
    if (!grow_stage(rs, cbytes)) {  // no pinned memory: the driver's pageable copies
      lk.unlock();
      rs = nullptr;
    }
  }
  if (rs) {
    advise_huge_pages(out, (size_t)n * sizeof(double2));
    // chunk q: interleave, DMA into half q % 2; then copy chunk q - 1 out of the other half
    int64_t prev0 = -1, prevc = 0;
    for (int64_t q0 = 0, b = 0; e == cudaSuccess && (q0 < n || prev0 >= 0); q0 += kChunk, b ^= 1) {
      const int64_t c = q0 < n ? std::min(kChunk, n - q0) : 0;
      if (c > 0) {
        e = launch_interleave(m.d_re + q0, m.d_im + q0, p->rd_scratch[b], c, p->d_rd_bad, s);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(rs->half[b], p->rd_scratch[b], (size_t)c * sizeof(double2),
                              cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaEventRecord(rs->ev[b], s);
      }
      if (e == cudaSuccess && prev0 >= 0) {
        e = cudaEventSynchronize(rs->ev[b ^ 1]);
        if (e == cudaSuccess)
          par_memcpy(reinterpret_cast<char*>(out + 2 * prev0), rs->half[b ^ 1],
                     (size_t)prevc * sizeof(double2));
      }
      prev0 = c > 0 ? q0 : -1;
      prevc = c;
    }
  } else {
    for (int64_t q0 = 0, b = 0; q0 < n && e == cudaSuccess; q0 += kChunk, b ^= 1) {
      const int64_t c = std::min(kChunk, n - q0);
      e = launch_interleave(m.d_re + q0, m.d_im + q0, p->rd_scratch[b], c, p->d_rd_bad, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(out + 2 * q0, p->rd_scratch[b], (size_t)c * sizeof(double2),
                            cudaMemcpyDeviceToHost, s);
    }
  }
  unsigned long long bad = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&bad, p->d_rd_bad, sizeof(bad), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_error(e, "read_monitor_interleaved");
  OEM_CUDA(cudaStreamSynchronize(s));
  p->rd_nonfinite += (int64_t)bad;
  return check_device_error(p);
}

int oem_plan_readout_nonfinite(oem_plan* p, int64_t* count) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (!count) return set_error(OEM_ERR_INVALID, "null output");
  *count = p->rd_nonfinite;
  p->rd_nonfinite = 0;
  return OEM_OK;
}

int oem_plan_read_time_monitor(oem_plan* p, int id, float* out, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (id < 0 || id >= (int)p->tmons.size()) return set_error(OEM_ERR_INVALID, "time monitor id out of range");
  if ((rc = use_device(p))) return rc;
  const TimeMon& m = p->tmons[id];
  const size_t n = (size_t)m.nc * m.nslots * m.ni * m.nj * m.nk;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n) OEM_CUDA(cudaMemcpyAsync(out, m.d_buf, n * sizeof(float), cudaMemcpyDeviceToHost, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  return OEM_OK;
}

int oem_plan_read_field(oem_plan* p, int comp, float* out, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (comp < 0 || comp > 5 || !out) return set_error(OEM_ERR_INVALID, "component must be 0..5");
  if ((rc = use_device(p))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  OEM_CUDA(cudaMemcpy2DAsync(out, (size_t)p->nz * sizeof(float), p->yp.f[comp],
                             (size_t)p->nzp * sizeof(float), (size_t)p->nz * sizeof(float),
                             (size_t)p->nx * p->ny, cudaMemcpyDeviceToHost, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  return check_device_error(p);
}

int oem_plan_read_field_complex(oem_plan* p, int comp, float* re, float* im, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (!p->is_complex) return set_error(OEM_ERR_STATE, "not a complex plan");
  if (comp < 0 || comp > 5 || !re || !im) return set_error(OEM_ERR_INVALID, "component must be 0..5");
  if ((rc = use_device(p))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float* src[2] = {p->yp.f[comp], p->yp.fi[comp]};
  float* dst[2] = {re, im};
  for (int q = 0; q < 2; ++q)
    OEM_CUDA(cudaMemcpy2DAsync(dst[q], (size_t)p->nz * sizeof(float), src[q],
                               (size_t)p->nzp * sizeof(float), (size_t)p->nz * sizeof(float),
                               (size_t)p->nx * p->ny, cudaMemcpyDeviceToHost, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  return check_device_error(p);
}

int oem_plan_read_time_monitor_complex(oem_plan* p, int id, float* re, float* im, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (!p->is_complex) return set_error(OEM_ERR_STATE, "not a complex plan");
  if (id < 0 || id >= (int)p->tmons.size()) return set_error(OEM_ERR_INVALID, "time monitor id out of range");
  if (!re || !im) return set_error(OEM_ERR_INVALID, "null output");
  if ((rc = use_device(p))) return rc;
  const TimeMon& m = p->tmons[id];
  const size_t n = (size_t)m.nc * m.nslots * m.ni * m.nj * m.nk;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n) {
    OEM_CUDA(cudaMemcpyAsync(re, m.d_buf, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    OEM_CUDA(cudaMemcpyAsync(im, m.d_buf_i, n * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  OEM_CUDA(cudaStreamSynchronize(s));
  return OEM_OK;
}

int oem_plan_write_field(oem_plan* p, int comp, const float* in, void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (comp < 0 || comp > 5 || !in) return set_error(OEM_ERR_INVALID, "component must be 0..5");
  if ((rc = use_device(p))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  OEM_CUDA(cudaMemcpy2DAsync(p->yp.f[comp], (size_t)p->nzp * sizeof(float), in,
                             (size_t)p->nz * sizeof(float), (size_t)p->nz * sizeof(float),
                             (size_t)p->nx * p->ny, cudaMemcpyHostToDevice, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  return OEM_OK;
}

int oem_plan_write_field_complex(oem_plan* p, int comp, const float* re, const float* im,
                                 void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (!p->is_complex) return set_error(OEM_ERR_STATE, "not a complex plan");
  if (comp < 0 || comp > 5 || !re || !im) return set_error(OEM_ERR_INVALID, "component must be 0..5");
  if ((rc = use_device(p))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float* dst[2] = {p->yp.f[comp], p->yp.fi[comp]};
  const float* src[2] = {re, im};
  for (int q = 0; q < 2; ++q)
    OEM_CUDA(cudaMemcpy2DAsync(dst[q], (size_t)p->nzp * sizeof(float), src[q],
                               (size_t)p->nz * sizeof(float), (size_t)p->nz * sizeof(float),
                               (size_t)p->nx * p->ny, cudaMemcpyHostToDevice, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  return OEM_OK;
}

int oem_plan_energy(oem_plan* p, double out[3], void* stream) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  if (!out) return set_error(OEM_ERR_INVALID, "null output");
  if ((rc = use_device(p))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = launch_energy(p->yp, p->d_dl, p->d_energy_part, p->energy_blocks, s);
  if (e != cudaSuccess) return cuda_error(e, "energy");
  std::vector<double> part(3 * (size_t)p->energy_blocks);
  OEM_CUDA(cudaMemcpyAsync(part.data(), p->d_energy_part, part.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, s));
  OEM_CUDA(cudaStreamSynchronize(s));
  out[0] = out[1] = out[2] = 0.0;
  for (int b = 0; b < p->energy_blocks; ++b)
    for (int c = 0; c < 3; ++c) out[c] += part[3 * (size_t)b + c];
  return check_device_error(p);
}

int oem_plan_field_ptrs(oem_plan* p, void* ptrs[6], int* nzp) {
  int rc = check_plan(p, true);
  if (rc) return rc;
  for (int c = 0; c < 6; ++c) ptrs[c] = p->yp.f[c];
  if (nzp) *nzp = p->nzp;
  return OEM_OK;
}

int oem_plan_enable_timing(oem_plan* p, int on) {
  if (!p) return set_error(OEM_ERR_INVALID, "null plan");
  p->timing = on != 0;
  p->trecs.clear();
  return OEM_OK;
}

int oem_plan_timing(oem_plan* p, int max, char* names, int64_t* counts, double* ms, int* n) {
  if (!p || !n) return set_error(OEM_ERR_INVALID, "null argument");
  int cnt = 0;
  for (const TimingRec& r : p->trecs) {
    if (cnt >= max) break;
    if (names) {
      strncpy(names + 32 * cnt, r.name.c_str(), 31);
      names[32 * cnt + 31] = 0;
    }
    if (counts) counts[cnt] = r.count;
    if (ms) ms[cnt] = r.ms;
    ++cnt;
  }
  *n = cnt;
  return OEM_OK;
}

}  // extern "C"
