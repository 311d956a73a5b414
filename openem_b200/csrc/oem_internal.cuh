// Internal declarations shared by the engine's translation units: device-side parameter
// blocks, the plan object, launch helpers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <thread>
#include <vector>

#include "../../include/oem_b200.h"

namespace oem {

// ---------------------------------------------------------------------------------------------
// Error reporting (thread-local last error, negative status codes)
// ---------------------------------------------------------------------------------------------
int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* what);

#define OEM_CUDA(call)                                               \
  do {                                                               \
    cudaError_t e_ = (call);                                         \
    if (e_ != cudaSuccess) return ::oem::cuda_error(e_, #call);      \
  } while (0)

// ---------------------------------------------------------------------------------------------
// Device-side views
// ---------------------------------------------------------------------------------------------

// One material tuple: update coefficients, permittivity and ADE pole set of the three E
// components at one cell. 64 bytes.
struct MatRec {
  float ca[3];
  float cb[3];
  float eps[3];
  int pset[3];  // -1 = not dispersive
  int np[3];    // poles of that set (0 when not dispersive)
  int reserved;  // np[0] + np[1] + np[2], filled by the plan
};
static_assert(sizeof(MatRec) == 64, "MatRec must be 16 words");

// One grid axis on the device. z tables are padded to nzp entries.
struct DevAxis {
  const float* idl_p;  // 1 / primal spacing
  const float* idl_d;  // 1 / dual spacing
  const int* nxt;      // forward neighbour
  const int* prv;      // backward neighbour
  const float* mnx;    // forward-neighbour mask (0 at an absorbing high wall)
  const float* mpv;    // backward-neighbour mask
  const float* ae;     // CPML (a, b, 1/kappa) at E positions
  const float* be;
  const float* ke;
  const float* ah;     // CPML at H positions
  const float* bh;
  const float* kh;
  const float* mnx_i;  // imaginary parts of the masks (complex plans: the Bloch phase at the
  const float* mpv_i;  // periodic seam), nullptr on the real path
  int n;
  int lo;  // psi slab cells at the low end  [0, lo)
  int hi;  // psi slab cells at the high end [n - hi, n)
};

// psi storage: [derivative axis][component slot][0 = low slab, 1 = high slab]; the component
// slots of derivative axis a are the two components != a in ascending order.
struct PsiSet {
  float* p[3][2][2];
};

// Everything the Yee kernels need.
struct YeeParams {
  float* f[6];  // Ex Ey Ez Hx Hy Hz, padded (nx, ny, nzp)
  float* fi[6];  // imaginary parts on a complex (Bloch) plan, nullptr otherwise
  DevAxis ax[3];
  PsiSet psih;
  PsiSet psie;
  PsiSet psih_i;  // imaginary psi on a complex plan
  PsiSet psie_i;
  int cplx;
  int nx, ny, nz, nzp;
  float ch;  // dt / mu0
  float cw;  // eps0 / dt
  const uint16_t* mat16;  // per-cell material index (padded layout), one of the two
  const uint32_t* mat32;
  const MatRec* mats;
  // ADE
  float2* P;               // pole states, cell order then component then pole
  float* J;                // pole-indexed polarisation currents of the separate pole pass
  const float4* pcoef;     // per pole of a set: (Re(A-1), Im(A-1), Re(B), Im(B))
  const int* pset_ofs;     // set -> first pole in pcoef
  const uint32_t* seg_ofs; // poles stored before each 32-cell segment
  uint32_t n_pole_total;
  int n_coef;              // entries of pcoef
  int n_sets;              // pole sets (pset_ofs holds n_sets + 1 entries)
  int has_ade;
  int expire_polls;        // > 0: the E update's consumers wait on a barrier nothing arrives at
                           // for this many polls (the check of the wait-expiry path)
};

// TMA descriptors of the field tiles the pipelined kernels load (see oem_yee_tma.cu):
// halo boxes 136 (z) x 5 (y) and tiles 128 x 4, plus the material-index tile.
struct TmaMaps {
  CUtensorMap e_wide[3];
  CUtensorMap h_tile[3];
  CUtensorMap h_wide[3];
  CUtensorMap e_tile[3];
  CUtensorMap m_tile;
};

// Tensor maps of the fused H + E kernel over one field bank: E boxes 136 x 6, E (y, z) and H
// tiles 128 x 5, the material tile 128 x 4.
struct FusedMaps {
  CUtensorMap e6[3];
  CUtensorMap e5[2];
  CUtensorMap h5[3];
  CUtensorMap m;
};

// Where the fused kernel writes: the other bank's fields and H-side psi.
struct FieldOut {
  float* f[6];
  PsiSet psih;
};

struct PlaneSrc {
  int pol, kh, ks;
  float coef_h, coef_e;
  int64_t ntab;
  double* d_ex = nullptr;
  double* d_hy = nullptr;
};

struct DipoleSet {
  int magnetic = 0;
  int n_targets = 0;
  int64_t nsteps1 = 0;
  int n_src = 0;
  int64_t* d_target = nullptr;  // padded flat index of each distinct (comp, cell)
  int* d_tcomp = nullptr;
  int* d_ofs = nullptr;         // target -> its points [ofs[t], ofs[t+1])
  float* d_coef = nullptr;
  int* d_src = nullptr;
  double* d_amp = nullptr;      // (n_src, nsteps1)
  double* d_amp_im = nullptr;   // imaginary part on a complex plan
};

// One mode-source injection entry (one-plane TF/SF with 2D complex profiles): the tangential
// pair t1 = axis+1, t2 = axis+2 (cyclic); profiles per term [8][n1][n2] = E_t1, E_t2, H_t1,
// H_t2 as (re, im) planes; amplitudes per term (ntab, 2).
struct ModeSrc {
  int axis = 0, kh = 0, ks = 0, n1 = 0, n2 = 0, nterms = 0;
  float ch1 = 0.f, ch2 = 0.f, ce1 = 0.f, ce2 = 0.f;
  int64_t ntab = 0;
  float* d_prof = nullptr;
  double* d_amp_e = nullptr;  // amp at n dt, paired with the E profiles on the H side
  double* d_amp_h = nullptr;  // amp at (n + 1/2) dt, paired with the H profiles on the E side
};

struct Monitor {
  int kind = 0;   // 0 = flux plane, 1 = box
  int axis = 0, km = 0;
  int i0 = 0, j0 = 0, k0 = 0, ni = 0, nj = 0, nk = 0;
  int n1 = 0, n2 = 0;  // plane extent (transverse axes ascending)
  int nf = 0, T = 1, ncomp = 0;
  int64_t cells = 0;
  int64_t n_total = 0;
  float* d_phase = nullptr;  // (n_total, nf, 4)
  float* d_snap = nullptr;   // (T, ncomp, cells)
  double* d_re = nullptr;    // (ncomp, nf, cells)
  double* d_im = nullptr;
  int* d_done = nullptr;     // last step already folded into the accumulators
  unsigned* d_count = nullptr;  // blocks of the running flush that have finished
  int cplx = 0;              // complex fields: the ring holds ncomp real then ncomp imaginary rows
};

// Box DFT monitors snapshotted by one launch (k_snap_boxes): block ranges per box.
constexpr int kMaxBoxSnap = 8;
struct BoxSnapSet {
  int n = 0;
  Monitor m[kMaxBoxSnap];
  uint32_t blk0[kMaxBoxSnap + 1] = {};  // first block of each box; blk0[n]: all blocks
  uint32_t cb[kMaxBoxSnap] = {};        // blocks of 256 points per plane of each box
};

// Box DFT monitors whose snapshot rows the warp-specialised E update writes itself: E^{n+1}
// from its registers, H^{n+1/2} from its staged tile, at the same positions and in the same
// ring row as k_snap_boxes (the ring holds six rows per step, components in order). The E-side
// dipole update then rewrites the rows of its few target cells that lie in a box.
constexpr int kMaxSnapBoxes = 4;
struct SnapBox {
  int i0 = 0, ni = 0, j0 = 0, nj = 0, k0 = 0, nk = 0, T = 1;
  int64_t cells = 0;
  float* snap = nullptr;  // (T, 6, cells)
};
struct SnapBoxes {
  int n = 0;
  const int* step = nullptr;
  SnapBox b[kMaxSnapBoxes];
};

// One absorber slab (Tidy3D's Absorber): the layers [g0, g0 + nlay) along `axis`, whole- and
// half-cell decay factors exp(-Gamma dt) per layer.
struct Absorber {
  int axis = 0, g0 = 0, nlay = 0;
  float* d_int = nullptr;
  float* d_half = nullptr;
};

// Time-modulated permittivity eps(t) = eps_s + amp cos(omega t - phi) on (comp, cell) entries:
// every step the D-form coefficients ca = (eps(t_n) - s) / (eps(t_n+1) + s + G),
// cb = (dt / eps0) / (eps(t_n+1) + s + G) are written into the cell's own material record (each
// modulated cell owns one). cs holds (cos w t_n, sin w t_n, cos w t_n+1, sin w t_n+1) per step.
struct Modulation {
  int n = 0, ntab = 0;
  float dte = 0.f;
  int* comp = nullptr;
  int64_t* cell = nullptr;  // padded index
  float* amp = nullptr;
  float* cph = nullptr;
  float* sph = nullptr;
  float* eps = nullptr;
  float* sd = nullptr;
  float* gg = nullptr;
  float4* cs = nullptr;
  MatRec* mats = nullptr;   // the plan's records (writable), set at finalize
};

// Instantaneous colocated flux of one plane (FluxTimeMonitor): per sample step m,
// s(m) = sum_planes w sum dS (E_t1 Hbar_t2 - E_t2 Hbar_t1), Hbar = (H^{m-1/2} + H^{m+1/2}) / 2,
// accumulated in two shots: at step m the E^m half with H^{m-1/2} (E colocated and kept), at step
// m + 1 the kept E with H^{m+1/2}. Per transverse axis: edge index, low / high interpolation
// cells, low weights of the two labels interpolated along it (E_t1, H_t2 along t1; E_t2, H_t1
// along t2) and high weights.
struct FluxTimeMon {
  int axis = 0, nplanes = 1;
  double w[2] = {1.0, 0.0};
  int ke[2] = {0, 0}, kh[2] = {0, 0};
  double wh[2][2] = {{1.0, 0.0}, {1.0, 0.0}};
  int n1 = 0, n2 = 0;
  int *e1 = nullptr, *lo1 = nullptr, *hi1 = nullptr;
  int *e2 = nullptr, *lo2 = nullptr, *hi2 = nullptr;
  double *wlo1 = nullptr, *whi1 = nullptr;  // wlo1: (2, n1) = (E_t1, H_t2)
  double *wlo2 = nullptr, *whi2 = nullptr;  // wlo2: (2, n2) = (E_t2, H_t1)
  double* dS = nullptr;                     // (n1, n2), signed
  double* ekeep = nullptr;                  // (nplanes, 2, n1, n2) colocated E of the last shot
  double* part = nullptr;                   // (nblocks, 2) block partial sums
  double* buf = nullptr;                    // (slots,)
  int nblocks = 0;
  int beg = 0, end = 0, iv = 1, slots = 0;
};

// TFSF box: faces (device copies) and the two incident tables; one launch per face group.
struct Tfsf {
  oem_tfsf_face* e_faces = nullptr;
  oem_tfsf_face* h_faces = nullptr;
  std::vector<std::pair<int, int>> e_groups, h_groups;  // [first face, count) per group
  std::vector<int64_t> e_points, h_points;             // points per group
  std::vector<std::vector<int64_t>> e_ofs_h, h_ofs_h;  // host prefix offsets per group
  int64_t* e_ofs = nullptr;                            // device prefix offsets, per face + 1
  int64_t* h_ofs = nullptr;
  double* ex_tab = nullptr;
  double* hy_tab = nullptr;
  int ex_rows = 0, ex_n = 0, hy_rows = 0, hy_n = 0;
};

// Fully anisotropic cells: per (component, cell) entry the rows of M1, M2 (n x 3) and the
// PEC-wall factor; rhs / enew hold M1 <E^n> and the new value between the passes.
struct TensorSet {
  int n = 0;
  int* comp = nullptr;
  int64_t* cell = nullptr;  // padded index
  float* m1 = nullptr;
  float* m2 = nullptr;
  float* pec = nullptr;
  float* rhs = nullptr;
  float* enew = nullptr;
};

// Slanted-interface entries (openem/kernels/dispersion_mix.cu): per entry the component, the
// padded cell, the pole ranges of the arithmetic (eps poles, P) and harmonic (1/eps poles, Q)
// branches, (k1, k2, 1 - beta, 1 / (k1 k2 + beta)), and the per-step state: SP / SQ of the first
// pass, the accumulated d_tot and the harmonic unknown d_h.
struct MixSet {
  int n = 0;
  float dte = 0.0f;  // dt / eps0
  int* comp = nullptr;
  int64_t* cell = nullptr;  // padded index
  int* p_ofs = nullptr;     // n + 1
  int* q_ofs = nullptr;
  float4* pc = nullptr;     // per pole (Re(A-1), Im(A-1), Re(B), Im(B))
  float4* qc = nullptr;
  float2* P = nullptr;      // pole states
  float2* Q = nullptr;
  float4* k = nullptr;
  float* sp = nullptr;
  float* sq = nullptr;
  float* dtot = nullptr;
  float* dh = nullptr;
};

// One face of Bloch seam cells of the split complex update: the cells whose index along
// `axis` is q, where the forward (H side) or backward (E side) neighbour mask has an
// imaginary part.
struct SeamFace {
  int axis = 0;
  int q = 0;
};

struct TimeMon {
  int nc = 0;
  int comps[6] = {0, 0, 0, 0, 0, 0};
  int i0 = 0, j0 = 0, k0 = 0, ni = 0, nj = 0, nk = 0;
  int beg = 0, end = 0, iv = 1, nslots = 0;
  float* d_buf = nullptr;  // (nc, nslots, ni, nj, nk)
  float* d_buf_i = nullptr;  // imaginary samples on a complex plan
};

struct AxisHost {
  std::vector<double> idl_p, idl_d, mnx, mpv, pml_e, pml_h;
  std::vector<double> mnx_i, mpv_i;  // complex plans: imaginary parts of the masks
  std::vector<int> nxt, prv;
  int lo = 0, hi = 0;
  bool set = false;
};

struct TimingRec {
  std::string name;
  int64_t count = 0;
  double ms = 0.0;
};

}  // namespace oem

struct oem_plan {
  int device = 0;
  int nx = 0, ny = 0, nz = 0, nzp = 0;
  double ch = 0.0, cw = 0.0;
  int64_t n_total = 0;
  int64_t steps = 0;
  bool finalized = false;

  oem::AxisHost axh[3];
  // materials (host staging until finalize)
  std::vector<oem::MatRec> mats;
  int index_bytes = 0;
  std::vector<uint8_t> mat_index;  // unpadded, index_bytes per cell
  // pole sets
  std::vector<int> pset_ofs;
  std::vector<float> pcoef;
  std::vector<uint32_t> seg_ofs;
  int64_t n_pole_total = 0;

  std::vector<oem::PlaneSrc> planes;
  std::vector<oem::DipoleSet> dipoles;
  std::vector<oem::ModeSrc> modesrcs;
  std::vector<oem::Absorber> absorbers;
  std::vector<oem::Modulation> mods;
  std::vector<std::vector<int64_t>> mod_cells;  // unpadded cells of each, kept until finalize
  // checkpoints of the state every ckpt_k steps (discrete adjoint): fields and CPML psi
  int ckpt_k = 0;
  // gradient box declared before the run: E of its cells after every step (step-major, the
  // three components, (steps + 1) rows), so the reverse pass needs no forward recompute
  int gbox[6] = {0, 0, 0, 0, 0, 0};
  bool gbox_set = false;
  float* hist = nullptr;
  std::vector<float*> ckpt;        // one buffer per checkpoint, ckpt_floats floats each
  size_t ckpt_floats = 0;
  std::vector<int64_t> ckpt_step;  // step held by each buffer (-1: empty)
  bool is_complex = false;  // Bloch / forced complex fields
  std::vector<oem::Monitor> mons;
  std::vector<oem::TimeMon> tmons;
  std::vector<oem::FluxTimeMon> ftmons;
  std::vector<oem::Tfsf> tfsfs;
  std::vector<oem::TensorSet> tensors;
  std::vector<oem::MixSet> mixes;
  // complex plans on large grids: the warp-specialised real kernels update the real and the
  // imaginary parts (tma / tma_i), the seam faces add the imaginary-mask terms
  bool cplx_ws = false;
  oem::TmaMaps tma_i{};
  std::vector<oem::SeamFace> seam_h, seam_e;
  double2* rd_scratch[2] = {nullptr, nullptr};  // readout interleave buffers (lazy)
  unsigned long long* d_rd_bad = nullptr;        // non-finite values seen by one readout
  int64_t rd_nonfinite = 0;                      // since the last oem_plan_readout_nonfinite
  int64_t rd_chunk = 0;
  std::thread stage_thread;  // grows the pinned readout stage after finalize (joined on use)

  // device state
  std::vector<void*> allocs;
  oem::YeeParams yp{};
  int* d_step = nullptr;
  double* d_energy_part = nullptr;
  int energy_blocks = 0;
  double* d_dl[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};  // primal, dual

  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t graph_many[2] = {nullptr, nullptr};  // per starting field bank
  cudaGraphExec_t graph_one[2] = {nullptr, nullptr};
  // pole pass one step ahead: a run of c >= 2 steps is one pole pass, c - 1 replays of
  // graph_mid (whose last branch runs the next step's pole pass beside the snapshots) and one
  // of graph_last (no pole pass), so no pole state is advanced past the run's last step
  bool ade_ahead = false;
  cudaGraphExec_t graph_mid = nullptr, graph_last = nullptr;
  int graph_steps = 1;
  int step_kernels = 0;  // kernel nodes of the one-step graph

  bool timing = false;
  std::vector<oem::TimingRec> trecs;

  bool dev_index = false;        // material index uploaded from device memory
  uint16_t* dev_mat16 = nullptr;
  uint32_t* dev_mat32 = nullptr;
  uint32_t* dev_seg = nullptr;   // segment offsets uploaded from device memory

  int basic_kernels = 3;  // 3: warp-specialised (default), 0: TMA, 1: one-thread-per-cell, 2: register-streaming
  oem::TmaMaps tma{};
  int* d_err = nullptr;   // set by a kernel whose bounded wait gave up
  int64_t* d_ade_segs = nullptr;  // segments with poles (separate pole pass)
  int64_t n_ade_segs = 0;
  oem::SnapBoxes snapk{};  // box monitors whose snapshots the E update writes (n = 0: none)
  cudaStream_t side_stream = nullptr;  // branch of the captured step that runs the pole pass
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int xch = 8;            // x planes per thread in the streaming kernels
  int xch_user = 0;       // tile shape chosen by the caller (0: automatic)
  // fused H + E step: two field banks (fields and H-side psi), swapped every step
  bool want_fused = true;
  bool fused = false;
  int bank = 0;
  float* bank_f[2][6] = {};
  oem::PsiSet bank_psih[2] = {};
  oem::FusedMaps fmaps[2];
};

namespace oem {

// Device allocation tracked by the plan (freed in oem_plan_destroy).
template <class T>
int dalloc(oem_plan* p, T** out, size_t count, bool zero = true) {
  void* ptr = nullptr;
  size_t bytes = count * sizeof(T);
  if (bytes == 0) bytes = sizeof(T);
  cudaError_t e = cudaMalloc(&ptr, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(OEM_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(bytes) +
                                         " bytes failed: " + cudaGetErrorString(e));
  }
  p->allocs.push_back(ptr);
  if (zero) {
    e = cudaMemset(ptr, 0, bytes);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemset");
  }
  *out = static_cast<T*>(ptr);
  return OEM_OK;
}

template <class T>
int dupload(oem_plan* p, T** out, const T* host, size_t count) {
  int rc = dalloc(p, out, count, false);
  if (rc) return rc;
  if (count) OEM_CUDA(cudaMemcpy(*out, host, count * sizeof(T), cudaMemcpyHostToDevice));
  return OEM_OK;
}

// Kernel launchers (defined in oem_kernels.cu). All return a cudaError_t of the launch.
cudaError_t launch_update_h(const YeeParams& P, cudaStream_t s);
cudaError_t launch_update_e(const YeeParams& P, cudaStream_t s);
cudaError_t launch_plane_h(const YeeParams& P, const PlaneSrc& src, const int* step,
                           cudaStream_t s);
cudaError_t launch_plane_e(const YeeParams& P, const PlaneSrc& src, const int* step,
                           cudaStream_t s);
cudaError_t launch_dipoles(const YeeParams& P, const DipoleSet& d, const int* step,
                           cudaStream_t s, const SnapBoxes* sb = nullptr);
cudaError_t launch_time_sample(const YeeParams& P, const TimeMon& m, const int* step, int add,
                               cudaStream_t s);
cudaError_t launch_snapshot(const YeeParams& P, const Monitor& m, const int* step,
                            cudaStream_t s);
cudaError_t launch_snapshot_boxes(const YeeParams& P, const Monitor* const* boxes, int n,
                                  const int* step, cudaStream_t s);
cudaError_t launch_flush(const Monitor& m, const int* step, int forced, cudaStream_t s);
cudaError_t launch_step_advance(int* step, cudaStream_t s);
int stream_xchunk(const YeeParams& P);
int tma_xchunk(const YeeParams& P);
cudaError_t tma_setup_kernels();
cudaError_t launch_update_h_tma(const TmaMaps& maps, const YeeParams& P, int xch, int* err,
                                cudaStream_t s);
cudaError_t launch_update_e_tma(const TmaMaps& maps, const YeeParams& P, int xch, int n_mats,
                                int* err, cudaStream_t s);
int make_tma_maps(oem_plan* p);
int make_tma_maps_of(oem_plan* p, TmaMaps& m, const YeeParams& P);
cudaError_t launch_pad_index(const void* in, int in_bytes, uint16_t* out16, uint32_t* out32,
                             int nx, int ny, int nz, int nzp, uint32_t n_mat, unsigned* bad,
                             cudaStream_t s);
cudaError_t launch_update_h_stream(const YeeParams& P, int xch, cudaStream_t s);
int ws_xchunk(const YeeParams& P);
int ws_max_xchunk();
cudaError_t ws_setup_kernels();
cudaError_t launch_update_h_ws(const TmaMaps& maps, const YeeParams& P, int xch, int* err,
                               cudaStream_t s);
cudaError_t launch_update_e_ws(const TmaMaps& maps, const YeeParams& P, int xch, int n_mats,
                               int* err, cudaStream_t s, const SnapBoxes* sb = nullptr);
cudaError_t launch_update_e_stream(const YeeParams& P, int xch, int n_mats, cudaStream_t s);
cudaError_t launch_list_pole_segments(const YeeParams& P, int64_t nseg, int64_t* list,
                                      unsigned long long* count, cudaStream_t s);
cudaError_t launch_ade_segments(const YeeParams& P, const int64_t* segs, int64_t nsegs,
                                int64_t nseg, int max_blocks, int n_mats, cudaStream_t s);
cudaError_t launch_update_h_c(const YeeParams& P, cudaStream_t s);
cudaError_t launch_update_e_c(const YeeParams& P, cudaStream_t s);
cudaError_t launch_seam_h(const YeeParams& P, const SeamFace& f, cudaStream_t s);
cudaError_t launch_seam_e(const YeeParams& P, const SeamFace& f, cudaStream_t s);
cudaError_t launch_absorb(const YeeParams& P, const Absorber& a, int is_e, cudaStream_t s);
cudaError_t launch_modulate(const YeeParams& P, const Modulation& m, const int* step,
                            cudaStream_t s);
cudaError_t launch_flux_time(const YeeParams& P, const FluxTimeMon& m, const int* step,
                             cudaStream_t s);
cudaError_t launch_update_he_fused(const FusedMaps& maps, const YeeParams& P, const FieldOut& out,
                                   int xch, int n_mats, int* err, cudaStream_t s);
cudaError_t launch_tfsf(const YeeParams& P, const Tfsf& t, int is_e, const int* step,
                        cudaStream_t s);
cudaError_t launch_tensor_pre(const YeeParams& P, const TensorSet& t, cudaStream_t s);
cudaError_t launch_tensor_post(const YeeParams& P, const TensorSet& t, cudaStream_t s);
cudaError_t launch_mix_pre(const YeeParams& P, const MixSet& m, cudaStream_t s);
cudaError_t launch_interleave(const double* re, const double* im, double2* out, int64_t n,
                              unsigned long long* bad, cudaStream_t s);
cudaError_t launch_mix_post(const YeeParams& P, const MixSet& m, cudaStream_t s);

// Discrete adjoint (oem_adjoint.cu): adjoint fields, their CPML psi, scratch for the transposed
// differences, and the gradient accumulators of ca and cb per component.
struct AdjState {
  float* lam[6];      // adjoint of Ex Ey Ez Hx Hy Hz (padded)
  PsiSet lpsih, lpsie;  // adjoint psi
  float* dbare[6];    // per-cell adjoint of the six differences of the E update
  float* dbarh[6];    // ... and of the H update
  int box[6];         // gradient box: i0, j0, k0, ni, nj, nk
  double* gca[3];     // per box cell: sum over steps of lambda_E^{n+1} E^n
  double* gcb[3];     // sum over steps of lambda_E^{n+1} T^n, T^n = (E^{n+1} - ca E^n) / cb
  float2* lps;        // adjoint of the ADE pole states (pole-indexed), nullptr without poles
};
struct AdjFlux {      // objective sources of one flux plane (see oem_adjoint.cu)
  int axis, km, n1, n2, nf;
  const float* phase;   // (n_total, nf, 4) forward phase table
  const double* coef;   // (4, nf, n1, n2, 2): per term and frequency the (cos, sin) weights
};
cudaError_t launch_adj_src(const YeeParams& P, const AdjFlux& a, const AdjState& S, int n,
                           cudaStream_t s);
cudaError_t launch_adj_step(const YeeParams& P, const AdjState& S, const float* en_box,
                            const float* en1_box, cudaStream_t s);
cudaError_t launch_hist_snap(const YeeParams& P, const int* box, float* hist, const int* step,
                             int64_t n_total, cudaStream_t s);
cudaError_t launch_adj_snap(const YeeParams& P, const AdjState& S, float* dst, cudaStream_t s);
cudaError_t launch_mode_h(const YeeParams& P, const ModeSrc& m, const int* step, cudaStream_t s);
cudaError_t launch_mode_e(const YeeParams& P, const ModeSrc& m, const int* step, cudaStream_t s);
cudaError_t launch_energy(const YeeParams& P, double* const dl[3][2], double* part, int nblocks,
                          cudaStream_t s);
// Block partials of the float64 energy sums: at most this many blocks of 256 threads, summed in
// block order. oem_plan_energy and oem_field_energy_noalloc share it, so both add the same
// partials in the same order.
constexpr int kEnergyMaxBlocks = 148 * 16;
int energy_block_count(const YeeParams& P);

}  // namespace oem
