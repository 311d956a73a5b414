/* C ABI of liboem_b200.so, the sm_100a FDTD step engine that replaces OpenEM's solver step loop.
 *
 * OpenEM drives its CUDA side through one Python module, openem/device.py (the Kernels
 * registry, openem/device.py:145-171, "the one entry point to the CUDA side", :3-10), with the
 * device tables built by openem/device_tables.py and the step loop in openem/solver.py. This
 * library is the replacement for that boundary: a *plan* owns every device buffer of one
 * simulation; the host computes every coefficient in float64 and hands plain host arrays to
 * the plan, which copies them to the device; stepping and readout are single calls.
 *
 * Conventions
 *   - Every function returns an int status: OEM_OK (0) or a negative OEM_ERR_* code. The text of
 *     the last error of the calling thread is returned by oem_last_error().
 *   - Host pointers are borrowed for the duration of the call only.
 *   - Field arrays are C-order (nx, ny, nz) on the host; on the device z is padded to a multiple
 *     of 32 floats.
 *   - A plan is used by one host thread at a time; different plans may run concurrently on
 *     different streams. The stream argument is a cudaStream_t passed as void* (NULL = the
 *     legacy default stream).
 */
#ifndef OEM_B200_H
#define OEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OEM_OK 0
#define OEM_ERR_INVALID (-1)     /* bad argument, shape or range (Python: ValueError) */
#define OEM_ERR_UNSUPPORTED (-2) /* physics this engine does not run (NotImplementedError) */
#define OEM_ERR_CUDA (-3)        /* CUDA runtime error (RuntimeError) */
#define OEM_ERR_TIMEOUT (-4)     /* a bounded device wait gave up (RuntimeError) */
#define OEM_ERR_STATE (-5)       /* call out of order, e.g. stepping before finalize */
#define OEM_ERR_NOMEM (-6)       /* device allocation failed */

typedef struct oem_plan oem_plan;

/* One face of a TFSF box correction (openem/kernels/tfsf.cu:49-86): for p < np, q < nq the
 * padded cell base + p sp + q sq of field component comp (0..5) gets coef x the incident table
 * row interpolated at column c0 + cp p + cq q (E faces also x the cell's cb). Faces of one group
 * touch disjoint cells; groups apply in order. */
typedef struct oem_tfsf_face {
  int32_t comp;
  int32_t group;
  float coef;
  float reserved;
  double c0, cp, cq;
  int64_t base, sp, sq;
  int32_t np, nq;
} oem_tfsf_face;

/* Library version (major*10000 + minor*100 + patch) and last error text of this thread. */
int oem_version(void);
const char* oem_last_error(void);

/* Create an empty plan for an (nx, ny, nz) grid on CUDA device `device`.
 * ch = dt/mu0 and cw = eps0/dt are the H-update and dispersion-history scalars
 * (openem/device_tables.py:174, :284). Replaces the allocation half of
 * openem/device_tables.py:42-84 (_alloc_fields). */
int oem_plan_create(int device, int nx, int ny, int nz, double ch, double cw, oem_plan** out);
int oem_plan_destroy(oem_plan* p);

/* One axis of the grid: 1/primal and 1/dual spacing, neighbour tables and masks
 * (openem/grid.py:219-304) and the CPML recursion coefficients at E and H positions, each an
 * (a | b | 1/kappa) triple of n values filled with the identity (0, 1, 1) outside the layers
 * (openem/coeffs.py:21-42). slab_lo / slab_hi are the numbers of cells at each end where psi
 * is stored; outside them the coefficients must be the identity. Replaces
 * openem/device_tables.py:118-165 (_axis_device_tables) and the psi allocation of
 * openem/coeffs.py:56-95. */
int oem_plan_set_axis(oem_plan* p, int axis, const double* idl_p, const double* idl_d,
                      const int32_t* nxt, const int32_t* prv, const double* mnx,
                      const double* mpv, const double* pml_e, const double* pml_h,
                      int slab_lo, int slab_hi);

/* Material tuples and the per-cell material index.
 * table: n_mat records of 16 32-bit words:
 *   float ca[3], float cb[3], float eps[3], int32 pole_set[3] (-1 = not dispersive),
 *   int32 pole_count[3], int32 reserved.
 * index: nx*ny*nz unpadded C-order cell indices into the table, 2 bytes each when
 * index_bytes == 2, 4 bytes when 4. Replaces the dense ca/cb arrays and the uint16 (ca, cb)
 * lookup table of openem/coeffs.py:98-208 and openem/device_tables.py:168-219. */
int oem_plan_set_materials(oem_plan* p, int n_mat, const uint32_t* table, int index_bytes,
                           const void* index);

/* Same as oem_plan_set_materials, with the per-cell index already in device memory
 * (unpadded (nx, ny, nz) C order, index_bytes each). The plan copies it. */
int oem_plan_set_materials_device(oem_plan* p, int n_mat, const uint32_t* table, int index_bytes,
                                  const void* d_index);

/* Pole sets of the ADE (openem/kernels/dispersion.cu:25-114): set s owns poles
 * set_ofs[s] .. set_ofs[s+1]-1; coef holds 4 floats per pole, (Re(A-1), Im(A-1), Re(B), Im(B)).
 * seg_ofs: one uint32 per 32-cell z segment of the padded grid, the number of poles stored
 * before that segment (cell order, then component, then pole). n_pole_total sizes P.
 * Replaces openem/device_tables.py:235-285 (_dispersion_tables). */
int oem_plan_set_pole_sets(oem_plan* p, int n_sets, const int32_t* set_ofs, const float* coef,
                           const uint32_t* seg_ofs, int64_t n_seg, int64_t n_pole_total);

/* Same as oem_plan_set_pole_sets, with seg_ofs already in device memory (copied). */
int oem_plan_set_pole_sets_device(oem_plan* p, int n_sets, const int32_t* set_ofs,
                                  const float* coef, const uint32_t* d_seg_ofs, int64_t n_seg,
                                  int64_t n_pole_total);

/* One-face TF/SF plane-wave group (openem/kernels/source_dft.cu:39-73,
 * openem/sources_setup.py:93-119): H correction on plane kh (Hy for pol 0, Hx for pol 1),
 * E correction on plane ks; tables hold n_tab >= n_total float64 samples. */
int oem_plan_add_plane_source(oem_plan* p, int pol, int kh, int ks, double coef_h,
                              double coef_e, int64_t n_tab, const double* ex_tab,
                              const double* hy_tab);

/* Point dipoles (openem/kernels/source_dft.cu:135-206, openem/sources_setup.py:419-457).
 * n_pts stencil points: cell (i, j, k) as three int32, component, coef = weight/dV, source
 * index. amp: (n_src, nsteps1) float64, half-step samples for electric dipoles, whole-step for
 * magnetic. Points that hit the same (component, cell) are summed in a fixed order. */
int oem_plan_add_dipoles(oem_plan* p, int magnetic, int n_pts, const int32_t* ijk,
                         const int32_t* comp, const float* coef, const int32_t* src, int n_src,
                         int64_t nsteps1, const double* amp);

/* Mode / Gaussian-beam / oblique plane-wave source: one-plane TF/SF injection with 2D complex
 * profiles (replaces inject_mode_h/_e, openem/kernels/source_dft.cu:84-128, their complex
 * variants inject_mode_h_c/_e_c, openem/kernels/bloch.cu:326-384, and the host tables of
 * openem/sources_setup.py:321-416). The tangential pair is cyclic, t1 = (axis+1)%3,
 * t2 = (axis+2)%3; n1 x n2 is the whole plane (n_t1, n_t2). profiles: (n_terms, 8, n1, n2)
 * float32 = E_t1 re, E_t1 im, E_t2 re, E_t2 im, H_t1 re, H_t1 im, H_t2 re, H_t2 im for the base
 * term then the broadband corrections; amp_e / amp_h: (n_terms, ntab, 2) float64 (re, im) of
 * amp(n dt) and amp((n+1/2) dt). After the H update of step n, H_t1[kh] += coef_h1 * E_t2 amp_e,
 * H_t2[kh] += coef_h2 * E_t1 amp_e; after the E update, E_t1[ks] += cb * coef_e1 * H_t2 amp_h,
 * E_t2[ks] += cb * coef_e2 * H_t1 amp_h. A real plan adds the real part of each product, a
 * complex plan the whole product. */
int oem_plan_add_mode_source(oem_plan* p, int axis, int kh, int ks, int n1, int n2,
                             double coef_h1, double coef_h2, double coef_e1, double coef_e2,
                             int n_terms, const float* profiles, int64_t ntab,
                             const double* amp_e, const double* amp_h);

/* Tile shape of the pipelined update kernels: x planes walked by one block (0 = the plan's
 * automatic choice; the warp-specialised kernels cap it at 64). No OpenEM counterpart: set by the
 * serving autotuner per grid-size class before oem_plan_finalize. */
int oem_plan_set_xchunk(oem_plan* p, int xch);

/* Check of the failure path of the bounded device waits (no OpenEM counterpart; OpenEM's
 * kernels have no waits). With polls > 0, before oem_plan_finalize, every consumer warp of the
 * warp-specialised E update additionally waits on a shared-memory barrier that no thread ever
 * arrives at, giving up after `polls` polls: the kernel records the expiry in the plan's error
 * word, every warp leaves its pipeline, the producers first wait for their own copies, and the
 * next oem_plan_status / readout returns OEM_ERR_TIMEOUT. The fields of such a run are invalid.
 * Nothing faults or hangs; the device and other plans stay usable. 0 (the default) = off. */
int oem_plan_set_wait_expiry_check(oem_plan* p, int polls);

/* Declare, before oem_plan_finalize, the box (i0, j0, k0, ni, nj, nk) a later
 * oem_plan_adjoint_flux_box will take gradients over. With checkpoints enabled the forward run
 * then records E of the box after every step ((steps + 1) x 3 x box floats, when that is at most
 * 8 GB and a quarter of the free memory), and the reverse pass over the same box reads it instead
 * of recomputing each segment from its checkpoint (the reference recomputes nothing: its
 * gradients come from a second solve, openem/nb/autograd_hook.py:184-221). The environment
 * variable OEM_B200_ADJ_HISTORY=0 keeps the recompute. */
int oem_plan_set_gradient_box(oem_plan* p, const int* box);

/* Discrete adjoint of a flux objective (the reference computes gradients with forward and
 * adjoint solves through tidy3d's VJP, openem/nb/autograd_hook.py:184-221; this engine adds a
 * time-reversed discrete adjoint with K-step checkpoints). oem_plan_enable_checkpoints (before
 * finalize) makes every oem_plan_run save the fields and CPML psi at steps 0, K, 2K, ...;
 * after the whole forward pass, oem_plan_adjoint_flux differentiates
 *   J = sum_f weights[f] * P_f,  P_f = 1/2 sum_plane [Re(E_t1 H_t2*) dA_1 - Re(E_t2 H_t1*) dA_2]
 * of flux monitor mon_id (the phasors it accumulated; dA1, dA2 the (n1, n2) face elements of the
 * two terms, transverse axes ascending) with respect to the E-update coefficients:
 * g_ca, g_cb receive dJ/dca and dJ/dcb per component and cell, (3, nx, ny, nz) float64 each. It
 * recomputes each segment from its checkpoint (the plan's fields are overwritten) and runs the
 * transposed step backward. Real, non-dispersive plans without absorbers. */
int oem_plan_enable_checkpoints(oem_plan* p, int k);
int oem_plan_adjoint_flux(oem_plan* p, int mon_id, const double* weights, const double* dA1,
                          const double* dA2, double* g_ca, double* g_cb, void* stream);
/* The same with the gradients kept for the cells of one box only, box = (i0, j0, k0, ni, nj, nk):
 * g_ca, g_cb are (3, ni, nj, nk); the box of a design region keeps the per-step gradient work
 * and the stored E of each segment to that region. */
int oem_plan_adjoint_flux_box(oem_plan* p, int mon_id, const double* weights, const double* dA1,
                              const double* dA2, const int* box, double* g_ca, double* g_cb,
                              void* stream);

/* Time-modulated permittivity (openem/kernels/modulation.cu:40-79,
 * openem/sources_setup.py:460-518, 640-650): eps(t) = eps_s + amp cos(omega t - phi) on n_entry
 * (comp, cell) entries, cell = (i ny + j) nz + k, each (comp, cell) at most once. Every step the
 * D-form coefficients ca = (eps(t_n) - sd) / (eps(t_n+1) + sd + gg), cb = dte / (same) replace
 * the cell's update coefficients before the E update; cph / sph are cos / sin of phi, cs_tab holds
 * ntab >= n_total rows (cos w t_n, sin w t_n, cos w t_n+1, sin w t_n+1), dte = dt / eps0. Each
 * modulated cell must own its material record (no other cell may use its material index). */
int oem_plan_add_modulation(oem_plan* p, int n_entry, const int* comp, const int64_t* cell,
                            const float* amp, const float* cph, const float* sph,
                            const float* eps_s, const float* sd, const float* gg, int ntab,
                            const float* cs_tab, double dte);

/* Instantaneous flux through a plane (FluxTimeMonitor; openem/readout.py:20-73,
 * openem/flux.py:146-164, 307-578): per sampled step m (m = beg + iv q < end, q < nslots)
 *   s(m) = sum_planes w sum_(u,v) dS[u,v] (E_t1 Hbar_t2 - E_t2 Hbar_t1),  Hbar = (H^{m-1/2} +
 * H^{m+1/2}) / 2, with the components colocated onto the samples: per plane q (1 or 2) E from
 * layer ke[q] of the normal axis, H from layers kh[q], kh[q] + 1 with weights wh[2q], wh[2q+1];
 * along t1 (the lower transverse axis) E_t1 and H_t2 interpolate between cells lo1[u] and hi1[u]
 * with low weights wlo1[0][u] (E) / wlo1[1][u] (H) and high weight whi1[u], the others sit on
 * edge e1[u]; the same along t2 with (E_t2, H_t1). dS is (n1, n2), signed. Read with
 * oem_plan_read_flux_time (nslots float64). */
int oem_plan_add_flux_time_monitor(oem_plan* p, int axis, int nplanes, const double* w,
                                   const int* ke, const int* kh, const double* wh, int n1,
                                   const int* e1, const int* lo1, const int* hi1,
                                   const double* wlo1, const double* whi1, int n2, const int* e2,
                                   const int* lo2, const int* hi2, const double* wlo2,
                                   const double* whi2, const double* dS, int beg, int end, int iv,
                                   int nslots, int* id);
int oem_plan_read_flux_time(oem_plan* p, int id, double* out, void* stream);

/* TFSF box (openem/sources_setup.py:120-318, openem/kernels/tfsf.cu): incident tables of the 1D
 * auxiliary line, ex_tab (ex_rows >= n_total + 1, ex_n columns) = E^n on the box edges read by
 * the H faces after the H update of step n, hy_tab (hy_rows >= n_total, hy_n) = H^{n+1/2} on the
 * box cells read by the E faces after the E update. Faces are grouped and ordered as described
 * at oem_tfsf_face; H-side corrections follow the plane waves, E-side ones likewise. */
int oem_plan_add_tfsf(oem_plan* p, int n_e, const oem_tfsf_face* e_faces, int n_h,
                      const oem_tfsf_face* h_faces, int ex_rows, int ex_n, const double* ex_tab,
                      int hy_rows, int hy_n, const double* hy_tab);

/* Fully anisotropic cells (openem/kernels/tensor.cu, openem/model.py:674-786): n_entry
 * (comp, cell) entries, cell = (i ny + j) nz + k, with the rows of M1 = A^-1 B and
 * M2 = (dt / eps0) A^-1 of their component (n x 3, A = eps + s, B = eps - s, s = sigma dt / 2eps0)
 * and the PEC-wall factor of the written value. The cells' material records must pass the curl
 * through (ca = 0, cb = 1); each step rhs = M1 <E^n> before the E update and
 * E^{n+1} = rhs + M2 <curl H - J> after the E-side injection, the other two components averaged
 * over four neighbours. The table must be closed under that stencil. */
int oem_plan_add_tensor(oem_plan* p, int n_entry, const int* comp, const int64_t* cell,
                        const float* m1, const float* m2, const float* pec);

/* Slanted-interface cells (openem/kernels/dispersion_mix.cu:41-135, openem/model.py:529-612,
 * tables of openem/device_tables.py:291-321): n_entry (comp, cell) entries, cell =
 * (i ny + j) nz + k, whose material records pass the curl through (ca = 0, cb = 1). Entry e owns
 * arithmetic-branch poles p_ofs[e]..p_ofs[e+1] (poles of eps, conjugate pairs counted by
 * 2 Re) and harmonic-branch poles q_ofs[e]..q_ofs[e+1] (poles of 1/eps, every root listed),
 * each pole a row (Re(A-1), Im(A-1), Re(B), Im(B)) of p_coef / q_coef; k holds per entry
 * (k1, k2, 1 - beta, 1 / (k1 k2 + beta)) with k1 = (1 - beta)(eps_inf + sum 2 Re(B_P)) and
 * k2 = zeta_inf + sum Re(B_Q); dte = dt / eps0. Each step SP / SQ come from E^n and d_h^n
 * before the E update; after the E-side injection d_tot += dte * E, d_h^{n+1} =
 * (d_tot - k1 SQ - (1 - beta) SP) / (k1 k2 + beta) and E^{n+1} = k2 d_h + SQ. */
int oem_plan_add_dispersion_mix(oem_plan* p, int n_entry, const int* comp, const int64_t* cell,
                                const int* p_ofs, const float* p_coef, int n_p, const int* q_ofs,
                                const float* q_coef, int n_q, const float* k, double dte);

/* Absorber boundary slab (Tidy3D's Absorber; replaces absorb_slab / absorb_batch,
 * openem/kernels/absorber.cu:20-70, absorb_batch.cu:15-110, and the host tables of
 * openem/dispersion_setup.py:89-120): layers [g0, g0 + nlay) along `axis`. After the H-side
 * sources of every step the H family in the layers is multiplied by the per-layer decay
 * exp(-Gamma dt) (tangential H at half-cell positions: decay_half, normal H: decay_int), after
 * the E-side updates the E family (normal E: decay_half, tangential E: decay_int). Several slabs
 * multiply in the order they were added. Factors must lie in (0, 1]. */
int oem_plan_add_absorber(oem_plan* p, int axis, int g0, int nlay, const double* decay_int,
                          const double* decay_half);

/* Complex (Bloch) plan: imaginary parts of the neighbour masks of one axis (the real parts come
 * from oem_plan_set_axis), exp(+-i 2 pi k) at the periodic seam of a Bloch axis
 * (openem/grid.py:219-252). The first call makes the plan complex: every field and psi gets an
 * imaginary array, the updates become openem/kernels/bloch.cu:38-221, and monitors and time
 * samples record complex values. Call after oem_plan_set_axis and before adding sources or
 * monitors. Complex plans take no dispersive media (OEM_ERR_UNSUPPORTED at finalize), the
 * subset of openem/solver.py:1221-1260. */
int oem_plan_set_axis_phase(oem_plan* p, int axis, const double* mnx_im, const double* mpv_im);

/* Point dipoles on a complex plan: as oem_plan_add_dipoles with the complex amplitude split in
 * two tables (openem/kernels/bloch.cu:226-278). */
int oem_plan_add_dipoles_complex(oem_plan* p, int magnetic, int n_pts, const int32_t* ijk,
                                 const int32_t* comp, const float* coef, const int32_t* src,
                                 int n_src, int64_t nsteps1, const double* amp_re,
                                 const double* amp_im);

/* DFT monitors (openem/kernels/source_dft.cu:208-779, openem/monitors_setup.py:74-255).
 * phase: (n_total, nf, 4) float32 rows (cos, sin at E time (n+1)dt, cos, sin at H time
 * (n+1/2)dt), apodisation window already multiplied in. Accumulators are float64.
 * A flux monitor records (E_t1, E_t2, H_t1, H_t2) on the plane km of normal `axis`
 * (transverse axes ascending) with H colocated as (H[km] + H[km-1]) / 2; a box monitor
 * records the six components at their Yee positions. batch: snapshot ring depth T (steps
 * per fp32 partial sum), 1..32. The id of the new monitor is written to *id. */
int oem_plan_add_flux_monitor(oem_plan* p, int axis, int km, int nf, int64_t n_total,
                              const float* phase, int batch, int* id);
int oem_plan_add_box_monitor(oem_plan* p, int i0, int j0, int k0, int ni, int nj, int nk,
                             int nf, int64_t n_total, const float* phase, int batch, int* id);

/* Field time monitor (openem/kernels/source_dft.cu:273-319): components comps[0..nc-1]
 * (0..5 = Ex..Hz) in a box, sampled at m = beg, beg+iv, ... < end into nslots slots, H averaged
 * over the two neighbouring half steps. */
int oem_plan_add_time_monitor(oem_plan* p, int nc, const int32_t* comps, int i0, int j0, int k0,
                              int ni, int nj, int nk, int beg, int end, int iv, int nslots,
                              int* id);

/* Allocate the fields and auxiliary state, upload everything, capture the step graph.
 * n_total is the nominal number of steps (bounds the source and phase tables). When the plan's
 * largest phasor readout takes 16 MB or more, a host thread started here grows the process's
 * pinned readout stage for this device (page locking of up to 128 MB); the first readout of
 * the plan, or oem_plan_destroy, joins it. */
int oem_plan_finalize(oem_plan* p, int64_t n_total);

/* Advance nsteps full time steps on `stream` (asynchronous). One step is
 * openem/solver.py:1145-1162 (_step_body): H update + H sources, E update with the ADE and
 * conductivity + E sources, time sampling, DFT. */
int oem_plan_run(oem_plan* p, int64_t nsteps, void* stream);

/* Fold the partly filled snapshot batch of every DFT monitor into its accumulator
 * (openem/readout.py:137-157). Idempotent until the next step. */
int oem_plan_flush(oem_plan* p, void* stream);

/* Synchronise `stream` and report OEM_ERR_TIMEOUT if a kernel's bounded pipeline wait gave up
 * since the last check (the readout calls report it too). */
int oem_plan_status(oem_plan* p, void* stream);

/* Number of kernel launches one time step of this plan makes (the kernel nodes of its
 * captured one-step graph). */
int oem_plan_launches_per_step(oem_plan* p, int* n);

/* Number of box DFT monitors whose per-step snapshot the E update kernel writes itself (0: one
 * snapshot launch covers every box monitor, the default). Decided at finalize when OEM_B200_SNAP=update
 * is set in the environment: a real plan on the warp-specialised kernels whose only E-side
 * work after the update is electric dipoles, with at most four box monitors. */
int oem_plan_box_snapshots_in_update(oem_plan* p, int* n);

/* 1 when this plan runs each step's pole pass one step early: a run of c >= 2 steps launches
 * the first step's pole pass, then every step but the last runs the next step's pole pass
 * beside its DFT snapshots and flushes (it reads E^{n+1} once every E-side source is in); the
 * last step runs none, so the pole states are those of the run's last step when the call
 * returns. Decided at finalize: a dispersive plan on the warp-specialised kernels without time
 * modulation, mixed-form or tensor entries; OEM_B200_ADE=inline in the environment turns it
 * off. The results are the same bit for bit either way. */
int oem_plan_pole_pass_ahead(oem_plan* p, int* on);

/* Steps taken so far (host-side count). */
int oem_plan_steps(oem_plan* p, int64_t* steps);

/* Complex plan readout: the real and imaginary (nx, ny, nz) float32 parts of one field
 * component; and the real and imaginary sample buffers of a time monitor
 * (openem/solver.py:1410-1436, _readout_c). */
int oem_plan_read_field_complex(oem_plan* p, int comp, float* re, float* im, void* stream);
int oem_plan_read_time_monitor_complex(oem_plan* p, int id, float* re, float* im, void* stream);

/* Readout, synchronous on `stream`: DFT accumulators (ncomp, nf, points) float64 real and
 * imaginary parts; time samples (nc, nslots, ni, nj, nk) float32; one field component
 * (0..5) as an unpadded (nx, ny, nz) float32 array. */
int oem_plan_read_monitor(oem_plan* p, int id, double* re, double* im, void* stream);

/* The same phasors as oem_plan_read_monitor, written as interleaved (re, im) pairs into one
 * host array of 2 x ncomp x nf x cells doubles: the memory layout of a complex128 array of the
 * monitor's shape, so the host assembles nothing (interleaved on the device, copied out in
 * chunks). */
int oem_plan_read_monitor_interleaved(oem_plan* p, int mon_id, double* out, void* stream);

/* Phasor values with a NaN or infinite part that oem_plan_read_monitor_interleaved has read out
 * since the previous call of this function (counted on the device while interleaving); the
 * count is reset. A caller warns of a diverged field from it without scanning the readout
 * (openem/solver.py:347-370 scans the host arrays). */
int oem_plan_readout_nonfinite(oem_plan* p, int64_t* count);
int oem_plan_read_time_monitor(oem_plan* p, int id, float* out, void* stream);
int oem_plan_read_field(oem_plan* p, int comp, float* out, void* stream);
int oem_plan_write_field(oem_plan* p, int comp, const float* in, void* stream);
/* Complex plan: set both parts of one field component from unpadded (nx, ny, nz) float32
 * arrays (the inverse of oem_plan_read_field_complex; OpenEM keeps re/im as separate arrays,
 * openem/device_tables.py:87-104). Synchronous. */
int oem_plan_write_field_complex(oem_plan* p, int comp, const float* re, const float* im,
                                 void* stream);

/* Volume-weighted float64 sums for the early-termination criteria
 * (openem/solver.py:107-121, :160-203): out[0] = sum V |E|^2, out[1] = sum V eps |E|^2,
 * out[2] = sum V |H|^2. V is the Yee dual volume of the E component of the same index
 * (openem/grid.py:350-366), for H too, as OpenEM weights them (openem/solver.py:176); a complex
 * plan sums re^2 + im^2. Synchronous. */
int oem_plan_energy(oem_plan* p, double out[3], void* stream);

/* Field sums for callers that cannot allocate device memory. This entry point has no
 * counterpart in OpenEM; it is the allocation-free form of oem_plan_energy, for code that owns
 * its fields in another framework's memory pool or must not let cudaMalloc synchronise the
 * device in its step loop. Inputs: six fp32 field arrays (device pointers, (nx, ny, nzp) with
 * z padded to nzp >= nz), three fp32 relative-permittivity arrays in the same layout (or NULL
 * for 1), and the host array `spacing` of 2*(nx+ny+nz) doubles: primal then dual spacing of x,
 * then of y, then of z. Output: out[0] = sum V|E|^2, out[1] = sum V eps|E|^2,
 * out[2] = sum V|H|^2 with the volumes of oem_plan_energy; synchronous on `stream`. Real
 * fields only: the imaginary parts of a complex (Bloch) plan are not summed, so such callers
 * use oem_plan_energy instead.
 * It allocates nothing: its only scratch is a file-scope device array of 581 KB (held on every
 * GPU that loads the library until exit), so nx + ny + nz is limited to 32768. The first call
 * on a device looks that array up (cudaGetSymbolAddress); under CUDA's lazy module loading
 * that first call also loads the library's module onto the device, which can allocate and
 * synchronise. Make one warm-up call per device outside the step loop and before any stream
 * capture. All calls share the array: calls that overlap on the GPU race. */
int oem_field_energy_noalloc(const float* const fields[6], const float* const eps[3], int nx,
                             int ny, int nz, int nzp, const double* spacing, double out[3],
                             void* stream);

/* Device pointers of the six field arrays (padded layout) and the padded z pitch, for
 * zero-copy interop with array libraries. */
int oem_plan_field_ptrs(oem_plan* p, void* ptrs[6], int* nzp);

/* Per-launch timing of the hot kernels accumulated by oem_plan_run when enabled (CUDA events
 * on the run stream): kernel names, launch counts and total milliseconds. */
int oem_plan_enable_timing(oem_plan* p, int on);
int oem_plan_timing(oem_plan* p, int max, char* names /* max*32 */, int64_t* counts,
                    double* ms, int* n);

#ifdef __cplusplus
}
#endif
#endif /* OEM_B200_H */
