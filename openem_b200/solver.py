"""Drop-in replacement of OpenEM's ``solver.run`` (``openem/solver.py:403-511``).

``run(sc, num_steps, use_shutoff, kernels, verbose, return_fields, policy, force_complex)``
takes the same ``Scene`` and returns the same ``Result``. The float64 tables are built on the
host (:mod:`openem_b200.tables`), handed to ``liboem_b200.so`` through its C ABI, and the step
loop runs there as a captured CUDA graph; Python only decides when to stop.

Physics this engine does not run yet raises ``NotImplementedError`` before anything is
allocated, the same fail-closed behaviour as OpenEM (``openem/solver.py:1221-1260``).
"""

from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from openem_b200 import flux as flux_mod
from openem_b200 import lib as L
from openem_b200 import shutoff as shutoff_mod
from openem_b200 import tables as T
from openem_b200.results import Phasors, Result

SHUTOFF_INTERVAL = 400
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")

_TOUCH_POOL = None


def host_array(shape, dtype) -> np.ndarray:
    """An output array for a device readout. A large one has its pages touched by eight threads
    first: a copy into fresh pages spends most of its time in page faults (a 403 MB phasor
    readout: 81 ms into fresh pages, 20 ms into touched ones), and the faults of separate
    threads run in parallel."""
    global _TOUCH_POOL
    out = np.empty(shape, dtype)
    flat = out.reshape(-1).view(np.uint8)
    if flat.size < (64 << 20):
        return out
    if _TOUCH_POOL is None:
        from concurrent.futures import ThreadPoolExecutor
        _TOUCH_POOL = ThreadPoolExecutor(max_workers=8)
    step = -(-flat.size // 8)
    list(_TOUCH_POOL.map(lambda q: flat[q * step:(q + 1) * step].fill(0), range(8)))
    return out


def refuse_unsupported(sc) -> None:
    """Fail closed on scene features outside this engine's real-field path."""
    checks = [
        (T.dispersion_in_absorbers(sc), "dispersive media inside Absorber layers"),
        (any(getattr(t, "k_hat", None) is None and getattr(t, "open_axes", ())
             for t in getattr(sc, "tfsf_sources", [])), "open-axis TFSF boxes at normal incidence"),
        (len(getattr(sc, "tfsf_sources", [])) > 1, "several TFSF boxes in one scene"),
        (sc.modulation is not None and sc.modulation.n_entry > 0
         and (sc.pec_ex is not None or sc.tensor is not None or sc.dispersion_mix is not None),
         "time-modulated media together with PEC, tensor or mixed media"),
        (sc.tensor is not None and sc.tensor.n_entry > 0
         and ((sc.dispersion is not None and sc.dispersion.n_entry > 0) or sc.pec_ex is not None
              or (sc.dispersion_mix is not None and sc.dispersion_mix.n_entry > 0)),
         "fully anisotropic media together with dispersion, PEC cells or mixed media"),
        (any(k != 0.0 for k in sc.bloch_k), "Bloch boundaries"),
    ]
    for bad, what in checks:
        if bad:
            raise NotImplementedError(f"{what} are not supported by the sm_100a engine yet")


def refuse_unsupported_bloch(sc) -> None:
    """Fail closed outside the complex-field subset (openem/solver.py:1221-1260): point dipoles,
    mode sources (oblique plane waves, beams), DFT and time monitors, CPML and periodic / Bloch
    axes; lossless, non-dispersive media without PEC."""
    bad = []
    if sc.sources:
        bad.append("plane wave sources")
    if getattr(sc, "tfsf_sources", None):
        bad.append("TFSF sources")
    if (sc.dispersion is not None and sc.dispersion.n_entry > 0) or \
            (sc.dispersion_mix is not None and sc.dispersion_mix.n_entry > 0):
        bad.append("dispersive media")
    if sc.modulation is not None and sc.modulation.n_entry > 0:
        bad.append("time-varying media")
    if sc.tensor is not None and sc.tensor.n_entry > 0:
        bad.append("tensor media")
    if sc.sigma_ex is not None:
        bad.append("conductivity")
    if sc.pec_ex is not None:
        bad.append("PEC cells")
    if getattr(sc, "flux_time_monitors", None):
        bad.append("FluxTimeMonitor")
    if bad:
        raise NotImplementedError(
            "the Bloch complex-field path does not support: " + ", ".join(bad)
            + ". The supported subset is point dipoles (electric/magnetic), mode sources, DFT "
            "and time monitors, CPML / periodic / Bloch boundaries")
    if not sc.dipoles and not getattr(sc, "mode_sources", None):
        raise NotImplementedError(
            "the Bloch complex-field path needs a point dipole source or an (oblique) mode "
            "source, and this scene has neither")


class Plan:
    """One simulation resident on the device: owns a ``oem_plan``."""

    def __init__(self, sc, n_total: int | None = None, device: int = 0, stream=None,
                 batch: int | None = None, cplx: bool = False, xchunk: int = 0,
                 checkpoint_every: int = 0, gradient_box=None, wait_expiry_polls: int = 0):
        self.cplx = bool(cplx)
        self.xchunk = int(xchunk)
        self.wait_expiry_polls = int(wait_expiry_polls)
        self.checkpoint_every = int(checkpoint_every)
        self.gradient_box = None if gradient_box is None else \
            np.ascontiguousarray(gradient_box, dtype=np.int32)
        if self.cplx:
            refuse_unsupported_bloch(sc)
        else:
            refuse_unsupported(sc)
        self.lib = L.load()
        self.sc = sc
        self.n_total = int(sc.num_time_steps if n_total is None else n_total)
        self.stream = stream
        self.device = int(device)
        self.shape = tuple(int(v) for v in sc.shape)
        nx, ny, nz = self.shape
        self._keep = []
        h = C.c_void_p()
        L.check(self.lib.oem_plan_create(int(device), nx, ny, nz, float(sc.dt / T.MU_0),
                                         float(T.EPSILON_0 / sc.dt), C.byref(h)), "plan_create")
        self.h = h
        self.h2d_bytes = 0
        try:
            self._build(batch)
        except Exception:
            self.close()
            raise

    # ---- construction ------------------------------------------------------------------
    def _device_tables(self) -> bool:
        """Build the per-cell tables on the GPU for large grids (host numpy otherwise)."""
        mode = os.environ.get("OEM_B200_TABLES", "auto")
        if mode == "host":
            return False
        from openem_b200 import tables_gpu
        if mode == "device":
            return True
        return int(np.prod(self.shape)) >= 100_000 and tables_gpu.available()

    @staticmethod
    def _warn_nonfinite_materials(table) -> None:
        """The deduplicated material records hold ca, cb and eps of every distinct cell: a NaN
        or Inf in eps or sigma shows here at no cost. Like OpenEM (openem/solver.py:347-370)
        the run goes ahead and the readout warns again; this names the cause up front."""
        coef = np.ascontiguousarray(table, dtype=np.uint32)[:, :9].view(np.float32)
        if not np.isfinite(coef).all():
            print("[openem_b200] warning: eps or sigma holds non-finite values (NaN/Inf): the "
                  "update coefficients of some cells are not finite and the fields will diverge",
                  flush=True)

    def _arr(self, a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        self._keep.append(a)
        self.h2d_bytes += a.nbytes
        return a

    def _build(self, batch):
        sc, lib, h = self.sc, self.lib, self.h
        if self.cplx:
            self.tabs = [T.axis_tables(sc, a, float(sc.bloch_k[a])) for a in range(3)]
        else:
            self.tabs = [T.axis_tables(sc, a) for a in range(3)]
        for a, t in enumerate(self.tabs):
            L.check(lib.oem_plan_set_axis(
                h, a, L.ptr(self._arr(t.idl_p, np.float64)), L.ptr(self._arr(t.idl_d, np.float64)),
                L.ptr(self._arr(t.nxt, np.int32)), L.ptr(self._arr(t.prv, np.int32)),
                L.ptr(self._arr(np.real(t.mnx), np.float64)),
                L.ptr(self._arr(np.real(t.mpv), np.float64)),
                L.ptr(self._arr(t.pml_e, np.float64)), L.ptr(self._arr(t.pml_h, np.float64)),
                int(t.lo), int(t.hi)), f"set_axis {a}")
        if self.cplx:
            for a, t in enumerate(self.tabs):
                L.check(lib.oem_plan_set_axis_phase(
                    h, a, L.ptr(self._arr(np.imag(t.mnx), np.float64)),
                    L.ptr(self._arr(np.imag(t.mpv), np.float64))), f"set_axis_phase {a}")
        mod = None if self.cplx else T.modulation_tables(sc, self.tabs, self.n_total)
        if self._device_tables():
            from openem_b200 import tables_gpu
            mt = tables_gpu.material_tables_device(sc, self.tabs, self.device)
            if mod is not None:
                tables_gpu.isolate_cells_device(mt, mod["cell"])
            self.h2d_bytes += int(mt.h2d_bytes)  # eps and sigma as copied (dense or sparse)
            self._warn_nonfinite_materials(mt.table)
            L.check(lib.oem_plan_set_materials_device(
                h, int(mt.n_mat), L.ptr(self._arr(mt.table, np.uint32)), int(mt.index_bytes),
                C.c_void_p(mt.index.data_ptr())), "set_materials_device")
            if mt.n_pole_total > 0:
                L.check(lib.oem_plan_set_pole_sets_device(
                    h, int(mt.set_ofs.size - 1), L.ptr(self._arr(mt.set_ofs, np.int32)),
                    L.ptr(self._arr(mt.coef, np.float32)), C.c_void_p(mt.seg_ofs.data_ptr()),
                    int(mt.seg_ofs.numel()), int(mt.n_pole_total)), "set_pole_sets_device")
            del mt
        else:
            mt = T.material_tables(sc, self.tabs)
            table, index, n_mat = mt.table, mt.index, mt.n_mat
            if mod is not None:
                table, index, n_mat = T.isolate_cells(table, index, mod["cell"])
            self._warn_nonfinite_materials(table)
            L.check(lib.oem_plan_set_materials(h, int(n_mat),
                                               L.ptr(self._arr(table, np.uint32)),
                                               int(index.dtype.itemsize),
                                               L.ptr(self._arr(index, index.dtype))),
                    "set_materials")
            if mt.n_pole_total > 0:
                L.check(lib.oem_plan_set_pole_sets(
                    h, int(mt.set_ofs.size - 1), L.ptr(self._arr(mt.set_ofs, np.int32)),
                    L.ptr(self._arr(mt.coef, np.float32)), L.ptr(self._arr(mt.seg_ofs, np.uint32)),
                    int(mt.seg_ofs.size), int(mt.n_pole_total)), "set_pole_sets")
        if mod is not None and mod["comp"].size:
            L.check(lib.oem_plan_add_modulation(
                h, int(mod["comp"].size), L.ptr(self._arr(mod["comp"], np.int32)),
                L.ptr(self._arr(mod["cell"], np.int64)), L.ptr(self._arr(mod["amp"], np.float32)),
                L.ptr(self._arr(mod["cph"], np.float32)), L.ptr(self._arr(mod["sph"], np.float32)),
                L.ptr(self._arr(mod["eps"], np.float32)), L.ptr(self._arr(mod["sd"], np.float32)),
                L.ptr(self._arr(mod["gg"], np.float32)), int(mod["cs"].shape[0]),
                L.ptr(self._arr(mod["cs"], np.float32)), float(mod["dte"])), "modulation")
        for ps in T.plane_sources(sc):
            if ps["ex"].size < self.n_total:
                raise ValueError(f"asked to run {self.n_total} steps, but the plane-wave table "
                                 f"holds {ps['ex'].size} samples")
            L.check(lib.oem_plan_add_plane_source(
                h, ps["pol"], ps["kh"], ps["ks"], ps["coef_h"], ps["coef_e"], int(ps["ex"].size),
                L.ptr(self._arr(ps["ex"], np.float64)), L.ptr(self._arr(ps["hy"], np.float64))),
                "add_plane_source")
        tt = None if self.cplx else T.tensor_tables(sc, self.tabs)
        if tt is not None:
            L.check(lib.oem_plan_add_tensor(
                h, int(tt["comp"].size), L.ptr(self._arr(tt["comp"], np.int32)),
                L.ptr(self._arr(tt["cell"], np.int64)), L.ptr(self._arr(tt["m1"], np.float32)),
                L.ptr(self._arr(tt["m2"], np.float32)), L.ptr(self._arr(tt["pec"], np.float32))),
                "add_tensor")
        mx = None if self.cplx else T.mix_tables(sc)
        if mx is not None:
            L.check(lib.oem_plan_add_dispersion_mix(
                h, int(mx["comp"].size), L.ptr(self._arr(mx["comp"], np.int32)),
                L.ptr(self._arr(mx["cell"], np.int64)), L.ptr(self._arr(mx["p_ofs"], np.int32)),
                L.ptr(self._arr(mx["pc"], np.float32)), int(mx["n_p"]),
                L.ptr(self._arr(mx["q_ofs"], np.int32)), L.ptr(self._arr(mx["qc"], np.float32)),
                int(mx["n_q"]), L.ptr(self._arr(mx["k"], np.float32)), float(mx["dte"])),
                "add_dispersion_mix")
        if getattr(sc, "tfsf_sources", None) and not self.cplx:
            from openem_b200 import tfsf as TF
            tb = TF.box_tables(sc, self.n_total)
            nzp = T.pad_z(self.shape[2])
            ef = self._arr(TF.device_faces(tb["e_faces"], self.shape[1], nzp), TF.FACE_DTYPE)
            hf = self._arr(TF.device_faces(tb["h_faces"], self.shape[1], nzp), TF.FACE_DTYPE)
            ex, hy = self._arr(tb["ex_tab"], np.float64), self._arr(tb["hy_tab"], np.float64)
            L.check(lib.oem_plan_add_tfsf(h, int(ef.size), L.ptr(ef), int(hf.size), L.ptr(hf),
                                          int(ex.shape[0]), int(ex.shape[1]), L.ptr(ex),
                                          int(hy.shape[0]), int(hy.shape[1]), L.ptr(hy)),
                    "add_tfsf")
        for mag in (False, True):
            dt_ = T.dipole_tables(sc, self.n_total, mag, complex_amp=self.cplx)
            if dt_ is None:
                continue
            head = (h, int(mag), int(dt_["comp"].size), L.ptr(self._arr(dt_["ijk"], np.int32)),
                    L.ptr(self._arr(dt_["comp"], np.int32)),
                    L.ptr(self._arr(dt_["coef"], np.float32)),
                    L.ptr(self._arr(dt_["src"], np.int32)), int(dt_["n_src"]),
                    int(dt_["nsteps1"]), L.ptr(self._arr(dt_["amp"], np.float64)))
            if self.cplx:
                L.check(lib.oem_plan_add_dipoles_complex(
                    *head, L.ptr(self._arr(dt_["amp_im"], np.float64))), "add_dipoles_complex")
            else:
                L.check(lib.oem_plan_add_dipoles(*head), "add_dipoles")
        for axis, g0, nlay, di, dh in T.absorber_tables(sc):
            L.check(lib.oem_plan_add_absorber(h, axis, g0, nlay, L.ptr(self._arr(di, np.float64)),
                                              L.ptr(self._arr(dh, np.float64))), "add_absorber")
        for ms in T.mode_tables(sc, self.n_total):
            L.check(lib.oem_plan_add_mode_source(
                h, ms["axis"], ms["kh"], ms["ks"], ms["n1"], ms["n2"], *ms["coef_h"],
                *ms["coef_e"], int(ms["prof"].shape[0]), L.ptr(self._arr(ms["prof"], np.float32)),
                ms["ntab"], L.ptr(self._arr(ms["amp_e"], np.float64)),
                L.ptr(self._arr(ms["amp_h"], np.float64))), "add_mode_source")
        nt = max(self.n_total, 1)
        self.flux_mons = []
        for m in sc.flux_monitors:
            t1, t2 = [a for a in range(3) if a != m.axis]
            n1, n2 = self.shape[t1], self.shape[t2]
            ph = T.phase_table(m.freqs, sc.dt, nt, m.apodization)
            Tb = batch or T.batch_depth(n1 * n2, 4)
            mid = C.c_int()
            L.check(lib.oem_plan_add_flux_monitor(h, int(m.axis), int(m.plane_index),
                                                  int(np.size(m.freqs)), nt,
                                                  L.ptr(self._arr(ph, np.float32)), int(Tb),
                                                  C.byref(mid)), f"flux monitor {m.name}")
            self.flux_mons.append((m, mid.value, (4, int(np.size(m.freqs)), n1, n2)))
        self.box_mons = []
        for m in sc.field_monitors:
            ni, nj, nk = (int(v) for v in m.box)
            ph = T.phase_table(m.freqs, sc.dt, nt, m.apodization)
            Tb = batch or T.batch_depth(ni * nj * nk, 6)
            mid = C.c_int()
            i0, j0, k0 = (int(v) for v in m.origin)
            L.check(lib.oem_plan_add_box_monitor(h, i0, j0, k0, ni, nj, nk,
                                                 int(np.size(m.freqs)), nt,
                                                 L.ptr(self._arr(ph, np.float32)), int(Tb),
                                                 C.byref(mid)), f"field monitor {m.name}")
            self.box_mons.append((m, mid.value, (6, int(np.size(m.freqs)), ni, nj, nk)))
        self.time_mons = []
        for m in sc.field_time_monitors:
            ni, nj, nk = (int(v) for v in m.box)
            comps = self._arr(np.asarray(m.comps, np.int32), np.int32)
            mid = C.c_int()
            i0, j0, k0 = (int(v) for v in m.origin)
            L.check(lib.oem_plan_add_time_monitor(h, int(comps.size), L.ptr(comps), i0, j0, k0,
                                                  ni, nj, nk, int(m.step_begin), int(m.step_end),
                                                  int(m.interval), int(m.num_slots),
                                                  C.byref(mid)), f"time monitor {m.name}")
            self.time_mons.append((m, mid.value, (int(comps.size), int(m.num_slots), ni, nj, nk)))
        self.ft_mons = []
        if not self.cplx:
            from openem_b200 import flux_time as FT
            for m in getattr(sc, "flux_time_monitors", []):
                t = FT.device_tables(FT.geometry(sc.grid, m))
                mid = C.c_int()
                a = lambda k, dt: L.ptr(self._arr(t[k], dt))
                L.check(lib.oem_plan_add_flux_time_monitor(
                    h, int(m.axis), int(t["nplanes"]), a("w", np.float64), a("ke", np.int32),
                    a("kh", np.int32), a("wh", np.float64), int(t["n1"]), a("e1", np.int32),
                    a("lo1", np.int32), a("hi1", np.int32), a("wlo1", np.float64),
                    a("whi1", np.float64), int(t["n2"]), a("e2", np.int32), a("lo2", np.int32),
                    a("hi2", np.int32), a("wlo2", np.float64), a("whi2", np.float64),
                    a("dS", np.float64), int(m.step_begin), int(m.step_end), int(m.interval),
                    int(m.num_slots), C.byref(mid)), f"flux time monitor {m.name}")
                self.ft_mons.append((m, mid.value))
        if self.xchunk:
            L.check(lib.oem_plan_set_xchunk(h, self.xchunk), "set_xchunk")
        if self.wait_expiry_polls:
            L.check(lib.oem_plan_set_wait_expiry_check(h, self.wait_expiry_polls),
                    "set_wait_expiry_check")
        if self.checkpoint_every:
            L.check(lib.oem_plan_enable_checkpoints(h, self.checkpoint_every), "checkpoints")
        if self.gradient_box is not None:
            L.check(lib.oem_plan_set_gradient_box(h, L.ptr(self.gradient_box)), "gradient box")
        L.check(lib.oem_plan_finalize(h, self.n_total), "finalize")
        self._keep.clear()

    # ---- stepping / readout ------------------------------------------------------------
    @property
    def _s(self):
        return L.stream_handle(self.stream)

    def run(self, nsteps: int) -> None:
        L.check(self.lib.oem_plan_run(self.h, int(nsteps), self._s), "run")

    def flush(self) -> None:
        L.check(self.lib.oem_plan_flush(self.h, self._s), "flush")

    @property
    def steps(self) -> int:
        v = C.c_int64()
        L.check(self.lib.oem_plan_steps(self.h, C.byref(v)))
        return int(v.value)

    def read_monitor(self, mid: int, shape) -> np.ndarray:
        # not pre-touched: the library's copy-out threads fault the pages in parallel
        out = np.empty(shape, np.complex128)
        L.check(self.lib.oem_plan_read_monitor_interleaved(self.h, int(mid), L.ptr(out), self._s),
                "read_monitor")
        return out

    def readout_nonfinite(self) -> int:
        """Phasor values with a non-finite part read out since the previous call (counted on
        the device)."""
        n = C.c_int64(0)
        L.check(self.lib.oem_plan_readout_nonfinite(self.h, C.byref(n)), "readout_nonfinite")
        return int(n.value)

    def adjoint_flux(self, mid: int, weights, dA1, dA2, box=None):
        """dJ/dca and dJ/dcb, (3, ni, nj, nk) float64 each, of ``J = sum_f weights[f] P_f``
        for the flux monitor ``mid`` (face elements ``dA1``, ``dA2`` of its two terms), over
        ``box = (i0, j0, k0, ni, nj, nk)`` (default: the whole grid)."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        a1 = np.ascontiguousarray(dA1, dtype=np.float64)
        a2 = np.ascontiguousarray(dA2, dtype=np.float64)
        b = np.asarray(box if box is not None else (0, 0, 0) + self.shape, dtype=np.int32)
        b = np.ascontiguousarray(b)
        g_ca = np.empty((3,) + tuple(int(v) for v in b[3:]), np.float64)
        g_cb = np.empty_like(g_ca)
        L.check(self.lib.oem_plan_adjoint_flux_box(self.h, int(mid), L.ptr(w), L.ptr(a1),
                                                   L.ptr(a2), L.ptr(b), L.ptr(g_ca),
                                                   L.ptr(g_cb), self._s), "adjoint_flux")
        return g_ca, g_cb

    def read_time_monitor(self, mid: int, shape) -> np.ndarray:
        out = np.empty(shape, np.float32)
        if self.cplx:
            im = np.empty(shape, np.float32)
            L.check(self.lib.oem_plan_read_time_monitor_complex(self.h, int(mid), L.ptr(out),
                                                                L.ptr(im), self._s),
                    "read_time_monitor_complex")
            return out + 1j * im
        L.check(self.lib.oem_plan_read_time_monitor(self.h, int(mid), L.ptr(out), self._s),
                "read_time_monitor")
        return out

    def read_field(self, comp: int) -> np.ndarray:
        out = host_array(self.shape, np.float32)
        if self.cplx:
            im = np.empty(self.shape, np.float32)
            L.check(self.lib.oem_plan_read_field_complex(self.h, int(comp), L.ptr(out),
                                                         L.ptr(im), self._s), "read_field_complex")
            return out + 1j * im
        L.check(self.lib.oem_plan_read_field(self.h, int(comp), L.ptr(out), self._s), "read_field")
        return out

    def write_field(self, comp: int, arr) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float32)
        if a.shape != self.shape:
            raise ValueError(f"field shape {a.shape} != {self.shape}")
        L.check(self.lib.oem_plan_write_field(self.h, int(comp), L.ptr(a), self._s), "write_field")

    def write_field_complex(self, comp: int, arr) -> None:
        """Set both parts of one field component of a complex plan."""
        arr = np.asarray(arr)
        re = np.ascontiguousarray(arr.real, dtype=np.float32)
        im = np.ascontiguousarray(arr.imag, dtype=np.float32)
        if re.shape != self.shape:
            raise ValueError(f"field shape {re.shape} != {self.shape}")
        L.check(self.lib.oem_plan_write_field_complex(self.h, int(comp), L.ptr(re), L.ptr(im),
                                                      self._s), "write_field_complex")

    def energy(self) -> np.ndarray:
        out = np.zeros(3, np.float64)
        L.check(self.lib.oem_plan_energy(self.h, L.ptr(out), self._s), "energy")
        return out

    def box_snapshots_in_update(self) -> int:
        """Box monitors whose snapshots the E update kernel writes (no launch of their own)."""
        n = C.c_int(0)
        L.check(self.lib.oem_plan_box_snapshots_in_update(self.h, C.byref(n)))
        return int(n.value)

    def pole_pass_ahead(self) -> bool:
        """Whether each step's pole pass runs at the end of the step before it (beside the DFT
        snapshots), within one ``run`` call."""
        n = C.c_int(0)
        L.check(self.lib.oem_plan_pole_pass_ahead(self.h, C.byref(n)))
        return bool(n.value)

    def launches_per_step(self) -> int:
        n = C.c_int()
        L.check(self.lib.oem_plan_launches_per_step(self.h, C.byref(n)))
        return int(n.value)

    def status(self) -> None:
        """Raise if a device pipeline wait timed out since the last check."""
        L.check(self.lib.oem_plan_status(self.h, self._s), "status")

    def enable_timing(self, on: bool = True) -> None:
        L.check(self.lib.oem_plan_enable_timing(self.h, int(bool(on))))

    def timing(self) -> dict:
        names = C.create_string_buffer(32 * 16)
        counts = np.zeros(16, np.int64)
        ms = np.zeros(16, np.float64)
        n = C.c_int()
        L.check(self.lib.oem_plan_timing(self.h, 16, names, L.ptr(counts), L.ptr(ms), C.byref(n)))
        out = {}
        for q in range(n.value):
            nm = names.raw[32 * q:32 * q + 32].split(b"\0", 1)[0].decode()
            out[nm] = (int(counts[q]), float(ms[q]))
        return out

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.oem_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- results -----------------------------------------------------------------------
    def flux_phasor(self, m, mid: int, shp) -> Phasors:
        return Phasors(name=m.name, data=self.read_monitor(mid, shp),
                       freqs=np.asarray(m.freqs, dtype=np.float64))

    def field_phasor(self, m, mid: int, shp) -> np.ndarray:
        return self.read_monitor(mid, shp)

    def flux_phasors(self) -> dict:
        return {m.name: self.flux_phasor(m, mid, shp) for m, mid, shp in self.flux_mons}

    def field_phasors(self) -> dict:
        return {m.name: self.field_phasor(m, mid, shp) for m, mid, shp in self.box_mons}

    def flux_time(self, steps_run: int) -> dict:
        """``{name: (filled,) float64}`` of the flux time monitors after ``steps_run`` steps."""
        out = {}
        for m, mid in self.ft_mons:
            buf = np.zeros(max(int(m.num_slots), 1), np.float64)
            L.check(self.lib.oem_plan_read_flux_time(self.h, int(mid), L.ptr(buf), self._s),
                    "read_flux_time")
            off = min(steps_run - 1, m.step_end - 1) - m.step_begin
            filled = 0 if off < 0 else min(m.num_slots, off // m.interval + 1)
            out[m.name] = buf[:filled].copy()
        return out

    def time_samples(self, steps_run: int):
        samples, slots = {}, {}
        for m, mid, shp in self.time_mons:
            buf = self.read_time_monitor(mid, shp)
            m_last = min(steps_run - 1, m.step_end - 1)
            off = m_last - m.step_begin
            filled = 0 if off < 0 else min(m.num_slots, off // m.interval + 1)
            samples[m.name] = buf[:, :filled].copy()
            slots[m.name] = filled
        return samples, slots


def _time_mon_guard(sc) -> int:
    tm = list(sc.field_time_monitors) + list(getattr(sc, "flux_time_monitors", []))
    return max([int(m.step_begin) + 1 for m in tm] + [0])


def run(sc, num_steps: int | None = None, use_shutoff: bool = True, kernels=None,
        verbose: bool = True, return_fields: bool = False, policy=None,
        force_complex: bool = False, device: int = 0, stream=None,
        stats: dict | None = None) -> Result:
    """Run one FDTD simulation on the GPU (signature of ``openem/solver.py:403-412``; the
    ``kernels`` argument is accepted for call compatibility and unused). ``stats``, when
    given, receives the host-to-device and device-to-host byte counts and the launches per
    step."""
    del kernels
    # the complex-field path (openem/solver.py:1263-1358, _run_bloch): fields and CPML psi as
    # real and imaginary float32 arrays, the Bloch phase exp(+-i 2 pi k) only in the seam
    # neighbour masks; with k = 0 (force_complex) the two parts are two independent real runs.
    # Its subset is OpenEM's (refuse_unsupported_bloch).
    cplx = bool(force_complex or any(k != 0.0 for k in sc.bloch_k))
    return run_plan(sc, num_steps, use_shutoff, verbose, return_fields, policy, device, stream,
                    stats, cplx=cplx)


def run_plan(sc, num_steps, use_shutoff, verbose, return_fields, policy, device, stream, stats,
             cplx: bool) -> Result:
    """Build a plan (real or complex fields), step it with the shutoff cadence, read out."""
    n_total = int(num_steps if num_steps is not None else sc.num_time_steps)
    t0 = time.perf_counter()
    plan = Plan(sc, n_total, device=device, stream=stream, cplx=cplx)
    t1 = time.perf_counter()
    try:
        res = _loop(plan, sc, n_total, use_shutoff, verbose, return_fields, policy)
        plan.status()
        t2 = time.perf_counter()
        if stats is not None:
            # host wall time of the three phases: tables + upload + graph capture, the steps
            # (with the shutoff checks), the readout of every monitor and field
            stats.update(setup_s=t1 - t0, step_s=res.wall_seconds,
                         readout_s=max(t2 - t1 - res.wall_seconds, 0.0))
            d2h = sum(np.asarray(p.data).size * 16 for p in res.phasors.values())
            d2h += sum(np.asarray(a).size * 16 for a in res.field_phasors.values())
            width = 8 if cplx else 4  # float32 parts read back per value
            d2h += sum(np.asarray(a).size * width for a in res.time_samples.values())
            d2h += sum(np.asarray(a).size * width for a in res.fields.values())
            stats.update(h2d_bytes=int(plan.h2d_bytes), d2h_bytes=int(d2h),
                         launches_per_step=plan.launches_per_step())
        return res
    finally:
        plan.close()


def _loop(plan: Plan, sc, n_total: int, use_shutoff: bool, verbose: bool, return_fields: bool,
          policy) -> Result:
    pol = policy or shutoff_mod.default_policy(sc.shutoff, interval=SHUTOFF_INTERVAL)
    interval = int(pol.interval)
    source_end = shutoff_mod.source_end_step(sc)
    guard = _time_mon_guard(sc)
    trace = []
    t0 = time.time()
    steps = 0
    triggered = False
    if not use_shutoff:
        plan.run(n_total)
        steps = n_total
    else:
        grid = sc.grid
        while steps < n_total:
            chunk = min(interval - steps % interval, n_total - steps)
            plan.run(chunk)
            steps += chunk
            if steps % interval:
                continue
            e = plan.energy()
            m_u = 0.5 * (T.EPSILON_0 * e[1] + T.MU_0 * e[2])
            fl = np.zeros(0)
            # the complex path checks no flux criterion (openem/solver.py:1325-1328)
            if plan.flux_mons and not plan.cplx:
                plan.flush()
                fl = np.concatenate([flux_mod.plane_flux(plan.read_monitor(mid, shp), grid,
                                                         axis=int(m.axis))
                                     for m, mid, shp in plan.flux_mons])
            stop = pol.check(steps, float(e[0]), float(m_u), fl) and steps > source_end \
                and steps >= guard
            trace.append((steps, shutoff_mod.trace_ratio(pol)))
            if stop:
                triggered = True
                if verbose:
                    print(f"  early termination at step {steps}: {pol.reason}", flush=True)
                break
    plan.flush()
    plan.status()  # waits for the stream: the steps are done when the clock stops
    wall = time.time() - t0
    # every monitor's readout counts its non-finite phasors on the device (no host scan)
    plan.readout_nonfinite()
    phasors, fphas = {}, {}
    for tag, d, read in (("mon", phasors, plan.flux_phasor), ("fld", fphas, plan.field_phasor)):
        for m, mid, shp in (plan.flux_mons if tag == "mon" else plan.box_mons):
            d[m.name] = read(m, mid, shp)
            if plan.readout_nonfinite():
                print(f"[openem_b200] warning: monitor {tag}:{m.name} holds non-finite values; "
                      "the field has most likely diverged", flush=True)
    tsamp, tslots = plan.time_samples(steps)
    fields = {}
    if return_fields:
        for c, nm in enumerate(COMPONENTS):
            fields[nm] = plan.read_field(c)
    return Result(phasors=phasors, steps_run=steps, shutoff_triggered=triggered,
                  decay_trace=trace,
                  energy_trace=shutoff_mod.energy_trace(pol),
                  source_end=int(source_end), wall_seconds=wall,
                  stop_reason=pol.reason, shutoff_summary=pol.summary(), fields=fields,
                  field_phasors=fphas, time_samples=tsamp, time_slots=tslots,
                  flux_time=plan.flux_time(steps))
