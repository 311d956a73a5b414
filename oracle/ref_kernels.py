"""OpenEM's own CUDA kernels driven step by step -- TEST INFRASTRUCTURE ONLY.

Loads the cubins that ``oracle/build_ref.py`` compiles from ``openem/kernels/{yee,dispersion,
source_dft}.cu`` (unchanged) and runs them in the launch order of OpenEM's two-pass step
(``openem/solver.py:876-969, 1026-1060, 1145-1162``):

    update_h -> dispersion_pre -> update_e -> inject_dipole -> dispersion_post -> step_advance

with the tables laid out as OpenEM's device builders lay them out (``openem/device_tables.py``):
dense float32 ``(nx, ny, nz)`` fields, twelve full-volume psi arrays, per-component dense ``ca`` /
``cb``, float32 axis tables, the dispersion CSR with a coefficient table indexed per pole, the
dipole stencil as flat indices with a float64 amplitude table. Device memory comes from torch;
kernels are launched through the CUDA driver API (``cuModuleLoad`` / ``cuLaunchKernel``).

Only ``tests/`` use this, to pin the FP64 oracle and the engine to the arithmetic of the
reference's kernels. The supported scenes are the real-field subset these kernels cover: CPML or
periodic axes, conductivity, PEC through the masks, pole-residue dispersion, electric dipoles.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from oracle import build_ref
from oracle.ref64 import EPSILON_0, MU_0, e_coeffs, pml_axis_arrays

_cuda = None
_mods: dict = {}


def _driver():
    global _cuda
    if _cuda is None:
        _cuda = C.CDLL("libcuda.so.1")
        _cuda.cuModuleLoad.argtypes = [C.POINTER(C.c_void_p), C.c_char_p]
        _cuda.cuModuleGetFunction.argtypes = [C.POINTER(C.c_void_p), C.c_void_p, C.c_char_p]
        _cuda.cuLaunchKernel.argtypes = [C.c_void_p, C.c_uint, C.c_uint, C.c_uint, C.c_uint,
                                         C.c_uint, C.c_uint, C.c_uint, C.c_void_p,
                                         C.POINTER(C.c_void_p), C.c_void_p]
    return _cuda


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"CUDA driver error {rc} in {what}")


def _function(file: str, name: str):
    cu = _driver()
    key = (file, name)
    if key not in _mods:
        path = build_ref.cubin_path(file)
        if not path.exists():
            raise FileNotFoundError(f"{path} is missing: run python -m oracle.build_ref")
        if file not in _mods:
            m = C.c_void_p()
            _check(cu.cuModuleLoad(C.byref(m), str(path).encode()), f"cuModuleLoad {file}")
            _mods[file] = m
        f = C.c_void_p()
        _check(cu.cuModuleGetFunction(C.byref(f), _mods[file], name.encode()),
               f"cuModuleGetFunction {name}")
        _mods[key] = f
    return _mods[key]


def _launch(file: str, name: str, grid, block, args, stream) -> None:
    """Launch with ``args``: torch tensors (passed as device pointers), ``np.int32`` and
    ``np.float32`` scalars, in the kernel's parameter order."""
    holders = []
    for a in args:
        if hasattr(a, "data_ptr"):
            holders.append(C.c_void_p(a.data_ptr()))
        elif isinstance(a, np.int32):
            holders.append(C.c_int(int(a)))
        elif isinstance(a, np.float32):
            holders.append(C.c_float(float(a)))
        else:
            raise TypeError(f"argument of type {type(a)} for {name}")
    params = (C.c_void_p * len(holders))(*[C.cast(C.pointer(h), C.c_void_p) for h in holders])
    _check(_driver().cuLaunchKernel(_function(file, name), *grid, *block, 0,
                                    C.c_void_p(stream), params, None), name)


class ReferenceKernels:
    """One scene resident on the GPU in OpenEM's layout, stepped by OpenEM's kernels."""

    def __init__(self, sc, n_total: int, device: str = "cuda:0"):
        import torch
        if sc.any_bloch or sc.sources or sc.tfsf_sources or getattr(sc, "mode_sources", None):
            raise NotImplementedError("reference-kernel runs cover dipole-driven real scenes")
        if (sc.modulation is not None and sc.modulation.n_entry) or \
                (sc.tensor is not None and sc.tensor.n_entry) or \
                (sc.dispersion_mix is not None and sc.dispersion_mix.n_entry) or \
                getattr(sc, "absorbers", None):
            raise NotImplementedError("reference-kernel runs cover CPML, sigma and poles only")
        self.torch, self.dev = torch, torch.device(device)
        self.sc = sc
        self.shape = nx, ny, nz = tuple(int(v) for v in sc.shape)
        self.n = 0
        f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=self.dev)
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=self.dev)
        zeros = lambda: torch.zeros(self.shape, dtype=torch.float32, device=self.dev)
        self.E = [zeros() for _ in range(3)]
        self.H = [zeros() for _ in range(3)]
        self.psi_h = [zeros() for _ in range(6)]  # hx_y hx_z hy_z hy_x hz_x hz_y
        self.psi_e = [zeros() for _ in range(6)]  # ex_y ex_z ey_z ey_x ez_x ez_y
        self.hist = [zeros() for _ in range(3)]
        tabs = [a.index_tables() for a in sc.grid.axes]
        self.on = [np.int32(int((a, "lo") in sc.pml or (a, "hi") in sc.pml)) for a in range(3)]
        self.idl_p = [f32(1.0 / a.dl) for a in sc.grid.axes]
        self.idl_d = [f32(1.0 / a.dl_dual) for a in sc.grid.axes]
        self.pml_h = [[f32(v) for v in pml_axis_arrays(sc, a, "H")] for a in range(3)]
        self.pml_e = [[f32(v) for v in pml_axis_arrays(sc, a, "E")] for a in range(3)]
        self.nxt = [i32(t["nxt"]) for t in tabs]
        self.prv = [i32(t["prv"]) for t in tabs]
        self.mnx = [f32(t["mnx"]) for t in tabs]
        self.mpv = [f32(t["mpv"]) for t in tabs]
        self.pec = [f32(t["pec"]) for t in tabs]
        ca, cb = e_coeffs(sc)
        self.ca = [f32(a) for a in ca]
        self.cb = [f32(b) for b in cb]
        self.ch = np.float32(sc.dt / MU_0)
        self.cw = np.float32(EPSILON_0 / sc.dt)
        d = sc.dispersion
        self.disp = None
        if d is not None and d.n_entry:
            cell = np.asarray(d.cell, dtype=np.int64)
            ofs = np.asarray(d.pole_ofs, dtype=np.int64)
            assert cell.min() >= 0 and cell.max() < nx * ny * nz and ofs[-1] == d.n_pole
            am1 = np.asarray(d.am1, dtype=np.complex128)
            b = np.asarray(d.b, dtype=np.complex128)
            self.disp = {"p_re": torch.zeros(d.n_pole, dtype=torch.float32, device=self.dev),
                         "p_im": torch.zeros(d.n_pole, dtype=torch.float32, device=self.dev),
                         "am1_re": f32(am1.real), "am1_im": f32(am1.imag),
                         "b_re": f32(b.real), "b_im": f32(b.imag),
                         "cidx": i32(np.arange(d.n_pole)), "comp": i32(d.comp),
                         "cell": i32(cell), "ofs": i32(ofs), "n": np.int32(d.n_entry),
                         "dec": torch.ones(d.n_entry, dtype=torch.float32, device=self.dev)}
        self.dip = None
        dips = [p for p in sc.dipoles if not p.magnetic]
        if any(p.magnetic for p in sc.dipoles):
            raise NotImplementedError("magnetic dipoles are not driven here")
        if dips:
            nsteps1 = min(len(p.waveform.amp_half) for p in dips)
            if n_total > nsteps1 - 1:
                raise ValueError("the dipole table is shorter than the run")
            flat, comp, coef, src = [], [], [], []
            for s, p in enumerate(dips):
                for (i, j, k), cf in zip(np.asarray(p.indices), np.asarray(p.coef)):
                    assert 0 <= i < nx and 0 <= j < ny and 0 <= k < nz
                    flat.append((int(i) * ny + int(j)) * nz + int(k))
                    comp.append(int(p.component))
                    coef.append(float(cf))
                    src.append(s)
            amp = np.stack([np.asarray(p.waveform.amp_half, dtype=np.float64)[:nsteps1]
                            for p in dips])
            self.dip = {"flat": i32(flat), "comp": i32(comp), "coef": f32(coef),
                        "src": i32(src), "amp": torch.as_tensor(amp, device=self.dev),
                        "nsteps1": np.int32(nsteps1), "n": np.int32(len(flat))}
        self.step_dev = torch.zeros(1, dtype=torch.int32, device=self.dev)

    def load_fields(self, fields) -> None:
        for F, v in zip((*self.E, *self.H), fields):
            F.copy_(self.torch.as_tensor(np.asarray(v, dtype=np.float32), device=self.dev))

    def step(self) -> None:
        nx, ny, nz = (np.int32(v) for v in self.shape)
        s = self.torch.cuda.current_stream().cuda_stream
        g3, b3 = ((int(nz) + 31) // 32, (int(ny) + 3) // 4, int(nx)), (32, 4, 1)
        ph, pe = self.pml_h, self.pml_e
        # openem/kernels/yee.cu:76 update_h
        _launch("yee.cu", "update_h", g3, b3,
                (*self.H, *self.E, *self.psi_h, *self.on, *self.idl_p,
                 *ph[0], *ph[1], *ph[2], *self.nxt, *self.mnx, self.ch, nx, ny, nz), s)
        d = self.disp
        if d is not None:
            # openem/kernels/dispersion.cu:68 dispersion_pre
            _launch("dispersion.cu", "dispersion_pre", ((int(d["n"]) + 255) // 256, 1, 1),
                    (256, 1, 1),
                    (d["p_re"], d["p_im"], *self.hist, d["am1_re"], d["am1_im"], d["b_re"],
                     d["b_im"], d["cidx"], d["comp"], d["cell"], d["ofs"], *self.E, d["n"]), s)
        # openem/kernels/yee.cu:154 update_e (hist box: the whole grid)
        _launch("yee.cu", "update_e", g3, b3,
                (*self.E, *self.H, *self.psi_e, *self.on, *self.ca, *self.cb, *self.idl_d,
                 *pe[0], *pe[1], *pe[2], *self.prv, *self.mpv, *self.pec, *self.hist, self.cw,
                 np.int32(0), nx, np.int32(0), ny, np.int32(0), nz, nx, ny, nz), s)
        if self.dip is not None:
            p = self.dip
            # openem/kernels/source_dft.cu:147 inject_dipole
            _launch("source_dft.cu", "inject_dipole", ((int(p["n"]) + 127) // 128, 1, 1),
                    (128, 1, 1),
                    (*self.E, *self.cb, p["flat"], p["comp"], p["coef"], p["src"], p["amp"],
                     self.step_dev, p["nsteps1"], p["n"]), s)
        if d is not None:
            # openem/kernels/dispersion.cu:135 dispersion_post
            _launch("dispersion.cu", "dispersion_post", ((int(d["n"]) + 255) // 256, 1, 1),
                    (256, 1, 1),
                    (d["p_re"], d["p_im"], d["b_re"], d["b_im"], d["cidx"], d["comp"],
                     d["cell"], d["ofs"], *self.E, d["dec"], np.int32(0), d["n"]), s)
        # openem/kernels/source_dft.cu:434 step_advance
        _launch("source_dft.cu", "step_advance", (1, 1, 1), (1, 1, 1), (self.step_dev,), s)
        self.n += 1

    def run(self, steps: int) -> dict:
        for _ in range(int(steps)):
            self.step()
        self.torch.cuda.synchronize()
        names = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
        return {nm: F.cpu().numpy() for nm, F in zip(names, (*self.E, *self.H))}
