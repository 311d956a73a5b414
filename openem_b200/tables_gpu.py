"""Device-side construction of the two per-cell tables of a large grid -- the material index and
the ADE segment offsets -- with torch used only as an array library at setup time.

The arithmetic is :func:`openem_b200.tables.material_tables` (float64 coefficient math, exact
float32 bit-pattern keys), run on the GPU instead of numpy: on a 512^3 grid the host version
spends over a minute hashing 134M cells, the device version well under a second. The results
(material records and the index, cell for cell) are identical up to the numbering of the
materials, which is sorted here and first-seen on the host.

The index and the segment offsets stay in device memory and are handed to the plan by pointer
(``oem_plan_set_materials_device`` / ``oem_plan_set_pole_sets_device``).
"""

from __future__ import annotations

import threading

import numpy as np

from openem_b200 import tables as T


def available() -> bool:
    try:
        import torch
        return bool(torch.cuda.is_available())
    except Exception:
        return False


class DeviceTables:
    """Material records (host), index and segment offsets (device tensors)."""

    def __init__(self, table, index, n_mat, set_ofs, coef, seg_ofs, n_pole_total):
        self.table = table
        self.index = index          # torch int16 / int32, (nx, ny, nz), on the device
        self.n_mat = n_mat
        self.set_ofs = set_ofs
        self.coef = coef
        self.seg_ofs = seg_ofs      # torch int32 (uint32 bits), (n_seg,), on the device
        self.n_pole_total = n_pole_total
        self.h2d_bytes = 0          # eps and sigma bytes copied to the device

    @property
    def index_bytes(self) -> int:
        return int(self.index.element_size())


def _to_dev(a, torch, dev, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(dev, non_blocking=False)


class _PinnedStager:
    """Host-to-device copies of large arrays through two halves of one pinned buffer: host
    threads copy chunk q into one half (numpy copies release the GIL, so the threads run in
    parallel) while the DMA of chunk q - 1 drains the other, so the transfer runs near the link
    rate instead of through the driver's single-threaded pageable staging. One buffer per
    process, made on first use; copies from several threads (a server building plans on
    worker threads) take turns through a lock."""

    CHUNK = 64 << 20
    THREADS = 8
    _buf = None
    _pool = None
    _lock = threading.Lock()

    @classmethod
    def copy(cls, a: np.ndarray, torch, dev):
        a = np.ascontiguousarray(a)
        if a.nbytes < 2 * cls.CHUNK:
            return torch.from_numpy(a).to(dev)
        with cls._lock:
            return cls._copy(a, torch, dev)

    @classmethod
    def _copy(cls, a: np.ndarray, torch, dev):
        if cls._buf is None or cls._buf.numel() < 2 * cls.CHUNK:
            cls._buf = torch.empty(2 * cls.CHUNK, dtype=torch.uint8, pin_memory=True)
        if cls.THREADS > 1 and cls._pool is None:
            from concurrent.futures import ThreadPoolExecutor
            cls._pool = ThreadPoolExecutor(max_workers=cls.THREADS)
        dst = torch.empty(a.shape, dtype=torch.from_numpy(a[:0]).dtype, device=dev)
        src = a.reshape(-1).view(np.uint8)
        buf = cls._buf.numpy()
        out = dst.view(-1).view(torch.uint8)
        stream = torch.cuda.current_stream(dev)
        done = [None, None]
        for q, off in enumerate(range(0, a.nbytes, cls.CHUNK)):
            half = q % 2
            n = min(cls.CHUNK, a.nbytes - off)
            if done[half] is not None:
                done[half].synchronize()  # the DMA out of this half has finished
            base = half * cls.CHUNK
            if cls.THREADS > 1:
                per = -(-n // cls.THREADS)  # bytes per thread, rounded up to whole pages
                step = (per + 4095) // 4096 * 4096
                list(cls._pool.map(
                    lambda r: np.copyto(buf[base + r:base + min(r + step, n)],
                                        src[off + r:off + min(r + step, n)]),
                    range(0, n, step)))
            else:
                np.copyto(buf[base:base + n], src[off:off + n])
            out[off:off + n].copy_(cls._buf[base:base + n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
            done[half] = ev
        stream.synchronize()
        return dst


_SCAN = threading.local()


def _differing(v: np.ndarray, v0, lo: int, hi: int, piece: int = 1 << 20):
    """Indices in [lo, hi) where v differs from v0 (int32) and v's values there, scanned a piece
    at a time through one reused mask per thread (no fresh pages per piece); pieces with no
    differing cell, the bulk of a background, cost one comparison and one any(). The values are
    gathered from the piece just compared, on the scanning thread."""
    b = getattr(_SCAN, "mask", None)
    if b is None:
        b = _SCAN.mask = np.empty(piece, dtype=bool)
    idx, val = [], []
    for q in range(lo, hi, piece):
        m = min(piece, hi - q)
        np.not_equal(v[q:q + m], v0, out=b[:m])
        if b[:m].any():
            k = np.flatnonzero(b[:m])
            val.append(v[q:q + m][k])
            idx.append((k + q).astype(np.int32))
    if not idx:
        return np.zeros(0, np.int32), np.zeros(0, v.dtype)
    return np.concatenate(idx), np.concatenate(val)


def _upload_material(a: np.ndarray, torch, dev):
    """One float64 per-cell array on the device, and the bytes that crossed the link.

    A scene's eps and sigma are mostly one background value with objects in it: the most
    common value among 4096 cells spread over the array is taken as the background, and when at
    most an eighth of the cells differ from it (compared bit for bit, so NaN and signed zeros
    count as different), only those cells' indices (int32) and values cross the link and the
    array is filled on the device; otherwise the whole array is copied. The same sample decides
    which path is tried (more than a quarter of it off the background: the whole array), and a
    scan that finds too many differing cells copies the whole array after all."""
    a = np.ascontiguousarray(a, np.float64).reshape(-1)
    n = a.size
    if n < (1 << 22) or n >= (1 << 31):
        return _PinnedStager.copy(a, torch, dev), a.nbytes
    v = a.view(np.uint64)
    # the background: the most common value among 4096 cells spread over the array
    u, cnt_u = np.unique(v[::max(1, n // 4096)], return_counts=True)
    top = int(np.argmax(cnt_u))
    v0 = u[top]
    if 4 * (int(cnt_u.sum()) - int(cnt_u[top])) > int(cnt_u.sum()):
        return _PinnedStager.copy(a, torch, dev), a.nbytes
    # four slices per pool thread: a slice that finds objects takes longer than a background one
    parts = T.par_map(lambda lo, hi: _differing(v, v0, lo, hi), n, parts=64)
    cnt = sum(int(p[0].size) for p in parts)
    if cnt > n // 8:
        return _PinnedStager.copy(a, torch, dev), a.nbytes
    # filled with the background's bits (a NaN keeps its payload, -0.0 its sign)
    out = torch.full((n,), int(np.array([v0], np.uint64).view(np.int64)[0]), dtype=torch.int64,
                     device=dev)
    if cnt:
        idx = np.concatenate([p[0] for p in parts])
        val = np.concatenate([p[1] for p in parts]).view(np.int64)
        out[torch.from_numpy(idx).to(dev).long()] = torch.from_numpy(val).to(dev)
    return out.view(torch.float64), 12 * cnt


class _Uploads:
    """The float64 eps and sigma arrays of each component put on the device by a worker thread
    (`_upload_material`: sparse or whole) while the caller turns the previous component into
    coefficients and keys: all three components queued back to back when the six arrays take
    under a quarter of the free device memory, otherwise one component ahead of the caller (at
    most two resident). The uploads run one at a time, each with its own host threads, and are
    synchronous on the worker's stream; the caller's stream is recorded on each tensor before
    use; `h2d` counts the bytes that crossed the link."""

    def __init__(self, sc, torch, dev):
        from concurrent.futures import ThreadPoolExecutor
        self.torch, self.dev = torch, dev
        self.eps = (sc.eps_ex, sc.eps_ey, sc.eps_ez)
        self.sig = (sc.sigma_ex, sc.sigma_ey, sc.sigma_ez)
        nbytes = sum(np.asarray(a).size * 8 for a in (*self.eps, *self.sig) if a is not None)
        free, _ = torch.cuda.mem_get_info(dev)
        self.depth = 3 if nbytes < free // 4 else 1
        self.stream = torch.cuda.Stream(device=dev)
        self.h2d = 0  # bytes copied to the device
        self.pool = ThreadPoolExecutor(max_workers=1)
        self.futs = [self.pool.submit(self._load, c) for c in range(self.depth)]

    def _load(self, c):
        torch, dev = self.torch, self.dev
        torch.cuda.set_device(dev)
        with torch.cuda.stream(self.stream):
            eps, nb = _upload_material(self.eps[c], torch, dev)
            sig = None
            if self.sig[c] is not None:
                sig, nb2 = _upload_material(self.sig[c], torch, dev)
                nb += nb2
            self.stream.synchronize()
        self.h2d += nb
        return eps, sig

    def get(self, c):
        if c + self.depth < 3:
            self.futs.append(self.pool.submit(self._load, c + self.depth))
        eps, sig = self.futs[c].result()
        self.futs[c] = None
        cur = self.torch.cuda.current_stream(self.dev)
        for t in (eps, sig):
            if t is not None:
                t.record_stream(cur)
        return eps, sig

    def close(self):
        self.pool.shutdown(wait=True, cancel_futures=True)


def material_tables_device(sc, tabs, device: int = 0) -> DeviceTables:
    import torch
    dev = torch.device("cuda", device)
    up = _Uploads(sc, torch, dev)
    try:
        mt = _material_tables_device(sc, tabs, torch, dev, up)
    finally:
        up.close()
    mt.h2d_bytes = up.h2d
    return mt


def _check_entries_device(name, shape, comp, cell, ofs_list, torch, dev):
    """The checks of ``model.check_csr`` (ranges, monotone offsets, (comp, cell) uniqueness, the
    same messages) made on the device; returns the entries' components and cells there."""
    comp = np.asarray(comp)
    cell = np.asarray(cell)
    n = int(comp.size)
    ncell = int(np.prod(shape))
    if comp.shape != (n,) or cell.shape != (n,):
        raise ValueError(f"{name}: comp/cell lengths differ")
    comp_d = _to_dev(comp, torch, dev, torch.int64)
    cell_d = _to_dev(cell, torch, dev, torch.int64)
    if n == 0:
        return comp_d, cell_d
    lo_c, hi_c, lo_k, hi_k = (int(v) for v in torch.stack(
        [comp_d.min(), comp_d.max(), cell_d.min(), cell_d.max()]).cpu())
    if lo_c < 0 or hi_c > 2:
        raise ValueError(f"{name}: comp out of range {lo_c}..{hi_c}")
    if lo_k < 0 or hi_k >= ncell:
        raise ValueError(f"{name}: cell out of range {hi_k} >= {ncell}")
    for oname, ofs, npole in ofs_list:
        ofs = np.asarray(ofs)
        if ofs.shape != (n + 1,):
            raise ValueError(f"{name}.{oname} has shape {ofs.shape}, expected ({n + 1},)")
        if ofs[0] != 0 or ofs[-1] != npole:
            raise ValueError(f"{name}.{oname} endpoints {ofs[0]}..{ofs[-1]}, expected 0..{npole}")
        od = _to_dev(ofs, torch, dev, torch.int64)
        if bool((od[1:] < od[:-1]).any()):
            raise ValueError(f"{name}.{oname} is not monotonic")
    key = comp_d * ncell + cell_d
    if n >= 2 and not bool((key[1:] > key[:-1]).all()):  # unordered: count the distinct keys
        nu = int(torch.unique(key).numel())
        if nu != n:
            raise ValueError(f"{name}: {n - nu} duplicate (comp, cell) entries")
    return comp_d, cell_d


def _material_tables_device(sc, tabs, torch, dev, up) -> DeviceTables:
    shape = tuple(int(v) for v in sc.shape)
    nx, ny, nz = shape
    ncell = nx * ny * nz
    d = sc.dispersion
    disp = d is not None and d.n_entry > 0
    pole_fut = pole_pool = None
    if disp:
        # the entry table checked on the device before any device indexing with it; the host
        # deduplicates the pole sets on a worker thread meanwhile (they are needed only for the
        # second key of each component, after the coefficients of all three)
        d.validate_shapes()
        comp_d, cell_d = _check_entries_device("Dispersion", shape, d.comp, d.cell,
                                               [("pole_ofs", d.pole_ofs, d.n_pole)], torch, dev)
        from concurrent.futures import ThreadPoolExecutor
        pole_pool = ThreadPoolExecutor(max_workers=1)
        pole_fut = pole_pool.submit(T.entry_pole_sets, sc, True, False)
        g_d = _to_dev(np.asarray(d.g, np.float64), torch, dev)
        sel = [torch.nonzero(comp_d == c).squeeze(1) for c in range(3)]  # entries per component
    try:
        return _material_tables_from(sc, tabs, torch, dev, up, shape, disp,
                                     (comp_d, cell_d, g_d, sel) if disp else None, pole_fut)
    finally:
        if pole_pool is not None:
            pole_pool.shutdown(wait=True)


def _lex_codes_hashed(keys, torch, dev):
    """Material codes from one sort: a 64-bit mix of each cell's key tuple is made unique, the
    distinct tuples (one representative cell each) are put in lexicographic order on the host,
    and every cell is checked against its code's tuple. Returns (n_mat, code), the same codes as
    the exact ranking, or None after a hash collision (the caller then ranks exactly)."""
    h = torch.zeros_like(keys[0])
    for k in keys:  # int64 arithmetic wraps; any deterministic mix will do, the check is exact
        h = (h ^ k) * -7046029254386353131
        h = h ^ (h >> 29)
    uu, code = torch.unique(h, return_inverse=True)
    del h
    n = int(uu.numel())
    rep = torch.empty(n, dtype=torch.int64, device=dev)
    rep.scatter_(0, code, torch.arange(code.numel(), device=dev))
    tup = []
    for k in keys:
        kr = k[rep]
        if bool((k != kr[code]).any()):
            return None
        tup.append(kr.cpu().numpy())
    order = np.lexsort(tuple(tup[::-1]))  # the first key is the primary one
    rank = np.empty(n, dtype=np.int64)
    rank[order] = np.arange(n, dtype=np.int64)
    return n, torch.from_numpy(rank).to(dev)[code]


def _lex_codes_exact(keys, torch):
    """Material codes as the rank of each cell's six key ranks in lexicographic order: one
    unique of their mixed-radix number when it fits in 62 bits, else a running code (the inverse
    of the unique of (previous code, next key rank)) -- the same codes either way."""
    invs, card = [], []
    for k in keys:
        u, inv = torch.unique(k, return_inverse=True)
        invs.append(inv)
        card.append(int(u.numel()))
    if float(np.prod(np.asarray(card, dtype=np.float64))) < 2.0 ** 62:
        comb = invs[0]
        for inv, nk in zip(invs[1:], card[1:]):
            comb = comb * nk + inv
        uu, code = torch.unique(comb, return_inverse=True)
    else:
        code = None
        for inv, nk in zip(invs, card):
            comb = inv if code is None else code * nk + inv
            uu, code = torch.unique(comb, return_inverse=True)
    return int(uu.numel()), code


def _material_tables_from(sc, tabs, torch, dev, up, shape, disp, ent, pole_fut) -> DeviceTables:
    nx, ny, nz = shape
    ncell = nx * ny * nz
    pecs = (sc.pec_ex, sc.pec_ey, sc.pec_ez)
    dt = float(sc.dt)
    # each key's rank among its distinct values: the coefficient key of a component while the
    # next one uploads, the (eps, pole set) key once the pole sets are known
    key1, key2, ca_l, cb_l, eps_l, ps_l = [], [], [], [], [], []
    mask32 = 0xFFFFFFFF
    for c in range(3):
        eps, sg = up.get(c)
        s = torch.zeros_like(eps) if sg is None else sg * dt / (2.0 * T.EPSILON_0)
        del sg
        gg = torch.zeros_like(eps)
        if disp:
            _, cell_d, g_d, sel = ent
            gg[cell_d[sel[c]]] = g_d[sel[c]]
        den = eps + s + gg
        ca = ((eps - s) / den).to(torch.float32)
        cb = ((dt / T.EPSILON_0) / den).to(torch.float32)
        del s, gg, den
        if pecs[c] is not None and np.asarray(pecs[c]).size:
            idx = np.asarray(pecs[c], np.int64)
            if idx.min() < 0 or idx.max() >= ncell:
                raise ValueError(f"pec_e{'xyz'[c]} index out of range")
            idd = _to_dev(idx, torch, dev)
            ca[idd] = 0.0
            cb[idd] = 0.0
        ca3 = ca.view(shape)
        cb3 = cb.view(shape)
        for a in range(3):
            if a == c:
                continue
            zero = np.flatnonzero(tabs[a].pec == 0.0)
            if zero.size == 0:
                continue
            zd = _to_dev(zero, torch, dev)
            sl = [slice(None)] * 3
            sl[a] = zd
            ca3[tuple(sl)] = 0.0
            cb3[tuple(sl)] = 0.0
        for ten in T.passthrough_tables(sc):  # curl passthrough (tables.e_coefficients)
            sel = np.asarray(ten.cell, np.int64)[np.asarray(ten.comp) == c]
            if sel.size:
                td = _to_dev(sel, torch, dev)
                ca[td] = 0.0
                cb[td] = torch.where(cb[td] != 0.0, torch.ones_like(cb[td]),
                                     torch.zeros_like(cb[td]))
        ef = eps.to(torch.float32)
        del eps
        key1.append(((ca.view(torch.int32).to(torch.int64) & mask32) << 32)
                    | (cb.view(torch.int32).to(torch.int64) & mask32))
        ca_l.append(ca)
        cb_l.append(cb)
        eps_l.append(ef)
    ep = pole_fut.result() if disp else None
    if ep is not None:
        _, _, set_e, set_ofs, coef, counts = ep
        set_d = _to_dev(set_e, torch, dev)
    else:
        set_ofs, coef, counts = np.zeros(1, np.int32), np.zeros((0, 4), np.float32), np.zeros(0, np.int32)
    for c in range(3):
        ps = torch.full((ncell,), -1, dtype=torch.int64, device=dev)
        if ep is not None:
            _, cell_d, _, sel = ent
            ps[cell_d[sel[c]]] = set_d[sel[c]]
        key2.append(((eps_l[c].view(torch.int32).to(torch.int64) & mask32) << 32) | (ps + 1))
        ps_l.append(ps)
    # the keys in component order, coefficient key first: (x1, x2, y1, y2, z1, z2); the material
    # code of a cell is the rank of its key tuple in lexicographic order
    keys = [k for c in range(3) for k in (key1[c], key2[c])]
    del key1, key2
    found = _lex_codes_hashed(keys, torch, dev)
    if found is not None:
        n_mat, code = found
        del keys
    else:
        n_mat, code = _lex_codes_exact(keys, torch)
        del keys
    rep = torch.empty(n_mat, dtype=torch.int64, device=dev)
    rep.scatter_(0, code, torch.arange(ncell, device=dev))
    rec = np.zeros((n_mat, 16), dtype=np.uint32)
    npc_mat = torch.zeros(n_mat, dtype=torch.int64, device=dev)
    counts_d = torch.as_tensor(np.concatenate([counts, [0]]).astype(np.int64), device=dev)
    for c in range(3):
        rec[:, c] = ca_l[c][rep].cpu().numpy().view(np.uint32)
        rec[:, 3 + c] = cb_l[c][rep].cpu().numpy().view(np.uint32)
        rec[:, 6 + c] = eps_l[c][rep].cpu().numpy().view(np.uint32)
        ps = ps_l[c][rep]
        rec[:, 9 + c] = ps.to(torch.int32).cpu().numpy().view(np.uint32)
        npl = torch.where(ps >= 0, counts_d[ps.clamp(min=0)], torch.zeros_like(ps))
        rec[:, 12 + c] = npl.to(torch.int32).cpu().numpy().view(np.uint32)
        npc_mat += npl
    del ca_l, cb_l, eps_l, ps_l
    idx_dtype = torch.int16 if n_mat <= 32767 else torch.int32
    index = code.to(idx_dtype).view(shape).contiguous()
    nzp = T.pad_z(nz)
    npc = torch.zeros((nx, ny, nzp), dtype=torch.int64, device=dev)
    npc[:, :, :nz] = npc_mat[code].view(shape)
    seg = npc.view(-1, 32).sum(dim=1)
    del npc
    total = int(seg.sum().item())
    if total > 0xFFFFFFFF:
        raise ValueError("more than 2^32 ADE poles")
    seg_ofs = (torch.cumsum(seg, 0) - seg).to(torch.int64) & mask32
    seg_ofs = seg_ofs.to(torch.int32).contiguous()
    # the stream the tables were built on, not the whole device: other plans may be stepping
    torch.cuda.current_stream(dev).synchronize()
    return DeviceTables(table=rec, index=index, n_mat=n_mat, set_ofs=set_ofs,
                        coef=np.ascontiguousarray(coef), seg_ofs=seg_ofs, n_pole_total=total)


def isolate_cells_device(mt: DeviceTables, cells) -> None:
    """:func:`openem_b200.tables.isolate_cells` on a device index, in place."""
    import torch
    cells = np.unique(np.asarray(cells, np.int64))
    flat = mt.index.view(-1)
    cd = torch.as_tensor(cells, device=flat.device)
    old = flat[cd].to(torch.int64).cpu().numpy()
    n0 = int(mt.n_mat)
    table = np.concatenate([mt.table, mt.table[old]])
    n_mat = int(table.shape[0])
    index = mt.index if (n_mat <= 32767 or mt.index.dtype == torch.int32) \
        else mt.index.to(torch.int32)
    index.view(-1)[cd] = torch.arange(n0, n_mat, device=flat.device, dtype=torch.int64) \
        .to(index.dtype)
    torch.cuda.current_stream(flat.device).synchronize()
    mt.table, mt.index, mt.n_mat = table, index, n_mat
