"""Sparsity pattern of the P1 global matrix in SELL-32 layout (host, NumPy).

Built once per mesh.  Replaces the reference's per-iteration COO fill +
``BCOO.sum_duplicates`` (src/numerics/assembly_re_v2.py:114-152): the
pattern (which node pairs share an element) never changes, so it is derived
once and every assembly writes values straight into fixed slots.

Layout (all int arrays little-endian, ready for device upload):
  rows are grouped in slices of 32; slice s has width w_s = max row length in
  the slice; entry k of row i is at slice_ptr[i//32] + 32*k + i%32.  Columns
  of a row are ascending; padding entries point at the row itself.
  The node -> element incidence uses the same sliced layout; each incidence
  packs the local vertex of the row's node (2 bits) and, for every vertex j
  of the element, the position of that vertex's column in the row (6 bits).

DIA variant (``layout="dia"``, chosen by ``"auto"`` when the matrix has at
most ``DIA_MAX`` distinct column offsets, i.e. on structured meshes): entry k
of row i is the k-th diagonal, stored at k*ld + i (ld = 32 * n_slices), with
column i + offsets[k]; rows hold zeros where a diagonal has no entry.  The
sparse kernels then read no column indices at all.
"""
import numpy as np

SLICE = 32
DIA_MAX = 16


class Pattern:
    """Host arrays of a SELL-32 (or DIA) pattern + node->element incidence."""

    def __init__(self, elements, n_nodes, layout="auto", extra_pairs=None, builder="native"):
        """``extra_pairs`` (k, 2): node pairs that must have matrix slots although no element
        contains both (boundary edges whose end points are not an element edge); both (i, j) and
        (j, i) are added.  ``builder``: "native" (``wspm_pattern_build`` in libwspm, host), "device" (the same
        arrays built on the GPU by ``wspm_pattern_device_count`` / ``_fill``; no ``extra_pairs``; the device
        arrays are kept in ``device_arrays`` for DeviceMesh) or "numpy" (the same arrays built with NumPy; kept as
        the restatement the native builders are tested against)."""
        if layout not in ("auto", "sell", "dia"):
            raise ValueError(f"unknown layout {layout!r}")
        if builder == "native":
            self._build_native(elements, n_nodes, layout, extra_pairs)
        elif builder == "device":
            if extra_pairs is not None and len(extra_pairs):
                raise ValueError("the device builder takes no extra pairs (use builder='native')")
            self._build_device(elements, n_nodes, layout)
        elif builder == "numpy":
            self._build_numpy(elements, n_nodes, layout, extra_pairs)
        else:
            raise ValueError(f"unknown builder {builder!r}")

    def _build_native(self, elements, n_nodes, layout, extra_pairs):
        import ctypes
        from . import _lib
        el = np.ascontiguousarray(elements, dtype=np.int64)
        if el.ndim != 2:
            raise ValueError("elements must be a 2D array")
        E, nv = el.shape
        N = int(n_nodes)
        ep = np.zeros((0, 2), dtype=np.int64)
        if extra_pairs is not None and len(extra_pairs):
            ep = np.ascontiguousarray(np.asarray(extra_pairs, dtype=np.int64).reshape(-1, 2))
        code = {"auto": 0, "sell": 1, "dia": 2}[layout]
        out = ctypes.POINTER(_lib.WspmPatternHost)()
        rc = _lib.lib.wspm_pattern_build(el.ctypes.data_as(ctypes.c_void_p), E, nv, N,
                                         ep.ctypes.data_as(ctypes.c_void_p) if len(ep) else None, len(ep), code,
                                         ctypes.byref(out))
        if rc == _lib.WSPM_UNSUPPORTED:
            raise ValueError("pattern not representable: more than 63 diagonals (DIA) or rows longer than 63 "
                             "(SELL-32)")
        if rc != _lib.WSPM_OK:
            raise ValueError("invalid mesh: element ids out of bounds or nodes that belong to no element")
        try:
            h = out.contents

            def arr(ptr, n):
                return np.ctypeslib.as_array(ptr, shape=(int(n),)).copy()
            self.n_rows, self.n_elems, self.nv = N, E, nv
            self.nnz, self.n_slices, self.nnz_padded = int(h.nnz), int(h.n_slices), int(h.nnz_padded)
            self.layout = "dia" if h.layout == 2 else "sell"
            self.ld = int(h.ld)
            self.max_width, self.max_inc, self.n_diags = int(h.max_width), int(h.max_inc), int(h.n_diags)
            ns = self.n_slices
            self.csr_indptr = arr(h.csr_indptr, N + 1)
            self.csr_indices = arr(h.csr_indices, self.nnz)
            self.sell_index = arr(h.sell_index, self.nnz)
            self.slice_ptr = arr(h.slice_ptr, ns + 1)
            self.slice_width = arr(h.slice_width, ns)
            self.cols = arr(h.cols, self.nnz_padded)
            self.diag_pos = arr(h.diag_pos, N)
            self.diag_offsets = arr(h.diag_offsets, self.n_diags) if self.n_diags else np.zeros(0, dtype=np.int32)
            self.inc_ptr = arr(h.inc_ptr, ns + 1)
            self.inc_width = arr(h.inc_width, ns)
            self.inc_elem = arr(h.inc_elem, h.n_inc)
            self.inc_slots = arr(h.inc_slots, h.n_inc)
        finally:
            _lib.lib.wspm_pattern_free(out)

    def _build_device(self, elements, n_nodes, layout, device=None):
        import ctypes
        import torch
        from . import _lib
        el = elements if isinstance(elements, torch.Tensor) else torch.as_tensor(np.asarray(elements))
        dev = torch.device(device or (el.device if el.is_cuda else "cuda"))
        conn = el.to(device=dev, dtype=torch.int32).contiguous()
        if conn.ndim != 2:
            raise ValueError("elements must be a 2D array")
        E, nv = conn.shape
        N = int(n_nodes)
        lib = _lib.lib
        nbytes = int(lib.wspm_pattern_device_scratch_bytes(E, nv, N))
        if nbytes <= 0:
            raise ValueError("invalid mesh sizes")
        scratch = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        sz = _lib.WspmPatternSizes()
        st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        code = {"auto": 0, "sell": 1, "dia": 2}[layout]
        rc = lib.wspm_pattern_device_count(conn.data_ptr(), E, nv, N, code, scratch.data_ptr(), nbytes,
                                           ctypes.byref(sz), st)
        if rc == _lib.WSPM_UNSUPPORTED:
            raise ValueError("pattern not representable (too many diagonals for DIA, rows longer than 63, or rows "
                             "that gather more than 128 element vertices: use builder='native')")
        if rc != _lib.WSPM_OK:
            raise ValueError("invalid mesh: element ids out of bounds or nodes that belong to no element")
        ns = int(sz.n_slices)
        i64 = dict(dtype=torch.int64, device=dev)
        i32 = dict(dtype=torch.int32, device=dev)
        d = {"csr_indptr": torch.empty(N + 1, **i64), "csr_indices": torch.empty(int(sz.nnz), **i32),
             "sell_index": torch.empty(int(sz.nnz), **i64), "slice_ptr": torch.empty(ns + 1, **i64),
             "slice_width": torch.empty(ns, **i32), "cols": torch.empty(int(sz.nnz_padded), **i32),
             "diag_pos": torch.empty(N, **i32), "diag_offsets": torch.zeros(max(1, int(sz.n_diags)), **i32),
             "inc_ptr": torch.empty(ns + 1, **i64), "inc_width": torch.empty(ns, **i32),
             "inc_elem": torch.empty(int(sz.n_inc), **i32), "inc_slots": torch.empty(int(sz.n_inc), **i32)}
        order = ("csr_indptr", "csr_indices", "sell_index", "slice_ptr", "slice_width", "cols", "diag_pos",
                 "diag_offsets", "inc_ptr", "inc_width", "inc_elem", "inc_slots")
        rc = lib.wspm_pattern_device_fill(conn.data_ptr(), E, nv, N, ctypes.byref(sz), scratch.data_ptr(), nbytes,
                                          *[d[k].data_ptr() for k in order], st)
        _lib.check("pattern_device_fill", rc)
        self.n_rows, self.n_elems, self.nv = N, E, nv
        self.nnz, self.n_slices, self.nnz_padded = int(sz.nnz), ns, int(sz.nnz_padded)
        self.layout = "dia" if sz.layout == 2 else "sell"
        self.ld = int(sz.ld)
        self.max_width, self.max_inc, self.n_diags = int(sz.max_width), int(sz.max_inc), int(sz.n_diags)
        host = {k: v.cpu().numpy() for k, v in d.items()}
        for k in order:
            setattr(self, k, host[k])
        self.inc_slots = host["inc_slots"].view(np.uint32)
        if not self.n_diags:
            self.diag_offsets = np.zeros(0, dtype=np.int32)
        self.device_arrays = d

    def _slot(self, rows, cols_):
        if self.layout == "dia":
            return np.searchsorted(self.diag_offsets.astype(np.int64), cols_ - rows)
        keys = self.__dict__.get("_keys")
        if keys is None:
            counts = np.diff(self.csr_indptr)
            keys = np.repeat(np.arange(self.n_rows, dtype=np.int64), counts) * self.n_rows + self.csr_indices
            self._keys = keys
        return np.searchsorted(keys, rows * self.n_rows + cols_) - self.csr_indptr[rows]

    def _build_numpy(self, elements, n_nodes, layout, extra_pairs):
        el = np.ascontiguousarray(elements, dtype=np.int64)
        E, nv = el.shape
        N = int(n_nodes)
        self.n_rows, self.n_elems, self.nv = N, E, nv
        # --- unique (row, col) pairs, ascending
        rows = np.repeat(el, nv, axis=1).ravel()
        cols = np.tile(el, (1, nv)).ravel()
        if extra_pairs is not None and len(extra_pairs):
            ep = np.asarray(extra_pairs, dtype=np.int64).reshape(-1, 2)
            rows = np.concatenate([rows, ep[:, 0], ep[:, 1]])
            cols = np.concatenate([cols, ep[:, 1], ep[:, 0]])
        keys = np.unique(rows * N + cols)
        r = keys // N
        c = keys - r * N
        counts = np.bincount(r, minlength=N)
        if np.any(counts == 0):
            raise ValueError("mesh has nodes that belong to no element")
        rowptr = np.zeros(N + 1, dtype=np.int64)
        np.cumsum(counts, out=rowptr[1:])
        self.csr_indptr, self.csr_indices = rowptr, c.astype(np.int32)
        self.nnz = int(keys.size)
        pos = np.arange(keys.size, dtype=np.int64) - rowptr[r]
        ns = (N + SLICE - 1) // SLICE
        self.n_slices = ns
        offs = np.unique(c - r)
        self.layout = "dia" if (layout == "dia" or (layout == "auto" and offs.size <= DIA_MAX)) else "sell"
        if self.layout == "dia":
            if offs.size > 63:
                raise ValueError("too many diagonals for the DIA layout")
            nd = int(offs.size)
            ld = ns * SLICE
            self.ld = ld
            self.diag_offsets = offs.astype(np.int32)
            self.slice_width = np.full(ns, nd, dtype=np.int32)
            self.slice_ptr = (np.arange(ns + 1, dtype=np.int64) * SLICE)
            self.nnz_padded = nd * ld
            self.max_width = nd
            kpos = np.searchsorted(offs, c - r)
            self.sell_index = kpos * ld + r
            all_i = np.arange(ld, dtype=np.int64)
            self.cols = np.clip(all_i[None, :] + offs[:, None], 0, N - 1).astype(np.int32).ravel()
            self.diag_pos = np.full(N, int(np.searchsorted(offs, 0)), dtype=np.int32)
        else:
            self.ld = 0
            self.diag_offsets = np.zeros(0, dtype=np.int32)
            pad_counts = np.zeros(ns * SLICE, dtype=np.int64)
            pad_counts[:N] = counts
            width = pad_counts.reshape(ns, SLICE).max(axis=1)
            if width.max() > 63:
                raise ValueError("row length above 63 is not supported by the SELL-32 kernels")
            self.slice_width = width.astype(np.int32)
            self.slice_ptr = np.zeros(ns + 1, dtype=np.int64)
            np.cumsum(width * SLICE, out=self.slice_ptr[1:])
            self.nnz_padded = int(self.slice_ptr[-1])
            self.max_width = int(width.max())
            lane = r % SLICE
            self.sell_index = self.slice_ptr[r // SLICE] + SLICE * pos + lane      # CSR entry -> SELL slot
            sell_cols = np.empty(self.nnz_padded, dtype=np.int32)
            all_rows = np.arange(ns * SLICE, dtype=np.int64)
            for_pad = np.minimum(all_rows, N - 1)                                   # padding: own row
            slot_row = np.repeat(for_pad.reshape(ns, SLICE), width, axis=0)
            sell_cols[:] = slot_row.ravel().astype(np.int32)
            sell_cols[self.sell_index] = c.astype(np.int32)
            self.cols = sell_cols
            self.diag_pos = np.empty(N, dtype=np.int32)
            dmask = r == c
            self.diag_pos[r[dmask]] = pos[dmask].astype(np.int32)
        self.n_diags = int(self.diag_offsets.size)
        # --- incidence: for each (node, element) in ascending element order
        inc_node = el.ravel()
        inc_elem = np.repeat(np.arange(E, dtype=np.int64), nv)
        inc_li = np.tile(np.arange(nv, dtype=np.int64), E)
        order = np.lexsort((inc_elem, inc_node))
        inc_node, inc_elem, inc_li = inc_node[order], inc_elem[order], inc_li[order]
        deg = np.bincount(inc_node, minlength=N)
        dptr = np.zeros(N + 1, dtype=np.int64)
        np.cumsum(deg, out=dptr[1:])
        ipos = np.arange(inc_node.size, dtype=np.int64) - dptr[inc_node]
        pad_deg = np.zeros(ns * SLICE, dtype=np.int64)
        pad_deg[:N] = deg
        iwidth = pad_deg.reshape(ns, SLICE).max(axis=1)
        self.inc_width = iwidth.astype(np.int32)
        self.inc_ptr = np.zeros(ns + 1, dtype=np.int64)
        np.cumsum(iwidth * SLICE, out=self.inc_ptr[1:])
        self.max_inc = int(iwidth.max())
        islot = self.inc_ptr[inc_node // SLICE] + SLICE * ipos + inc_node % SLICE
        inc_e = np.full(int(self.inc_ptr[-1]), -1, dtype=np.int32)
        inc_e[islot] = inc_elem.astype(np.int32)
        packed = inc_li.astype(np.uint32)
        node_rows = inc_node
        for j in range(nv):
            colj = el[inc_elem, j]
            kj = self._slot(node_rows, colj)
            packed |= (kj.astype(np.uint32) & 63) << np.uint32(2 + 6 * j)
        inc_s = np.zeros(int(self.inc_ptr[-1]), dtype=np.uint32)
        inc_s[islot] = packed
        self.inc_elem, self.inc_slots = inc_e, inc_s

    def tri_levels(self, lower=True):
        """Level schedule of a triangular sweep over this pattern: (level_ptr, rows), rows grouped so that row i
        only depends on rows of earlier levels (lower: columns j < i, swept upwards; upper: j > i, downwards)."""
        cache = self.__dict__.setdefault("_levels", {})
        if lower in cache:
            return cache[lower]
        import ctypes
        from . import _lib
        n = self.n_rows
        ptr = np.ascontiguousarray(self.csr_indptr, dtype=np.int64)
        idx = np.ascontiguousarray(self.csr_indices, dtype=np.int32)
        lv = np.empty(n, dtype=np.int32)
        nl = ctypes.c_int32(0)
        _lib.check("pattern_levels", _lib.lib.wspm_pattern_levels(
            ptr.ctypes.data_as(ctypes.c_void_p), idx.ctypes.data_as(ctypes.c_void_p), n, int(bool(lower)),
            lv.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nl)))
        level = lv.astype(np.int64)
        rows = np.argsort(level, kind="stable").astype(np.int32)
        counts = np.bincount(level, minlength=int(level.max()) + 1 if n else 0)
        level_ptr = np.zeros(counts.size + 1, dtype=np.int32)
        np.cumsum(counts, out=level_ptr[1:])
        cache[lower] = (level_ptr, rows)
        return cache[lower]

    def slot(self, i, j):
        """Row position k of column j in row i (i, j arrays)."""
        return np.asarray(self._slot(np.asarray(i, dtype=np.int64), np.asarray(j, dtype=np.int64)))

    def entry_pos(self, i, k):
        """Storage index of entry k of row i."""
        if self.layout == "dia":
            return k * self.ld + i
        return self.slice_ptr[i // SLICE] + SLICE * k + i % SLICE

    # ---- conversions used by tests and by the reference-API shims ----------
    def sell_from_csr_values(self, data):
        out = np.zeros(self.nnz_padded, dtype=np.asarray(data).dtype)
        out[self.sell_index] = data
        return out

    def csr_values_from_sell(self, vals):
        return np.asarray(vals)[self.sell_index]

    def to_scipy(self, vals):
        import scipy.sparse as sp
        return sp.csr_matrix((self.csr_values_from_sell(vals), self.csr_indices, self.csr_indptr),
                             shape=(self.n_rows, self.n_rows))
