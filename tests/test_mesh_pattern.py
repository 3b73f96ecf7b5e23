"""Mesh generators against the reference meshes, and SELL-32 pattern invariants (CPU)."""
import hashlib
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from wspm_b200 import mesh
from wspm_b200.pattern import Pattern

GOLD = os.path.join(os.path.dirname(__file__), "golden")
DIGESTS = json.load(open(os.path.join(GOLD, "mesh_digests.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("n", [25, 50, 100, 200])
def test_structured_triangles_match_reference_files(n):
    p, t = mesh.structured_triangles(n, 15.24)
    assert sha(p) == DIGESTS[f"richards/p{n}"]["sha256"]
    assert sha(t) == DIGESTS[f"richards/t{n}"]["sha256"]


@pytest.mark.parametrize("n", [25, 50, 100])
def test_unit_square_matches_nitrogen_meshes(n):
    p, t = mesh.structured_triangles(n, 1.0)
    assert sha(p) == DIGESTS[f"nitrogen/p_{n}"]["sha256"]
    assert sha(t) == DIGESTS[f"nitrogen/t_{n}"]["sha256"]


def test_kuhn_tetrahedra_match_reference_file():
    p, t = mesh.kuhn_tetrahedra(20, 15.24)
    assert sha(p) == DIGESTS["richards/p_3D"]["sha256"]
    assert sha(t) == DIGESTS["richards/t_3D"]["sha256"]
    J = p[t[:, 1:]] - p[t[:, :1]]
    assert np.all(np.linalg.det(J) > 0)


def test_auto_layout_choice():
    p, t = mesh.structured_triangles(12)
    P = Pattern(t, len(p))
    assert P.layout == "dia" and P.n_diags == 7
    p, t = mesh.kuhn_tetrahedra(4)
    P = Pattern(t, len(p))
    assert P.layout == "dia" and P.n_diags == 15


@pytest.mark.parametrize("n", [1, 3, 8, 33])
def test_nnz_formula_2d(n):
    p, t = mesh.structured_triangles(n)
    P = Pattern(t, len(p))
    assert P.nnz == 7 * n * n + 6 * n + 1


@pytest.mark.parametrize("n", [1, 2, 5])
def test_nnz_formula_3d(n):
    p, t = mesh.kuhn_tetrahedra(n)
    P = Pattern(t, len(p))
    assert P.nnz == (n + 1) ** 3 + 2 * (3 * n * (n + 1) ** 2 + 3 * n * n * (n + 1) + n ** 3)


@pytest.mark.parametrize("kind,layout", [("tri", "sell"), ("tri", "dia"), ("tet", "sell"), ("tet", "dia"),
                                         ("ragged", "sell"), ("ragged", "auto")])
def test_pattern_roundtrip_and_incidence(kind, layout):
    rng = np.random.default_rng(0)
    if kind == "tri":
        p, t = mesh.structured_triangles(7)
    elif kind == "tet":
        p, t = mesh.kuhn_tetrahedra(3)
    else:  # unstructured: permuted nodes and elements (ragged slices)
        p, t = mesh.structured_triangles(9)
        perm = rng.permutation(len(p))
        inv = np.argsort(perm)
        p, t = p[perm], inv[t][rng.permutation(len(t))]
    P = Pattern(t, len(p), layout=layout)
    if kind == "ragged":
        assert P.layout == "sell"          # permuted numbering: offsets are not a small set
    nv = t.shape[1]
    rows = np.repeat(t, nv, axis=1).ravel()
    cols = np.tile(t, (1, nv)).ravel()
    ref = sp.coo_matrix((np.ones(rows.size), (rows, cols)), shape=(len(p), len(p))).tocsr()
    ref.sum_duplicates()
    ref.sort_indices()
    np.testing.assert_array_equal(P.csr_indptr, ref.indptr)
    np.testing.assert_array_equal(P.csr_indices, ref.indices)
    vals = rng.standard_normal(P.nnz)
    np.testing.assert_array_equal(P.csr_values_from_sell(P.sell_from_csr_values(vals)), vals)
    # every incidence decodes to the right columns, elements ascending per node
    for i in range(len(p)):
        s, lane = divmod(i, 32)
        prev = -1
        for k in range(P.inc_width[s]):
            o = P.inc_ptr[s] + 32 * k + lane
            e = P.inc_elem[o]
            if e < 0:
                break
            assert e > prev
            prev = e
            pk = int(P.inc_slots[o])
            assert t[e, pk & 3] == i
            for j in range(nv):
                kj = (pk >> (2 + 6 * j)) & 63
                assert P.cols[P.entry_pos(i, kj)] == t[e, j]
        assert P.cols[P.entry_pos(i, P.diag_pos[i])] == i


def test_loader_errors(tmp_path):
    pf, tf = tmp_path / "p.csv", tmp_path / "t.csv"
    with pytest.raises(FileNotFoundError):
        mesh.load_csv_mesh(str(pf), str(tf), 2)
    pf.write_text("0,0\n1,0\n0,1\n")
    tf.write_text("1,2,4\n")
    with pytest.raises(ValueError, match="out of bounds"):
        mesh.load_csv_mesh(str(pf), str(tf), 2)
    tf.write_text("1,2,3\n")
    pts, el = mesh.load_csv_mesh(str(pf), str(tf), 2)
    assert el.tolist() == [[0, 1, 2]]


ATTRS = ("csr_indptr", "csr_indices", "sell_index", "slice_ptr", "slice_width", "cols", "diag_pos", "diag_offsets",
         "inc_ptr", "inc_width", "inc_elem", "inc_slots")


def _shuffled_triangles(n, seed):
    """A structured grid with permuted node and element ids: an unstructured-looking mesh (SELL rows)."""
    pts, tri = mesh.structured_triangles(n, 1.0)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(len(pts))
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    return pts[perm], inv[tri][rng.permutation(len(tri))]


@pytest.mark.parametrize("case", ["tri-auto", "tri-sell", "tri-dia", "tet-auto", "tet-sell", "shuffled-auto",
                                  "extra-pairs"])
def test_native_pattern_builder_matches_numpy(case):
    """wspm_pattern_build (libwspm, C++) produces the NumPy builder's arrays element for element, dtypes included."""
    extra = None
    if case.startswith("tri"):
        pts, el = mesh.structured_triangles(13, 1.0)
    elif case.startswith("tet"):
        pts, el = mesh.kuhn_tetrahedra(5, 1.0)
    elif case.startswith("shuffled"):
        pts, el = _shuffled_triangles(11, 7)
    else:
        pts, el = mesh.structured_triangles(9, 1.0)
        extra = np.array([[0, 20], [5, 77]])
    layout = case.split("-")[1] if case.split("-")[1] in ("auto", "sell", "dia") else "auto"
    a = Pattern(el, len(pts), layout=layout, extra_pairs=extra, builder="native")
    b = Pattern(el, len(pts), layout=layout, extra_pairs=extra, builder="numpy")
    for k in ("layout", "n_rows", "nnz", "n_slices", "nnz_padded", "ld", "max_width", "max_inc", "n_diags"):
        assert getattr(a, k) == getattr(b, k), k
    for k in ATTRS:
        x, y = getattr(a, k), getattr(b, k)
        assert x.dtype == y.dtype and np.array_equal(x, y), k
    if case == "shuffled-auto":
        assert a.layout == "sell"
    rows = np.array([0, 3, len(pts) - 1])
    np.testing.assert_array_equal(a.slot(rows, rows), b.slot(rows, rows))


def test_native_pattern_builder_errors():
    pts, el = mesh.structured_triangles(4, 1.0)
    with pytest.raises(ValueError):
        Pattern(el, len(pts) + 1, builder="native")            # a node in no element
    bad = el.copy()
    bad[0, 0] = len(pts)
    with pytest.raises(ValueError):
        Pattern(bad, len(pts), builder="native")               # id out of range


@pytest.mark.parametrize("lower", [True, False])
def test_native_level_schedule_matches_row_loop(lower):
    """wspm_pattern_levels against the row-by-row definition (row i waits for every row it depends on)."""
    pts, el = _shuffled_triangles(9, 5)
    P = Pattern(el, len(pts))
    level_ptr, rows = P.tri_levels(lower)
    n, ptr, idx = P.n_rows, P.csr_indptr, P.csr_indices
    level = np.zeros(n, dtype=np.int64)
    for i in (range(n) if lower else range(n - 1, -1, -1)):
        c = idx[ptr[i]:ptr[i + 1]]
        dep = c[c < i] if lower else c[c > i]
        if dep.size:
            level[i] = level[dep].max() + 1
    np.testing.assert_array_equal(rows, np.argsort(level, kind="stable"))
    np.testing.assert_array_equal(np.diff(level_ptr), np.bincount(level))
