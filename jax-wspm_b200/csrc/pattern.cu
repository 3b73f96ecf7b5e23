// Host-side builder of the sparsity pattern and node -> element incidence.
//
// The reference assembles every Picard iteration into a COO list of 9E
// (16E in 3D) entries and merges duplicates with BCOO.sum_duplicates
// (src/numerics/assembly_re_v2.py:114-152, assembly_re_3D.py:118-151); the
// pattern of which node pairs share an element never changes, so it is built
// here once per mesh and every assembly writes values into fixed slots.
//
// Output (all host arrays, owned by the returned handle):
//   * CSR of the unique (row, col) pairs, columns ascending per row;
//   * DIA (every row's column offsets in one set of at most 16) or SELL-32
//     storage: slice_ptr / slice_width / cols / diag_pos and the CSR entry ->
//     storage slot map sell_index;
//   * incidence: per node the elements that contain it, ascending element id,
//     in the same sliced layout; each slot packs the node's local vertex
//     (2 bits) and, per element vertex j, that vertex's position in the row
//     (6 bits).  Padding slots: element -1, word 0.
// The arrays are the ones the NumPy builder of the Python package produces,
// element for element (tests compare them).
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "wspm.h"

namespace {

constexpr int kSlice = 32;
constexpr int kDiaMax = 16;

template <typename T>
T *dup_array(const std::vector<T> &v) {
    T *p = static_cast<T *>(std::malloc(std::max<size_t>(1, v.size()) * sizeof(T)));
    if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

}  // namespace

extern "C" void wspm_pattern_free(wspm_pattern_host *p) {
    if (!p) return;
    void *arrays[] = {p->csr_indptr, p->csr_indices, p->sell_index, p->slice_ptr, p->slice_width, p->cols,
                      p->diag_pos,   p->diag_offsets, p->inc_ptr,   p->inc_width, p->inc_elem,    p->inc_slots};
    for (void *a : arrays) std::free(a);
    std::free(p);
}

extern "C" int wspm_pattern_build(const int64_t *elements, int64_t n_elems, int32_t nv, int32_t n_nodes,
                                  const int64_t *extra_pairs, int64_t n_extra, int32_t layout,
                                  wspm_pattern_host **out) {
    if (!out) return WSPM_BAD_ARG;
    *out = nullptr;
    if (!elements || n_elems <= 0 || nv < 2 || nv > 4 || n_nodes <= 0 || n_extra < 0 || (n_extra > 0 && !extra_pairs))
        return WSPM_BAD_ARG;
    if (layout < WSPM_LAYOUT_AUTO || layout > WSPM_LAYOUT_DIA) return WSPM_BAD_ARG;
    const int64_t N = n_nodes, E = n_elems;
    for (int64_t t = 0; t < E * nv; ++t)
        if (elements[t] < 0 || elements[t] >= N) return WSPM_BAD_ARG;
    for (int64_t t = 0; t < 2 * n_extra; ++t)
        if (extra_pairs[t] < 0 || extra_pairs[t] >= N) return WSPM_BAD_ARG;
    try {
        // ---- incidence lists: node -> (element, local vertex), elements ascending (counting sort)
        std::vector<int64_t> deg_ptr(N + 1, 0);
        for (int64_t t = 0; t < E * nv; ++t) ++deg_ptr[elements[t] + 1];
        for (int64_t i = 0; i < N; ++i) deg_ptr[i + 1] += deg_ptr[i];
        std::vector<int32_t> inc_e_flat(E * nv), inc_li_flat(E * nv);
        {
            std::vector<int64_t> fill(deg_ptr.begin(), deg_ptr.end() - 1);
            for (int64_t e = 0; e < E; ++e)
                for (int j = 0; j < nv; ++j) {
                    const int64_t node = elements[e * nv + j];
                    const int64_t q = fill[node]++;
                    inc_e_flat[q] = (int32_t)e;
                    inc_li_flat[q] = j;
                }
        }
        // extra pairs per row (both directions)
        std::vector<int64_t> ex_ptr(N + 1, 0);
        std::vector<int64_t> ex_col(2 * n_extra);
        for (int64_t t = 0; t < n_extra; ++t) {
            ++ex_ptr[extra_pairs[2 * t] + 1];
            ++ex_ptr[extra_pairs[2 * t + 1] + 1];
        }
        for (int64_t i = 0; i < N; ++i) ex_ptr[i + 1] += ex_ptr[i];
        {
            std::vector<int64_t> fill(ex_ptr.begin(), ex_ptr.end() - 1);
            for (int64_t t = 0; t < n_extra; ++t) {
                const int64_t a = extra_pairs[2 * t], b = extra_pairs[2 * t + 1];
                ex_col[fill[a]++] = b;
                ex_col[fill[b]++] = a;
            }
        }
        // ---- CSR: per row the sorted unique vertices of its elements and extra partners
        std::vector<int64_t> indptr(N + 1, 0);
        std::vector<int32_t> indices;
        indices.reserve((size_t)E * nv * 2 + 2 * n_extra);
        std::vector<int64_t> buf;
        for (int64_t i = 0; i < N; ++i) {
            buf.clear();
            for (int64_t q = deg_ptr[i]; q < deg_ptr[i + 1]; ++q) {
                const int64_t e = inc_e_flat[q];
                for (int j = 0; j < nv; ++j) buf.push_back(elements[e * nv + j]);
            }
            for (int64_t q = ex_ptr[i]; q < ex_ptr[i + 1]; ++q) buf.push_back(ex_col[q]);
            std::sort(buf.begin(), buf.end());
            buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
            if (buf.empty()) return WSPM_BAD_ARG;                 // a node that belongs to no element
            for (int64_t c : buf) indices.push_back((int32_t)c);
            indptr[i + 1] = (int64_t)indices.size();
        }
        const int64_t nnz = (int64_t)indices.size();
        // ---- distinct column offsets (DIA when at most kDiaMax, unless SELL is asked for)
        std::vector<int64_t> offs;
        bool many = false;
        for (int64_t i = 0; i < N && !many; ++i)
            for (int64_t q = indptr[i]; q < indptr[i + 1]; ++q) {
                const int64_t o = indices[q] - i;
                if (std::find(offs.begin(), offs.end(), o) == offs.end()) {
                    offs.push_back(o);
                    if ((int)offs.size() > 64) { many = true; break; }
                }
            }
        std::sort(offs.begin(), offs.end());
        const bool dia = layout == WSPM_LAYOUT_DIA || (layout == WSPM_LAYOUT_AUTO && !many && (int)offs.size() <= kDiaMax);
        if (dia && (many || offs.size() > 63)) return WSPM_UNSUPPORTED;   // too many diagonals for DIA
        const int64_t ns = (N + kSlice - 1) / kSlice;
        std::vector<int64_t> slice_ptr(ns + 1, 0), sell_index(nnz);
        std::vector<int32_t> slice_width(ns), diag_pos(N), cols, diag_offsets;
        int64_t nnz_padded = 0, ld = 0;
        int max_width = 0;
        auto offset_index = [&](int64_t o) { return (int)(std::lower_bound(offs.begin(), offs.end(), o) - offs.begin()); };
        if (dia) {
            const int nd = (int)offs.size();
            ld = ns * kSlice;
            for (int64_t s = 0; s <= ns; ++s) slice_ptr[s] = s * kSlice;
            std::fill(slice_width.begin(), slice_width.end(), nd);
            nnz_padded = nd * ld;
            max_width = nd;
            diag_offsets.assign(offs.begin(), offs.end());
            for (int64_t i = 0; i < N; ++i)
                for (int64_t q = indptr[i]; q < indptr[i + 1]; ++q)
                    sell_index[q] = (int64_t)offset_index(indices[q] - i) * ld + i;
            cols.resize(nnz_padded);
            for (int k = 0; k < nd; ++k)
                for (int64_t i = 0; i < ld; ++i) {
                    int64_t c = i + offs[k];
                    c = c < 0 ? 0 : (c > N - 1 ? N - 1 : c);
                    cols[k * ld + i] = (int32_t)c;
                }
            std::fill(diag_pos.begin(), diag_pos.end(), offset_index(0));
        } else {
            for (int64_t s = 0; s < ns; ++s) {
                int64_t w = 0;
                for (int64_t i = s * kSlice; i < std::min<int64_t>(N, (s + 1) * kSlice); ++i)
                    w = std::max(w, indptr[i + 1] - indptr[i]);
                if (w > 63) return WSPM_UNSUPPORTED;              // 6-bit row positions in the incidence word
                slice_width[s] = (int32_t)w;
                slice_ptr[s + 1] = slice_ptr[s] + w * kSlice;
                max_width = std::max<int>(max_width, (int)w);
            }
            nnz_padded = slice_ptr[ns];
            cols.resize(nnz_padded);
            for (int64_t s = 0; s < ns; ++s)                       // padding slots point at the own row
                for (int k = 0; k < slice_width[s]; ++k)
                    for (int l = 0; l < kSlice; ++l)
                        cols[slice_ptr[s] + (int64_t)kSlice * k + l] = (int32_t)std::min<int64_t>(s * kSlice + l, N - 1);
            for (int64_t i = 0; i < N; ++i) {
                for (int64_t q = indptr[i]; q < indptr[i + 1]; ++q) {
                    const int64_t pos = q - indptr[i];
                    const int64_t slot = slice_ptr[i / kSlice] + kSlice * pos + i % kSlice;
                    sell_index[q] = slot;
                    cols[slot] = indices[q];
                    if (indices[q] == i) diag_pos[i] = (int32_t)pos;
                }
            }
        }
        // ---- incidence in the sliced layout with packed row positions
        std::vector<int32_t> inc_width(ns);
        std::vector<int64_t> inc_ptr(ns + 1, 0);
        int max_inc = 0;
        for (int64_t s = 0; s < ns; ++s) {
            int64_t w = 0;
            for (int64_t i = s * kSlice; i < std::min<int64_t>(N, (s + 1) * kSlice); ++i)
                w = std::max(w, deg_ptr[i + 1] - deg_ptr[i]);
            inc_width[s] = (int32_t)w;
            inc_ptr[s + 1] = inc_ptr[s] + w * kSlice;
            max_inc = std::max<int>(max_inc, (int)w);
        }
        const int64_t n_inc = inc_ptr[ns];
        std::vector<int32_t> inc_elem(n_inc, -1);
        std::vector<uint32_t> inc_slots(n_inc, 0u);
        for (int64_t i = 0; i < N; ++i) {
            const int32_t *row_cols = indices.data() + indptr[i];
            const int64_t rl = indptr[i + 1] - indptr[i];
            for (int64_t q = deg_ptr[i]; q < deg_ptr[i + 1]; ++q) {
                const int64_t e = inc_e_flat[q];
                uint32_t packed = (uint32_t)inc_li_flat[q];
                for (int j = 0; j < nv; ++j) {
                    const int64_t c = elements[e * nv + j];
                    int kj;
                    if (dia) kj = offset_index(c - i);
                    else kj = (int)(std::lower_bound(row_cols, row_cols + rl, (int32_t)c) - row_cols);
                    packed |= ((uint32_t)kj & 63u) << (2 + 6 * j);
                }
                const int64_t slot = inc_ptr[i / kSlice] + kSlice * (q - deg_ptr[i]) + i % kSlice;
                inc_elem[slot] = (int32_t)e;
                inc_slots[slot] = packed;
            }
        }
        // ---- hand over
        wspm_pattern_host *p = static_cast<wspm_pattern_host *>(std::calloc(1, sizeof(wspm_pattern_host)));
        if (!p) return WSPM_BAD_ARG;
        p->n_rows = (int32_t)N;
        p->n_slices = (int32_t)ns;
        p->max_width = max_width;
        p->max_inc = max_inc;
        p->n_diags = dia ? (int32_t)offs.size() : 0;
        p->layout = dia ? WSPM_LAYOUT_DIA : WSPM_LAYOUT_SELL;
        p->nnz = nnz;
        p->nnz_padded = nnz_padded;
        p->n_inc = n_inc;
        p->ld = ld;
        p->csr_indptr = dup_array(indptr);
        p->csr_indices = dup_array(indices);
        p->sell_index = dup_array(sell_index);
        p->slice_ptr = dup_array(slice_ptr);
        p->slice_width = dup_array(slice_width);
        p->cols = dup_array(cols);
        p->diag_pos = dup_array(diag_pos);
        p->diag_offsets = dup_array(diag_offsets);
        p->inc_ptr = dup_array(inc_ptr);
        p->inc_width = dup_array(inc_width);
        p->inc_elem = dup_array(inc_elem);
        p->inc_slots = dup_array(inc_slots);
        if (!p->csr_indptr || !p->csr_indices || !p->sell_index || !p->slice_ptr || !p->slice_width || !p->cols ||
            !p->diag_pos || !p->diag_offsets || !p->inc_ptr || !p->inc_width || !p->inc_elem || !p->inc_slots) {
            wspm_pattern_free(p);
            return WSPM_BAD_ARG;
        }
        *out = p;
        return WSPM_OK;
    } catch (const std::bad_alloc &) {
        return WSPM_BAD_ARG;
    }
}

// Level schedule of a triangular sweep: level[i] = 1 + max level of the rows
// row i depends on (columns j < i for the lower sweep, j > i for the upper
// one), 0 without dependencies.  Rows of one level can be processed together.
extern "C" int wspm_pattern_levels(const int64_t *indptr, const int32_t *indices, int32_t n_rows, int32_t lower,
                                   int32_t *level, int32_t *n_levels) {
    if (!indptr || !indices || n_rows <= 0 || !level || !n_levels) return WSPM_BAD_ARG;
    int32_t top = -1;
    for (int32_t t = 0; t < n_rows; ++t) {
        const int32_t i = lower ? t : n_rows - 1 - t;
        int32_t lv = 0;
        for (int64_t q = indptr[i]; q < indptr[i + 1]; ++q) {
            const int32_t j = indices[q];
            if (j < 0 || j >= n_rows) return WSPM_BAD_ARG;
            if (lower ? j < i : j > i) lv = std::max(lv, level[j] + 1);
        }
        level[i] = lv;
        top = std::max(top, lv);
    }
    *n_levels = top + 1;
    return WSPM_OK;
}
