// Device-side builder of the sparsity pattern and node -> element incidence
// (wspm_pattern_device_*, declared in include/wspm.h).
//
// The same arrays as the host builder (pattern.cu), element for element, from
// the element connectivity already on the device: the reference rebuilds its
// COO pattern and sorts it (BCOO.sum_duplicates) at every assembly
// (src/numerics/assembly_re_v2.py:114-152); the host builder does it once per
// mesh in O(E nv^2 log) on one core, which dominates the start-up of large
// ensembles.  Here every node is one thread:
//   count:  degree histogram -> exclusive scan -> incidence lists (atomic
//           cursors, then each node's list sorted by element id) -> each row's
//           sorted unique columns (length, DIA offset set) -> scans of row
//           lengths, slice widths and incidence widths; the host reads the sizes;
//   fill:   CSR, storage layout (DIA or SELL-32), diagonal positions and the
//           packed incidence words, written into the caller's arrays.
// The library allocates nothing: the caller sizes a scratch buffer with
// wspm_pattern_device_scratch_bytes and the outputs from the counts.
#include <algorithm>
#include <cstring>
#include <vector>
#include "common.cuh"

namespace wspm {
namespace {

constexpr int kPS = 32;              // slice height
constexpr int kDiaCap = 16;          // DIA when at most this many offsets
constexpr int kSetCap = 64;          // offsets tracked before giving up on DIA
constexpr int kRowCap = 128;         // max (element vertices) gathered per row
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;        // items per thread in a scan block
constexpr int64_t kScanBlockItems = (int64_t)kScanThreads * kScanItems;

// ---- exclusive scan of int64 (two levels: block sums scanned by one block) ----
__global__ void __launch_bounds__(kScanThreads) scan_blocks_kernel(const int64_t *__restrict__ in, int64_t n,
                                                                  int64_t *out, int64_t *block_sums) {
    __shared__ int64_t s[kScanThreads];
    const int64_t base = blockIdx.x * kScanBlockItems + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems], t = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        v[q] = base + q < n ? in[base + q] : 0;
        t += v[q];
    }
    s[threadIdx.x] = t;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {       // inclusive Hillis-Steele over thread totals
        const int64_t a = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += a;
        __syncthreads();
    }
    int64_t run = s[threadIdx.x] - t;                          // exclusive prefix of this thread
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        if (base + q < n) out[base + q] = run;
        run += v[q];
    }
    if (threadIdx.x == kScanThreads - 1) block_sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(int64_t *block_sums, int nb, int64_t *total) {
    __shared__ int64_t s[kScanThreads];
    const int64_t v = threadIdx.x < nb ? block_sums[threadIdx.x] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {
        const int64_t a = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += a;
        __syncthreads();
    }
    if (threadIdx.x < nb) block_sums[threadIdx.x] = s[threadIdx.x] - v;
    if (threadIdx.x == kScanThreads - 1) *total = s[threadIdx.x];
}

__global__ void scan_add_kernel(int64_t *out, int64_t n, const int64_t *block_sums) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] += block_sums[i / kScanBlockItems];
}

// out[0..n) = exclusive scan of in[0..n), out[n] = total (n <= kScanThreads * kScanBlockItems)
void scan_i64(const int64_t *in, int64_t n, int64_t *out, int64_t *block_sums, cudaStream_t st) {
    const int nb = (int)((n + kScanBlockItems - 1) / kScanBlockItems);
    scan_blocks_kernel<<<nb > 0 ? nb : 1, kScanThreads, 0, st>>>(in, n, out, block_sums);
    scan_sums_kernel<<<1, kScanThreads, 0, st>>>(block_sums, nb, out + n);
    if (n > 0) scan_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, block_sums);
}

// ---- incidence ------------------------------------------------------------------
__global__ void degree_kernel(const int32_t *__restrict__ conn, int64_t n_entries, int n_nodes, int64_t *deg,
                              int *bad) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_entries;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int v = conn[t];
        if (v < 0 || v >= n_nodes) { atomicOr(bad, 1); continue; }
        atomicAdd(reinterpret_cast<unsigned long long *>(deg + v), 1ull);
    }
}

// incidence entries (element, local vertex) packed as e * 4 + j, in any order
__global__ void incidence_fill_kernel(const int32_t *__restrict__ conn, int64_t n_entries, int nv,
                                      const int64_t *__restrict__ deg_ptr, int32_t *cursor, int64_t *inc) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_entries;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int v = conn[t];
        const int64_t e = t / nv;
        const int j = (int)(t - e * nv);
        const int q = atomicAdd(cursor + v, 1);
        inc[deg_ptr[v] + q] = e * 4 + j;
    }
}

// each node's list sorted by element id (the host builder's counting sort order)
__global__ void incidence_sort_kernel(int n_nodes, const int64_t *__restrict__ deg_ptr, int64_t *inc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    int64_t *a = inc + deg_ptr[i];
    const int m = (int)(deg_ptr[i + 1] - deg_ptr[i]);
    for (int x = 1; x < m; ++x) {
        const int64_t key = a[x];
        int y = x - 1;
        while (y >= 0 && a[y] > key) { a[y + 1] = a[y]; --y; }
        a[y + 1] = key;
    }
}

// row i's sorted unique columns into buf; returns the count (-1: more than kRowCap vertices)
__device__ int row_columns(int i, const int32_t *__restrict__ conn, int nv, const int64_t *__restrict__ deg_ptr,
                           const int64_t *__restrict__ inc, int (&buf)[kRowCap]) {
    int m = 0;
    for (int64_t q = deg_ptr[i]; q < deg_ptr[i + 1]; ++q) {
        const int64_t e = inc[q] >> 2;
        for (int j = 0; j < nv; ++j) {
            if (m >= kRowCap) return -1;
            const int c = conn[e * nv + j];
            int y = m - 1;                                 // insertion into the sorted prefix, duplicates dropped
            while (y >= 0 && buf[y] > c) --y;
            if (y >= 0 && buf[y] == c) continue;
            for (int z = m - 1; z > y; --z) buf[z + 1] = buf[z];
            buf[y + 1] = c;
            ++m;
        }
    }
    return m;
}

// Insert offset o into the device set (kSetCap slots of int64, empty = INT64_MIN); overflow sets *many.
__device__ void offset_insert(unsigned long long *set, int *count, int *many, long long o) {
    const unsigned long long key = (unsigned long long)o;
    const unsigned long long empty = 0x8000000000000000ull;
    unsigned h = (unsigned)(((unsigned long long)o * 0x9E3779B97F4A7C15ull) >> 58);   // 6 bits: 0..63
    for (int probe = 0; probe < kSetCap; ++probe) {
        const unsigned slot = (h + probe) & (kSetCap - 1);
        const unsigned long long prev = atomicCAS(set + slot, empty, key);
        if (prev == empty) {
            if (atomicAdd(count, 1) + 1 > kSetCap - 1) atomicOr(many, 1);
            return;
        }
        if (prev == key) return;
    }
    atomicOr(many, 1);
}

__global__ void row_count_kernel(int n_nodes, const int32_t *__restrict__ conn, int nv,
                                 const int64_t *__restrict__ deg_ptr, const int64_t *__restrict__ inc,
                                 int64_t *row_len, unsigned long long *set, int *set_count, int *many, int *bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    int buf[kRowCap];
    const int m = row_columns(i, conn, nv, deg_ptr, inc, buf);
    if (m <= 0) { atomicOr(bad, m < 0 ? 2 : 1); row_len[i] = 0; return; }   // 1: node in no element
    row_len[i] = m;
    if (*(volatile int *)many) return;
    for (int q = 0; q < m; ++q) offset_insert(set, set_count, many, (long long)buf[q] - i);
}

// per slice: max over its rows of len[] (row lengths or incidence degrees)
__global__ void slice_max_kernel(int n_nodes, int ns, const int64_t *__restrict__ ptr, int64_t *width) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    int64_t w = 0;
    for (int i = s * kPS; i < min(n_nodes, (s + 1) * kPS); ++i) w = max(w, ptr[i + 1] - ptr[i]);
    width[s] = w;
}

__global__ void times_slice_kernel(int ns, const int64_t *__restrict__ w, int64_t *out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < ns) out[s] = w[s] * kPS;
}

__global__ void max_kernel(int n, const int64_t *__restrict__ v, unsigned long long *out) {
    unsigned long long m = 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        m = max(m, (unsigned long long)v[s]);
    atomicMax(out, m);
}

// ---- fill ------------------------------------------------------------------------
struct FillArgs {
    int n_nodes, nv, ns, dia, nd;
    int64_t ld;
    const int32_t *conn;
    const int64_t *deg_ptr, *inc, *indptr, *slice_ptr, *inc_ptr;
    const int32_t *offs;               // [nd] sorted (DIA)
    int32_t *indices, *cols, *diag_pos, *inc_elem;
    int64_t *sell_index;
    uint32_t *inc_slots;
};

__device__ __forceinline__ int offset_index(const FillArgs &a, int o) {
    int k = 0;
    while (k < a.nd && a.offs[k] < o) ++k;
    return k;
}

__global__ void rows_fill_kernel(FillArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_nodes) return;
    int buf[kRowCap];
    const int m = row_columns(i, a.conn, a.nv, a.deg_ptr, a.inc, buf);
    const int64_t p0 = a.indptr[i];
    for (int q = 0; q < m; ++q) {
        a.indices[p0 + q] = buf[q];
        int64_t slot;
        if (a.dia) {
            slot = (int64_t)offset_index(a, buf[q] - i) * a.ld + i;
        } else {
            slot = a.slice_ptr[i / kPS] + (int64_t)kPS * q + i % kPS;
            a.cols[slot] = buf[q];
            if (buf[q] == i) a.diag_pos[i] = q;
        }
        a.sell_index[p0 + q] = slot;
    }
    if (a.dia) a.diag_pos[i] = offset_index(a, 0);
    // incidence: the node's elements in ascending id, packed row positions of every vertex
    const int64_t ib = a.inc_ptr[i / kPS] + i % kPS;
    int r = 0;
    for (int64_t q = a.deg_ptr[i]; q < a.deg_ptr[i + 1]; ++q, ++r) {
        const int64_t ent = a.inc[q];
        const int64_t e = ent >> 2;
        uint32_t packed = (uint32_t)(ent & 3);
        for (int j = 0; j < a.nv; ++j) {
            const int c = a.conn[e * a.nv + j];
            int kj;
            if (a.dia) {
                kj = offset_index(a, c - i);
            } else {
                int lo = 0, hi = m;                        // lower_bound in the sorted row
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (buf[mid] < c) lo = mid + 1; else hi = mid;
                }
                kj = lo;
            }
            packed |= ((uint32_t)kj & 63u) << (2 + 6 * j);
        }
        a.inc_elem[ib + (int64_t)kPS * r] = (int32_t)e;
        a.inc_slots[ib + (int64_t)kPS * r] = packed;
    }
}

// SELL padding: every slot of a slice points at the slot's own row (rows_fill overwrites the real entries)
__global__ void sell_pad_kernel(int n_nodes, int ns, const int64_t *__restrict__ slice_ptr, int32_t *cols) {
    const int s = blockIdx.x;
    if (s >= ns) return;
    const int64_t b = slice_ptr[s], e = slice_ptr[s + 1];
    for (int64_t t = b + threadIdx.x; t < e; t += blockDim.x) {
        const int lane = (int)((t - b) % kPS);
        cols[t] = min(s * kPS + lane, n_nodes - 1);
    }
}

__global__ void dia_cols_kernel(int n_nodes, int nd, int64_t ld, const int32_t *__restrict__ offs, int32_t *cols) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nd * ld) return;
    const int k = (int)(t / ld);
    const int64_t i = t - k * ld;
    int64_t c = i + offs[k];
    c = c < 0 ? 0 : (c > n_nodes - 1 ? n_nodes - 1 : c);
    cols[t] = (int32_t)c;
}

__global__ void fill_i32_kernel(int32_t *p, int64_t n, int32_t v) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        p[t] = v;
}

__global__ void widths_i32_kernel(int ns, const int64_t *__restrict__ w, int32_t *out, int dia, int nd) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < ns) out[s] = dia ? nd : (int32_t)w[s];
}

// ---- scratch layout (in int64 words) ----------------------------------------------
struct Scratch {
    int64_t *deg, *deg_ptr, *inc, *row_len, *row_ptr, *sw, *sw_ptr, *iw, *iw_ptr, *bsum, *totals;
    unsigned long long *set, *maxes;
    int32_t *cursor;
    int *flags;          // [0] bad, [1] many, [2] set count
};

int64_t scratch_words(int64_t E, int nv, int64_t N) {
    const int64_t ns = (N + kPS - 1) / kPS;
    return (N + 1) * 2 + E * nv + (N + 1) * 2 + (ns + 1) * 4 + kScanThreads + 8 + kSetCap + 8 + (N + 1) / 2 + 1 + 8 +
           16 * 8;
}

Scratch carve(void *base, int64_t E, int nv, int64_t N) {
    const int64_t ns = (N + kPS - 1) / kPS;
    int64_t *p = reinterpret_cast<int64_t *>(base);
    Scratch s;
    s.deg = p; p += N + 1;
    s.deg_ptr = p; p += N + 1;
    s.inc = p; p += E * nv;
    s.row_len = p; p += N + 1;
    s.row_ptr = p; p += N + 1;
    s.sw = p; p += ns + 1;
    s.sw_ptr = p; p += ns + 1;
    s.iw = p; p += ns + 1;
    s.iw_ptr = p; p += ns + 1;
    s.bsum = p; p += kScanThreads;
    s.totals = p; p += 8;
    s.set = reinterpret_cast<unsigned long long *>(p); p += kSetCap;
    s.maxes = reinterpret_cast<unsigned long long *>(p); p += 8;
    s.cursor = reinterpret_cast<int32_t *>(p); p += (N + 1) / 2 + 1;
    s.flags = reinterpret_cast<int *>(p); p += 8;
    return s;
}

}  // namespace
}  // namespace wspm

namespace wspm {
namespace {
__global__ void set_init_kernel(unsigned long long *set, int n) {
    for (int t = threadIdx.x; t < n; t += blockDim.x) set[t] = 0x8000000000000000ull;
}
__global__ void slice_ptr_dia_kernel(int ns, int64_t *slice_ptr) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s <= ns) slice_ptr[s] = (int64_t)s * kPS;
}
inline unsigned grid_for(int64_t n, int tb = 256) {
    int64_t b = (n + tb - 1) / tb;
    if (b > 148 * 64) b = 148 * 64;
    return (unsigned)(b > 0 ? b : 1);
}
}  // namespace
}  // namespace wspm

using namespace wspm;

extern "C" int64_t wspm_pattern_device_scratch_bytes(int64_t n_elems, int32_t nv, int32_t n_nodes) {
    if (n_elems <= 0 || nv < 2 || nv > 4 || n_nodes <= 0) return -1;
    return 8 * scratch_words(n_elems, nv, n_nodes) + 256;
}

extern "C" int wspm_pattern_device_count(const int32_t *conn, int64_t n_elems, int32_t nv, int32_t n_nodes,
                                         int32_t layout, void *scratch, int64_t scratch_bytes,
                                         wspm_pattern_sizes *sizes, void *stream) {
    if (!conn || !scratch || !sizes || n_elems <= 0 || nv < 2 || nv > 4 || n_nodes <= 0) return WSPM_BAD_ARG;
    if (layout < WSPM_LAYOUT_AUTO || layout > WSPM_LAYOUT_DIA) return WSPM_BAD_ARG;
    if (scratch_bytes < wspm_pattern_device_scratch_bytes(n_elems, nv, n_nodes)) return WSPM_BAD_ARG;
    const int64_t N = n_nodes, E = n_elems;
    if (N + 1 > (int64_t)kScanThreads * kScanBlockItems || E * nv > (int64_t)INT32_MAX) return WSPM_UNSUPPORTED;
    const int ns = (int)((N + kPS - 1) / kPS);
    cudaStream_t st = (cudaStream_t)stream;
    Scratch w = carve(scratch, E, nv, N);
    WSPM_CUDA_TRY(cudaMemsetAsync(w.deg, 0, sizeof(int64_t) * (N + 1), st));
    WSPM_CUDA_TRY(cudaMemsetAsync(w.cursor, 0, sizeof(int32_t) * (N + 1), st));
    WSPM_CUDA_TRY(cudaMemsetAsync(w.flags, 0, sizeof(int) * 8, st));
    WSPM_CUDA_TRY(cudaMemsetAsync(w.maxes, 0, sizeof(unsigned long long) * 8, st));
    set_init_kernel<<<1, 64, 0, st>>>(w.set, kSetCap);
    degree_kernel<<<grid_for(E * nv), 256, 0, st>>>(conn, E * nv, n_nodes, w.deg, w.flags);
    scan_i64(w.deg, N, w.deg_ptr, w.bsum, st);
    incidence_fill_kernel<<<grid_for(E * nv), 256, 0, st>>>(conn, E * nv, nv, w.deg_ptr, w.cursor, w.inc);
    incidence_sort_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(n_nodes, w.deg_ptr, w.inc);
    row_count_kernel<<<(unsigned)((N + 127) / 128), 128, 0, st>>>(n_nodes, conn, nv, w.deg_ptr, w.inc, w.row_len,
                                                                  w.set, w.flags + 2, w.flags + 1, w.flags);
    scan_i64(w.row_len, N, w.row_ptr, w.bsum, st);
    slice_max_kernel<<<(ns + 255) / 256, 256, 0, st>>>(n_nodes, ns, w.row_ptr, w.sw);
    slice_max_kernel<<<(ns + 255) / 256, 256, 0, st>>>(n_nodes, ns, w.deg_ptr, w.iw);
    max_kernel<<<grid_for(ns), 256, 0, st>>>(ns, w.sw, w.maxes);
    max_kernel<<<grid_for(ns), 256, 0, st>>>(ns, w.iw, w.maxes + 1);
    // slice pointers: scan of width * 32 (the scan input reuses the pointer arrays' tails is avoided: own buffers)
    times_slice_kernel<<<(ns + 255) / 256, 256, 0, st>>>(ns, w.sw, w.sw_ptr);
    times_slice_kernel<<<(ns + 255) / 256, 256, 0, st>>>(ns, w.iw, w.iw_ptr);
    WSPM_CUDA_TRY(cudaMemcpyAsync(w.row_len, w.sw_ptr, sizeof(int64_t) * ns, cudaMemcpyDeviceToDevice, st));
    scan_i64(w.row_len, ns, w.sw_ptr, w.bsum, st);
    WSPM_CUDA_TRY(cudaMemcpyAsync(w.row_len, w.iw_ptr, sizeof(int64_t) * ns, cudaMemcpyDeviceToDevice, st));
    scan_i64(w.row_len, ns, w.iw_ptr, w.bsum, st);
    WSPM_CUDA_TRY(cudaGetLastError());
    // the sizes come back to the host (synchronous: the caller allocates the outputs from them)
    int flags[8];
    unsigned long long set[kSetCap], maxes[2];
    int64_t nnz = 0, sell_total = 0, n_inc = 0;
    WSPM_CUDA_TRY(cudaMemcpyAsync(flags, w.flags, sizeof(flags), cudaMemcpyDeviceToHost, st));
    WSPM_CUDA_TRY(cudaMemcpyAsync(set, w.set, sizeof(set), cudaMemcpyDeviceToHost, st));
    WSPM_CUDA_TRY(cudaMemcpyAsync(maxes, w.maxes, sizeof(maxes), cudaMemcpyDeviceToHost, st));
    WSPM_CUDA_TRY(cudaMemcpyAsync(&nnz, w.row_ptr + N, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    WSPM_CUDA_TRY(cudaMemcpyAsync(&sell_total, w.sw_ptr + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    WSPM_CUDA_TRY(cudaMemcpyAsync(&n_inc, w.iw_ptr + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    WSPM_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags[0] & 1) return WSPM_BAD_ARG;            // an element id out of range, or a node in no element
    if (flags[0] & 2) return WSPM_UNSUPPORTED;        // a row gathers more than kRowCap element vertices
    const bool many = flags[1] != 0;
    std::vector<int> offs;
    for (int t = 0; t < kSetCap && !many; ++t)
        if (set[t] != 0x8000000000000000ull) offs.push_back((int)(long long)set[t]);
    std::sort(offs.begin(), offs.end());
    const bool dia = layout == WSPM_LAYOUT_DIA || (layout == WSPM_LAYOUT_AUTO && !many && (int)offs.size() <= kDiaCap);
    if (dia && (many || offs.size() > 63)) return WSPM_UNSUPPORTED;
    if (!dia && maxes[0] > 63) return WSPM_UNSUPPORTED;
    std::memset(sizes, 0, sizeof(*sizes));
    sizes->n_rows = n_nodes;
    sizes->n_slices = ns;
    sizes->max_inc = (int32_t)maxes[1];
    sizes->nnz = nnz;
    sizes->n_inc = n_inc;
    sizes->layout = dia ? WSPM_LAYOUT_DIA : WSPM_LAYOUT_SELL;
    if (dia) {
        sizes->n_diags = (int32_t)offs.size();
        sizes->ld = (int64_t)ns * kPS;
        sizes->nnz_padded = sizes->n_diags * sizes->ld;
        sizes->max_width = sizes->n_diags;
        for (size_t k = 0; k < offs.size(); ++k) sizes->diag_offsets[k] = offs[k];
    } else {
        sizes->nnz_padded = sell_total;
        sizes->max_width = (int32_t)maxes[0];
    }
    return WSPM_OK;
}

extern "C" int wspm_pattern_device_fill(const int32_t *conn, int64_t n_elems, int32_t nv, int32_t n_nodes,
                                        const wspm_pattern_sizes *sizes, void *scratch, int64_t scratch_bytes,
                                        int64_t *csr_indptr, int32_t *csr_indices, int64_t *sell_index,
                                        int64_t *slice_ptr, int32_t *slice_width, int32_t *cols, int32_t *diag_pos,
                                        int32_t *diag_offsets, int64_t *inc_ptr, int32_t *inc_width,
                                        int32_t *inc_elem, uint32_t *inc_slots, void *stream) {
    if (!conn || !scratch || !sizes || sizes->n_rows != n_nodes || n_elems <= 0 || nv < 2 || nv > 4) return WSPM_BAD_ARG;
    if (scratch_bytes < wspm_pattern_device_scratch_bytes(n_elems, nv, n_nodes)) return WSPM_BAD_ARG;
    if (!csr_indptr || !csr_indices || !sell_index || !slice_ptr || !slice_width || !cols || !diag_pos || !inc_ptr ||
        !inc_width || !inc_elem || !inc_slots || (sizes->n_diags > 0 && !diag_offsets))
        return WSPM_BAD_ARG;
    const int64_t N = n_nodes, E = n_elems;
    const int ns = sizes->n_slices;
    const bool dia = sizes->layout == WSPM_LAYOUT_DIA;
    cudaStream_t st = (cudaStream_t)stream;
    Scratch w = carve(scratch, E, nv, N);
    WSPM_CUDA_TRY(cudaMemcpyAsync(csr_indptr, w.row_ptr, sizeof(int64_t) * (N + 1), cudaMemcpyDeviceToDevice, st));
    WSPM_CUDA_TRY(cudaMemcpyAsync(inc_ptr, w.iw_ptr, sizeof(int64_t) * (ns + 1), cudaMemcpyDeviceToDevice, st));
    widths_i32_kernel<<<(ns + 255) / 256, 256, 0, st>>>(ns, w.iw, inc_width, 0, 0);
    fill_i32_kernel<<<grid_for(sizes->n_inc), 256, 0, st>>>(inc_elem, sizes->n_inc, -1);
    WSPM_CUDA_TRY(cudaMemsetAsync(inc_slots, 0, sizeof(uint32_t) * sizes->n_inc, st));
    if (dia) {
        WSPM_CUDA_TRY(cudaMemcpyAsync(diag_offsets, sizes->diag_offsets, sizeof(int32_t) * sizes->n_diags,
                                      cudaMemcpyHostToDevice, st));
        slice_ptr_dia_kernel<<<(ns + 256) / 256, 256, 0, st>>>(ns, slice_ptr);
        widths_i32_kernel<<<(ns + 255) / 256, 256, 0, st>>>(ns, w.sw, slice_width, 1, sizes->n_diags);
        dia_cols_kernel<<<grid_for(sizes->nnz_padded), 256, 0, st>>>(n_nodes, sizes->n_diags, sizes->ld, diag_offsets,
                                                                     cols);
    } else {
        WSPM_CUDA_TRY(cudaMemcpyAsync(slice_ptr, w.sw_ptr, sizeof(int64_t) * (ns + 1), cudaMemcpyDeviceToDevice, st));
        widths_i32_kernel<<<(ns + 255) / 256, 256, 0, st>>>(ns, w.sw, slice_width, 0, 0);
        sell_pad_kernel<<<ns, 256, 0, st>>>(n_nodes, ns, slice_ptr, cols);
    }
    FillArgs a;
    a.n_nodes = n_nodes; a.nv = nv; a.ns = ns; a.dia = dia ? 1 : 0; a.nd = sizes->n_diags; a.ld = sizes->ld;
    a.conn = conn; a.deg_ptr = w.deg_ptr; a.inc = w.inc; a.indptr = w.row_ptr; a.slice_ptr = slice_ptr;
    a.inc_ptr = w.iw_ptr; a.offs = diag_offsets;
    a.indices = csr_indices; a.cols = cols; a.diag_pos = diag_pos; a.inc_elem = inc_elem;
    a.sell_index = sell_index; a.inc_slots = inc_slots;
    rows_fill_kernel<<<(unsigned)((N + 127) / 128), 128, 0, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? WSPM_OK : WSPM_CUDA_ERROR;
}
