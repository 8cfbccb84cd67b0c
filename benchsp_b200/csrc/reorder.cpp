// Matrix reordering (no reference counterpart: the reference's SMaT path
// blocks the matrix in its given order, src/smat.cu:116-120, so scattered
// nonzeros give one nonzero per 16x16 tile).  Reverse Cuthill-McKee on the
// symmetrized pattern gathers nonzeros near the diagonal, which raises the
// fill of BSR blocks and SMaT tiles for matrices whose rows were numbered
// without locality.  Host code (a one-time preprocessing step); the device
// entry points copy in, reorder on the host and copy back.
//
// RCM: for every connected component, start from a pseudo-peripheral vertex
// (the George-Liu search: repeat a BFS from the farthest, lowest-degree
// vertex of the last level while the eccentricity grows), visit the BFS
// levels taking each vertex's unvisited neighbours in increasing degree
// (ties by index), and reverse the whole order at the end.
#include <cuda_runtime.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/bsp.h"

namespace bsp {
void set_error(const std::string &msg);
void clear_error();
}  // namespace bsp

namespace {

bsp_status fail(bsp_status st, const char *msg) {
  bsp::set_error(msg);
  return st;
}

struct Graph {
  std::vector<int64_t> ptr;
  std::vector<int32_t> adj;
};

// Pattern of A + A^T without the diagonal, neighbours sorted and distinct.
Graph symmetrize(int32_t n, const int32_t *rp, const int32_t *ci) {
  std::vector<int64_t> deg(n + 1, 0);
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
      const int32_t c = ci[j];
      if (c == i || c < 0 || c >= n) continue;
      ++deg[i];
      ++deg[c];
    }
  Graph g;
  g.ptr.assign(n + 1, 0);
  for (int32_t i = 0; i < n; ++i) g.ptr[i + 1] = g.ptr[i] + deg[i];
  g.adj.resize(g.ptr[n]);
  std::vector<int64_t> fill(g.ptr.begin(), g.ptr.end() - 1);
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
      const int32_t c = ci[j];
      if (c == i || c < 0 || c >= n) continue;
      g.adj[fill[i]++] = c;
      g.adj[fill[c]++] = i;
    }
  // sort + unique each list, then compact
  std::vector<int64_t> np(n + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t i = 0; i < n; ++i) {
    auto b = g.adj.begin() + g.ptr[i], e = g.adj.begin() + g.ptr[i + 1];
    std::sort(b, e);
    np[i + 1] = std::unique(b, e) - b;
  }
  for (int32_t i = 0; i < n; ++i) np[i + 1] += np[i];
  std::vector<int32_t> adj(np[n]);
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < n; ++i)
    std::copy(g.adj.begin() + g.ptr[i], g.adj.begin() + g.ptr[i] + (np[i + 1] - np[i]), adj.begin() + np[i]);
  g.ptr.swap(np);
  g.adj.swap(adj);
  return g;
}

// BFS from s over unvisited-by-order vertices of s's component; returns the
// last level's vertices and the number of levels.
int bfs_levels(const Graph &g, int32_t s, std::vector<int32_t> &level, std::vector<int32_t> &queue,
               std::vector<int32_t> &last) {
  queue.clear();
  queue.push_back(s);
  level[s] = 0;
  int depth = 0;
  size_t head = 0;
  while (head < queue.size()) {
    const int32_t v = queue[head++];
    for (int64_t k = g.ptr[v]; k < g.ptr[v + 1]; ++k) {
      const int32_t w = g.adj[k];
      if (level[w] < 0) {
        level[w] = level[v] + 1;
        depth = std::max(depth, level[w]);
        queue.push_back(w);
      }
    }
  }
  last.clear();
  for (int32_t v : queue)
    if (level[v] == depth) last.push_back(v);
  for (int32_t v : queue) level[v] = -1;  // reset for the next search
  return depth;
}

void rcm(int32_t n, const int32_t *rp, const int32_t *ci, int32_t *perm) {
  const Graph g = symmetrize(n, rp, ci);
  auto degree = [&](int32_t v) { return g.ptr[v + 1] - g.ptr[v]; };
  std::vector<int32_t> level(n, -1), queue, last, order;
  order.reserve(n);
  std::vector<char> placed(n, 0);
  std::vector<int32_t> nb;
  for (int32_t seed = 0; seed < n; ++seed) {
    if (placed[seed]) continue;
    // pseudo-peripheral start (a few George-Liu steps)
    int32_t s = seed;
    int depth = bfs_levels(g, s, level, queue, last);
    for (int it = 0; it < 8; ++it) {
      int32_t best = last[0];
      for (int32_t v : last)
        if (degree(v) < degree(best) || (degree(v) == degree(best) && v < best)) best = v;
      const int d2 = bfs_levels(g, best, level, queue, last);
      if (d2 <= depth) break;
      s = best;
      depth = d2;
    }
    // Cuthill-McKee BFS from s
    size_t head = order.size();
    order.push_back(s);
    placed[s] = 1;
    while (head < order.size()) {
      const int32_t v = order[head++];
      nb.clear();
      for (int64_t k = g.ptr[v]; k < g.ptr[v + 1]; ++k)
        if (!placed[g.adj[k]]) nb.push_back(g.adj[k]);
      std::sort(nb.begin(), nb.end(), [&](int32_t a, int32_t b) {
        return degree(a) != degree(b) ? degree(a) < degree(b) : a < b;
      });
      for (int32_t w : nb) {
        placed[w] = 1;
        order.push_back(w);
      }
    }
  }
  for (int32_t i = 0; i < n; ++i) perm[i] = order[n - 1 - i];
}

// P A P^T: new row i = old row perm[i], columns renumbered by the inverse and
// sorted.
void permute(int32_t n, const int32_t *rp, const int32_t *ci, const double *va, const int32_t *perm,
             int32_t *orp, int32_t *oci, double *ova) {
  std::vector<int32_t> inv(n);
  for (int32_t i = 0; i < n; ++i) inv[perm[i]] = i;
  orp[0] = 0;
  for (int32_t i = 0; i < n; ++i) orp[i + 1] = orp[i] + (rp[perm[i] + 1] - rp[perm[i]]);
#pragma omp parallel
  {
    std::vector<std::pair<int32_t, double>> row;
#pragma omp for schedule(dynamic, 512)
    for (int32_t i = 0; i < n; ++i) {
      const int32_t o = perm[i];
      row.clear();
      for (int32_t j = rp[o]; j < rp[o + 1]; ++j) row.emplace_back(inv[ci[j]], va ? va[j] : 0.0);
      std::sort(row.begin(), row.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
      for (size_t k = 0; k < row.size(); ++k) {
        oci[orp[i] + k] = row[k].first;
        if (ova) ova[orp[i] + k] = row[k].second;
      }
    }
  }
}

// Row-similarity order for tile formats: rows whose nonzeros fall in the
// same column blocks are placed in the same group of `G` consecutive rows,
// so a G x BC tiling of the reordered matrix needs few tiles.  Signature of
// a row = its distinct column blocks (col / BC), ascending.  A group starts
// at the first unplaced row (row order) and grows one row at a time: the
// candidates are the unplaced rows that share a block with the group's
// union of blocks U, found through an inverted index (block -> rows,
// ascending).  The scans are bounded: a joining row's new blocks are read
// shortest list first (rare blocks say the most), at most kScanBlocks blocks
// and kScanEntries entries per block, until a group has kTouched
// candidates.  The next row is the candidate of highest Jaccard similarity
// |S_c & U| / |S_c | U| (ties by row index; compared by exact integer
// cross-multiplication), and its blocks join U.  A group left short is
// filled with the next unplaced rows in row order.  Empty rows go last.
// Deterministic; O(nnz log) for the signatures plus O(rows * kTouched) for
// the grouping.
constexpr int32_t kScanBlocks = 64;
constexpr int64_t kScanEntries = 1024;
constexpr size_t kTouched = 512;

void similarity_order(int32_t n, int32_t cols, const int32_t *rp, const int32_t *ci, int32_t G, int32_t BC,
                      int32_t *perm) {
  const int32_t nb = (int32_t)(((int64_t)cols + BC - 1) / BC);
  std::vector<int32_t> len(n);
#pragma omp parallel
  {
    std::vector<int32_t> t;
#pragma omp for schedule(dynamic, 1024)
    for (int32_t i = 0; i < n; ++i) {
      t.assign(ci + rp[i], ci + rp[i + 1]);
      for (int32_t &c : t) c /= BC;
      std::sort(t.begin(), t.end());
      len[i] = (int32_t)(std::unique(t.begin(), t.end()) - t.begin());
    }
  }
  std::vector<int64_t> sp(n + 1, 0);
  for (int32_t i = 0; i < n; ++i) sp[i + 1] = sp[i] + len[i];
  std::vector<int32_t> sig(sp[n]);
#pragma omp parallel
  {
    std::vector<int32_t> t;
#pragma omp for schedule(dynamic, 1024)
    for (int32_t i = 0; i < n; ++i) {
      t.assign(ci + rp[i], ci + rp[i + 1]);
      for (int32_t &c : t) c /= BC;
      std::sort(t.begin(), t.end());
      t.erase(std::unique(t.begin(), t.end()), t.end());
      std::copy(t.begin(), t.end(), sig.begin() + sp[i]);
    }
  }
  // inverted index, rows ascending within a block
  std::vector<int64_t> bp(nb + 1, 0);
  for (int64_t k = 0; k < sp[n]; ++k) ++bp[sig[k] + 1];
  for (int32_t b = 0; b < nb; ++b) bp[b + 1] += bp[b];
  std::vector<int32_t> brow(sp[n]);
  {
    std::vector<int64_t> fill(bp.begin(), bp.end() - 1);
    for (int32_t i = 0; i < n; ++i)
      for (int64_t k = sp[i]; k < sp[i + 1]; ++k) brow[fill[sig[k]]++] = i;
  }
  std::vector<int64_t> head(bp.begin(), bp.end() - 1);
  std::vector<char> placed(n, 0);
  std::vector<int32_t> shared(n, 0), touched, fresh, in_u(nb, -1);
  int32_t out = 0, next = 0, group = 0;
  auto place = [&](int32_t r) {
    placed[r] = 1;
    perm[out++] = r;
  };
  auto next_unplaced = [&]() {
    while (next < n && (placed[next] || len[next] == 0)) ++next;
    return next;
  };
  while (next_unplaced() < n) {
    int64_t ulen = 0;
    int32_t scanned = 0, size = 0;
    touched.clear();
    // row r joins the group: its new blocks join U and bring their rows in
    auto join = [&](int32_t r) {
      place(r);
      ++size;
      fresh.clear();
      for (int64_t k = sp[r]; k < sp[r + 1]; ++k) {
        const int32_t b = sig[k];
        if (in_u[b] == group) continue;
        in_u[b] = group;
        ++ulen;
        fresh.push_back(b);
      }
      std::sort(fresh.begin(), fresh.end(), [&](int32_t a, int32_t b) {
        const int64_t la = bp[a + 1] - head[a], lb = bp[b + 1] - head[b];
        return la != lb ? la < lb : a < b;
      });
      for (int32_t b : fresh) {
        if (scanned >= kScanBlocks || touched.size() >= kTouched) break;
        ++scanned;
        while (head[b] < bp[b + 1] && placed[brow[head[b]]]) ++head[b];
        for (int64_t e = head[b], lim = std::min<int64_t>(bp[b + 1], head[b] + kScanEntries); e < lim; ++e) {
          const int32_t c = brow[e];
          if (placed[c]) continue;
          if (shared[c]++ == 0) {
            touched.push_back(c);
            if (touched.size() >= kTouched) break;
          }
        }
      }
    };
    join(next);
    while (size < G) {
      // highest |S_c & U| / (|U| + |S_c| - |S_c & U|), then lower index
      int32_t best = -1;
      for (int32_t c : touched) {
        if (placed[c]) continue;
        if (best < 0) {
          best = c;
          continue;
        }
        const int64_t sc = shared[c], sb = shared[best];
        const int64_t lhs = sc * (ulen + len[best] - sb), rhs = sb * (ulen + len[c] - sc);
        if (lhs > rhs || (lhs == rhs && c < best)) best = c;
      }
      if (best < 0) break;
      join(best);
    }
    for (int32_t c : touched) shared[c] = 0;
    while (size < G && next_unplaced() < n) {
      place(next);
      ++size;
    }
    ++group;
  }
  for (int32_t i = 0; i < n; ++i)
    if (!placed[i]) place(i);  // the empty rows
}

// P A (rows only): new row i = old row perm[i], its entries as stored.
void permute_rows(int32_t n, const int32_t *rp, const int32_t *ci, const double *va, const int32_t *perm,
                  int32_t *orp, int32_t *oci, double *ova) {
  orp[0] = 0;
  for (int32_t i = 0; i < n; ++i) orp[i + 1] = orp[i] + (rp[perm[i] + 1] - rp[perm[i]]);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t i = 0; i < n; ++i) {
    const int32_t o = perm[i], m = rp[o + 1] - rp[o];
    std::copy(ci + rp[o], ci + rp[o] + m, oci + orp[i]);
    if (ova) std::copy(va + rp[o], va + rp[o] + m, ova + orp[i]);
  }
}

// 16 x 16 tiles of A with its rows in the order `perm` (null: as given):
// the distinct column blocks of every 16-row block, summed.
int64_t count_tiles(int32_t n, const int32_t *rp, const int32_t *ci, const int32_t *perm) {
  const int32_t nbr = (int32_t)(((int64_t)n + 15) / 16);
  int64_t total = 0;
#pragma omp parallel reduction(+ : total)
  {
    std::vector<int32_t> t;
#pragma omp for schedule(dynamic, 256)
    for (int32_t br = 0; br < nbr; ++br) {
      t.clear();
      for (int32_t i = br * 16; i < std::min<int32_t>(n, br * 16 + 16); ++i) {
        const int32_t r = perm ? perm[i] : i;
        for (int32_t j = rp[r]; j < rp[r + 1]; ++j) t.push_back(ci[j] >> 4);
      }
      std::sort(t.begin(), t.end());
      total += (int64_t)(std::unique(t.begin(), t.end()) - t.begin());
    }
  }
  return total;
}

// SpMM engine cost model, seconds per unit per column of B, from the B200
// measurements of the SMaT and CSR SpMM at N = 128 (dense-tile and
// row-shuffled 524,288-row matrices, power-law graph): the persistent
// tcgen05 kernel 163 us for 262,144 tiles at N = 128 (4.9e-12 s per
// tile-column, 64-column slabs below N = 128), the grouped CSR kernel
// 1.93 ms for 67.1M nonzeros (2.3e-13 s per nonzero-column).
constexpr double kTileColSecTc = 4.9e-12;
constexpr double kNnzColSecCsr = 2.3e-13;
// Gathered-tile tcgen05 kernel (bsp_gtile): 366,808 chunks of a
// column-permuted 27-point stencil (48^3 x 4 dof) in 0.668 ms at N = 128 and
// 1.33 ms at N = 256, 2.01M chunks of a power-law graph in 4.30 ms at N = 128:
// 1.45e-11 s per chunk-column; below N = 128 the slab is 64 columns and a
// chunk took 1.2-1.5 ns at N = 32 (counted as 96 columns).
constexpr double kChunkColSecGt = 1.45e-11;

// Chunks of the gathered-tile form with A's rows in the order `perm` (null:
// as given): every 16-row group's distinct columns, in chunks of 16, summed.
int64_t count_chunks(int32_t n, const int32_t *rp, const int32_t *ci, const int32_t *perm) {
  const int32_t ng = (int32_t)(((int64_t)n + 15) / 16);
  int64_t total = 0;
#pragma omp parallel reduction(+ : total)
  {
    std::vector<int32_t> t;
#pragma omp for schedule(dynamic, 256)
    for (int32_t g = 0; g < ng; ++g) {
      t.clear();
      for (int32_t i = g * 16; i < std::min<int32_t>(n, g * 16 + 16); ++i) {
        const int32_t r = perm ? perm[i] : i;
        t.insert(t.end(), ci + rp[r], ci + rp[r + 1]);
      }
      std::sort(t.begin(), t.end());
      total += ((int64_t)(std::unique(t.begin(), t.end()) - t.begin()) + 15) / 16;
    }
  }
  return total;
}

bool valid_csr(int32_t n, int32_t nnz, const int32_t *rp) {
  if (rp[0] != 0 || rp[n] != nnz) return false;
  for (int32_t i = 0; i < n; ++i)
    if (rp[i + 1] < rp[i]) return false;
  return true;
}

bool valid_perm(int32_t n, const int32_t *perm) {
  std::vector<char> seen(n, 0);
  for (int32_t i = 0; i < n; ++i) {
    if (perm[i] < 0 || perm[i] >= n || seen[perm[i]]) return false;
    seen[perm[i]] = 1;
  }
  return true;
}

template <typename T>
bool d2h(std::vector<T> &h, const T *d, size_t n) {
  h.resize(n);
  return n == 0 || cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess;
}

template <typename T>
bool h2d(T *d, const std::vector<T> &h) {
  return h.empty() || cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
}

}  // namespace

extern "C" bsp_status bsp_reorder_rcm_host(int32_t rows, int32_t nnz, const int32_t *rowPtr,
                                           const int32_t *colIdx, int32_t *perm) {
  bsp::clear_error();
  if (rows < 0 || nnz < 0 || !rowPtr || !perm || (nnz > 0 && !colIdx))
    return fail(BSP_ERR_INVALID, "bsp_reorder_rcm: bad argument");
  if (!valid_csr(rows, nnz, rowPtr)) return fail(BSP_ERR_INVALID, "bsp_reorder_rcm: malformed row pointers");
  if (rows > 0) rcm(rows, rowPtr, colIdx, perm);
  return BSP_OK;
}

extern "C" bsp_status bsp_permute_csr_host(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                                           const double *values, const int32_t *perm, int32_t *outRowPtr,
                                           int32_t *outColIdx, double *outValues) {
  bsp::clear_error();
  if (rows < 0 || nnz < 0 || !rowPtr || !perm || !outRowPtr || (nnz > 0 && (!colIdx || !outColIdx)))
    return fail(BSP_ERR_INVALID, "bsp_permute_csr: bad argument");
  if (!valid_csr(rows, nnz, rowPtr)) return fail(BSP_ERR_INVALID, "bsp_permute_csr: malformed row pointers");
  if (!valid_perm(rows, perm)) return fail(BSP_ERR_INVALID, "bsp_permute_csr: perm is not a permutation");
  for (int32_t j = 0; j < nnz; ++j)
    if (colIdx[j] < 0 || colIdx[j] >= rows)
      return fail(BSP_ERR_INVALID, "bsp_permute_csr: column out of range (square matrices only)");
  permute(rows, rowPtr, colIdx, values, perm, outRowPtr, outColIdx, outValues);
  return BSP_OK;
}

extern "C" bsp_status bsp_reorder_rcm(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                                      int32_t *perm, bsp_stream_t stream) {
  bsp::clear_error();
  if (rows < 0 || nnz < 0) return fail(BSP_ERR_INVALID, "bsp_reorder_rcm: negative size");
  if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
    return fail(BSP_ERR_CUDA, "bsp_reorder_rcm: stream synchronize failed");
  std::vector<int32_t> rp, ci, p(rows > 0 ? rows : 0);
  if (!d2h(rp, rowPtr, (size_t)rows + 1) || !d2h(ci, colIdx, (size_t)nnz))
    return fail(BSP_ERR_CUDA, "bsp_reorder_rcm: copy to the host failed");
  const bsp_status st = bsp_reorder_rcm_host(rows, nnz, rp.data(), ci.data(), p.data());
  if (st != BSP_OK) return st;
  return h2d(perm, p) ? BSP_OK : fail(BSP_ERR_CUDA, "bsp_reorder_rcm: copy to the device failed");
}

extern "C" bsp_status bsp_permute_csr(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                                      const double *values, const int32_t *perm, int32_t *outRowPtr,
                                      int32_t *outColIdx, double *outValues, bsp_stream_t stream) {
  bsp::clear_error();
  if (rows < 0 || nnz < 0) return fail(BSP_ERR_INVALID, "bsp_permute_csr: negative size");
  if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
    return fail(BSP_ERR_CUDA, "bsp_permute_csr: stream synchronize failed");
  std::vector<int32_t> rp, ci, p, orp((size_t)rows + 1), oci(nnz);
  std::vector<double> va, ova(values ? nnz : 0);
  if (!d2h(rp, rowPtr, (size_t)rows + 1) || !d2h(ci, colIdx, (size_t)nnz) || !d2h(p, perm, (size_t)rows) ||
      (values && !d2h(va, values, (size_t)nnz)))
    return fail(BSP_ERR_CUDA, "bsp_permute_csr: copy to the host failed");
  const bsp_status st = bsp_permute_csr_host(rows, nnz, rp.data(), ci.data(), values ? va.data() : nullptr,
                                             p.data(), orp.data(), oci.data(), values ? ova.data() : nullptr);
  if (st != BSP_OK) return st;
  if (!h2d(outRowPtr, orp) || !h2d(outColIdx, oci) || (values && outValues && !h2d(outValues, ova)))
    return fail(BSP_ERR_CUDA, "bsp_permute_csr: copy to the device failed");
  return BSP_OK;
}

extern "C" bsp_status bsp_reorder_similarity_host(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                                  const int32_t *colIdx, int32_t group_rows, int32_t block_cols,
                                                  int32_t *perm) {
  bsp::clear_error();
  if (rows < 0 || cols < 0 || nnz < 0 || !rowPtr || !perm || (nnz > 0 && !colIdx))
    return fail(BSP_ERR_INVALID, "bsp_reorder_similarity: bad argument");
  if (group_rows < 1 || group_rows > 4096 || block_cols < 1)
    return fail(BSP_ERR_INVALID, "bsp_reorder_similarity: group_rows must be in [1, 4096], block_cols >= 1");
  if (!valid_csr(rows, nnz, rowPtr)) return fail(BSP_ERR_INVALID, "bsp_reorder_similarity: malformed row pointers");
  for (int32_t j = 0; j < nnz; ++j)
    if (colIdx[j] < 0 || colIdx[j] >= cols) return fail(BSP_ERR_INVALID, "bsp_reorder_similarity: column out of range");
  if (rows > 0) similarity_order(rows, cols, rowPtr, colIdx, group_rows, block_cols, perm);
  return BSP_OK;
}

extern "C" bsp_status bsp_permute_rows_csr_host(int32_t rows, int32_t nnz, const int32_t *rowPtr,
                                                const int32_t *colIdx, const double *values, const int32_t *perm,
                                                int32_t *outRowPtr, int32_t *outColIdx, double *outValues) {
  bsp::clear_error();
  if (rows < 0 || nnz < 0 || !rowPtr || !perm || !outRowPtr || (nnz > 0 && (!colIdx || !outColIdx)))
    return fail(BSP_ERR_INVALID, "bsp_permute_rows_csr: bad argument");
  if (!valid_csr(rows, nnz, rowPtr)) return fail(BSP_ERR_INVALID, "bsp_permute_rows_csr: malformed row pointers");
  if (!valid_perm(rows, perm)) return fail(BSP_ERR_INVALID, "bsp_permute_rows_csr: perm is not a permutation");
  permute_rows(rows, rowPtr, colIdx, values && outValues ? values : nullptr, perm, outRowPtr, outColIdx,
               values && outValues ? outValues : nullptr);
  return BSP_OK;
}

extern "C" bsp_status bsp_reorder_similarity(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                             const int32_t *colIdx, int32_t group_rows, int32_t block_cols,
                                             int32_t *perm, bsp_stream_t stream) {
  bsp::clear_error();
  if (rows < 0 || nnz < 0) return fail(BSP_ERR_INVALID, "bsp_reorder_similarity: negative size");
  if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
    return fail(BSP_ERR_CUDA, "bsp_reorder_similarity: stream synchronize failed");
  std::vector<int32_t> rp, ci, p(rows > 0 ? rows : 0);
  if (!d2h(rp, rowPtr, (size_t)rows + 1) || !d2h(ci, colIdx, (size_t)nnz))
    return fail(BSP_ERR_CUDA, "bsp_reorder_similarity: copy to the host failed");
  const bsp_status st =
      bsp_reorder_similarity_host(rows, cols, nnz, rp.data(), ci.data(), group_rows, block_cols, p.data());
  if (st != BSP_OK) return st;
  return h2d(perm, p) ? BSP_OK : fail(BSP_ERR_CUDA, "bsp_reorder_similarity: copy to the device failed");
}

extern "C" bsp_status bsp_permute_rows_csr(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                                           const double *values, const int32_t *perm, int32_t *outRowPtr,
                                           int32_t *outColIdx, double *outValues, bsp_stream_t stream) {
  bsp::clear_error();
  if (rows < 0 || nnz < 0) return fail(BSP_ERR_INVALID, "bsp_permute_rows_csr: negative size");
  if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
    return fail(BSP_ERR_CUDA, "bsp_permute_rows_csr: stream synchronize failed");
  std::vector<int32_t> rp, ci, p, orp((size_t)rows + 1), oci(nnz);
  std::vector<double> va, ova(values ? nnz : 0);
  if (!d2h(rp, rowPtr, (size_t)rows + 1) || !d2h(ci, colIdx, (size_t)nnz) || !d2h(p, perm, (size_t)rows) ||
      (values && !d2h(va, values, (size_t)nnz)))
    return fail(BSP_ERR_CUDA, "bsp_permute_rows_csr: copy to the host failed");
  const bsp_status st = bsp_permute_rows_csr_host(rows, nnz, rp.data(), ci.data(), values ? va.data() : nullptr,
                                                  p.data(), orp.data(), oci.data(), values ? ova.data() : nullptr);
  if (st != BSP_OK) return st;
  if (!h2d(outRowPtr, orp) || !h2d(outColIdx, oci) || (values && outValues && !h2d(outValues, ova)))
    return fail(BSP_ERR_CUDA, "bsp_permute_rows_csr: copy to the device failed");
  return BSP_OK;
}

extern "C" bsp_status bsp_spmm_choose_host(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                           const int32_t *colIdx, int32_t N, int32_t *perm, bsp_spmm_choice *out) {
  bsp::clear_error();
  if (rows < 0 || cols < 0 || nnz < 0 || N <= 0 || !rowPtr || !out || (nnz > 0 && !colIdx))
    return fail(BSP_ERR_INVALID, "bsp_spmm_choose: bad argument");
  if (!valid_csr(rows, nnz, rowPtr)) return fail(BSP_ERR_INVALID, "bsp_spmm_choose: malformed row pointers");
  for (int32_t j = 0; j < nnz; ++j)
    if (colIdx[j] < 0 || colIdx[j] >= cols) return fail(BSP_ERR_INVALID, "bsp_spmm_choose: column out of range");
  bsp_spmm_choice c{};
  const bool smat_ok = N % 32 == 0;
  c.smat_path = BSP_SMAT_TCGEN05;
  // the tensor-core path works in slabs of 64 or 128 C columns
  const double per_tile = kTileColSecTc * (double)(((int64_t)N + 63) / 64 * 64);
  c.tiles_given = count_tiles(rows, rowPtr, colIdx, nullptr);
  c.tiles_reordered = -1;
  if (perm && rows > 0) {
    similarity_order(rows, cols, rowPtr, colIdx, 16, 16, perm);
    c.tiles_reordered = count_tiles(rows, rowPtr, colIdx, perm);
  }
  c.est_seconds_csr = kNnzColSecCsr * N * (double)nnz;
  c.est_seconds_smat_given = smat_ok ? per_tile * (double)c.tiles_given : -1.0;
  c.est_seconds_smat_reordered = smat_ok && c.tiles_reordered >= 0 ? per_tile * (double)c.tiles_reordered : -1.0;
  // the gathered-tile kernel: N % 8 == 0, slabs of 64 or 128 C columns
  const bool gt_ok = N % 8 == 0;
  const double per_chunk = kChunkColSecGt * (double)std::max<int64_t>(96, ((int64_t)N + 63) / 64 * 64);
  c.chunks_given = count_chunks(rows, rowPtr, colIdx, nullptr);
  c.chunks_reordered = c.tiles_reordered >= 0 ? count_chunks(rows, rowPtr, colIdx, perm) : -1;
  c.est_seconds_gtile_given = gt_ok ? per_chunk * (double)c.chunks_given : -1.0;
  c.est_seconds_gtile_reordered = gt_ok && c.chunks_reordered >= 0 ? per_chunk * (double)c.chunks_reordered : -1.0;
  c.engine = BSP_SPMM_ENGINE_CSR;
  double best = c.est_seconds_csr;
  auto take = [&](double est, int32_t engine, int32_t reorder) {
    if (est >= 0 && est < best) {
      best = est;
      c.engine = engine;
      c.reorder = reorder;
    }
  };
  take(c.est_seconds_smat_given, BSP_SPMM_ENGINE_SMAT, 0);
  take(c.est_seconds_smat_reordered, BSP_SPMM_ENGINE_SMAT, 1);
  take(c.est_seconds_gtile_given, BSP_SPMM_ENGINE_GTILE, 0);
  take(c.est_seconds_gtile_reordered, BSP_SPMM_ENGINE_GTILE, 1);
  *out = c;
  return BSP_OK;
}
