// Host-side CSR utilities of the engine library: CSR1 file I/O, validation and
// the seeded synthetic generators used by the CLI, the tests and the bench.
//
// CSR1 layout (little-endian), as written by write_bin (src/export_bin.py:20-29)
// and read by load_bin (src/spgemm_engine.cuh:21-32):
//   char[4] "CSR1"; int32 n; int32 pad; int64 nnz;
//   int32 indptr[n+1]; int32 indices[nnz]; double data[nnz]
//
// Random streams: std::mt19937_64, a fully specified engine, with our own
// conversions (never a <random> distribution, whose output is library-defined):
//   u01(x)  = (x >> 11) · 2^-53            ∈ [0, 1)
//   um11(x) = 2·u01(x) − 1                 ∈ [−1, 1)   (exact in binary64)
//   below(x, m) = floor(u01(x) · m)        ∈ [0, m)
#include "internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

namespace spg {

static inline double u01(std::mt19937_64& g) {
  return (double)(g() >> 11) * 0x1.0p-53;
}
static inline double um11(std::mt19937_64& g) { return 2.0 * u01(g) - 1.0; }
static inline int64_t below(std::mt19937_64& g, int64_t m) {
  int64_t r = (int64_t)(u01(g) * (double)m);
  return r < m ? r : m - 1;
}

static spg_status alloc_host(spg_host_csr* out, int32_t n, int64_t nnz) {
  out->n = n;
  out->nnz = nnz;
  out->rowptr = (int32_t*)std::malloc(sizeof(int32_t) * ((size_t)n + 1));
  out->col = (int32_t*)std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(nnz, 1));
  out->val = (double*)std::malloc(sizeof(double) * (size_t)std::max<int64_t>(nnz, 1));
  if (!out->rowptr || !out->col || !out->val) {
    spg_host_csr_free(out);
    return set_error(SPG_ERR_OOM, "host allocation of a %d x %d CSR with %lld entries failed",
                     n, n, (long long)nnz);
  }
  return SPG_OK;
}

// Build a host CSR from per-row column lists already sorted and unique.
struct RowBuilder {
  std::vector<int32_t> rowptr, col;
  std::vector<double> val;
  explicit RowBuilder(int32_t n) { rowptr.reserve((size_t)n + 1); rowptr.push_back(0); }
  void end_row() { rowptr.push_back((int32_t)col.size()); }
  spg_status finish(spg_host_csr* out) {
    int32_t n = (int32_t)rowptr.size() - 1;
    if (col.size() > (size_t)INT32_MAX)
      return set_error(SPG_ERR_UNSUPPORTED, "generated matrix exceeds int32 row pointers");
    spg_status st = alloc_host(out, n, (int64_t)col.size());
    if (st != SPG_OK) return st;
    std::memcpy(out->rowptr, rowptr.data(), sizeof(int32_t) * rowptr.size());
    if (!col.empty()) {
      std::memcpy(out->col, col.data(), sizeof(int32_t) * col.size());
      std::memcpy(out->val, val.data(), sizeof(double) * val.size());
    }
    return SPG_OK;
  }
};

}  // namespace spg

using namespace spg;

extern "C" {

void spg_host_csr_free(spg_host_csr* A) {
  if (!A) return;
  std::free(A->rowptr);
  std::free(A->col);
  std::free(A->val);
  A->rowptr = nullptr;
  A->col = nullptr;
  A->val = nullptr;
  A->n = 0;
  A->nnz = 0;
}

spg_status spg_host_csr_validate(const spg_host_csr* A) {
  clear_error();
  if (!A || A->n < 0 || A->nnz < 0) return set_error(SPG_ERR_INVALID_ARG, "null or negative CSR");
  if (A->n > 0 && !A->rowptr) return set_error(SPG_ERR_INVALID_ARG, "null rowptr");
  if (A->nnz > 0 && (!A->col || !A->val)) return set_error(SPG_ERR_INVALID_ARG, "null col/val");
  if (A->n == 0) return A->nnz == 0 ? SPG_OK : set_error(SPG_ERR_INVALID_CSR, "n=0 with nnz>0");
  if (A->rowptr[0] != 0) return set_error(SPG_ERR_INVALID_CSR, "rowptr[0] = %d, expected 0", A->rowptr[0]);
  if ((int64_t)A->rowptr[A->n] != A->nnz)
    return set_error(SPG_ERR_INVALID_CSR, "rowptr[n] = %d but nnz = %lld", A->rowptr[A->n],
                     (long long)A->nnz);
  for (int32_t i = 0; i < A->n; ++i) {
    int32_t s = A->rowptr[i], e = A->rowptr[i + 1];
    if (e < s) return set_error(SPG_ERR_INVALID_CSR, "rowptr decreases at row %d", i);
    for (int32_t p = s; p < e; ++p) {
      int32_t j = A->col[p];
      if (j < 0 || j >= A->n)
        return set_error(SPG_ERR_INVALID_CSR, "column %d out of range in row %d", j, i);
      if (p > s && A->col[p - 1] >= j)
        return set_error(SPG_ERR_INVALID_CSR, "row %d columns not strictly increasing at %d", i, p);
    }
  }
  return SPG_OK;
}

spg_status spg_csr1_read(const char* path, spg_host_csr* out) {
  clear_error();
  if (!path || !out) return set_error(SPG_ERR_INVALID_ARG, "null argument");
  std::memset(out, 0, sizeof(*out));
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(SPG_ERR_IO, "cannot open %s", path);
  char magic[4];
  int32_t n = 0, pad = 0;
  int64_t nnz = 0;
  spg_status st = SPG_OK;
  if (std::fread(magic, 1, 4, f) != 4 || std::memcmp(magic, "CSR1", 4) != 0) {
    st = set_error(SPG_ERR_IO, "%s: bad magic (expected CSR1)", path);
  } else if (std::fread(&n, 4, 1, f) != 1 || std::fread(&pad, 4, 1, f) != 1 ||
             std::fread(&nnz, 8, 1, f) != 1) {
    st = set_error(SPG_ERR_IO, "%s: truncated header", path);
  } else if (n < 0 || nnz < 0 || nnz > INT32_MAX) {
    st = set_error(SPG_ERR_IO, "%s: bad sizes n=%d nnz=%lld", path, n, (long long)nnz);
  } else if ((st = alloc_host(out, n, nnz)) == SPG_OK) {
    if (std::fread(out->rowptr, 4, (size_t)n + 1, f) != (size_t)n + 1 ||
        std::fread(out->col, 4, (size_t)nnz, f) != (size_t)nnz ||
        std::fread(out->val, 8, (size_t)nnz, f) != (size_t)nnz) {
      spg_host_csr_free(out);
      st = set_error(SPG_ERR_IO, "%s: truncated arrays", path);
    }
  }
  std::fclose(f);
  return st;
}

spg_status spg_csr1_write(const char* path, const spg_host_csr* A) {
  clear_error();
  if (!path || !A) return set_error(SPG_ERR_INVALID_ARG, "null argument");
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(SPG_ERR_IO, "cannot create %s", path);
  int32_t pad = 0;
  bool ok = std::fwrite("CSR1", 1, 4, f) == 4 && std::fwrite(&A->n, 4, 1, f) == 1 &&
            std::fwrite(&pad, 4, 1, f) == 1 && std::fwrite(&A->nnz, 8, 1, f) == 1 &&
            std::fwrite(A->rowptr, 4, (size_t)A->n + 1, f) == (size_t)A->n + 1 &&
            (A->nnz == 0 || (std::fwrite(A->col, 4, (size_t)A->nnz, f) == (size_t)A->nnz &&
                             std::fwrite(A->val, 8, (size_t)A->nnz, f) == (size_t)A->nnz));
  ok = (std::fclose(f) == 0) && ok;
  return ok ? SPG_OK : set_error(SPG_ERR_IO, "write to %s failed", path);
}

spg_status spg_gen_laplace2d(int32_t side, spg_host_csr* out) {
  clear_error();
  if (!out || side < 1 || (int64_t)side * side > INT32_MAX / 5)
    return set_error(SPG_ERR_INVALID_ARG, "bad side %d", side);
  int32_t n = side * side;
  RowBuilder rb(n);
  for (int32_t y = 0; y < side; ++y)
    for (int32_t x = 0; x < side; ++x) {
      int32_t i = y * side + x;
      if (y > 0) { rb.col.push_back(i - side); rb.val.push_back(-1.0); }
      if (x > 0) { rb.col.push_back(i - 1); rb.val.push_back(-1.0); }
      rb.col.push_back(i); rb.val.push_back(4.0);
      if (x + 1 < side) { rb.col.push_back(i + 1); rb.val.push_back(-1.0); }
      if (y + 1 < side) { rb.col.push_back(i + side); rb.val.push_back(-1.0); }
      rb.end_row();
    }
  return rb.finish(out);
}

spg_status spg_gen_stencil27(int32_t side, uint64_t seed, spg_host_csr* out) {
  clear_error();
  if (!out || side < 1 || (int64_t)side * side * side * 27 > INT32_MAX)
    return set_error(SPG_ERR_INVALID_ARG, "bad side %d", side);
  int64_t s = side;
  int32_t n = (int32_t)(s * s * s);
  std::mt19937_64 g(seed);
  RowBuilder rb(n);
  rb.col.reserve((size_t)n * 27);
  rb.val.reserve((size_t)n * 27);
  for (int64_t z = 0; z < s; ++z)
    for (int64_t y = 0; y < s; ++y)
      for (int64_t x = 0; x < s; ++x) {
        for (int dz = -1; dz <= 1; ++dz) {
          int64_t zz = z + dz;
          if (zz < 0 || zz >= s) continue;
          for (int dy = -1; dy <= 1; ++dy) {
            int64_t yy = y + dy;
            if (yy < 0 || yy >= s) continue;
            for (int dx = -1; dx <= 1; ++dx) {
              int64_t xx = x + dx;
              if (xx < 0 || xx >= s) continue;
              rb.col.push_back((int32_t)((zz * s + yy) * s + xx));
              rb.val.push_back(um11(g));
            }
          }
        }
        rb.end_row();
      }
  return rb.finish(out);
}

spg_status spg_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                        uint64_t seed, spg_host_csr* out) {
  clear_error();
  if (!out || scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 ||
      a + b + c > 1.0)
    return set_error(SPG_ERR_INVALID_ARG, "bad R-MAT parameters");
  const int64_t n = (int64_t)1 << scale;
  const int64_t draws = (int64_t)edge_factor * n;
  std::mt19937_64 g(seed);
  std::vector<uint64_t> keys((size_t)draws);
  const double ab = a + b, abc = a + b + c;
  for (int64_t e = 0; e < draws; ++e) {
    uint64_t r = 0, cc = 0;
    for (int lvl = 0; lvl < scale; ++lvl) {
      double u = u01(g);
      uint64_t br = (u >= ab) ? 1u : 0u;                         // quadrants c, d
      uint64_t bc = (u >= a && u < ab) || (u >= abc) ? 1u : 0u;  // quadrants b, d
      r = (r << 1) | br;
      cc = (cc << 1) | bc;
    }
    keys[(size_t)e] = (r << 32) | cc;
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  if (keys.size() > (size_t)INT32_MAX) return set_error(SPG_ERR_UNSUPPORTED, "R-MAT too large");
  spg_status st = alloc_host(out, (int32_t)n, (int64_t)keys.size());
  if (st != SPG_OK) return st;
  size_t p = 0;
  for (int64_t i = 0; i < n; ++i) {
    out->rowptr[i] = (int32_t)p;
    while (p < keys.size() && (int64_t)(keys[p] >> 32) == i) {
      out->col[p] = (int32_t)(keys[p] & 0xffffffffu);
      out->val[p] = u01(g);
      ++p;
    }
  }
  out->rowptr[n] = (int32_t)p;
  return SPG_OK;
}

spg_status spg_gen_banded(int32_t n, int32_t bw, double fill, uint64_t seed, spg_host_csr* out) {
  clear_error();
  if (!out || n < 1 || bw < 0 || fill < 0 || fill > 1)
    return set_error(SPG_ERR_INVALID_ARG, "bad banded parameters");
  std::mt19937_64 g(seed);
  RowBuilder rb(n);
  for (int32_t i = 0; i < n; ++i) {
    int32_t lo = std::max(0, i - bw), hi = std::min(n - 1, i + bw);
    for (int32_t j = lo; j <= hi; ++j) {
      bool keep = (j == i) || (u01(g) < fill);
      if (keep) {
        rb.col.push_back(j);
        rb.val.push_back(um11(g));
      }
    }
    rb.end_row();
    if (rb.col.size() > (size_t)INT32_MAX)
      return set_error(SPG_ERR_UNSUPPORTED, "banded matrix too large");
  }
  return rb.finish(out);
}

// Distinct sorted columns by rejection into a sorted vector (k << n) or a
// shuffle-free complement selection when k is a large fraction of n.
static void draw_columns(std::mt19937_64& g, int32_t n, int32_t k, std::vector<int32_t>& cols) {
  cols.clear();
  if (k <= 0) return;
  if ((int64_t)k * 4 > n) {
    // selection sampling (Knuth's algorithm S): exactly k of n in order
    int32_t need = k;
    for (int32_t j = 0; j < n && need > 0; ++j) {
      if (below(g, (int64_t)n - j) < need) {
        cols.push_back(j);
        --need;
      }
    }
    return;
  }
  while ((int32_t)cols.size() < k) {
    int32_t j = (int32_t)below(g, n);
    auto it = std::lower_bound(cols.begin(), cols.end(), j);
    if (it == cols.end() || *it != j) cols.insert(it, j);
  }
}

spg_status spg_gen_er(int32_t n, double lambda, uint64_t seed, spg_host_csr* out) {
  clear_error();
  if (!out || n < 1 || !(lambda >= 0) || lambda > 1e6)
    return set_error(SPG_ERR_INVALID_ARG, "bad Erdos-Renyi parameters");
  std::mt19937_64 g(seed);
  RowBuilder rb(n);
  std::vector<int32_t> cols;
  const double e = std::exp(-lambda);
  for (int32_t i = 0; i < n; ++i) {
    // Poisson(lambda) by inversion with sequential search
    double u = u01(g), p = e, F = p;
    int32_t k = 0;
    while (u > F && k < n && p > 0) {
      ++k;
      p *= lambda / k;
      F += p;
    }
    k = std::min(k, n);
    draw_columns(g, n, k, cols);
    for (int32_t j : cols) {
      rb.col.push_back(j);
      rb.val.push_back(um11(g));
    }
    rb.end_row();
    if (rb.col.size() > (size_t)INT32_MAX) return set_error(SPG_ERR_UNSUPPORTED, "ER too large");
  }
  return rb.finish(out);
}

spg_status spg_gen_uniform(int32_t n, int32_t per_row, uint64_t seed, spg_host_csr* out) {
  clear_error();
  if (!out || n < 0 || per_row < 0) return set_error(SPG_ERR_INVALID_ARG, "bad parameters");
  std::mt19937_64 g(seed);
  RowBuilder rb(n);
  std::vector<int32_t> cols;
  int32_t k = std::min(per_row, n);
  for (int32_t i = 0; i < n; ++i) {
    draw_columns(g, n, k, cols);
    for (int32_t j : cols) {
      rb.col.push_back(j);
      rb.val.push_back(um11(g));
    }
    rb.end_row();
    if (rb.col.size() > (size_t)INT32_MAX) return set_error(SPG_ERR_UNSUPPORTED, "too large");
  }
  return rb.finish(out);
}

}  // extern "C"
