/*
 * CPU oracle for the SpGEMM hot path — TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
 * this file, as the checker and the timed CPU baseline.  The engine never
 * links or calls it.
 *
 * It restates, in plain C, what the reference computes:
 *  - Gustavson's row-wise product C = A·B (report/REPORT.md:56-62): row i of C
 *    is Σ_{k in row i of A} A[i,k]·B[k,:]; B = A for "AA", B = Aᵀ for "AAt"
 *    and "AAtS" (src/spgemm_engine.cuh:3-5, :134).
 *  - Structural semantics: every (i,j) reached by some product is an entry,
 *    also when its value cancels to 0.0 (report/CORRECTNESS_NOTES.md:3-16;
 *    the reference keeps them, cuSPARSE keeps them, scipy prunes them).
 *  - Column indices sorted within each row: the reference's canonical order
 *    after its radix sort on i·n+j (src/spgemm_engine.cuh:178-195).
 *  - Order-independent checksums Σv, Σ|v|, Σv² summed in index order
 *    (checksum(), src/spgemm_engine.cuh:116-118).
 *  - Product counts: A·A Σ_{(i,k)} nnz(A_k), A·Aᵀ Σ_k colcount(k)²
 *    (k_flops, src/spgemm_engine.cuh:47-50; est_outputs,
 *    bench/run_baseline.py:38-44).
 * The reference accumulates with atomicAdd(double) in run-dependent order
 * (src/spgemm_engine.cuh:104).  This oracle fixes one order: each value is
 * acc = 0.0, then acc = acc + round(a_ik·b_kj) for k in increasing position
 * of row i of A.  Built with -ffp-contract=off so no multiply-add is fused.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  int32_t* mark;
  double* acc;
  int32_t* list;
} spa_t;

static int spa_init(spa_t* s, int32_t n) {
  s->mark = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  s->acc = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  s->list = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  if (!s->mark || !s->acc || !s->list) return -1;
  for (int32_t j = 0; j < n; ++j) s->mark[j] = -1;
  return 0;
}

static void spa_free(spa_t* s) {
  free(s->mark);
  free(s->acc);
  free(s->list);
}

static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

static void sort_cols(int32_t* v, int64_t m) {
  if (m > 48) {
    qsort(v, (size_t)m, sizeof(int32_t), cmp_i32);
    return;
  }
  for (int64_t i = 1; i < m; ++i) {
    int32_t x = v[i];
    int64_t j = i - 1;
    while (j >= 0 && v[j] > x) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = x;
  }
}

/* Number of distinct columns of row i of A·B.  `stamp` marks the columns
 * seen in this visit: distinct for every visit made with one accumulator. */
static int64_t row_count(spa_t* s, int32_t i, int32_t stamp, const int32_t* Ap,
                         const int32_t* Ai, const int32_t* Bp, const int32_t* Bi) {
  int64_t c = 0;
  for (int32_t p = Ap[i]; p < Ap[i + 1]; ++p) {
    int32_t k = Ai[p];
    for (int32_t q = Bp[k]; q < Bp[k + 1]; ++q) {
      int32_t j = Bi[q];
      if (s->mark[j] != stamp) {
        s->mark[j] = stamp;
        ++c;
      }
    }
  }
  return c;
}

/* Row i of A·B: sorted columns into cols, values into vals; returns count. */
static int64_t row_fill(spa_t* s, int32_t i, int32_t stamp, const int32_t* Ap,
                        const int32_t* Ai, const double* Ax, const int32_t* Bp,
                        const int32_t* Bi, const double* Bx, int32_t* cols, double* vals) {
  int64_t m = 0;
  for (int32_t p = Ap[i]; p < Ap[i + 1]; ++p) {
    int32_t k = Ai[p];
    double a = Ax[p];
    for (int32_t q = Bp[k]; q < Bp[k + 1]; ++q) {
      int32_t j = Bi[q];
      double v = a * Bx[q];
      if (s->mark[j] != stamp) {
        s->mark[j] = stamp;
        s->acc[j] = 0.0;
        s->list[m++] = j;
      }
      s->acc[j] = s->acc[j] + v;
    }
  }
  sort_cols(s->list, m);
  for (int64_t t = 0; t < m; ++t) {
    cols[t] = s->list[t];
    vals[t] = s->acc[s->list[t]];
  }
  return m;
}

/* Per-row distinct counts of C = A·B (rownnz: n entries); returns nnz(C). */
int64_t oracle_count(int32_t n, const int32_t* Ap, const int32_t* Ai, const int32_t* Bp,
                     const int32_t* Bi, int64_t* rownnz, int nthreads) {
  int64_t total = 0;
  int failed = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel reduction(+ : total) reduction(| : failed)
#endif
  {
    spa_t s;
    if (spa_init(&s, n) != 0) {
      failed = 1;
    } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
      for (int32_t i = 0; i < n; ++i) {
        int64_t c = row_count(&s, i, i, Ap, Ai, Bp, Bi);
        rownnz[i] = c;
        total += c;
      }
    }
    spa_free(&s);
  }
  return failed ? -1 : total;
}

/* Fill C given its row pointers Cp (n+1, from the counts). Returns 0 or -1. */
int oracle_fill(int32_t n, const int32_t* Ap, const int32_t* Ai, const double* Ax,
                const int32_t* Bp, const int32_t* Bi, const double* Bx, const int64_t* Cp,
                int32_t* Ci, double* Cx, int nthreads) {
  int failed = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel reduction(| : failed)
#endif
  {
    spa_t s;
    if (spa_init(&s, n) != 0) {
      failed = 1;
    } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
      for (int32_t i = 0; i < n; ++i) {
        int64_t m = row_fill(&s, i, i, Ap, Ai, Ax, Bp, Bi, Bx, Ci + Cp[i], Cx + Cp[i]);
        if (m != Cp[i + 1] - Cp[i]) failed = 1;
      }
    }
    spa_free(&s);
  }
  return failed ? -1 : 0;
}

/* Aᵀ by a sequential stable counting sort: rows of Aᵀ list i ascending. */
void oracle_transpose(int32_t n, const int32_t* Ap, const int32_t* Ai, const double* Ax,
                      int32_t* Tp, int32_t* Ti, double* Tx) {
  int64_t nnz = Ap[n];
  for (int32_t k = 0; k <= n; ++k) Tp[k] = 0;
  for (int64_t p = 0; p < nnz; ++p) Tp[Ai[p] + 1]++;
  for (int32_t k = 0; k < n; ++k) Tp[k + 1] += Tp[k];
  int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  for (int32_t k = 0; k < n; ++k) cur[k] = Tp[k];
  for (int32_t i = 0; i < n; ++i)
    for (int32_t p = Ap[i]; p < Ap[i + 1]; ++p) {
      int32_t d = cur[Ai[p]]++;
      Ti[d] = i;
      Tx[d] = Ax[p];
    }
  free(cur);
}

/* Σ_{(i,k)} nnz(B_k): intermediate products of A·B. */
int64_t oracle_products(int32_t n, const int32_t* Ap, const int32_t* Ai, const int32_t* Bp) {
  int64_t f = 0;
  int64_t nnz = Ap[n];
  for (int64_t p = 0; p < nnz; ++p) f += Bp[Ai[p] + 1] - Bp[Ai[p]];
  return f;
}

/* Σv, Σ|v|, Σv² in index order. */
void oracle_checksum(const double* v, int64_t m, double* out3) {
  double s = 0, as = 0, sq = 0;
  for (int64_t t = 0; t < m; ++t) {
    double x = v[t];
    s += x;
    as += x < 0 ? -x : x;
    sq += x * x;
  }
  out3[0] = s;
  out3[1] = as;
  out3[2] = sq;
}

/*
 * CPU baseline: compute rows [r0, r1) of C = A·B, each row into a per-thread
 * buffer reused across rows, so any size streams through bounded memory.
 * Returns nnz of the rows, or -1; checksums of their values into chk3 (summed
 * per thread, so they are for reporting, not for parity).
 */
int64_t oracle_rows_stream(int32_t n, const int32_t* Ap, const int32_t* Ai, const double* Ax,
                           const int32_t* Bp, const int32_t* Bi, const double* Bx, int32_t r0,
                           int32_t r1, int nthreads, double* chk3) {
  int64_t total = 0;
  int failed = 0;
  double s = 0, as = 0, sq = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel reduction(+ : total, s, as, sq) reduction(| : failed)
#endif
  {
    spa_t sp;
    int32_t* cols = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    double* vals = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (spa_init(&sp, n) != 0 || !cols || !vals) {
      failed = 1;
    } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
      for (int32_t i = r0; i < r1; ++i) {
        int64_t m = row_fill(&sp, i, i, Ap, Ai, Ax, Bp, Bi, Bx, cols, vals);
        total += m;
        for (int64_t t = 0; t < m; ++t) {
          double x = vals[t];
          s += x;
          as += x < 0 ? -x : x;
          sq += x * x;
        }
      }
    }
    spa_free(&sp);
    free(cols);
    free(vals);
  }
  if (chk3) {
    chk3[0] = s;
    chk3[1] = as;
    chk3[2] = sq;
  }
  return failed ? -1 : total;
}

/*
 * A sample of rows of C = A·B (rows[0..m), any order, for checking products
 * too large to hold whole): their distinct counts into rownnz[0..m); returns
 * the total, or -1.
 */
int64_t oracle_rows_count(int32_t n, const int32_t* Ap, const int32_t* Ai, const int32_t* Bp,
                          const int32_t* Bi, const int32_t* rows, int32_t m, int64_t* rownnz,
                          int nthreads) {
  int64_t total = 0;
  int failed = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel reduction(+ : total) reduction(| : failed)
#endif
  {
    spa_t s;
    if (spa_init(&s, n) != 0) {
      failed = 1;
    } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
      for (int32_t t = 0; t < m; ++t) {
        int64_t c = row_count(&s, rows[t], t, Ap, Ai, Bp, Bi);
        rownnz[t] = c;
        total += c;
      }
    }
    spa_free(&s);
  }
  return failed ? -1 : total;
}

/* The sampled rows themselves, into Ci/Cx at offsets Cp (m+1, from the
 * counts).  Returns 0 or -1. */
int oracle_rows_fill(int32_t n, const int32_t* Ap, const int32_t* Ai, const double* Ax,
                     const int32_t* Bp, const int32_t* Bi, const double* Bx, const int32_t* rows,
                     int32_t m, const int64_t* Cp, int32_t* Ci, double* Cx, int nthreads) {
  int failed = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel reduction(| : failed)
#endif
  {
    spa_t s;
    if (spa_init(&s, n) != 0) {
      failed = 1;
    } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
      for (int32_t t = 0; t < m; ++t) {
        int64_t c = row_fill(&s, rows[t], t, Ap, Ai, Ax, Bp, Bi, Bx, Ci + Cp[t], Cx + Cp[t]);
        if (c != Cp[t + 1] - Cp[t]) failed = 1;
      }
    }
    spa_free(&s);
  }
  return failed ? -1 : 0;
}

/*
 * The 27-point stencil on a side³ grid as the benchmark defines it, for the
 * CPU legs that must not load the engine library: rows in z, y, x order,
 * neighbours in dz, dy, dx order (each −1..1, inside the grid), so columns
 * ascend; values um11(x) = 2·((x >> 11)·2^-53) − 1 of consecutive draws x of
 * MT19937-64 (Matsumoto and Nishimura's 64-bit Mersenne Twister, the engine of
 * C++'s std::mt19937_64) seeded with `seed`, one draw per entry in CSR order.
 * rowptr has side³+1 entries; col and val (3·side − 2)³.
 */
typedef struct {
  uint64_t mt[312];
  int i;
} mt64_t;

static void mt64_seed(mt64_t* g, uint64_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 312; ++i)
    g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
  g->i = 312;
}

static uint64_t mt64_next(mt64_t* g) {
  const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
  const uint64_t mat = 0xB5026F5AA96619E9ULL;
  if (g->i >= 312) {
    for (int k = 0; k < 312; ++k) {
      uint64_t y = (g->mt[k] & upper) | (g->mt[(k + 1) % 312] & lower);
      g->mt[k] = g->mt[(k + 156) % 312] ^ (y >> 1) ^ ((y & 1ULL) ? mat : 0ULL);
    }
    g->i = 0;
  }
  uint64_t x = g->mt[g->i++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= x >> 43;
  return x;
}

int64_t oracle_gen_stencil27(int32_t side, uint64_t seed, int32_t* rowptr, int32_t* col,
                             double* val) {
  const int64_t s = side;
  mt64_t g;
  mt64_seed(&g, seed);
  int64_t p = 0, row = 0;
  rowptr[0] = 0;
  for (int64_t z = 0; z < s; ++z)
    for (int64_t y = 0; y < s; ++y)
      for (int64_t x = 0; x < s; ++x) {
        for (int dz = -1; dz <= 1; ++dz) {
          const int64_t zz = z + dz;
          if (zz < 0 || zz >= s) continue;
          for (int dy = -1; dy <= 1; ++dy) {
            const int64_t yy = y + dy;
            if (yy < 0 || yy >= s) continue;
            for (int dx = -1; dx <= 1; ++dx) {
              const int64_t xx = x + dx;
              if (xx < 0 || xx >= s) continue;
              col[p] = (int32_t)((zz * s + yy) * s + xx);
              val[p] = 2.0 * ((double)(mt64_next(&g) >> 11) * 0x1.0p-53) - 1.0;
              ++p;
            }
          }
        }
        rowptr[++row] = (int32_t)p;
      }
  return p;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
