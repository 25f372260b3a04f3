/*
 * CPU oracle for the sparse x dense execute path — TEST INFRASTRUCTURE ONLY.
 * See plsparse_oracle.h for the contract, the pinning strategy, and the
 * reference file:line each routine restates. Only tests/, bench.py's
 * CPU-baseline leg and __graft_entry__.smoke() may load this library.
 */
#include "plsparse_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ CSR -- */

/* compressed_sparse_rows.cpp:1114-1138 (mode 0) and 1215-1321 (mode 1).
 * Mode 1 keeps the reference's per-row accumulator split: positions at even
 * offsets from the row start go to s0, odd to s1, and s0 + s1 is formed
 * before scaling. The reference's pairing of two rows per iteration does not
 * change any row's arithmetic, so rows are processed independently here. */
#define ORC_CSR_SPMV(NAME, T)                                                  \
  void NAME(int32_t m, const int32_t *row_ptr, const int32_t *col,             \
            const T *vals, const T *x, T *y, T alpha, T beta, int mode) {      \
    const int32_t off = row_ptr[0];                                            \
    _Pragma("omp parallel for schedule(static)") for (int32_t i = 0; i < m;    \
                                                      ++i) {                   \
      const int32_t s = row_ptr[i] - off, e = row_ptr[i + 1] - off;            \
      if (mode == 0) {                                                         \
        T sum = 0;                                                             \
        for (int32_t j = s; j < e; ++j)                                        \
          sum += x[col[j] - off] * vals[j];                                    \
        y[i] = (beta != (T)0) ? y[i] * beta + alpha * sum : alpha * sum;       \
      } else {                                                                 \
        T s0 = 0, s1 = 0;                                                      \
        int32_t j = s;                                                         \
        for (; j < e - 1; j += 2) {                                            \
          s0 += vals[j] * x[col[j] - off];                                     \
          s1 += vals[j + 1] * x[col[j + 1] - off];                             \
        }                                                                      \
        for (; j < e; ++j)                                                     \
          s0 += vals[j] * x[col[j] - off];                                     \
        s0 += s1;                                                              \
        s0 *= alpha;                                                           \
        if (beta != (T)0)                                                      \
          s0 += beta * y[i];                                                   \
        y[i] = s0;                                                             \
      }                                                                        \
    }                                                                          \
  }

ORC_CSR_SPMV(orc_csr_spmv_d, double)
ORC_CSR_SPMV(orc_csr_spmv_s, float)

/* compressed_sparse_rows.cpp:1558-1676: beta scaling (or zeroing) of y,
 * then a scatter of alpha*val*x[row] into y[col], rows in order. */
void orc_csr_spmv_trans_d(int32_t m, int32_t n, const int32_t *row_ptr,
                          const int32_t *col, const double *vals,
                          const double *x, double *y, double alpha,
                          double beta) {
  const int32_t off = row_ptr[0];
  for (int32_t i = 0; i < n; ++i)
    y[i] = (beta == 0.0) ? 0.0 : y[i] * beta;
  for (int32_t i = 0; i < m; ++i)
    for (int32_t j = row_ptr[i] - off; j < row_ptr[i + 1] - off; ++j)
      y[col[j] - off] += alpha * vals[j] * x[i];
}

void orc_csr_absdot_d(int32_t m, const int32_t *row_ptr, const int32_t *col,
                      const double *vals, const double *x, double *out) {
  const int32_t off = row_ptr[0];
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < m; ++i) {
    double s = 0;
    for (int32_t j = row_ptr[i] - off; j < row_ptr[i + 1] - off; ++j)
      s += fabs(vals[j] * x[col[j] - off]);
    out[i] = s;
  }
}

/* ------------------------------------------------------- SELL-C-sigma -- */

typedef struct {
  int64_t key_len; /* row length */
  int64_t row;     /* input row index */
} orc_pair;

/* Descending lexicographic order on (length, row): the order std::sort with
 * std::greater<> gives the reference's std::pair<len, row> elements
 * (sell_c_sigma.cpp:186-202). Ties cannot remain, so qsort's instability
 * does not matter. */
static int orc_pair_desc(const void *a, const void *b) {
  const orc_pair *p = (const orc_pair *)a, *q = (const orc_pair *)b;
  if (p->key_len != q->key_len)
    return p->key_len > q->key_len ? -1 : 1;
  if (p->row != q->row)
    return p->row > q->row ? -1 : 1;
  return 0;
}

static int64_t orc_div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }

void orc_scs_sizes(int32_t m, const int32_t *row_ptr, int32_t C,
                   int32_t sigma, int64_t *out) {
  /* Only the chunk widths are needed: run the permutation part of the
   * builder without the data vectors. */
  const int64_t nC = orc_div_up(m, C);
  int64_t *cs = (int64_t *)malloc(sizeof(int64_t) * (nC ? nC : 1));
  int64_t *cl = (int64_t *)malloc(sizeof(int64_t) * (nC ? nC : 1));
  int64_t *cm = (int64_t *)malloc(sizeof(int64_t) * (nC ? nC : 1));
  int64_t *p1 = (int64_t *)malloc(sizeof(int64_t) * (nC * C ? nC * C : 1));
  int64_t *p2 = (int64_t *)malloc(sizeof(int64_t) * (nC * C ? nC * C : 1));
  int64_t info[3];
  /* col is only read for the column range: pass row_ptr-only mode by a
   * NULL col; the builder skips the range scan then. */
  orc_scs_build_d(m, 0, row_ptr, NULL, NULL, C, sigma, cs, cl, cm, p1, p2,
                  NULL, NULL, info);
  out[0] = nC;
  out[1] = nC ? cs[nC - 1] + cl[nC - 1] * C : 0;
  free(cs);
  free(cl);
  free(cm);
  free(p1);
  free(p2);
}

/* csr2scs (sell_c_sigma.cpp:145-336) followed by gen_data_vectors
 * (sell_c_sigma.cpp:584-705), NOTRANS. */
int orc_scs_build_d(int32_t m, int32_t n, const int32_t *row_ptr,
                    const int32_t *col, const double *vals, int32_t C,
                    int32_t sigma, int64_t *cs, int64_t *cl, int64_t *col_min,
                    int64_t *permd2in, int64_t *in2permd, double *out_vals,
                    int64_t *offsets, int64_t *info) {
  (void)n;
  const int64_t rows = m;
  const int64_t nC = orc_div_up(rows, C);
  int do_sort = 1;
  if (sigma == 0) { /* :175-178 */
    sigma = C;
    do_sort = 0;
  }
  const int64_t sigma_chunks = sigma / C;
  const int64_t nschunks = orc_div_up(rows, sigma);
  const int32_t base = row_ptr[0];

  /* :186-196 windows of sigma (length, row) pairs; unused slots of the last
   * window stay (0, 0), exactly as the reference's value-initialised
   * pairs. */
  orc_pair *w = (orc_pair *)calloc((size_t)(nschunks * sigma ? nschunks * sigma : 1),
                                   sizeof(orc_pair));
  for (int64_t i = 0; i < rows; ++i) {
    w[i].key_len = row_ptr[i + 1] - row_ptr[i];
    w[i].row = i;
  }
  if (do_sort) /* :198-202 */
    for (int64_t s = 0; s < nschunks; ++s)
      qsort(w + s * sigma, (size_t)sigma, sizeof(orc_pair), orc_pair_desc);

  /* :204-225 chunk widths */
  for (int64_t ic = 0; ic < nC; ++ic) {
    const int64_t sid = ic / sigma_chunks, rid = (ic * C) % sigma;
    if (do_sort) {
      cl[ic] = w[sid * sigma + rid].key_len;
    } else {
      int64_t mx = 0;
      for (int64_t r = 0; r < sigma; ++r)
        if (w[sid * sigma + r].key_len > mx)
          mx = w[sid * sigma + r].key_len;
      cl[ic] = mx;
    }
  }
  /* :227-231 chunk starts */
  if (nC > 0)
    cs[0] = 0;
  for (int64_t ic = 1; ic < nC; ++ic)
    cs[ic] = cs[ic - 1] + cl[ic - 1] * C;

  for (int64_t i = 0; i < nC * C; ++i) {
    permd2in[i] = -1;
    in2permd[i] = -1;
  }

  /* :236-250 per-row column range (INT32_MAX / 0 for empty rows) */
  int32_t *rmin = (int32_t *)malloc(sizeof(int32_t) * (rows ? rows : 1));
  int32_t *rmax = (int32_t *)malloc(sizeof(int32_t) * (rows ? rows : 1));
  for (int64_t i = 0; i < rows; ++i) {
    rmin[i] = INT32_MAX;
    rmax[i] = 0;
    if (!col)
      continue;
    for (int32_t j = row_ptr[i] - base; j < row_ptr[i + 1] - base; ++j) {
      const int32_t c = col[j] - base;
      if (c < rmin[i])
        rmin[i] = c;
      if (c > rmax[i])
        rmax[i] = c;
    }
  }

  /* :254-305 chunk column minimum, permutations, global range */
  int64_t range = 0;
  for (int64_t ic = 0; ic < nC; ++ic) {
    const int64_t sid = ic / sigma_chunks, rid = (ic * C) % sigma;
    const orc_pair *cur = &w[sid * sigma + rid];
    const int64_t nr = (rows - ic * C) < C ? (rows - ic * C) : C;
    int32_t cmin = INT32_MAX, cmax = 0;
    for (int64_t r = 0; r < nr; ++r) {
      const int64_t in = cur[r].row;
      if (rmin[in] < cmin)
        cmin = rmin[in];
      if (rmax[in] > cmax)
        cmax = rmax[in];
    }
    const int64_t cr = (int64_t)cmax - (int64_t)cmin;
    if (cr > range)
      range = cr;
    col_min[ic] = cmin;
    for (int64_t r = 0; r < nr; ++r) {
      in2permd[cur[r].row] = ic * C + r;
      permd2in[ic * C + r] = cur[r].row;
    }
  }

  /* :309-320 offset width (signed: a range of 127 fits one byte) */
  int bits = 0;
  while (range) {
    range >>= 1;
    bits++;
  }
  int bytes = bits / 8 + 1;
  if (bytes == 3)
    bytes = 4;
  else if (bytes > 4)
    bytes = 8;

  /* :322-332 full chunks and tidy-up rows */
  int64_t n_full = nC;
  int64_t ntidy = 0;
  if (nC > 0) {
    n_full = permd2in[nC * C - 1] < 0 ? nC - 1 : nC;
    int64_t pad = 0;
    while (pad < C && permd2in[nC * C - pad - 1] < 0)
      pad++;
    ntidy = pad == 0 ? 0 : C - pad;
  }
  info[0] = bytes;
  info[1] = n_full;
  info[2] = ntidy;

  /* gen_data_vectors (:611-704): column-major within chunks; padding columns
   * of a row, and padding rows of the last chunk, hold value 0, offset 0. */
  if (out_vals && offsets && col && vals) {
    for (int64_t ic = 0; ic < nC; ++ic) {
      const int64_t width = cl[ic];
      for (int64_t r = 0; r < C; ++r) {
        const int64_t in = permd2in[ic * C + r];
        int64_t rs = 0, rl = 0;
        if (in >= 0) {
          rs = row_ptr[in] - base;
          rl = row_ptr[in + 1] - row_ptr[in];
        }
        for (int64_t j = 0; j < width; ++j) {
          const int64_t o = cs[ic] + j * C + r;
          if (in >= 0 && j < rl) {
            out_vals[o] = vals[rs + j];
            offsets[o] = (int64_t)(col[rs + j] - base) - col_min[ic];
          } else {
            out_vals[o] = 0.0;
            offsets[o] = 0;
          }
        }
      }
    }
  }
  free(rmin);
  free(rmax);
  free(w);
  return 0;
}

/* sell_c_sigma.cpp:719-797 */
void orc_scs_spmv_d(int64_t nC, int32_t C, const int64_t *cs,
                    const int64_t *cl, const int64_t *col_min,
                    const int64_t *permd2in, const double *vals,
                    const int64_t *offsets, const double *x, double *y,
                    double alpha, double beta) {
#pragma omp parallel for schedule(static)
  for (int64_t ic = 0; ic < nC; ++ic) {
    for (int32_t r = 0; r < C; ++r) {
      double wk = 0.0;
      for (int64_t j = 0; j < cl[ic]; ++j) {
        const int64_t o = cs[ic] + j * C + r;
        wk += vals[o] * x[offsets[o] + col_min[ic]];
      }
      const int64_t dst = permd2in[ic * C + r];
      if (dst > -1)
        y[dst] = (beta != 0.0) ? alpha * wk + beta * y[dst] : alpha * wk;
    }
  }
}

/* sell_c_sigma.cpp:369-379 */
double orc_scs_beta(int64_t nC, int32_t C, const int64_t *cs,
                    const int64_t *cl, int32_t ntidyup, int64_t nnz) {
  const int no_tidy = ntidyup == 0;
  const int64_t par = cs[nC - 1] + no_tidy * cl[nC - 1] * C;
  const int64_t tot = par + cl[nC - 1] * ntidyup;
  return (double)nnz / (double)tot;
}

/* ---------------------------------------------------------------- BSR -- */

/* block_sparse_rows.cpp:458-515 (vanilla; any block size) and 607-742
 * (generic<N>). Each scalar row's sum runs block by block, left to right;
 * the reference's generic kernels keep one partial per (i, j) and reduce at
 * the end, which differs from this only in summation order. Then
 * y = beta*y (or 0) + alpha*sum. */
void orc_bsr_spmv_d(int32_t nrowsb, int32_t bs, int32_t layout,
                    const int32_t *row_ptr, const int32_t *col,
                    const double *vals, const double *x, double *y,
                    double alpha, double beta) {
  const int32_t off = row_ptr[0];
  const int64_t be = (int64_t)bs * bs;
#pragma omp parallel for schedule(static)
  for (int32_t br = 0; br < nrowsb; ++br) {
    for (int32_t i = 0; i < bs; ++i) {
      double sum = 0.0;
      for (int32_t b = row_ptr[br] - off; b < row_ptr[br + 1] - off; ++b) {
        const int64_t c0 = (int64_t)(col[b] - off) * bs;
        for (int32_t j = 0; j < bs; ++j) {
          const double v = layout == 91 ? vals[b * be + (int64_t)i * bs + j]
                                        : vals[b * be + (int64_t)j * bs + i];
          sum += v * x[c0 + j];
        }
      }
      const int64_t r = (int64_t)br * bs + i;
      y[r] = (beta != 0.0 ? y[r] * beta : 0.0) + alpha * sum;
    }
  }
}

/* compressed_sparse_rows.cpp:966-1056 */
int64_t orc_bsr2csr_d(int32_t nrowsb, int32_t bs, int32_t layout,
                      const int32_t *row_ptr, const int32_t *col,
                      const double *vals, int32_t *out_row_ptr,
                      int32_t *out_col, double *out_vals) {
  const int32_t base = row_ptr[0];
  const int64_t be = (int64_t)bs * bs;
  int64_t cnt = 0;
  if (out_row_ptr)
    out_row_ptr[0] = base;
  int64_t rows_done = 0;
  for (int32_t br = 0; br < nrowsb; ++br) {
    const int32_t b0 = row_ptr[br] - base, b1 = row_ptr[br + 1] - base;
    for (int32_t i = 0; i < bs; ++i) {
      for (int32_t b = b0; b < b1; ++b) {
        for (int32_t j = 0; j < bs; ++j) {
          const double v = layout == 91 ? vals[b * be + (int64_t)i * bs + j]
                                        : vals[b * be + (int64_t)j * bs + i];
          if (v == 0.0)
            continue;
          if (out_col) {
            out_col[cnt] = bs * (col[b] - base) + base + j;
            out_vals[cnt] = v;
          }
          cnt++;
        }
      }
      rows_done++;
      if (out_row_ptr)
        out_row_ptr[rows_done] = (int32_t)(cnt + base);
    }
  }
  return cnt;
}

/* General-block-size CSR -> BSR (the canonical layout the B200 converter
 * produces; see header). */
int64_t orc_csr2bsr_d(int32_t m, int32_t n, int32_t bs, int32_t layout,
                      const int32_t *row_ptr, const int32_t *col,
                      const double *vals, int32_t *out_row_ptr,
                      int32_t *out_col, double *out_vals) {
  const int32_t base = row_ptr[0];
  const int32_t nrowsb = m / bs, ncolsb = n / bs;
  const int64_t be = (int64_t)bs * bs;
  int32_t *mark = (int32_t *)malloc(sizeof(int32_t) * (ncolsb ? ncolsb : 1));
  int32_t *list = (int32_t *)malloc(sizeof(int32_t) * (ncolsb ? ncolsb : 1));
  int32_t *slot = (int32_t *)malloc(sizeof(int32_t) * (ncolsb ? ncolsb : 1));
  for (int32_t c = 0; c < ncolsb; ++c)
    mark[c] = -1;
  int64_t nnzb = 0;
  if (out_row_ptr)
    out_row_ptr[0] = base;
  for (int32_t br = 0; br < nrowsb; ++br) {
    int32_t nb = 0;
    for (int32_t i = br * bs; i < (br + 1) * bs; ++i)
      for (int32_t p = row_ptr[i] - base; p < row_ptr[i + 1] - base; ++p) {
        const int32_t cb = (col[p] - base) / bs;
        if (mark[cb] != br) {
          mark[cb] = br;
          list[nb++] = cb;
        }
      }
    /* ascending block columns (insertion sort: block rows are short) */
    for (int32_t a = 1; a < nb; ++a) {
      int32_t v = list[a], b = a - 1;
      while (b >= 0 && list[b] > v) {
        list[b + 1] = list[b];
        b--;
      }
      list[b + 1] = v;
    }
    for (int32_t a = 0; a < nb; ++a)
      slot[list[a]] = a;
    if (out_col) {
      for (int32_t a = 0; a < nb; ++a) {
        out_col[nnzb + a] = list[a] + base;
        memset(out_vals + (nnzb + a) * be, 0, sizeof(double) * be);
      }
      for (int32_t i = br * bs; i < (br + 1) * bs; ++i)
        for (int32_t p = row_ptr[i] - base; p < row_ptr[i + 1] - base; ++p) {
          const int32_t c = col[p] - base;
          const int32_t li = i - br * bs, lj = c % bs;
          const int64_t blk = nnzb + slot[c / bs];
          const int64_t at = layout == 91 ? (int64_t)li * bs + lj
                                          : (int64_t)lj * bs + li;
          out_vals[blk * be + at] = vals[p];
        }
    }
    nnzb += nb;
    if (out_row_ptr)
      out_row_ptr[br + 1] = (int32_t)(nnzb + base);
  }
  free(mark);
  free(list);
  free(slot);
  return nnzb;
}

/* ---------------------------------------------------------------- SpMM -- */

/* compressed_sparse_rows.cpp:1699-1745 */
#define ORC_CSR_SPMM(NAME, T)                                                  \
  void NAME(int32_t m, const int32_t *row_ptr, const int32_t *col,             \
            const T *vals, const T *B, int64_t ldb, T *Cm, int64_t ldc,        \
            int32_t k, T alpha, T beta) {                                      \
    const int32_t off = row_ptr[0];                                            \
    const int use_beta = beta != (T)0 && beta != (T)1;                         \
    _Pragma("omp parallel for schedule(static)") for (int32_t i = 0; i < m;    \
                                                      ++i) {                   \
      T *crow = Cm + (int64_t)i * ldc;                                         \
      if (use_beta)                                                            \
        for (int32_t j = 0; j < k; ++j)                                        \
          crow[j] *= beta;                                                     \
      for (int32_t p = row_ptr[i] - off; p < row_ptr[i + 1] - off; ++p) {      \
        T a = vals[p];                                                         \
        a *= alpha;                                                            \
        const T *brow = B + (int64_t)(col[p] - off) * ldb;                     \
        for (int32_t j = 0; j < k; ++j)                                        \
          crow[j] += a * brow[j];                                              \
      }                                                                        \
    }                                                                          \
  }

ORC_CSR_SPMM(orc_csr_spmm_d, double)
ORC_CSR_SPMM(orc_csr_spmm_s, float)

/* inf_norm_csr.cpp:12-30 */
double orc_csr_inf_norm_d(int32_t m, const int32_t *row_ptr,
                          const double *vals) {
  const int32_t off = row_ptr[0];
  double mx = 0.0;
  for (int32_t i = 0; i < m; ++i) {
    double s = 0.0;
    for (int32_t j = row_ptr[i] - off; j < row_ptr[i + 1] - off; ++j)
      s += fabs(vals[j]);
    if (s > mx || isnan(s))
      mx = s;
  }
  return mx;
}

/* ------------------------------------------------------- COO / CSC input -- */

/* coo2csr (compressed_sparse_rows.cpp:591-640): entries ordered by the key
 * row*n + col, every entry kept (duplicates too), row_ptr from the row
 * counts. The reference sorts (value, key) pairs with std::sort on the key,
 * which leaves the order of equal keys unspecified; this restatement keeps
 * equal keys in input order (two stable counting passes: by column, then by
 * row). Indices are 0-based (the C interface's COO base). */
void orc_coo2csr_d(int32_t m, int32_t n, int64_t nnz, const int32_t *row,
                   const int32_t *col, const double *vals, int32_t *row_ptr,
                   int32_t *col_out, double *vals_out) {
  int64_t *cnt = (int64_t *)calloc((size_t)(n > m ? n : m) + 1, sizeof(int64_t));
  int64_t *tmp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nnz > 0 ? nnz : 1));
  int64_t *ord = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nnz > 0 ? nnz : 1));
  /* pass 1: stable by column */
  for (int64_t i = 0; i < nnz; ++i)
    cnt[col[i] + 1]++;
  for (int32_t j = 0; j < n; ++j)
    cnt[j + 1] += cnt[j];
  for (int64_t i = 0; i < nnz; ++i)
    tmp[cnt[col[i]]++] = i;
  /* pass 2: stable by row */
  memset(cnt, 0, sizeof(int64_t) * ((size_t)(n > m ? n : m) + 1));
  for (int64_t i = 0; i < nnz; ++i)
    cnt[row[i] + 1]++;
  for (int32_t r = 0; r < m; ++r)
    cnt[r + 1] += cnt[r];
  for (int32_t r = 0; r <= m; ++r)
    row_ptr[r] = (int32_t)cnt[r];
  for (int64_t t = 0; t < nnz; ++t) {
    const int64_t i = tmp[t];
    ord[cnt[row[i]]++] = i;
  }
  for (int64_t t = 0; t < nnz; ++t) {
    col_out[t] = col[ord[t]];
    vals_out[t] = vals[ord[t]];
  }
  free(cnt);
  free(tmp);
  free(ord);
}

/* csc2csr (compressed_sparse_rows.cpp:750-800): count entries per row, scan,
 * then walk the columns in order and append each entry to its row, so the
 * columns of every row come out ascending. Index base from col_ptr[0]; the
 * output keeps that base. */
void orc_csc2csr_d(int32_t m, int32_t n, const int32_t *row_indx,
                   const int32_t *col_ptr, const double *vals, int32_t *row_ptr,
                   int32_t *col_out, double *vals_out) {
  const int32_t base = col_ptr[0];
  const int64_t nnz = (int64_t)col_ptr[n] - base;
  int64_t *next = (int64_t *)calloc((size_t)m + 1, sizeof(int64_t));
  for (int64_t k = 0; k < nnz; ++k)
    next[row_indx[k] - base + 1]++;
  for (int32_t r = 0; r < m; ++r)
    next[r + 1] += next[r];
  for (int32_t r = 0; r <= m; ++r)
    row_ptr[r] = (int32_t)next[r] + base;
  for (int32_t j = 0; j < n; ++j)
    for (int64_t k = col_ptr[j] - base; k < col_ptr[j + 1] - base; ++k) {
      const int32_t r = row_indx[k] - base;
      const int64_t o = next[r]++;
      col_out[o] = j + base;
      vals_out[o] = vals[k];
    }
  free(next);
}
