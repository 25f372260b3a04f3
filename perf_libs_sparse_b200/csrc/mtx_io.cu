// Matrix Market reader (host only): coordinate files -> 0-based CSR.
//
// Reads what the reference's benchmark driver reads
// (bench/pl_bench_sparse_x_dense.c:124-240): a "%%MatrixMarket matrix
// coordinate <field> <symmetry>" header, '%' comment lines, a size line
// "m n entries", then 1-based "row col [value]" entries. Fields real,
// integer and pattern (value 1.0); symmetric and hermitian files add the
// mirrored entry of every off-diagonal entry, skew-symmetric ones add it
// negated. Entries are ordered by (row, column); entries at the same
// position are all kept, in file order.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/perflibs_b200.h"

namespace {

struct Entry {
  int32_t r, c;
  double v;
};

bool lower_eq(const char *a, const char *b) {
  for (; *a && *b; ++a, ++b)
    if (std::tolower((unsigned char)*a) != std::tolower((unsigned char)*b))
      return false;
  return *a == *b;
}

struct FileCloser {
  void operator()(FILE *f) const { std::fclose(f); }
};

perflibs_status_t read_mtx_file(const char *path, int32_t *m, int32_t *n, int64_t *nnz,
                                 int32_t **row_ptr, int32_t **col_indx, double **vals) {
  std::unique_ptr<FILE, FileCloser> fh(std::fopen(path, "r"));  // closed on every exit
  FILE *f = fh.get();
  if (!f)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  std::vector<Entry> e;
  perflibs_status_t st = PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  char line[1024];
  char obj[64], fmt[64], field[64], sym[64];
  long long mm = 0, nn = 0, ne = 0;
  do {
    if (!std::fgets(line, sizeof line, f) ||
        std::sscanf(line, "%%%%MatrixMarket %63s %63s %63s %63s", obj, fmt, field, sym) != 4 ||
        !lower_eq(obj, "matrix") || !lower_eq(fmt, "coordinate") || lower_eq(field, "complex"))
      break;
    const bool pattern = lower_eq(field, "pattern");
    const bool general = lower_eq(sym, "general");
    const bool skew = lower_eq(sym, "skew-symmetric");
    if (!general && !skew && !lower_eq(sym, "symmetric") && !lower_eq(sym, "hermitian"))
      break;
    bool sized = false;
    while (std::fgets(line, sizeof line, f)) {
      if (line[0] == '%')
        continue;
      sized = std::sscanf(line, "%lld %lld %lld", &mm, &nn, &ne) == 3;
      break;
    }
    if (!sized || mm < 0 || nn < 0 || ne < 0 || mm > INT32_MAX || nn > INT32_MAX)
      break;
    e.reserve((size_t)ne * (general ? 1 : 2));
    bool ok = true;
    for (long long i = 0; i < ne && ok; ++i) {
      long long r = 0, c = 0;
      double v = 1.0;
      ok = pattern ? std::fscanf(f, "%lld %lld", &r, &c) == 2
                   : std::fscanf(f, "%lld %lld %lf", &r, &c, &v) == 3;
      ok = ok && r >= 1 && r <= mm && c >= 1 && c <= nn;
      if (!ok)
        break;
      e.push_back({(int32_t)(r - 1), (int32_t)(c - 1), v});
      if (!general && r != c)
        e.push_back({(int32_t)(c - 1), (int32_t)(r - 1), skew ? -v : v});
    }
    if (!ok)
      break;
    st = PERFLIBS_STATUS_SUCCESS;
  } while (false);
  fh.reset();
  if (st != PERFLIBS_STATUS_SUCCESS)
    return st;

  std::stable_sort(e.begin(), e.end(), [](const Entry &a, const Entry &b) {
    return a.r != b.r ? a.r < b.r : a.c < b.c;
  });
  const size_t cnt = e.size();
  int32_t *rp = (int32_t *)std::calloc((size_t)mm + 1, sizeof(int32_t));
  int32_t *ci = (int32_t *)std::malloc(sizeof(int32_t) * std::max<size_t>(cnt, 1));
  double *vv = (double *)std::malloc(sizeof(double) * std::max<size_t>(cnt, 1));
  if (!rp || !ci || !vv || cnt > (size_t)INT32_MAX) {
    std::free(rp);
    std::free(ci);
    std::free(vv);
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
  for (size_t i = 0; i < cnt; ++i) {
    rp[e[i].r + 1]++;
    ci[i] = e[i].c;
    vv[i] = e[i].v;
  }
  for (long long r = 0; r < mm; ++r)
    rp[r + 1] += rp[r];
  *m = (int32_t)mm;
  *n = (int32_t)nn;
  *nnz = (int64_t)cnt;
  *row_ptr = rp;
  *col_indx = ci;
  *vals = vv;
  return PERFLIBS_STATUS_SUCCESS;
}

}  // namespace

// A size line asking for more entries than host memory holds is an
// execution failure, as is any other host allocation failure: no exception
// leaves the C interface.
extern "C" perflibs_status_t perflibs_b200_read_mtx(const char *path, int32_t *m, int32_t *n,
                                                    int64_t *nnz, int32_t **row_ptr,
                                                    int32_t **col_indx, double **vals) {
  if (!path || !m || !n || !nnz || !row_ptr || !col_indx || !vals)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  *row_ptr = nullptr;
  *col_indx = nullptr;
  *vals = nullptr;
  try {
    return read_mtx_file(path, m, n, nnz, row_ptr, col_indx, vals);
  } catch (...) {
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
}
