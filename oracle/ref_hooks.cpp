/*
 * C-linkage hooks into the reference library's internals, compiled together
 * with the reference sources into oracle/_ref/libplsparse_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ (golden data, parity checks) and by
 * bench.py's CPU-baseline leg. Nothing in the shipped B200 library links it.
 *
 * The hooks reach three deterministic modes of the reference that its public
 * API cannot select on its own:
 *   - the CSR -> SELL-C-sigma conversion for any chunk height C (including
 *     C=32, which the reference never executes), via csr2scs +
 *     gen_parallel_decomp + gen_data_vectors (src/sell_c_sigma.cpp:145-336,
 *     464-552, 584-705);
 *   - forcing the SELL path at optimize time, via the internal knobs set_C /
 *     set_sigma / set_time_limit (src/matrix_state.cpp:434-457);
 *   - reading back which format and SELL parameters the auditioner chose
 *     (src/types.hpp:97-125).
 */
#include "matrix_state.hpp"
#include "sell_c_sigma.hpp"
#include "types.hpp"

#include <cstdint>
#include <cstring>

using perflibs::sparse::perflibs_scs;

namespace {
struct ref_scs_box {
  perflibs_scs<double> scs;
};
} // namespace

extern "C" {

/* Build a SELL-C-sigma layout with the reference's own builder.
 * sigma is in rows (a multiple of C, or 0 for no sorting). nthreads fixes the
 * decomposition used for the first-touch copy; it does not change the
 * layout. */
void *ref_scs_build_d(int32_t m, int32_t n, const int32_t *row_ptr,
                      const int32_t *col_indx, const double *vals, int32_t C,
                      int32_t sigma, int32_t nthreads) {
  auto box = new ref_scs_box;
  box->scs = perflibs::sparse::csr2scs<double>(
      PERFLIBS_OPERATION_NOTRANS, m, n, vals, col_indx, row_ptr, C, sigma,
      nthreads, {nullptr, nullptr});
  box->scs.gen_parallel_decomp(
      perflibs::sparse::perflibs_scs_parallel_chunk_division);
  box->scs.gen_data_vectors(PERFLIBS_OPERATION_NOTRANS, row_ptr, col_indx,
                            vals);
  return box;
}

/* Scalars: nC, C, sigma, col_indx_bytes, n_full_chunks, ntidyup, data size. */
void ref_scs_info(void *h, int64_t *out7) {
  auto &s = static_cast<ref_scs_box *>(h)->scs;
  out7[0] = s.nC;
  out7[1] = s.C;
  out7[2] = s.sigma;
  out7[3] = s.col_indx_bytes;
  out7[4] = s.n_full_chunks;
  out7[5] = s.ntidyup;
  out7[6] = (int64_t)s.vals.size();
}

double ref_scs_beta(void *h, int32_t nnz) {
  return static_cast<ref_scs_box *>(h)->scs.get_beta(nnz);
}

/* Copy out the arrays. cs, cl, col_min have nC entries; perm has nC*C;
 * vals has data-size entries; offsets has data-size * col_indx_bytes bytes. */
void ref_scs_arrays(void *h, int64_t *cs, int64_t *cl, int64_t *col_min,
                    int64_t *permd2in, int64_t *in2permd, double *vals,
                    void *offsets) {
  auto &s = static_cast<ref_scs_box *>(h)->scs;
  std::memcpy(cs, s.cs.data(), sizeof(int64_t) * s.nC);
  std::memcpy(cl, s.cl.data(), sizeof(int64_t) * s.nC);
  std::memcpy(col_min, s.col_indx_min.data(), sizeof(int64_t) * s.nC);
  std::memcpy(permd2in, s.row_permd2in.data(),
              sizeof(int64_t) * (size_t)s.nC * s.C);
  std::memcpy(in2permd, s.row_in2permd.data(),
              sizeof(int64_t) * (size_t)s.nC * s.C);
  std::memcpy(vals, s.vals.data(), sizeof(double) * s.vals.size());
  std::memcpy(offsets, s.col_indx_offsets.data(),
              (size_t)s.col_indx_bytes * s.vals.size());
}

/* Run the reference's generic C++ SELL kernel spmv_scs<double, C> for
 * C in 2..16 (even). Returns 0 on success, 1 for an unsupported C. */
int ref_scs_spmv_d(void *h, const double *x, double *y, double alpha,
                   double beta) {
  auto &s = static_cast<ref_scs_box *>(h)->scs;
  if (s.C < 2 || s.C > 16 || (s.C % 2) != 0)
    return 1;
  perflibs::sparse::spmv_scs_opt<double>(s, x, y, alpha, beta);
  return 0;
}

void ref_scs_free(void *h) { delete static_cast<ref_scs_box *>(h); }

/* Internal knobs of the reference handle. */
void ref_set_C_sigma_d(perflibs_spmat_t A, int C, int sigma_mult) {
  perflibs::sparse::set_C<double>(A, C);
  perflibs::sparse::set_sigma<double>(A, sigma_mult);
}
void ref_set_time_limit_d(perflibs_spmat_t A, double tl) {
  perflibs::sparse::set_time_limit<double>(A, tl);
}

/* Current live format of a double handle (the reference's spmat_format_t
 * value), plus C / sigma when it is SELL-C-sigma. */
int ref_format_d(perflibs_spmat_t A, int *C, int *sigma) {
  auto impl = reinterpret_cast<perflibs_spmat_impl_t<double> *>(A->impl);
  if (C)
    *C = impl->scs.C;
  if (sigma)
    *sigma = impl->scs.sigma;
  return (int)impl->spmat_format;
}
}
