// CPU replay of the TMA-staged diagonal-form SpMM (k_spmm_dia_tma in
// perf_libs_sparse_b200/csrc/spmm_dia.cu) over the plan the library computes
// (dia_tma_shape in csrc/dia_plan.hpp), before any GPU runs it. For each
// matrix shape (diagonal offsets, rows), k and element sizes it follows
// every CTA's sequence of work items, copies and waits as the kernel issues
// them, and every thread's reads, and checks that
//   * every copy fits its slot or slab, starts 128-byte (windows) or
//     16-byte (values) aligned, with the tensor copy's inner coordinate on a
//     16-byte boundary and at most 256 rows per box;
//   * a copy is only issued into a slot whose previous copy was waited for
//     and whose window no later group of the tile still reads, and every
//     copy is waited for exactly once, before its first read;
//   * every window row a thread reads lies inside the slot and holds B's row
//     row + offset for the entry it is used with;
//   * every value read lies inside its slab, and every slab copy inside the
//     padded diagonal-form buffer;
//   * every element of C (row < m, column < k) is written exactly once;
//   * shared memory fits one CTA.
// It also replays the line-patch plan of the kernel that reads B through L1
// (k_spmm_dia: dia_patch_plan / dia_patch_unit in the same header) over
// every CTA and thread: every unit of rows is computed exactly once, and
// each patch CTA holds whole line segments.
// Prints "ok <cases>" or the first violation (exit status 1).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "dia_plan.hpp"

using namespace pls;

// Rows per thread of the kernel.
static const int kTR = kDiaTmaThreadRows;

static int g_fail = 0;
#define CHECK(cond, ...)                                   \
  do {                                                     \
    if (!(cond)) {                                         \
      std::fprintf(stderr, "violation: %s | ", #cond);     \
      std::fprintf(stderr, __VA_ARGS__);                   \
      std::fprintf(stderr, "\n");                          \
      std::exit(1);                                        \
    }                                                      \
  } while (0)

struct Case {
  std::string name;
  int32_t m;
  std::vector<int32_t> offs;
  std::vector<int> ks = {4, 8, 16, 24, 32, 40, 128, 200};
};

static std::vector<int32_t> stencil3d(int g, bool full27) {
  std::vector<int32_t> o;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        if (!full27 && (dz != 0) + (dy != 0) + (dx != 0) > 1)
          continue;
        o.push_back(dz * g * g + dy * g + dx);
      }
  std::sort(o.begin(), o.end());
  return o;
}

static std::vector<int32_t> stencil2d(int g, bool nine) {
  std::vector<int32_t> o;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      if (!nine && dy != 0 && dx != 0)
        continue;
      o.push_back(dy * g + dx);
    }
  std::sort(o.begin(), o.end());
  return o;
}

static std::vector<int32_t> band(int lo, int hi) {
  std::vector<int32_t> o;
  for (int i = lo; i <= hi; ++i)
    o.push_back(i);
  return o;
}

// One (case, k, element sizes) replay. Returns whether the plan applied.
static bool replay(const Case &cs, int k, int xb, int vb, int sms) {
  const int nd = (int)cs.offs.size();
  const DiaTmaShape sh = dia_tma_shape(cs.offs.data(), nd, cs.m, k, xb, vb, sms);
  if (!sh.ok)
    return false;
  const DiaTmaArgs &a = sh.a;
  // RB: rows of a value block; TR: rows per thread (the kernel's
  // kDiaTmaThreadRows), 4 * 256 / TR threads.
  const int VEC = 16 / xb, NV = sh.NV, KS = NV * VEC, RB = kDiaRows, L = sh.L, TR = kTR;
  const int NT = kDiaRows * kDiaTmaThreads / TR;
  const int row_bytes = KS * xb;
  const int64_t slot_rows = (int64_t)a.NB * a.BR;
  const char *nm = cs.name.c_str();
  CHECK(L == kDiaTmaThreads / NV * RB && L == NT / NV * TR, "%s", nm);
  CHECK(sh.smem + 128 <= 227 * 1024, "%s smem %zu", nm, sh.smem);  // + alignment room
  CHECK(a.S >= 1 && a.S <= kDiaTmaMaxSlots && a.G >= 1 && a.G <= a.S, "%s S %d G %d", nm, a.S, a.G);
  CHECK(a.BR >= 1 && a.BR <= 256, "%s BR %d", nm, a.BR);
  CHECK(a.slot_bytes == slot_rows * row_bytes, "%s", nm);
  CHECK(((int64_t)a.BR * row_bytes) % 128 == 0, "%s box bytes", nm);
  CHECK(row_bytes % 16 == 0, "%s row bytes", nm);
  CHECK(a.vslab_bytes % 16 == 0, "%s vslab", nm);
  // the slab: values (copied from the 16-byte boundary below their start),
  // then from f_at the blocks' masks (copied the same way)
  const int64_t f_at = (((int64_t)L * nd * vb + 15) / 16) * 16 + 16;
  CHECK(((int64_t)a.S * a.slot_bytes) % 128 == 0, "%s slab base", nm);
  CHECK(a.grp_run0[0] == 0 && a.grp_run0[a.G] <= kDiaMax, "%s runs", nm);
  const int64_t dia_elems = plan_div_up((int64_t)cs.m + kDiaPadRows, RB) * nd * RB;
  const int64_t dia_bytes = dia_elems * vb + 16;  // the allocation, with its slack
  const int64_t full_bytes = plan_div_up((int64_t)cs.m + kDiaPadRows, RB) * 4 + 16;
  const bool early = a.S > a.G;
  const unsigned grid = (unsigned)std::min<int64_t>(a.n_items, sms);
  // Every run's diagonals and window rows.
  int runs_seen = 0;
  for (int g = 0; g < a.G; ++g)
    for (int r = a.grp_run0[g]; r < a.grp_run0[g + 1]; ++r) {
      CHECK(a.run_len[r] >= 1 && a.run_len[r] <= kDiaRun, "%s run len", nm);
      for (int l = 0; l < a.run_len[r]; ++l) {
        CHECK(a.run_d0[r] + l == runs_seen, "%s diagonals in order", nm);
        ++runs_seen;
      }
    }
  CHECK(runs_seen == nd, "%s every diagonal once (%d of %d)", nm, runs_seen, nd);

  std::vector<uint8_t> written((size_t)cs.m * (size_t)plan_div_up(k, VEC), 0);
  for (unsigned cta = 0; cta < grid; ++cta) {
    // slot -> window held (-1 none), issued-not-waited, waited
    std::vector<int64_t> slot_win(a.S, INT64_MIN);
    std::vector<int> slot_pending(a.S, 0), slot_ready(a.S, 0);
    int64_t vslab_tile[2] = {INT64_MIN, INT64_MIN};
    int vpending[2] = {0, 0}, vready[2] = {0, 0};
    for (int64_t item = cta; item < a.n_items; item += grid) {
      const int slice = (int)(item % a.n_slices);
      const int64_t rest = item / a.n_slices;
      const int chain = (int)(rest % a.n_chains);
      const int seg = (int)(rest / a.n_chains);
      const int k0 = slice * KS;
      const int64_t b = (int64_t)chain * L;
      const int rows_tile = (int)std::min<int64_t>(L, (int64_t)a.P - b);
      CHECK(rows_tile > 0, "%s rows_tile", nm);
      const int64_t tiles = b < a.m ? ((int64_t)a.m - b + a.P - 1) / a.P : 0;
      const int t0 = seg * a.Z;
      const int t1 = (int)std::min<int64_t>((int64_t)t0 + a.Z, tiles);
      if (t0 >= t1)
        continue;
      // window ids are unique per (item, w)
      const int64_t wid_base = item * 1000000;
      auto issue_window = [&](int w) {
        const int s = w % a.S;
        CHECK(!slot_pending[s], "%s issue into a pending slot", nm);
        CHECK(((int64_t)k0 * xb) % 16 == 0, "%s inner coordinate", nm);
        const int64_t row0 = b + (int64_t)w * a.P + a.win0;
        CHECK(row0 > INT32_MIN / 2 && row0 + slot_rows < INT32_MAX / 2, "%s coordinate range", nm);
        slot_win[s] = wid_base + w;
        slot_pending[s] = 1;
        slot_ready[s] = 0;
      };
      auto issue_vals = [&](int t) {
        const int s = t & 1;
        CHECK(!vpending[s], "%s vals issue into a pending slab", nm);
        const int64_t R = b + (int64_t)t * a.P;
        CHECK(R % RB == 0, "%s tile start on a block", nm);
        const int64_t v0 = R * nd * vb;
        const int64_t lo = v0 & ~(int64_t)15;
        const int64_t hi = (v0 + (int64_t)L * nd * vb + 15) & ~(int64_t)15;
        CHECK(lo >= 0 && hi <= dia_bytes, "%s vals copy inside the buffer", nm);
        CHECK(hi - lo <= f_at && (hi - lo) % 16 == 0, "%s vals copy fits before the masks", nm);
        CHECK((v0 - lo) + (int64_t)L * nd * vb <= hi - lo, "%s vals inside the copy", nm);
        const int64_t f0 = (R / RB) * 4;
        const int64_t flo = f0 & ~(int64_t)15;
        const int64_t fhi = (f0 + (L / RB) * 4 + 15) & ~(int64_t)15;
        CHECK(flo >= 0 && fhi <= full_bytes, "%s mask copy inside the buffer", nm);
        CHECK(f_at + (fhi - flo) <= a.vslab_bytes && f_at % 16 == 0, "%s mask copy fits the slab", nm);
        CHECK((f0 - flo) % 4 == 0, "%s mask alignment", nm);
        vslab_tile[s] = wid_base + t;
        vpending[s] = 1;
        vready[s] = 0;
      };
      auto wait_window = [&](int s) {
        CHECK(slot_pending[s], "%s wait on a slot with no copy", nm);
        slot_pending[s] = 0;
        slot_ready[s] = 1;
      };
      for (int g = 0; g < a.G; ++g)
        issue_window(t0 + g);
      issue_vals(t0);
      for (int t = t0; t < t1; ++t) {
        const int64_t R = b + (int64_t)t * a.P;
        if (t + 1 < t1) {
          if (early)
            issue_window(t + a.G);
          issue_vals(t + 1);
        }
        const int vs = t & 1;
        CHECK(vpending[vs] && vslab_tile[vs] == wid_base + t, "%s vals wait", nm);
        vpending[vs] = 0;
        vready[vs] = 1;
        for (int g = 0; g < a.G; ++g) {
          const int s = (t + g) % a.S;
          if (t == t0 || g == a.G - 1)
            wait_window(s);
          CHECK(slot_ready[s] && slot_win[s] == wid_base + t + g, "%s slot holds PW(t+g)", nm);
          const int64_t row0 = b + (int64_t)(t + g) * a.P + a.win0;
          for (int rg = 0; rg < NT / NV; ++rg) {
            const int i0 = rg * TR;
            const int64_t fskew = (R / RB) * 4 - (((R / RB) * 4) & ~(int64_t)15);
            CHECK(f_at + fskew + (i0 / RB) * 4 + 4 <= a.vslab_bytes, "%s mask read", nm);
            for (int r = a.grp_run0[g]; r < a.grp_run0[g + 1]; ++r) {
              const int q0 = a.run_q0[r], len = a.run_len[r], d0 = a.run_d0[r];
              for (int j = 0; j < TR + len - 1; ++j) {
                const int64_t idx = (int64_t)i0 + q0 + j;
                CHECK(idx >= 0 && idx < slot_rows, "%s window row %lld of %lld", nm, (long long)idx,
                      (long long)slot_rows);
              }
              for (int l = 0; l < len; ++l) {
                const int d = d0 + l;
                const int64_t vofs = (R * nd * vb & 15) + ((int64_t)(i0 / RB) * nd * RB + d * RB + i0 % RB) * vb;
                CHECK(vofs + TR * vb <= f_at, "%s vals read inside the values part", nm);
                CHECK(vofs % (TR * vb >= 16 ? 16 : TR * vb) == 0, "%s vals read alignment", nm);
                for (int i = 0; i < TR; ++i) {
                  // bv[i + l] is window row i0 + q0 + i + l
                  const int64_t brow = row0 + i0 + q0 + i + l;
                  CHECK(brow == R + i0 + i + cs.offs[d], "%s window row holds B row %lld, needs %lld", nm,
                        (long long)brow, (long long)(R + i0 + i + cs.offs[d]));
                }
              }
            }
          }
          if (g == 0 && !early && t + 1 < t1) {
            // after the CTA barrier: PW(t)'s slot takes PW(t + G); no later
            // group of this tile reads PW(t)
            for (int g2 = 1; g2 < a.G; ++g2)
              CHECK((t + g2) % a.S != s, "%s slot reused while read", nm);
            issue_window(t + a.G);
          }
        }
        for (int rg = 0; rg < NT / NV; ++rg)
          for (int cl = 0; cl < NV; ++cl) {
            const int col = k0 + cl * VEC;
            if (col >= k)
              continue;
            for (int i = 0; i < TR; ++i) {
              const int64_t row = R + rg * TR + i;
              if (rg * TR + i < rows_tile && row < a.m) {
                uint8_t &w = written[(size_t)row * (size_t)plan_div_up(k, VEC) + col / VEC];
                CHECK(w == 0, "%s C(%lld, %d) written twice", nm, (long long)row, col);
                w = 1;
              }
            }
          }
      }
      for (int s = 0; s < a.S; ++s)
        CHECK(!slot_pending[s], "%s copy never waited for", nm);
      CHECK(!vpending[0] && !vpending[1], "%s values copy never waited for", nm);
    }
  }
  for (size_t i = 0; i < written.size(); ++i)
    CHECK(written[i] == 1, "%s C element %zu not written", nm, i);
  (void)g_fail;
  return true;
}

// The line-patch plan of the diagonal-form kernel that reads B through L1
// (k_spmm_dia): over every CTA and thread of the launch, every unit of rb
// rows below the row count is computed by exactly one thread group, units at
// or past it only by the consecutive tail (where the kernel's row guard
// drops them), and each patch CTA holds kDiaLines whole line segments of the
// detected line stride. Returns whether patches applied.
static bool replay_patches(const Case &cs, int lg_tk, int rb) {
  const DiaRuns runs = dia_runs(cs.offs.data(), (int)cs.offs.size());
  const int64_t nunits = plan_div_up(cs.m, rb);
  const DiaPatchPlan p = dia_patch_plan(runs, rb, nunits, lg_tk);
  CHECK(p.units % (256 >> lg_tk) == 0 && p.units <= nunits, "%s lg_tk=%d: %lld patch units",
        cs.name.c_str(), lg_tk, (long long)p.units);
  const int64_t grid = plan_div_up(nunits << lg_tk, 256);
  std::vector<unsigned char> seen((size_t)nunits, 0);
  for (int64_t b = 0; b < grid; ++b) {
    int64_t first = -1;
    for (int tid = 0; tid < 256; tid += 1 << lg_tk) {
      const int64_t u = dia_patch_unit(b, tid, lg_tk, p);
      const bool in_patch = (b * 256 >> lg_tk) < p.units;
      if (u >= nunits) {
        CHECK(!in_patch, "%s lg_tk=%d: patch unit %lld past %lld", cs.name.c_str(), lg_tk, (long long)u,
              (long long)nunits);
        continue;
      }
      CHECK(u >= 0 && seen[(size_t)u] == 0, "%s lg_tk=%d: unit %lld twice", cs.name.c_str(), lg_tk,
            (long long)u);
      seen[(size_t)u] = 1;
      if (in_patch) {
        // thread group t of the CTA: line t >> lg_seg of the patch, the
        // (t & (seg - 1))-th unit of the segment
        const int t = tid >> lg_tk, seg = 1 << p.lg_seg;
        if (t == 0)
          first = u;
        CHECK(u == first + (int64_t)(t / seg) * p.ly_u + t % seg, "%s lg_tk=%d: patch shape",
              cs.name.c_str(), lg_tk);
      }
    }
  }
  for (int64_t u = 0; u < nunits; ++u)
    CHECK(seen[(size_t)u] == 1, "%s lg_tk=%d: unit %lld not computed", cs.name.c_str(), lg_tk,
          (long long)u);
  return p.units > 0;
}

int main() {
  std::vector<Case> cases = {
      {"27pt-128", 128 * 128 * 128, stencil3d(128, true), {8, 32, 128}},
      {"27pt-24", 24 * 24 * 24, stencil3d(24, true)},
      {"27pt-20", 20 * 20 * 20, stencil3d(20, true)},
      {"27pt-12", 12 * 12 * 12, stencil3d(12, true)},
      {"27pt-5", 125, stencil3d(5, true)},
      {"7pt-64", 64 * 64 * 64, stencil3d(64, false)},
      {"7pt-30", 30 * 30 * 30, stencil3d(30, false)},
      {"27pt-22", 22 * 22 * 22, stencil3d(22, true)},
      {"9pt-150", 150 * 150, stencil2d(150, true)},
      {"5pt-200", 200 * 200, stencil2d(200, false)},
      {"7pt-40x", 40 * 40 * 40 - 7, stencil3d(40, false)},
      {"5pt-512", 512 * 512, stencil2d(512, false), {8, 24, 128}},
      {"5pt-64", 64 * 64, stencil2d(64, false)},
      {"5pt-32", 32 * 32, stencil2d(32, false)},
      {"9pt-100", 100 * 100, stencil2d(100, true)},
      {"9pt-1024", 1024 * 1024, stencil2d(1024, true), {8, 40}},
      {"band9", 5000, band(-9, 9)},
      {"band2", 4001, band(-2, 2)},
      {"tri1", 1, band(-1, 1)},
      {"upper", 777, band(0, 3)},
      {"lower", 1003, band(-5, 0)},
      {"diag", 10, band(0, 0)},
  };
  int applied = 0, tried = 0;
  for (const Case &cs : cases)
    for (int k : cs.ks)
      for (int xb : {8, 4})
        for (int vb : {8, 4, 2}) {
          if (vb > xb || (k * xb) % 16 != 0)
            continue;  // the diagonal form needs 16-byte vectors of B and C
          ++tried;
          applied += replay(cs, k, xb, vb, 148) ? 1 : 0;
        }
  // The C3 configuration must be covered by the plan.
  const Case &c3 = cases[0];
  for (int k : {8, 32, 128})
    for (int vb : {8})
      CHECK(dia_tma_shape(c3.offs.data(), (int)c3.offs.size(), c3.m, k, 8, vb, 148).ok, "C3 k=%d FP64", k);
  for (int k : {8, 32, 128})
    for (int vb : {4, 2})
      CHECK(dia_tma_shape(c3.offs.data(), (int)c3.offs.size(), c3.m, k, 4, vb, 148).ok, "C3 k=%d FP32", k);
  int patched = 0, ptried = 0;
  for (const Case &cs : cases)
    for (int lg_tk = 0; lg_tk <= 5; ++lg_tk)
      for (int rb : {4, 2}) {
        ++ptried;
        patched += replay_patches(cs, lg_tk, rb) ? 1 : 0;
      }
  // The C3 matrix gets patches at the lane counts of k = 8 / 32 / 128 (FP64).
  for (int lg_tk : {2, 4, 5}) {
    const DiaRuns r = dia_runs(c3.offs.data(), (int)c3.offs.size());
    CHECK(dia_patch_plan(r, kDiaRows, plan_div_up(c3.m, kDiaRows), lg_tk).units ==
              plan_div_up(c3.m, kDiaRows),
          "C3 line patches, lg_tk=%d", lg_tk);
  }
  std::printf("ok %d of %d configurations applied and replayed; line patches in %d of %d\n",
              applied, tried, patched, ptried);
  return 0;
}
