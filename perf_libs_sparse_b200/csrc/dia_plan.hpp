// Diagonal form of a CSR matrix: constants, and the launch plan of the
// diagonal-form SpMM whose B rows are staged in shared memory by tensor-map
// copies (k_spmm_dia_tma in spmm_dia.cu). Host-only C++ with no CUDA
// dependency, so that the plan can also be checked by a CPU program that
// replays the kernel's indexing (tests/dia_plan_check.cpp).
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace pls {

// The diagonal form (DiaDev): for every block of kDiaRows rows and every
// diagonal, the block's kDiaRows values; at most kDiaMax diagonals; the
// blocks continue kDiaPadRows rows past the matrix's last row, all absent.
constexpr int kDiaRows = 4;
constexpr int kDiaMax = 32;
constexpr int kDiaPadRows = 1024;
// Consecutive diagonals handled together (their B rows loaded once).
constexpr int kDiaRun = 3;

// The staged kernel's tile is kDiaTmaThreads / NV value blocks of
// kDiaRows rows; its threads take kDiaTmaThreadRows rows each, so it runs
// kDiaRows * kDiaTmaThreads / kDiaTmaThreadRows threads.
constexpr int kDiaTmaThreads = 256;
constexpr int kDiaTmaThreadRows = 4;
constexpr int kDiaTmaMaxSlots = 8;
constexpr int kDiaTmaMaxSmem = 220 * 1024;  // + 128 bytes of alignment room at launch

// Kernel arguments of the staged diagonal-form SpMM.
struct DiaTmaArgs {
  int32_t m, k;
  int32_t P;            // rows between consecutive tiles of a chain
  int32_t win0;         // first window row of group 0, relative to the tile's first row
  int32_t BR, NB;       // TMA box rows; boxes per window (NB * BR >= L + 2h)
  int32_t slot_bytes;   // one window slot
  int32_t vslab_bytes;  // one tile's values and blocks' full-diagonal masks (see below)
  int32_t S, G, nd;
  int32_t n_chains, n_slices, Z;
  int64_t n_items;
  int32_t grp_run0[kDiaTmaMaxSlots + 1];  // runs of group g: [grp_run0[g], grp_run0[g + 1])
  int32_t run_q0[kDiaMax], run_len[kDiaMax], run_d0[kDiaMax];
  int32_t tx_extra;  // failure-path tests: bytes expected beyond the copies
  int32_t wait_limit;
};

inline int64_t plan_div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }

#ifdef __CUDACC__
#define PLS_PLAN_HD __host__ __device__
#else
#define PLS_PLAN_HD
#endif

// Runs of consecutive diagonals (at most kDiaRun each) over the ascending
// offsets: run q starts at offset o0[q], diagonal d0[q], and has len[q]
// diagonals.
struct DiaRuns {
  int n = 0;
  int o0[kDiaMax], len[kDiaMax], d0[kDiaMax];
};

inline DiaRuns dia_runs(const int32_t *offs, int nd) {
  DiaRuns r{};
  for (int i = 0; i < nd;) {
    int len = 1;
    while (i + len < nd && len < kDiaRun && offs[i + len] == offs[i] + len)
      ++len;
    r.o0[r.n] = offs[i];
    r.len[r.n] = len;
    r.d0[r.n] = i;
    ++r.n;
    i += len;
  }
  return r;
}

// Line patches of the diagonal-form SpMM (k_spmm_dia). On a grid stencil
// the runs come one grid line (Ly rows) apart, so the runs of row r at
// offset +Ly read the rows of B that row r + Ly reads at offset 0. Where the
// run centres show such a stride (the smallest gap of at least 16 rows
// between consecutive centres), each CTA takes kDiaLines lines x (its units
// / kDiaLines) consecutive units (a unit is one thread's rb rows) instead of
// consecutive units, so the lines it holds read each other's rows of B from
// L1. The patches tile the first `units` units (whole groups of kDiaLines
// lines, ly_u units per line, segments of 2^lg_seg units); the rest keep
// consecutive units. 256-thread CTAs, 2^lg_tk threads per unit.
constexpr int kDiaLines = 4;

struct DiaPatchPlan {
  int64_t units = 0;  // units covered by patches (0: none)
  int32_t ly_u = 0;   // units per grid line
  int lg_seg = 0;     // log2(units per CTA / kDiaLines)
};

inline DiaPatchPlan dia_patch_plan(const DiaRuns &runs, int rb, int64_t nunits, int lg_tk) {
  DiaPatchPlan p;
  p.lg_seg = 8 - lg_tk - 2;
  int64_t ly = 0;
  for (int q = 1; q < runs.n; ++q) {
    const int64_t gap = ((int64_t)runs.o0[q] + (runs.len[q] - 1) / 2) -
                        ((int64_t)runs.o0[q - 1] + (runs.len[q - 1] - 1) / 2);
    if (gap >= 16 && (ly == 0 || gap < ly))
      ly = gap;
  }
  if (p.lg_seg >= 0 && ly > 0 && ly % rb == 0 && ly / rb <= INT32_MAX &&
      (ly / rb) % ((int64_t)1 << p.lg_seg) == 0) {
    p.ly_u = (int32_t)(ly / rb);
    p.units = nunits / ((int64_t)kDiaLines * p.ly_u) * ((int64_t)kDiaLines * p.ly_u);
  }
  return p;
}

// The unit that thread `tid` (of 256) of CTA `block` computes.
PLS_PLAN_HD inline int64_t dia_patch_unit(int64_t block, int tid, int lg_tk,
                                          const DiaPatchPlan &p) {
  const int64_t u = (block * 256 + tid) >> lg_tk;
  if ((block * 256 >> lg_tk) >= p.units)
    return u;
  const int64_t nseg = p.ly_u >> p.lg_seg;
  const int64_t lg = block / nseg, xs = block - lg * nseg;
  const int t = tid >> lg_tk;
  return (lg * kDiaLines + (t >> p.lg_seg)) * p.ly_u + (xs << p.lg_seg) +
         (t & ((1 << p.lg_seg) - 1));
}

inline int64_t floor_mid(int64_t lo, int64_t hi) {
  const int64_t s = lo + hi;
  return s >= 0 ? s / 2 : -((-s + 1) / 2);
}

// Grouping of the diagonal offsets (ascending) for the staged kernel: groups
// split where the gap between neighbouring offsets is more than half the
// largest gap; the staged form needs their centres evenly spaced (P apart)
// for a chain of windows, otherwise all offsets form one group.
struct DiaGroups {
  int G = 1;
  int64_t P = 0;   // 0: one group
  int64_t c0 = 0;  // centre of group 0
  int64_t h = 0;   // every offset within h of its group's centre
  int grp[kDiaMax] = {};
};

// All offsets as one group (a band): the centre of the span.
inline DiaGroups one_group(const int32_t *o, int nd) {
  DiaGroups r;
  r.c0 = floor_mid(o[0], o[nd - 1]);
  r.h = std::max(r.c0 - o[0], (int64_t)o[nd - 1] - r.c0);
  return r;
}

inline DiaGroups dia_groups(const int32_t *o, int nd) {
  DiaGroups r;
  int64_t maxgap = 0;
  for (int i = 0; i + 1 < nd; ++i)
    maxgap = std::max<int64_t>(maxgap, (int64_t)o[i + 1] - o[i]);
  std::vector<int> start{0};
  for (int i = 0; i + 1 < nd; ++i)
    if (2 * ((int64_t)o[i + 1] - o[i]) > maxgap)
      start.push_back(i + 1);
  start.push_back(nd);
  const int G = (int)start.size() - 1;
  std::vector<int64_t> centre(G);
  for (int g = 0; g < G; ++g)
    centre[g] = floor_mid(o[start[g]], o[start[g + 1] - 1]);
  bool ap = G >= 2 && G <= kDiaTmaMaxSlots;
  for (int g = 2; ap && g < G; ++g)
    ap = centre[g] - centre[g - 1] == centre[1] - centre[0];
  if (ap) {
    r.G = G;
    r.P = centre[1] - centre[0];
    r.c0 = centre[0];
    for (int g = 0; g < G; ++g)
      for (int i = start[g]; i < start[g + 1]; ++i) {
        r.grp[i] = g;
        r.h = std::max(r.h, std::max(centre[g] - o[i], (int64_t)o[i] - centre[g]));
      }
    if (2 * r.h < r.P)  // windows of neighbouring groups must not overlap
      return r;
  }
  return one_group(o, nd);
}

// Launch shape of the staged kernel for one call: column lanes NV (slices
// of KS = NV * VEC columns, VEC = 16 / x_bytes), rows per tile L, the
// window boxes, the slots and the work items. ok = false when no shape fits
// shared memory or the copies' alignment rules. x_bytes: the size of B's
// and C's elements; v_bytes: the size of the values; sms: the SM count.
struct DiaTmaShape {
  bool ok = false;
  int NV = 0, L = 0;
  DiaTmaArgs a{};
  size_t smem = 0;
};

inline DiaTmaShape dia_tma_shape(const int32_t *offs, int nd, int32_t m, int k, int x_bytes,
                                 int v_bytes, int sms) {
  const int VEC = 16 / x_bytes;
  DiaTmaShape out;
  if (nd <= 0 || nd > kDiaMax || m <= 0 || k <= 0)
    return out;
  const DiaGroups gr = dia_groups(offs, nd);
  for (int NV : {8, 4, 2}) {
    if (NV > 2 && NV * VEC > k)
      continue;  // narrower slices waste fewer columns
    const int KS = NV * VEC;
    const int L = kDiaTmaThreads / NV * kDiaRows;
    const int row_bytes = KS * x_bytes;
    // A chain needs P >= L (tiles of one chain must not overlap) and tile
    // starts on whole blocks of values; otherwise the band of all offsets.
    const DiaGroups g =
        gr.G >= 2 && gr.P >= L && gr.P % kDiaRows == 0 ? gr : one_group(offs, nd);
    const int64_t P = g.G >= 2 ? g.P : L;
    const int64_t W = L + 2 * g.h;
    const int NB = (int)plan_div_up(W, 256);
    int BR = (int)plan_div_up(W, NB);
    const int align_rows = std::max(1, 128 / row_bytes);  // 128-byte aligned boxes
    BR = (int)plan_div_up(BR, align_rows) * align_rows;
    if (BR > 256)
      continue;
    const int64_t slot = (int64_t)NB * BR * row_bytes;
    const int S = g.G >= 2 ? g.G : 2;
    // A tile's slab: its values (from byte R * nd * v_bytes of the diagonal
    // form, not always on a 16-byte boundary: copied from the boundary below,
    // so up to 16 bytes more), then from the next 16-byte boundary on its
    // L / 4 blocks' 32-bit full-diagonal masks (copied the same way).
    const int64_t vslab = plan_div_up((int64_t)L * nd * v_bytes, 16) * 16 + 16 + (L / kDiaRows) * 4 + 16;
    const int64_t smem = S * slot + 2 * vslab;
    if (smem > kDiaTmaMaxSmem)
      continue;
    DiaTmaArgs &a = out.a;
    a = DiaTmaArgs{};
    a.m = m;
    a.k = k;
    a.P = (int32_t)P;
    a.win0 = (int32_t)(g.c0 - g.h);
    a.BR = BR;
    a.NB = NB;
    a.slot_bytes = (int32_t)slot;
    a.vslab_bytes = (int32_t)vslab;
    a.S = S;
    a.G = g.G;
    a.nd = nd;
    a.n_chains = (int32_t)plan_div_up(P, L);
    a.n_slices = (int32_t)plan_div_up(k, KS);
    // Runs of consecutive offsets (at most kDiaRun) within each group, and
    // each run's first row in the group's window for tile row 0.
    int nr = 0;
    for (int gi = 0; gi < g.G; ++gi) {
      a.grp_run0[gi] = nr;
      const int64_t cg = g.c0 + (int64_t)gi * (g.G >= 2 ? g.P : 0);
      for (int i = 0; i < nd;) {
        if ((g.G >= 2 ? g.grp[i] : 0) != gi) {
          ++i;
          continue;
        }
        int len = 1;
        while (i + len < nd && len < kDiaRun && offs[i + len] == offs[i] + len &&
               (g.G >= 2 ? g.grp[i + len] : 0) == gi)
          ++len;
        a.run_q0[nr] = (int32_t)(offs[i] - cg + g.h);
        a.run_len[nr] = len;
        a.run_d0[nr] = i;
        ++nr;
        i += len;
      }
    }
    a.grp_run0[g.G] = nr;
    // Tiles per work item: whole chains when that gives enough items,
    // otherwise halved down to 4 (each item re-reads G - 1 windows first).
    const int64_t tiles = plan_div_up(m, P);
    int64_t Z = tiles;
    auto items = [&](int64_t z) { return a.n_chains * plan_div_up(tiles, z) * a.n_slices; };
    while (Z > 4 && items(Z) < 8 * (int64_t)sms)
      Z = plan_div_up(Z, 2);
    a.Z = (int32_t)Z;
    a.n_items = items(Z);
    out.ok = true;
    out.NV = NV;
    out.L = L;
    out.smem = (size_t)smem;
    return out;
  }
  return out;
}

}  // namespace pls
