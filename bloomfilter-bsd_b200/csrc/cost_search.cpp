// cost_search.cpp -- the exhaustive calibrated configuration search.
//
// The reference picks a filter for (n, tw) by minimising, for every valid
// configuration, overhead(m) = t_lookup(m) + tw * fpr(m, n, config) over the
// filter size m (cost_fn.hpp:150-160, optimizer.hpp:25-140), then taking the
// configuration with the least overhead (skyline_matrix_builder.cpp:88-115).
// Here the same search runs over a tabulated grid of bits per key, with the
// lookup time read from GPU calibration runs (t per key at log2-spaced filter
// sizes, linearly interpolated) instead of per-cache-level deltas:
//
//   cost(c, m) = t_c(m / 8 bytes, f, h) + ns_per_match * (h + (1 - h) * f)
//                + work_ns * (1 - h) * f,        f = fpr_c(m / n)
//
// where t_c is the first half of a block's probe plus, for the keys that go
// on (members, and non-members passing the first half), the second half:
// t_c = first_c(m) + (h + (1 - h) sqrt(f)) second_c(m).
//
// subject to f <= fpr_target and, for L2-resident queries, m / 8 <=
// l2_budget_bytes.  Queries are split over host threads.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <thread>
#include <vector>

#include "../../include/dtlg.h"

namespace {

double lookup_row(const dtlg_cost_tables* t, const double* table, uint32_t c, double log2_bytes) {
  const double* row = table + static_cast<size_t>(c) * t->n_size;
  if (t->n_size == 1) return row[0];
  double x = (log2_bytes - t->log2_bytes_first) / t->log2_bytes_step;
  x = std::min(std::max(x, 0.0), static_cast<double>(t->n_size - 1));
  uint32_t i = static_cast<uint32_t>(x);
  if (i > t->n_size - 2) i = t->n_size - 2;
  const double f = x - i;
  return row[i] * (1.0 - f) + row[i + 1] * f;
}

// Probe time per key of candidate c at a filter of 2^log2_bytes bytes, for a
// filter whose false-positive rate is f, at hit ratio h: the first half of the
// block always, the second half for members and for the non-members that pass
// the first half (probability sqrt(f)).
double lookup_ns(const dtlg_cost_tables* t, uint32_t c, double log2_bytes, double f, double h) {
  double ns = lookup_row(t, t->ns_per_key, c, log2_bytes);
  if (t->ns_second) {
    const double q = std::min(1.0, std::sqrt(std::max(0.0, f)));
    ns += (h + (1.0 - h) * q) * lookup_row(t, t->ns_second, c, log2_bytes);
  }
  return ns;
}

void search_range(const dtlg_cost_tables* t, const dtlg_cost_query* q, uint32_t q0, uint32_t q1, double* cand_cost,
                  double* cand_bpk, int32_t* best, double* best_cost, double* best_bpk) {
  const double inf = std::numeric_limits<double>::infinity();
  const uint32_t C = t->n_cand, K = t->n_bpk;
  std::vector<double> log2_bpk(K);
  for (uint32_t k = 0; k < K; k++) log2_bpk[k] = std::log2(t->bits_per_key[k]);
  for (uint32_t qi = q0; qi < q1; qi++) {
    const dtlg_cost_query& Q = q[qi];
    const double h = Q.hit_ratio, miss = 1.0 - Q.hit_ratio;
    const double n = std::exp2(Q.log2_n);
    double b_cost = inf, b_bpk = std::nan("");
    int32_t b_idx = -1;
    for (uint32_t c = 0; c < C; c++) {
      double c_cost = inf, c_bpk = std::nan("");
      const double* fr = t->fpr + static_cast<size_t>(c) * K;
      for (uint32_t k = 0; k < K; k++) {
        const double f = fr[k];
        if (!(f <= Q.fpr_target)) continue;
        const double bytes = n * t->bits_per_key[k] / 8.0;
        if (Q.l2_resident && bytes > t->l2_budget_bytes) continue;
        const double cost = lookup_ns(t, c, Q.log2_n + log2_bpk[k] - 3.0, f, h) +
                            t->ns_per_match * (h + miss * f) + Q.work_ns * miss * f;
        if (cost < c_cost) {
          c_cost = cost;
          c_bpk = t->bits_per_key[k];
        }
      }
      if (cand_cost) cand_cost[static_cast<size_t>(qi) * C + c] = c_cost;
      if (cand_bpk) cand_bpk[static_cast<size_t>(qi) * C + c] = c_bpk;
      if (c_cost < b_cost) {
        b_cost = c_cost;
        b_bpk = c_bpk;
        b_idx = static_cast<int32_t>(c);
      }
    }
    if (best) best[qi] = b_idx;
    if (best_cost) best_cost[qi] = b_cost;
    if (best_bpk) best_bpk[qi] = b_bpk;
  }
}

}  // namespace

extern "C" {

dtlg_status dtlg_cost_search(const dtlg_cost_tables* t, const dtlg_cost_query* queries, uint32_t n_queries,
                             double* cand_cost, double* cand_bpk, int32_t* best, double* best_cost,
                             double* best_bpk, int threads) {
  if (!t || (n_queries && !queries)) return DTLG_ERR_NULL;
  if (!t->n_cand || !t->n_bpk || !t->n_size || !t->bits_per_key || !t->fpr || !t->ns_per_key ||
      !(t->log2_bytes_step > 0.0))
    return DTLG_ERR_INVALID_CONFIG;
  if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  threads = static_cast<int>(std::min<uint32_t>(static_cast<uint32_t>(threads), std::max(1u, n_queries)));
  if (threads <= 1) {
    search_range(t, queries, 0, n_queries, cand_cost, cand_bpk, best, best_cost, best_bpk);
    return DTLG_OK;
  }
  std::vector<std::thread> pool;
  const uint32_t per = (n_queries + threads - 1) / threads;
  for (int i = 0; i < threads; i++) {
    const uint32_t a = std::min(n_queries, per * i), b = std::min(n_queries, per * (i + 1));
    if (a < b) pool.emplace_back(search_range, t, queries, a, b, cand_cost, cand_bpk, best, best_cost, best_bpk);
  }
  for (auto& th : pool) th.join();
  return DTLG_OK;
}

dtlg_status dtlg_cost_eval(const dtlg_cost_tables* t, const dtlg_cost_query* queries, uint32_t n_queries,
                           const int32_t* cand, const uint32_t* bpk_index, double* cost) {
  if (!t || (n_queries && (!queries || !cand || !bpk_index || !cost))) return DTLG_ERR_NULL;
  const double inf = std::numeric_limits<double>::infinity();
  for (uint32_t qi = 0; qi < n_queries; qi++) {
    const dtlg_cost_query& Q = queries[qi];
    const int32_t c = cand[qi];
    const uint32_t k = bpk_index[qi];
    if (c < 0 || static_cast<uint32_t>(c) >= t->n_cand || k >= t->n_bpk) {
      cost[qi] = inf;
      continue;
    }
    const double f = t->fpr[static_cast<size_t>(c) * t->n_bpk + k];
    const double bytes = std::exp2(Q.log2_n) * t->bits_per_key[k] / 8.0;
    if (!(f <= Q.fpr_target) || (Q.l2_resident && bytes > t->l2_budget_bytes)) {
      cost[qi] = inf;
      continue;
    }
    const double miss = 1.0 - Q.hit_ratio;
    cost[qi] = lookup_ns(t, static_cast<uint32_t>(c), Q.log2_n + std::log2(t->bits_per_key[k]) - 3.0, f,
                         Q.hit_ratio) +
               t->ns_per_match * (Q.hit_ratio + miss * f) + Q.work_ns * miss * f;
  }
  return DTLG_OK;
}

}  // extern "C"
