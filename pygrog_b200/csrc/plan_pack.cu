// plan_pack.cu -- host-side packing steps of the brick plans (no device code).
//
// The brick plans of the fused gridders (pygrog_b200/calib/_plan6.py) sort
// the valid replicas on the GPU; three steps of the plan are sequential per
// sub-chunk or per plan and run here, in C++ on the host, one call each:
//   * pgb_plan_pack_quarter_warps: first-fit packing of a sub-chunk's
//     replicas into quarter-warps whose lanes read operators that are equal
//     or in distinct shared-memory bank classes (the lane-per-replica v8
//     kernels);
//   * pgb_plan_pack_rows: next-fit packing of a sub-chunk's cell runs into
//     16-row m-tiles (the tensor-core forward), padding a run to the next
//     m-tile when it would cross one and the sub-chunk's capacity allows;
//   * pgb_plan_lpt: largest-first assignment of work items to the least
//     loaded CTA.
// Sub-chunks are independent, so the first two split their sub-chunks over
// host threads.  The same functions serve plans of host and device tensors.
#include <algorithm>
#include <queue>
#include <thread>
#include <utility>
#include <vector>

#include "common.cuh"

namespace {

// Run f(begin, end) over [0, n) in contiguous ranges on up to hardware
// concurrency threads (one thread for small n).
template <typename F>
void parallel_ranges(int64_t n, int64_t grain, F f) {
  unsigned hw = std::thread::hardware_concurrency();
  int64_t nt = std::max<int64_t>(1, std::min<int64_t>(hw ? hw : 1, n / std::max<int64_t>(grain, 1)));
  nt = std::min<int64_t>(nt, 64);
  if (nt <= 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> th;
  for (int64_t i = 0; i < nt; ++i) {
    const int64_t b = n * i / nt, e = n * (i + 1) / nt;
    th.emplace_back([=]() { f(b, e); });
  }
  for (auto& t : th) t.join();
}

}  // namespace

using namespace pgb;

extern "C" {

int pgb_plan_pack_quarter_warps(const int64_t* sub_ptr, const int64_t* q, const int64_t* k, int64_t n_subs,
                                int64_t per, int64_t* lane, int64_t* nq_out) {
  clear_error();
  PGB_REQUIRE(n_subs >= 0 && (per == 4 || per == 8), PGB_ERR_INVALID,
              "plan_pack_quarter_warps: per must be 4 or 8, n_subs >= 0");
  PGB_REQUIRE(n_subs == 0 || (sub_ptr && nq_out), PGB_ERR_INVALID, "plan_pack_quarter_warps: null pointer");
  const int64_t n = n_subs ? sub_ptr[n_subs] : 0;
  PGB_REQUIRE(n == 0 || (q && k && lane), PGB_ERR_INVALID, "plan_pack_quarter_warps: null pointer");
  for (int64_t s = 0; s < n_subs; ++s)
    PGB_REQUIRE(sub_ptr[s + 1] >= sub_ptr[s], PGB_ERR_INVALID, "plan_pack_quarter_warps: sub_ptr not ascending");
  const int nres = static_cast<int>(per);
  parallel_ranges(n_subs, 256, [&](int64_t s0, int64_t s1) {
    std::vector<int64_t> used, res_q, res_k;
    for (int64_t s = s0; s < s1; ++s) {
      const int64_t b = sub_ptr[s], cnt = sub_ptr[s + 1] - b;
      const int64_t nq = (cnt + per - 1) / per;
      nq_out[s] = nq;
      used.assign(nq, 0);
      res_q.assign(nq * nres, -1);
      res_k.assign(nq * nres, -1);
      for (int64_t i = 0; i < cnt; ++i) {
        const int64_t qq = q[b + i], kk = k[b + i];
        const int rq = static_cast<int>(((qq % nres) + nres) % nres), rk = static_cast<int>(((kk % nres) + nres) % nres);
        // first quarter-warp with a free lane that (1) already reads this
        // inner operator, else (2) has its inner residue free, both with a
        // compatible outer residue, else (3) has a compatible inner residue,
        // else (4) has the fewest lanes taken
        int64_t pick = -1;
        for (int pass = 0; pass < 3 && pick < 0; ++pass) {
          for (int64_t w = 0; w < nq; ++w) {
            if (used[w] >= per) continue;
            const int64_t cq = res_q[w * nres + rq], ck = res_k[w * nres + rk];
            const bool ok_k = ck < 0 || ck == kk;
            const bool same_q = cq == qq;
            const bool hit = pass == 0 ? (same_q && ok_k) : pass == 1 ? (cq < 0 && ok_k) : (cq < 0 || same_q);
            if (hit) {
              pick = w;
              break;
            }
          }
        }
        if (pick < 0) {
          int64_t best = per + 1;
          for (int64_t w = 0; w < nq; ++w)
            if (used[w] < per && used[w] < best) {
              best = used[w];
              pick = w;
            }
        }
        lane[b + i] = pick * per + used[pick];
        used[pick] += 1;
        if (res_q[pick * nres + rq] < 0) res_q[pick * nres + rq] = qq;
        if (res_k[pick * nres + rk] < 0) res_k[pick * nres + rk] = kk;
      }
    }
  });
  return PGB_OK;
}

int pgb_plan_pack_rows(const int64_t* run_len, const int64_t* run_ptr, int64_t n_subs, int64_t rows, int64_t cap,
                       int64_t* run_start, int64_t* n_entries) {
  clear_error();
  PGB_REQUIRE(n_subs >= 0 && rows >= 1 && cap >= 1, PGB_ERR_INVALID, "plan_pack_rows: invalid sizes");
  PGB_REQUIRE(n_subs == 0 || (run_ptr && n_entries), PGB_ERR_INVALID, "plan_pack_rows: null pointer");
  const int64_t nr = n_subs ? run_ptr[n_subs] : 0;
  PGB_REQUIRE(nr == 0 || (run_len && run_start), PGB_ERR_INVALID, "plan_pack_rows: null pointer");
  parallel_ranges(n_subs, 1024, [&](int64_t s0, int64_t s1) {
    for (int64_t s = s0; s < s1; ++s) {
      const int64_t b = run_ptr[s], e = run_ptr[s + 1];
      int64_t rem = 0;
      for (int64_t r = b; r < e; ++r) rem += run_len[r];  // rows of this and the later runs
      int64_t cur = 0;
      for (int64_t r = b; r < e; ++r) {
        const int64_t ln = run_len[r];
        const int64_t off = cur % rows;
        int64_t pad = (ln > 0 && ln <= rows && off + ln > rows) ? rows - off : 0;
        if (cur + pad + rem > cap) pad = 0;  // the padding budget of the sub-chunk is spent
        cur += pad;
        run_start[r] = cur;
        cur += ln;
        rem -= ln;
      }
      n_entries[s] = cur;
    }
  });
  return PGB_OK;
}

int pgb_plan_lpt(const double* cost, int64_t n, int64_t bins, int32_t* out) {
  clear_error();
  PGB_REQUIRE(n >= 0 && bins >= 1, PGB_ERR_INVALID, "plan_lpt: n >= 0 and bins >= 1 required");
  PGB_REQUIRE(n == 0 || (cost && out), PGB_ERR_INVALID, "plan_lpt: null pointer");
  std::vector<int64_t> order(n);
  for (int64_t i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
  using Slot = std::pair<double, int64_t>;  // (load, bin): least load first, then lowest bin
  std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> heap;
  for (int64_t b = 0; b < bins; ++b) heap.push({0.0, b});
  for (int64_t i : order) {
    Slot s = heap.top();
    heap.pop();
    out[i] = static_cast<int32_t>(s.second);
    heap.push({s.first + cost[i], s.second});
  }
  return PGB_OK;
}

}  // extern "C"
