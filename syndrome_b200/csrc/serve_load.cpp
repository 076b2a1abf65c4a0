// Open-loop load driver for the serving engine (syndrome_serve_run_load).
//
// Transport blocks arrive as a Poisson process; each arrival takes the next entry of a
// pool of pre-encoded transport blocks (device-resident LLRs of its four redundancy
// versions) and is submitted at its arrival time.  A failed transmission is
// retransmitted at once with the next redundancy version (0, 2, 3, 1) until its CRCs
// pass or max_transmissions is reached.  A transport block's latency runs from its
// scheduled arrival (so a driver that falls behind counts the delay) to the result of
// its last transmission.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <random>
#include <thread>
#include <vector>

#include "../../include/syndrome_ldpc.h"
#include "serve.h"

namespace syn {

int run_load(ServeEngine& eng, const SyndromeLoadTb* pool, size_t pool_n, const SyndromeLoadSpec& spec,
             SyndromeLoadReport* rep, double* lat_out, size_t lat_cap, std::string* err) {
  static const int kRv[4] = {0, 2, 3, 1};
  using clock = std::chrono::steady_clock;
  const int max_tx = std::max(1, std::min<int>((int)spec.max_transmissions, 4));
  std::mt19937_64 rng(spec.seed);
  std::exponential_distribution<double> gap(spec.offered_tb_per_s);
  std::vector<double> arrivals;
  for (double t = gap(rng); t < spec.duration_s; t += gap(rng)) arrivals.push_back(t);
  const size_t n = arrivals.size();
  std::vector<int> tx(n, 0);
  std::vector<double> latency(n, -1.0);
  std::vector<char> ok(n, 0);
  std::vector<ServeResult> res(1024);
  std::vector<double> tx_lat;
  tx_lat.reserve(n * 2);
  double sum_queue = 0.0, sum_step = 0.0;
  size_t next = 0, finished = 0;
  long long transmissions = 0;
  double info_ok = 0.0, info_decoded = 0.0;
  const auto t0 = clock::now();
  auto now_s = [&] { return std::chrono::duration<double>(clock::now() - t0).count(); };
  auto send = [&](size_t i) -> int {
    const SyndromeLoadTb& p = pool[i % pool_n];
    const int k = tx[i];
    std::string e;
    const int r = eng.submit((uint64_t)i, (long long)p.tb_size, p.target_rate, (int)p.qm, (long long)p.g, kRv[k],
                             p.llr[k], (long long)p.llr_len, true, &e);
    if (r != SYNDROME_OK) {
      if (err) *err = e;
      return r;
    }
    tx[i] = k + 1;
    ++transmissions;
    info_decoded += (double)p.tb_size;
    return SYNDROME_OK;
  };
  while (finished < n) {
    const double t = now_s();
    while (next < n && arrivals[next] <= t) {
      const int r = send(next);
      if (r != SYNDROME_OK) return r;
      ++next;
    }
    const double wait_s = next < n ? std::max(0.0, arrivals[next] - now_s()) : 0.002;
    const int got = eng.poll(res.data(), (int)res.size(), (long long)std::min(wait_s * 1e6, 2000.0));
    for (int j = 0; j < got; ++j) {
      const size_t i = (size_t)res[j].id;
      tx_lat.push_back(res[j].latency_us);
      sum_queue += res[j].queue_us;
      sum_step += res[j].step_us;
      if (res[j].crc_ok || tx[i] >= max_tx) {
        latency[i] = (now_s() - arrivals[i]) * 1e6;
        ok[i] = res[j].crc_ok ? 1 : 0;
        if (ok[i]) info_ok += (double)pool[i % pool_n].tb_size;
        std::string e;
        eng.release((uint64_t)i, &e);
        ++finished;
      } else {
        const int r = send(i);
        if (r != SYNDROME_OK) return r;
      }
    }
  }
  const double wall = now_s();
  std::vector<double> sorted(latency);
  std::sort(sorted.begin(), sorted.end());
  auto pct = [&](double q) {
    if (sorted.empty()) return 0.0;
    const size_t k = std::min(sorted.size() - 1, (size_t)std::floor(q * (double)(sorted.size() - 1) + 0.5));
    return sorted[k];
  };
  double mean = 0.0;
  for (double v : latency) mean += v;
  rep->tbs = n;
  rep->tbs_ok = 0;
  for (char c : ok) rep->tbs_ok += c;
  rep->transmissions = (uint64_t)transmissions;
  rep->wall_s = wall;
  rep->info_bits_ok = info_ok;
  rep->info_bits_decoded = info_decoded;
  rep->p50_us = pct(0.50);
  rep->p99_us = pct(0.99);
  rep->mean_us = n ? mean / (double)n : 0.0;
  rep->max_us = sorted.empty() ? 0.0 : sorted.back();
  std::sort(tx_lat.begin(), tx_lat.end());
  auto tpct = [&](double q) {
    if (tx_lat.empty()) return 0.0;
    return tx_lat[std::min(tx_lat.size() - 1, (size_t)std::floor(q * (double)(tx_lat.size() - 1) + 0.5))];
  };
  rep->tx_p50_us = tpct(0.50);
  rep->tx_p99_us = tpct(0.99);
  rep->tx_mean_queue_us = tx_lat.empty() ? 0.0 : sum_queue / (double)tx_lat.size();
  rep->tx_mean_step_us = tx_lat.empty() ? 0.0 : sum_step / (double)tx_lat.size();
  if (lat_out)
    for (size_t i = 0; i < std::min(lat_cap, n); ++i) lat_out[i] = latency[i];
  return SYNDROME_OK;
}

}  // namespace syn
