// gen.cc -- deterministic synthetic graph generators (COO pairs, 0-indexed uint32).
//
// The reference ships no generator; its evaluation reads public datasets.  These
// produce the synthetic workloads the engine is measured on: R-MAT (a/b/c/d, no
// noise), Chung-Lu power law, Erdos-Renyi G(n,p) by geometric skipping, and
// planted cliques.  Every draw comes from a counter-based SplitMix64 stream, so
// output is identical for any thread count.  Pairs are emitted raw: self-loops
// and duplicates are left for the loader to drop, as the reference loader does
// (src/graph.cc:88-111).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "internal.h"

namespace {

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;

inline uint64_t mix64(uint64_t x) {
  uint64_t z = x + kGolden;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// key of stream `s` under `seed`; draw t of that stream is mix64(key + t)
inline uint64_t stream_key(uint64_t seed, uint64_t s) {
  return mix64(seed * kGolden ^ mix64(s + 0x632BE59BD9B4E019ULL));
}

inline double unit(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

inline uint64_t thresh53(double p) {
  if (p <= 0) return 0;
  if (p >= 1) return 1ULL << 53;
  return (uint64_t)std::llround(p * 9007199254740992.0);
}

int pick_threads(int threads) {
  if (threads > 0) return threads;
  unsigned hc = std::thread::hardware_concurrency();
  return hc ? (int)std::min(hc, 64u) : 1;
}

template <class F>
void parallel_for(uint64_t n, int threads, F f) {
  threads = pick_threads(threads);
  if (n < 65536 || threads == 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> th;
  uint64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    uint64_t b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    th.emplace_back([=]() { f(b, e); });
  }
  for (auto &x : th) x.join();
}

struct Sink {
  uint32_t *u, *v;
  uint64_t cap, n;
  void push(uint32_t a, uint32_t b) {
    if (n < cap && u && v) {
      u[n] = a;
      v[n] = b;
    }
    n++;
  }
};

// Erdos-Renyi G(n,p) over pairs (w < x) by geometric skipping
// (Batagelj & Brandes, Phys. Rev. E 71, 2005).
void gnp(uint32_t n, double p, uint64_t seed, Sink &out) {
  if (n < 2 || p <= 0) return;
  const uint64_t key = stream_key(seed, 0);
  uint64_t t = 0;
  if (p >= 1) {
    for (uint32_t x = 1; x < n; x++)
      for (uint32_t w = 0; w < x; w++) out.push(w, x);
    return;
  }
  const double lq = std::log(1.0 - p);
  int64_t x = 1, w = -1;
  while (x < (int64_t)n) {
    double r = unit(mix64(key + t++));
    w += 1 + (int64_t)std::floor(std::log(1.0 - r) / lq);
    while (w >= x && x < (int64_t)n) {
      w -= x;
      x++;
    }
    if (x < (int64_t)n) out.push((uint32_t)w, (uint32_t)x);
  }
}

// `count` cliques, sizes uniform in [lo, hi] (clamped to n), members uniform
// distinct vertices of [0, n); all pairs of each clique are emitted.
void planted(uint32_t n, uint32_t count, uint32_t lo, uint32_t hi, uint64_t seed, Sink &out) {
  if (n == 0) return;
  std::vector<uint32_t> mem;
  for (uint32_t c = 0; c < count; c++) {
    const uint64_t key = stream_key(seed, (1ULL << 40) + c);
    uint64_t t = 0;
    uint32_t span = hi >= lo ? hi - lo + 1 : 1;
    uint32_t k = lo + (uint32_t)(mix64(key + t++) % span);
    k = std::min(k, n);
    mem.clear();
    while (mem.size() < k) {
      uint32_t x = (uint32_t)(mix64(key + t++) % n);
      if (std::find(mem.begin(), mem.end(), x) == mem.end()) mem.push_back(x);
    }
    for (uint32_t i = 0; i < k; i++)
      for (uint32_t j = i + 1; j < k; j++) out.push(mem[i], mem[j]);
  }
}

mce_status finish(const Sink &s, uint64_t *out_count) {
  if (out_count) *out_count = s.n;
  if (!s.u || !s.v) return MCE_OK;  // size query
  return s.n > s.cap ? MCE_ERR_CAPACITY : MCE_OK;
}

}  // namespace

extern "C" {

uint64_t mce_mix64(uint64_t x) { return mix64(x); }

mce_status mce_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                        uint32_t *u, uint32_t *v, uint64_t capacity, uint64_t *out_count, int threads) {
  if (scale == 0 || scale > 31 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 + 1e-12)
    return MCE_ERR_INVALID_ARG;
  const uint64_t ne = (uint64_t)edge_factor << scale;
  if (out_count) *out_count = ne;
  if (!u || !v) return MCE_OK;
  if (capacity < ne) return MCE_ERR_CAPACITY;
  const uint64_t ta = thresh53(a), tab = thresh53(a + b), tabc = thresh53(a + b + c);
  parallel_for(ne, threads, [&](uint64_t e0, uint64_t e1) {
    for (uint64_t e = e0; e < e1; e++) {
      const uint64_t key = stream_key(seed, e);
      uint32_t x = 0, y = 0;
      for (uint32_t l = 0; l < scale; l++) {
        uint64_t r = mix64(key + l) >> 11;
        uint32_t bx = 0, by = 0;
        if (r < ta) {
        } else if (r < tab) {
          by = 1;
        } else if (r < tabc) {
          bx = 1;
        } else {
          bx = by = 1;
        }
        x = (x << 1) | bx;
        y = (y << 1) | by;
      }
      u[e] = x;
      v[e] = y;
    }
  });
  return MCE_OK;
}

mce_status mce_gen_chung_lu(uint32_t n, double avg_degree, double gamma, uint64_t seed, uint32_t *u, uint32_t *v,
                            uint64_t capacity, uint64_t *out_count, int threads) {
  if (n < 2 || avg_degree <= 0 || gamma <= 1.0) return MCE_ERR_INVALID_ARG;
  const uint64_t ns = (uint64_t)std::llround((double)n * avg_degree / 2.0);
  if (out_count) *out_count = ns;
  if (!u || !v) return MCE_OK;
  if (capacity < ns) return MCE_ERR_CAPACITY;
  // w_i proportional to (i+1)^(-1/(gamma-1)); endpoints drawn proportional to w
  std::vector<double> cum(n);
  double acc = 0;
  const double ex = -1.0 / (gamma - 1.0);
  for (uint32_t i = 0; i < n; i++) {
    acc += std::pow((double)(i + 1), ex);
    cum[i] = acc;
  }
  auto pick = [&](double r) {
    double target = r * acc;
    uint32_t i = (uint32_t)(std::upper_bound(cum.begin(), cum.end(), target) - cum.begin());
    return i >= n ? n - 1 : i;
  };
  parallel_for(ns, threads, [&](uint64_t s0, uint64_t s1) {
    for (uint64_t s = s0; s < s1; s++) {
      const uint64_t key = stream_key(seed, s);
      u[s] = pick(unit(mix64(key)));
      v[s] = pick(unit(mix64(key + 1)));
    }
  });
  return MCE_OK;
}

mce_status mce_gen_gnp(uint32_t n, double avg_degree, uint64_t seed, uint32_t *u, uint32_t *v, uint64_t capacity,
                       uint64_t *out_count) {
  if (n < 2 || avg_degree < 0) return MCE_ERR_INVALID_ARG;
  Sink s{u, v, capacity, 0};
  gnp(n, std::min(1.0, avg_degree / (double)(n - 1)), seed, s);
  return finish(s, out_count);
}

mce_status mce_gen_planted(uint32_t n, uint32_t num_cliques, uint32_t size_lo, uint32_t size_hi, uint64_t seed,
                           uint32_t *u, uint32_t *v, uint64_t capacity, uint64_t *out_count) {
  if (n == 0 || size_lo > size_hi) return MCE_ERR_INVALID_ARG;
  Sink s{u, v, capacity, 0};
  planted(n, num_cliques, size_lo, size_hi, seed, s);
  return finish(s, out_count);
}

mce_status mce_gen_batch_member(uint32_t index, uint64_t base_seed, uint32_t *u, uint32_t *v, uint64_t capacity,
                                uint64_t *out_count, uint32_t *out_n) {
  // member `index` of the many-instance batch: n log-uniform in [64, 4096],
  // mean degree uniform in [8, 64], seed base_seed + index, 0-3 planted
  // cliques of size uniform in [8, 32]
  const uint64_t seed = base_seed + index;
  const uint64_t key = stream_key(seed, 1ULL << 50);
  const double ln_lo = std::log(64.0), ln_hi = std::log(4096.0);
  uint32_t n = (uint32_t)std::floor(std::exp(ln_lo + unit(mix64(key)) * (ln_hi - ln_lo)));
  n = std::min<uint32_t>(std::max<uint32_t>(n, 64), 4096);
  const double deg = 8.0 + unit(mix64(key + 1)) * 56.0;
  const uint32_t ncl = (uint32_t)(mix64(key + 2) % 4);
  if (out_n) *out_n = n;
  Sink s{u, v, capacity, 0};
  gnp(n, std::min(1.0, deg / (double)(n - 1)), seed, s);
  planted(n, ncl, 8, 32, seed ^ 0x5bd1e995ULL, s);
  return finish(s, out_count);
}

}  // extern "C"
