// hostio.cc -- host-side graph file formats.
//
//  * COO text as Graph::LoadFromFile reads it (src/graph.cc:82-104): the file
//    is a stream of unsigned decimal tokens; each record is `>> u >> v`
//    (white space, newlines included, may separate the two), the rest of the
//    line after v is ignored, and a failed extraction discards the rest of the
//    current line.  '%' / '#' header lines therefore fall out as bad lines.
//  * the reference .bin container (src/graph.cc:154-213): four native-endian
//    size_t (n, m, max_degree, degeneracy), then per vertex a size_t degree and
//    that many uint32 neighbours, then n uint32 original labels.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "hostio.h"

namespace mce {

namespace {

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

// one `std::istream >> unsigned int`: returns false on failure (no digits or
// overflow); `pos` ends after the consumed characters
bool extract_u32(const char *s, size_t len, size_t &pos, uint32_t &out) {
  size_t p = pos;
  while (p < len && is_space(s[p])) p++;
  bool neg = false;
  if (p < len && (s[p] == '+' || s[p] == '-')) {
    neg = s[p] == '-';
    p++;
  }
  if (p >= len || s[p] < '0' || s[p] > '9') {
    pos = p;
    return false;
  }
  uint64_t val = 0;
  bool overflow = false;
  for (; p < len && s[p] >= '0' && s[p] <= '9'; p++) {
    if (!overflow) {
      val = val * 10 + (uint64_t)(s[p] - '0');
      overflow = val > 0xFFFFFFFFULL;
    }
  }
  pos = p;
  if (overflow) return false;
  out = neg ? (uint32_t)(0u - (uint32_t)val) : (uint32_t)val;
  return true;
}

}  // namespace

namespace {

// One record attempt from a line start: `>> u >> v` (either may cross line
// breaks), then the rest of the current line is skipped.  Returns the next
// record start, which is again a line start (or len).
inline size_t parse_record(const char *s, size_t len, size_t pos, std::vector<uint32_t> &u,
                           std::vector<uint32_t> &v) {
  uint32_t a = 0, b = 0;
  const bool ok = extract_u32(s, len, pos, a) && extract_u32(s, len, pos, b);
  if (ok) {
    u.push_back(a);
    v.push_back(b);
  }
  const void *nl = std::memchr(s + pos, '\n', len - pos);
  return nl ? (size_t)((const char *)nl - s) + 1 : len;
}

// Parse [from, ...) until the first record start at or past `stop`; returns it.
size_t parse_span(const char *s, size_t len, size_t from, size_t stop, std::vector<uint32_t> &u,
                  std::vector<uint32_t> &v) {
  size_t pos = from;
  while (pos < stop && pos < len) pos = parse_record(s, len, pos, u, v);
  return pos;
}

constexpr size_t kChunkBytes = 4u << 20;  // below this a file is parsed by one thread

}  // namespace

// Record starts form a chain: each is a line start fixed by the one before,
// and a record normally ends at its own line end.  The file is cut at line
// starts into chunks parsed in parallel, each assuming a record starts at its
// first byte.  Then, in order, a chunk whose true first record start (where
// the previous chunk's chain left off) differs from its cut -- a record ran
// across the cut -- is parsed again from the true start.  The output is
// exactly the sequential parse.
mce_status parse_coo_text(const char *path, std::vector<uint32_t> &u, std::vector<uint32_t> &v) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return MCE_ERR_IO;
  if (std::fseek(f, 0, SEEK_END) != 0) {
    std::fclose(f);
    return MCE_ERR_IO;
  }
  long len = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (len < 0) {
    std::fclose(f);
    return MCE_ERR_IO;
  }
  std::unique_ptr<char[]> buf(new (std::nothrow) char[(size_t)len + 1]);  // not zero-filled
  if (!buf) {
    std::fclose(f);
    return MCE_ERR_OUT_OF_MEMORY;
  }
  if (len > 0 && std::fread(buf.get(), 1, (size_t)len, f) != (size_t)len) {
    std::fclose(f);
    return MCE_ERR_IO;
  }
  std::fclose(f);
  const char *s = buf.get();
  const size_t L = (size_t)len;
  u.clear();
  v.clear();
  size_t nt = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), L / kChunkBytes));
  if (nt == 1) {
    u.reserve(L / 8);
    v.reserve(L / 8);
    parse_span(s, L, 0, L, u, v);
    return MCE_OK;
  }
  // cuts at line starts
  std::vector<size_t> cut(nt + 1);
  cut[0] = 0;
  cut[nt] = L;
  for (size_t j = 1; j < nt; j++) {
    size_t c = std::max(cut[j - 1], L * j / nt);
    const void *nl = std::memchr(s + c, '\n', L - c);
    cut[j] = nl ? (size_t)((const char *)nl - s) + 1 : L;
  }
  std::vector<std::vector<uint32_t>> cu(nt), cv(nt);
  std::vector<size_t> end(nt);
  std::vector<std::thread> th;
  for (size_t j = 0; j < nt; j++)
    th.emplace_back([&, j]() {
      // thread-local vectors: neighbouring vector headers share cache lines
      std::vector<uint32_t> lu, lv;
      lu.reserve((cut[j + 1] - cut[j]) / 8);
      lv.reserve((cut[j + 1] - cut[j]) / 8);
      const size_t e = parse_span(s, L, cut[j], cut[j + 1], lu, lv);
      cu[j] = std::move(lu);
      cv[j] = std::move(lv);
      end[j] = e;
    });
  for (auto &t : th) t.join();
  for (size_t j = 1; j < nt; j++) {
    if (end[j - 1] == cut[j]) continue;
    // a record ran across the cut: this chunk restarts where the chain is
    cu[j].clear();
    cv[j].clear();
    end[j] = end[j - 1] >= cut[j + 1] ? end[j - 1] : parse_span(s, L, end[j - 1], cut[j + 1], cu[j], cv[j]);
  }
  std::vector<size_t> at(nt + 1, 0);
  for (size_t j = 0; j < nt; j++) at[j + 1] = at[j] + cu[j].size();
  u.resize(at[nt]);
  v.resize(at[nt]);
  th.clear();
  for (size_t j = 0; j < nt; j++)
    th.emplace_back([&, j]() {
      if (!cu[j].empty()) {
        std::memcpy(u.data() + at[j], cu[j].data(), cu[j].size() * 4);
        std::memcpy(v.data() + at[j], cv[j].data(), cv[j].size() * 4);
      }
    });
  for (auto &t : th) t.join();
  return MCE_OK;
}

mce_status read_bin(const char *path, BinGraph &g) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return MCE_ERR_IO;
  uint64_t hdr[4];
  if (std::fread(hdr, 8, 4, f) != 4) {
    std::fclose(f);
    return MCE_ERR_FORMAT;
  }
  g.n = hdr[0];
  g.m = hdr[1];
  g.max_degree = hdr[2];
  g.degeneracy = hdr[3];
  if (2 * g.m >= (1ULL << 32) || g.n >= (1ULL << 32)) {
    std::fclose(f);
    return MCE_ERR_TOO_LARGE;
  }
  g.off.assign(g.n + 1, 0);
  g.adj.resize(2 * g.m);
  uint64_t e = 0;
  for (uint64_t x = 0; x < g.n; x++) {
    uint64_t d = 0;
    if (std::fread(&d, 8, 1, f) != 1 || e + d > 2 * g.m) {
      std::fclose(f);
      return MCE_ERR_FORMAT;
    }
    if (d && std::fread(g.adj.data() + e, 4, d, f) != d) {
      std::fclose(f);
      return MCE_ERR_FORMAT;
    }
    e += d;
    g.off[x + 1] = (uint32_t)e;
  }
  if (e != 2 * g.m) {
    std::fclose(f);
    return MCE_ERR_FORMAT;
  }
  g.labels.resize(g.n);
  if (g.n && std::fread(g.labels.data(), 4, g.n, f) != g.n) {
    std::fclose(f);
    return MCE_ERR_FORMAT;
  }
  std::fclose(f);
  return MCE_OK;
}

mce_status write_bin(const char *path, const BinGraph &g) {
  FILE *f = std::fopen(path, "wb");
  if (!f) return MCE_ERR_IO;
  uint64_t hdr[4] = {g.n, g.m, g.max_degree, g.degeneracy};
  bool ok = std::fwrite(hdr, 8, 4, f) == 4;
  for (uint64_t x = 0; ok && x < g.n; x++) {
    uint64_t d = g.off[x + 1] - g.off[x];
    ok = std::fwrite(&d, 8, 1, f) == 1 && (d == 0 || std::fwrite(g.adj.data() + g.off[x], 4, d, f) == d);
  }
  if (ok && g.n) ok = std::fwrite(g.labels.data(), 4, g.n, f) == g.n;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? MCE_OK : MCE_ERR_IO;
}

bool has_bin_suffix(const char *path) {
  size_t L = std::strlen(path);
  return L >= 4 && std::strcmp(path + L - 4, ".bin") == 0;
}

}  // namespace mce

extern "C" {

mce_status mce_parse_text(const char *path, uint32_t **u, uint32_t **v, uint64_t *n_pairs) {
  if (!path || !u || !v || !n_pairs) return MCE_ERR_INVALID_ARG;
  std::vector<uint32_t> a, b;
  mce_status s = mce::parse_coo_text(path, a, b);
  if (s != MCE_OK) return s;
  *n_pairs = a.size();
  *u = (uint32_t *)std::malloc(std::max<size_t>(a.size(), 1) * 4);
  *v = (uint32_t *)std::malloc(std::max<size_t>(b.size(), 1) * 4);
  if (!*u || !*v) {
    std::free(*u);
    std::free(*v);
    return MCE_ERR_OUT_OF_MEMORY;
  }
  if (!a.empty()) {
    std::memcpy(*u, a.data(), a.size() * 4);
    std::memcpy(*v, b.data(), b.size() * 4);
  }
  return MCE_OK;
}

void mce_free_host(void *p) { std::free(p); }

}  // extern "C"
