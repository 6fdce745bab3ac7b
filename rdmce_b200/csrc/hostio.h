// hostio.h -- host-side graph file formats (COO text, reference .bin).
#pragma once
#include <cstdint>
#include <vector>

#include "internal.h"

namespace mce {

struct BinGraph {
  uint64_t n = 0, m = 0, max_degree = 0, degeneracy = 0;
  std::vector<uint32_t> off;  // n + 1
  std::vector<uint32_t> adj;  // 2m
  std::vector<uint32_t> labels;
};

mce_status parse_coo_text(const char *path, std::vector<uint32_t> &u, std::vector<uint32_t> &v);
mce_status read_bin(const char *path, BinGraph &g);
mce_status write_bin(const char *path, const BinGraph &g);
bool has_bin_suffix(const char *path);

}  // namespace mce
