// rdmce_graph.h -- C++ facade with the reference's host API names over the C ABI.
//
// Mirrors class Graph (include/graph.h:12-52) and class MceGpuSolver
// (include/mce_gpu.cuh:15-24) so host code written against the reference
// compiles against this engine.  Differences: errors throw rdmce::Error instead
// of calling exit(); Solve() also fills mce_count_ (the reference leaves it 0,
// src/mce_gpu.cu:14-22) and result_ (histogram, checksum, phase times).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rdmce.h"

using vid_t = uint32_t;
using acc_t = uint64_t;

namespace rdmce {

class Error : public std::runtime_error {
 public:
  Error(mce_status s, const std::string &what) : std::runtime_error(what), status(s) {}
  mce_status status;
};

enum class OrderType { UNCHANGED, ASC, DES, DEG };

class Graph {
 public:
  Graph() = default;
  Graph(const Graph &) = delete;
  Graph &operator=(const Graph &) = delete;
  Graph(Graph &&other) noexcept;
  ~Graph();

  // COO text, src/graph.cc:64-152 (parsed on the GPU when SortByOrder or the
  // first use builds the device graph)
  void LoadFromFile(const std::string &path);
  // the reference .bin container, already ordered (src/graph.cc:178-213)
  void LoadFromBin(const std::string &path);
  // writes <path without extension>.bin, as src/graph.cc:154-176 does
  void StoreIntoBin(const std::string &path);
  // fills the host CSR returned by GetRowOffset / GetColIdx (src/graph.cc:216-236)
  void ConvertToCsr();
  void SortByOrder(OrderType order);

  const std::string &GetName() const { return name_; }
  size_t GetNumVertices() const;
  size_t GetNumEdges() const;
  size_t GetMaxDegree() const;
  size_t GetDegeneracy() const;
  vid_t *GetRowOffset() { return rowoffset_.empty() ? nullptr : rowoffset_.data(); }
  vid_t *GetColIdx() { return colidx_.empty() ? nullptr : colidx_.data(); }
  const std::vector<uint32_t> &Labels() const { return labels_; }

  void SetDevice(int device) { device_ = device; }
  // the device-resident graph (built on first use with the current order)
  mce_graph *Handle();

 private:
  void Require(mce_status s, const char *what) const;
  std::string name_;
  int device_ = 0;
  OrderType order_ = OrderType::DEG;
  std::string text_path_;        // pending COO text file (parsed on the GPU at build)
  std::vector<uint32_t> u_, v_;  // pending COO pairs
  std::vector<uint32_t> rowoffset_, colidx_, labels_;
  mce_graph *g_ = nullptr;
};

class MceGpuSolver {
 public:
  explicit MceGpuSolver(Graph &g, int device_id = 0);
  // prints "MC numbers: N" and "MCE GPU Time: t" as src/mce_gpu.cu:20-21 does
  void Solve();
  acc_t mce_count_ = 0;
  mce_result result_{};
  mce_options options_{};

 private:
  int device_id_;
  Graph &g_;
};

// Multi-device solve: roots are split into contiguous ranges, one per device,
// each device holding its own copy of the graph; results are summed on the host.
mce_result SolveOnDevices(Graph &g, const std::vector<int> &devices, const mce_options &base);

std::string ExtractName(const std::string &path);

}  // namespace rdmce
