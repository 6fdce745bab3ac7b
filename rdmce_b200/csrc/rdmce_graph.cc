// rdmce_graph.cc -- the reference-named C++ facade over the C ABI.
#include "rdmce_graph.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <memory>
#include <thread>

namespace rdmce {

std::string ExtractName(const std::string &path) {
  // file name without directory and extension (src/common.cu:2-17)
  size_t slash = path.find_last_of("/\\");
  std::string f = slash == std::string::npos ? path : path.substr(slash + 1);
  size_t dot = f.find_last_of('.');
  return dot == std::string::npos ? f : f.substr(0, dot);
}

Graph::Graph(Graph &&o) noexcept
    : name_(std::move(o.name_)),
      device_(o.device_),
      order_(o.order_),
      u_(std::move(o.u_)),
      v_(std::move(o.v_)),
      rowoffset_(std::move(o.rowoffset_)),
      colidx_(std::move(o.colidx_)),
      labels_(std::move(o.labels_)),
      g_(o.g_) {
  o.g_ = nullptr;
}

Graph::~Graph() { mce_graph_free(g_); }

void Graph::Require(mce_status s, const char *what) const {
  if (s != MCE_OK) throw Error(s, std::string(what) + ": " + mce_status_str(s));
}

void Graph::LoadFromFile(const std::string &path) {
  name_ = ExtractName(path);
  // the text is parsed on the GPU when the device graph is built (Handle),
  // with the order chosen by then; only its readability is checked here, so a
  // missing file still fails at load time as the reference's does
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) throw Error(MCE_ERR_IO, "cannot read " + path);
  std::fclose(f);
  text_path_ = path;
  u_.clear();
  v_.clear();
  mce_graph_free(g_);
  g_ = nullptr;
  rowoffset_.clear();
  colidx_.clear();
}

void Graph::LoadFromBin(const std::string &path) {
  name_ = ExtractName(path);
  mce_options o;
  mce_default_options(&o);
  o.device = device_;
  mce_graph_free(g_);
  g_ = nullptr;
  Require(mce_graph_load_file(path.c_str(), &o, &g_), ("cannot load " + path).c_str());
  text_path_.clear();
  u_.clear();
  v_.clear();
  rowoffset_.clear();
  colidx_.clear();
}

mce_graph *Graph::Handle() {
  if (!g_) {
    mce_options o;
    mce_default_options(&o);
    o.device = device_;
    switch (order_) {
      case OrderType::UNCHANGED: o.order = MCE_ORDER_UNCHANGED; break;
      case OrderType::ASC: o.order = MCE_ORDER_DEGREE_ASC; break;
      case OrderType::DES: o.order = MCE_ORDER_DEGREE_DESC; break;
      case OrderType::DEG: o.order = MCE_ORDER_DEGENERACY; break;
    }
    if (!text_path_.empty())
      Require(mce_graph_load_file(text_path_.c_str(), &o, &g_), ("cannot load " + text_path_).c_str());
    else
      Require(mce_graph_from_coo(u_.data(), v_.data(), u_.size(), &o, &g_), "graph build");
  }
  return g_;
}

void Graph::SortByOrder(OrderType order) {
  if (!text_path_.empty() || !u_.empty() || !g_) {
    order_ = order;
    mce_graph_free(g_);
    g_ = nullptr;
    Handle();
  }
  // a graph loaded from .bin keeps its stored order, as main.cc:26 skips the sort
}

void Graph::ConvertToCsr() {
  mce_graph_info info;
  Require(mce_graph_info_get(Handle(), &info), "graph info");
  rowoffset_.assign(info.num_vertices + 1, 0);
  colidx_.assign(2 * info.num_edges, 0);
  labels_.assign(info.num_vertices, 0);
  Require(mce_graph_export_csr(g_, rowoffset_.data(), colidx_.data(), labels_.data()), "CSR export");
}

void Graph::StoreIntoBin(const std::string &path) {
  size_t dot = path.find_last_of('.');
  Require(mce_graph_store_bin(Handle(), (path.substr(0, dot) + ".bin").c_str()), "store .bin");
}

size_t Graph::GetNumVertices() const {
  mce_graph_info i{};
  return g_ && mce_graph_info_get(g_, &i) == MCE_OK ? i.num_vertices : 0;
}
size_t Graph::GetNumEdges() const {
  mce_graph_info i{};
  return g_ && mce_graph_info_get(g_, &i) == MCE_OK ? i.num_edges : 0;
}
size_t Graph::GetMaxDegree() const {
  mce_graph_info i{};
  return g_ && mce_graph_info_get(g_, &i) == MCE_OK ? i.max_degree : 0;
}
size_t Graph::GetDegeneracy() const {
  mce_graph_info i{};
  return g_ && mce_graph_info_get(g_, &i) == MCE_OK ? i.degeneracy : 0;
}

MceGpuSolver::MceGpuSolver(Graph &g, int device_id) : device_id_(device_id), g_(g) {
  mce_default_options(&options_);
  options_.device = device_id;
  g_.SetDevice(device_id);
}

void MceGpuSolver::Solve() {
  mce_graph *h = g_.Handle();
  auto t0 = std::chrono::steady_clock::now();
  mce_status s = mce_solve(h, &options_, &result_);
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (s != MCE_OK) throw Error(s, std::string("solve: ") + mce_status_str(s));
  mce_count_ = result_.count;
  std::cout << "\nMC numbers: " << result_.count << std::endl;
  std::cout << "MCE GPU Time: " << sec << std::endl;
}

mce_result SolveOnDevices(Graph &g, const std::vector<int> &devices, const mce_options &base) {
  mce_result total{};
  mce_graph_info info{};
  if (mce_graph_info_get(g.Handle(), &info) != MCE_OK) throw Error(MCE_ERR_INTERNAL, "graph info");
  std::vector<uint32_t> off(info.num_vertices + 1), adj(2 * info.num_edges), lab(info.num_vertices);
  mce_status s = mce_graph_export_csr(g.Handle(), off.data(), adj.data(), lab.data());
  if (s != MCE_OK) throw Error(s, "CSR export");
  const size_t k = devices.size();
  std::vector<std::unique_ptr<mce_result>> parts(k);
  std::vector<mce_status> st(k, MCE_OK);
  std::vector<std::thread> th;
  for (size_t i = 0; i < k; i++) {
    parts[i].reset(new mce_result());
    th.emplace_back([&, i]() {
      mce_options o = base;
      o.device = devices[i];
      o.root_begin = info.num_edges * i / k;
      o.root_end = info.num_edges * (i + 1) / k;
      mce_graph *h = nullptr;
      st[i] = mce_graph_from_csr(info.num_vertices, off.data(), adj.data(), lab.data(), 1, &o, &h);
      if (st[i] == MCE_OK) st[i] = mce_solve(h, &o, parts[i].get());
      mce_graph_free(h);
    });
  }
  for (auto &t : th) t.join();
  for (size_t i = 0; i < k; i++) {
    if (st[i] != MCE_OK) throw Error(st[i], "device " + std::to_string(devices[i]) + ": " + mce_status_str(st[i]));
    total.count += parts[i]->count;
    total.checksum += parts[i]->checksum;
    total.max_size = std::max(total.max_size, parts[i]->max_size);
    total.roots += parts[i]->roots;
    for (int b = 0; b < MCE_HIST_LEN; b++) total.hist[b] += parts[i]->hist[b];
  }
  total.num_vertices = info.num_vertices;
  total.num_edges = info.num_edges;
  total.max_degree = info.max_degree;
  total.degeneracy = info.degeneracy;
  return total;
}

}  // namespace rdmce
