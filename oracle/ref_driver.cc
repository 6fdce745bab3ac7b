// ref_driver.cc -- a driver around the UNMODIFIED reference CPU code
// (RDMCE src/graph.cc, src/mce.cc, src/common.cu), compiled out-of-tree by
// oracle/Makefile into oracle/_ref/ref_cpu.  Test infrastructure only: it pins
// the oracle (loader conventions, degeneracy value, clique counts) and is the
// "reference" CPU baseline that bench.py --impl reference times.
//
// Modes:
//   ref_cpu count <graph>            MceSolver::Solve(BKFixedMemPivotBit), 1 thread
//   ref_cpu pivot <graph>            MceSolver::Solve(BKPivot), 1 thread
//   ref_cpu par <graph> <threads> [max_roots]
//                                    root-parallel: one MceSolver per thread, the
//                                    vertex roots of src/mce.cc:64-95 handed out in
//                                    chunks, each solved by BKFixedMemPivotBit2
//   ref_cpu steps <graph> <threads> <seconds> <warmup> <steps>
//                                    bench steps: each step (a forked child)
//                                    solves vertex roots in a seeded random order
//                                    with all threads until <seconds>, then
//                                    reports the cliques found so far and exits
//   ref_cpu stats <graph>            n, m, max degree, degeneracy after the sort
//   ref_cpu csr <graph> <out>        CSR + labels after the sort (binary dump)
//   ref_cpu storebin <graph> <out>   Graph::StoreIntoBin of the loaded (sorted) graph
//   ref_cpu edge_roots <graph> <threads> <rootfile>
//                                    the listed EDGE roots (ids = edges v0 < v1 in CSR
//                                    order of the graph as loaded), each solved to
//                                    completion by BKFixedMemPivotBit2 with R = {v0, v1},
//                                    P = common neighbours > v1, X = the others, as the
//                                    reference's own edge-root loop does (src/mce.cc:96-131,
//                                    kept there as a comment); prints per-root counts
//   ref_cpu edge_steps <graph> <threads> <rootfile> <seconds> <warmup> <steps>
//                                    bench steps over those edge roots in file order:
//                                    all threads until <seconds> (forked child per step,
//                                    as `steps`), cliques counted at the deadline
// <graph> is COO text (sorted by degeneracy as main.cc:26-27 does) or a .bin
// (used in stored order: main.cc:26 sorts only non-.bin input).
#include <atomic>
#include <random>
#include <sys/wait.h>
#include <unistd.h>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <string>
#include <thread>
#include <vector>
#include <algorithm>
#include <memory>
#include <sstream>
#include <unordered_map>
#include <queue>
#include <cassert>
#include <limits>
// The per-root solver entry points are private members of MceSolver; the
// root-parallel harness needs them, so open the class for this driver only.
#define private public
#include "mce.h"
#undef private

static void load(Graph &g, const std::string &path) {
  if (path.size() >= 4 && path.substr(path.size() - 4) == ".bin") {
    g.LoadFromBin(path);
  } else {
    g.LoadFromFile(path);
    g.SortByOrder(OrderType::DEG);
  }
}

// Edge roots in CSR order: root r is the r-th pair (v0, v1), v0 < v1, walking
// the rows in id order.  upper[v] = index of v's first root.
struct EdgeRoots {
  std::vector<uint64_t> upper;
  explicit EdgeRoots(const Graph &g) {
    const uint64_t n = g.GetNumVertices();
    upper.assign(n + 1, 0);
    for (uint64_t v = 0; v < n; v++) {
      uint64_t up = 0;
      for (vid_t w : g.N((vid_t)v)) up += w > v;
      upper[v + 1] = upper[v] + up;
    }
  }
  bool get(const Graph &g, uint64_t r, vid_t *v0, vid_t *v1) const {
    if (r >= upper.back()) return false;
    const uint64_t v = (uint64_t)(std::upper_bound(upper.begin(), upper.end(), r) - upper.begin()) - 1;
    const vlist_t &row = g.N((vid_t)v);
    const uint64_t lower = row.size() - (upper[v + 1] - upper[v]);
    *v0 = (vid_t)v;
    *v1 = row[lower + (r - upper[v])];
    return true;
  }
};

// One edge root through the reference solver, as its edge-root loop does.
static void solve_edge_root(MceSolver &s, const Graph &g, vid_t v0, vid_t v1) {
  vlist_t cand;
  std::set_intersection(g.N(v0).begin(), g.N(v0).end(), g.N(v1).begin(), g.N(v1).end(), std::back_inserter(cand));
  vlist_t R, P, X;
  R.emplace_back(v0);
  R.emplace_back(v1);
  for (auto c : cand) {
    if (c > v1) P.emplace_back(c);
    else X.emplace_back(c);
  }
  if (P.empty()) {
    if (X.empty()) s.IncrementMceCount();
    return;
  }
  if (X.size() > (P.size() + 1) * 16) X = s.Partition(P, X);
  s.BKFixedMemPivotBit2(R, P, X);
}

static std::vector<uint64_t> read_roots(const char *path) {
  std::vector<uint64_t> roots;
  std::ifstream f(path);
  uint64_t r;
  while (f >> r) roots.push_back(r);
  return roots;
}

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s count|pivot|par|stats|csr <graph> [...]\n", argv[0]);
    return 2;
  }
  std::string mode = argv[1];
  Graph g;
  load(g, argv[2]);
  if (mode == "stats") {
    std::printf("n %zu m %zu max_degree %zu degeneracy %zu\n", g.GetNumVertices(), g.GetNumEdges(),
                g.GetMaxDegree(), g.GetDegeneracy());
    return 0;
  }
  if (mode == "csr") {
    if (argc < 4) return 2;
    g.ConvertToCsr();
    FILE *f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    uint64_t n = g.GetNumVertices(), m = g.GetNumEdges();
    std::fwrite(&n, 8, 1, f);
    std::fwrite(&m, 8, 1, f);
    std::fwrite(g.GetRowOffset(), 4, n + 1, f);
    std::fwrite(g.GetColIdx(), 4, 2 * m, f);
    // labels are not exposed by Graph; recover them through the operator<< dump
    std::ostringstream os;
    os << g;
    std::istringstream is(os.str());
    std::string line;
    std::vector<uint32_t> labels(n, 0);
    while (std::getline(is, line)) {
      if (line.size() < 2 || line[0] != 'v') continue;
      unsigned long id = 0, lab = 0;
      if (std::sscanf(line.c_str(), "v%lu(%lu)", &id, &lab) == 2 && id < n) labels[id] = (uint32_t)lab;
    }
    std::fwrite(labels.data(), 4, n, f);
    std::fclose(f);
    return 0;
  }
  if (mode == "storebin") {
    if (argc < 4) return 2;
    g.StoreIntoBin(argv[3]);  // writes <argv[3] without its extension>.bin
    return 0;
  }
  if (mode == "edge_roots" || mode == "edge_steps") {
    if (argc < 5) return 2;
    const int threads = std::max(1, std::atoi(argv[3]));
    const std::vector<uint64_t> roots = read_roots(argv[4]);
    const EdgeRoots er(g);
    for (uint64_t r : roots) {
      vid_t a, b;
      if (!er.get(g, r, &a, &b)) {
        std::fprintf(stderr, "root %llu out of range\n", (unsigned long long)r);
        return 1;
      }
    }
    const uint64_t nr = roots.size();
    if (mode == "edge_roots") {
      std::vector<uint64_t> counts(nr, 0);
      std::atomic<uint64_t> next(0);
      auto t0 = std::chrono::steady_clock::now();
      std::vector<std::thread> th;
      for (int t = 0; t < threads; t++) {
        th.emplace_back([&]() {
          MceSolver s(g);
          for (;;) {
            const uint64_t k = next.fetch_add(1);
            if (k >= nr) break;
            vid_t v0, v1;
            er.get(g, roots[k], &v0, &v1);
            const acc_t c0 = s.mce_count_;
            solve_edge_root(s, g, v0, v1);
            counts[k] = s.mce_count_ - c0;
          }
        });
      }
      for (auto &x : th) x.join();
      double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      uint64_t total = 0;
      for (uint64_t k = 0; k < nr; k++) {
        std::printf("ROOT %llu %llu\n", (unsigned long long)roots[k], (unsigned long long)counts[k]);
        total += counts[k];
      }
      std::printf("RESULT count %llu seconds %.6f threads %d roots %llu\n", (unsigned long long)total, sec, threads,
                  (unsigned long long)nr);
      return 0;
    }
    if (argc < 8) return 2;
    const double seconds = std::atof(argv[5]);
    const int total_steps = std::atoi(argv[6]) + std::atoi(argv[7]);
    for (int step = 0; step < total_steps; step++) {
      std::fflush(stdout);
      pid_t pid = fork();
      if (pid < 0) return 1;
      if (pid == 0) {
        // one edge root can take far longer than a step: threads are detached
        // and the child reports the cliques counted by the deadline, then exits
        std::atomic<uint64_t> next(0), done(0);
        std::vector<std::unique_ptr<MceSolver>> solvers;
        for (int t = 0; t < threads; t++) solvers.emplace_back(new MceSolver(g));
        auto t0 = std::chrono::steady_clock::now();
        for (int t = 0; t < threads; t++) {
          std::thread([&, t]() {
            MceSolver &s = *solvers[t];
            for (;;) {
              const uint64_t k = next.fetch_add(1);
              if (k >= nr) break;
              vid_t v0, v1;
              er.get(g, roots[k], &v0, &v1);
              solve_edge_root(s, g, v0, v1);
              done.fetch_add(1);
            }
          }).detach();
        }
        for (;;) {
          std::this_thread::sleep_for(std::chrono::milliseconds(20));
          double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
          if (el >= seconds || done.load() >= nr) {
            uint64_t total = 0;
            for (auto &sv : solvers) total += *(volatile acc_t *)&sv->mce_count_;
            std::printf("STEP %d cliques %llu seconds %.6f roots_done %llu of %llu\n", step,
                        (unsigned long long)total, el, (unsigned long long)done.load(), (unsigned long long)nr);
            std::fflush(stdout);
            _exit(0);
          }
        }
      }
      int status = 0;
      waitpid(pid, &status, 0);
    }
    return 0;
  }
  if (mode == "count" || mode == "pivot") {
    MceSolver s(g);
    auto t0 = std::chrono::steady_clock::now();
    s.Solve(mode == "count" ? MceAlgorithm::BKFixedMemPivotBit : MceAlgorithm::BKPivot);
    double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("RESULT count %llu seconds %.6f threads 1\n", (unsigned long long)s.mce_count_, sec);
    return 0;
  }
  if (mode == "par") {
    int threads = argc > 3 ? std::atoi(argv[3]) : (int)std::thread::hardware_concurrency();
    if (threads < 1) threads = 1;
    uint64_t n = g.GetNumVertices();
    uint64_t limit = argc > 4 ? std::strtoull(argv[4], nullptr, 10) : n;
    if (limit > n) limit = n;
    std::atomic<uint64_t> next(0);
    std::vector<uint64_t> counts(threads, 0);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int t = 0; t < threads; t++) {
      th.emplace_back([&, t]() {
        MceSolver s(g);
        for (;;) {
          uint64_t k0 = next.fetch_add(16);
          if (k0 >= limit) break;
          uint64_t k1 = std::min(limit, k0 + 16);
          for (uint64_t k = k0; k < k1; k++) {
            // heavy (late) vertices first, as the GPU kernel orders its roots
            vid_t v0 = (vid_t)(n - 1 - k);
            vlist_t R, P, X;
            R.emplace_back(v0);
            for (vid_t v1 : g.N(v0)) {
              if (v0 > v1) X.emplace_back(v1);
              else P.emplace_back(v1);
            }
            if (P.empty()) {
              if (X.empty()) s.IncrementMceCount();
              continue;
            }
            s.BKFixedMemPivotBit2(R, P, X);
          }
        }
        counts[t] = s.mce_count_;
      });
    }
    for (auto &x : th) x.join();
    double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    uint64_t total = 0;
    for (auto c : counts) total += c;
    std::printf("RESULT count %llu seconds %.6f threads %d roots %llu\n", (unsigned long long)total, sec,
                threads, (unsigned long long)limit);
    return 0;
  }
  if (mode == "steps") {
    if (argc < 7) return 2;
    const int threads = std::max(1, std::atoi(argv[3]));
    const double seconds = std::atof(argv[4]);
    const int total_steps = std::atoi(argv[5]) + std::atoi(argv[6]);
    const uint64_t n = g.GetNumVertices();
    std::vector<vid_t> order(n);
    for (uint64_t i = 0; i < n; i++) order[i] = (vid_t)i;
    std::mt19937_64 rng(12345);
    std::shuffle(order.begin(), order.end(), rng);
    for (int step = 0; step < total_steps; step++) {
      std::fflush(stdout);
      pid_t pid = fork();
      if (pid < 0) return 1;
      if (pid == 0) {
        // a single vertex root can take hours: threads are detached and the
        // child reports the cliques counted so far at the deadline, then exits
        std::atomic<uint64_t> next(0);
        std::vector<std::unique_ptr<MceSolver>> solvers;
        for (int t = 0; t < threads; t++) solvers.emplace_back(new MceSolver(g));
        auto t0 = std::chrono::steady_clock::now();
        for (int t = 0; t < threads; t++) {
          std::thread([&, t]() {
            MceSolver &s = *solvers[t];
            for (;;) {
              uint64_t k = next.fetch_add(1);
              if (k >= n) break;
              vid_t v0 = order[k];
              vlist_t R, P, X;
              R.emplace_back(v0);
              for (vid_t v1 : g.N(v0)) {
                if (v0 > v1) X.emplace_back(v1);
                else P.emplace_back(v1);
              }
              if (P.empty()) {
                if (X.empty()) s.IncrementMceCount();
                continue;
              }
              s.BKFixedMemPivotBit2(R, P, X);
            }
          }).detach();
        }
        for (;;) {
          std::this_thread::sleep_for(std::chrono::milliseconds(50));
          double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
          if (el >= seconds || next.load() >= n + (uint64_t)threads) {
            uint64_t total = 0;
            for (auto &sv : solvers) total += *(volatile acc_t *)&sv->mce_count_;
            std::printf("STEP %d cliques %llu seconds %.6f roots %llu\n", step, (unsigned long long)total, el,
                        (unsigned long long)std::min<uint64_t>(next.load(), n));
            std::fflush(stdout);
            _exit(0);
          }
        }
      }
      int status = 0;
      waitpid(pid, &status, 0);
    }
    return 0;
  }
  std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 2;
}
