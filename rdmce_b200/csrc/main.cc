// main.cc -- `RDMCE -i <graph> [-o a|d|deg|unchange] [-d id[,id..]] [-c]`
//
// The reference command line (main.cc:13-138): same options, same exit on a
// bad option, and the same result lines ("MC numbers: N", "MCE GPU Time: t")
// that scripts/analyze.sh parses.  Extra lines report the clique-size
// histogram and the checksum.  `-d` with several ids splits the roots over
// those devices (each holds a copy of the graph).
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "rdmce_graph.h"

namespace {

void usage(const char *argv0) {
  std::cerr << "Usage: " << argv0 << " -i <input_graph_file> -o <order_option> -d <device_ids> [-c]" << std::endl;
  std::cerr << "Order options: a (ascending), d (descending), deg (degeneracy),  unchange (unchanged)" << std::endl;
  std::cerr << "e.g., " << argv0 << " -i data/zachary.txt -o deg -d 0" << std::endl;
  std::exit(1);
}

bool ends_with_bin(const std::string &s) { return s.size() >= 4 && s.substr(s.size() - 4) == ".bin"; }

void print_result(const mce_result &r) {
  std::printf("MC checksum: 0x%016llx\n", (unsigned long long)r.checksum);
  std::printf("MC max size: %u\n", r.max_size);
  std::printf("MC histogram:");
  for (int s = 0; s < MCE_HIST_LEN; s++)
    if (r.hist[s]) std::printf(" %d:%llu", s, (unsigned long long)r.hist[s]);
  std::printf("\n");
}

}  // namespace

int main(int argc, char *argv[]) {
  std::string input;
  rdmce::OrderType order = rdmce::OrderType::DEG;
  std::vector<int> devices;
  bool convert_only = false;
  bool bad = false;
  int opt;
  while ((opt = getopt(argc, argv, "i:o:d:c")) != -1) {
    switch (opt) {
      case 'i': input = optarg; break;
      case 'o':
        if (!std::strcmp(optarg, "a")) order = rdmce::OrderType::ASC;
        else if (!std::strcmp(optarg, "d")) order = rdmce::OrderType::DES;
        else if (!std::strcmp(optarg, "deg")) order = rdmce::OrderType::DEG;
        else if (!std::strcmp(optarg, "unchange")) order = rdmce::OrderType::UNCHANGED;
        else bad = true;
        break;
      case 'd': {
        std::stringstream ss(optarg);
        std::string tok;
        devices.clear();
        while (std::getline(ss, tok, ',')) {
          char *end = nullptr;
          long id = std::strtol(tok.c_str(), &end, 10);
          if (tok.empty() || *end || id < 0) {
            std::cerr << "invalid device ID: " << tok << std::endl;
            return 1;
          }
          devices.push_back((int)id);
        }
        if (devices.empty()) {
          std::cerr << "-d option must provide at least one device ID" << std::endl;
          return 1;
        }
        break;
      }
      case 'c': convert_only = true; break;
      default: bad = true;
    }
  }
  if (input.empty() || bad) usage(argv[0]);
  try {
    rdmce::Graph g;
    g.SetDevice(devices.empty() ? 0 : devices[0]);
    auto t0 = std::chrono::steady_clock::now();
    if (ends_with_bin(input)) g.LoadFromBin(input);
    else g.LoadFromFile(input);
    std::cout << "Load time: " << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
              << "s" << std::endl;
    if (!ends_with_bin(input)) {
      t0 = std::chrono::steady_clock::now();
      g.SortByOrder(order);
      std::cout << "Sort time: " << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
                << "s" << std::endl;
      if (convert_only) {
        g.StoreIntoBin(input);
        std::cout << "preprocess " << input << " done" << std::endl;
      }
    }
    g.Handle();
    std::cout << "vertices: " << g.GetNumVertices() << " \tedges: " << g.GetNumEdges() << std::endl;
    std::cout << "max degree: " << g.GetMaxDegree() << " \tdegeneracy: " << g.GetDegeneracy() << std::endl;
    if (convert_only) {
      std::cout << "Convert only mode (-c) enabled, exiting after conversion." << std::endl;
      return 0;
    }
    if (devices.size() < 2) {
      rdmce::MceGpuSolver solver(g, devices.empty() ? 0 : devices[0]);
      solver.Solve();
      print_result(solver.result_);
    } else {
      mce_options o;
      mce_default_options(&o);
      auto t1 = std::chrono::steady_clock::now();
      mce_result r = rdmce::SolveOnDevices(g, devices, o);
      double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
      std::cout << "\nMC numbers: " << r.count << std::endl;
      std::cout << "MCE GPU Time: " << sec << std::endl;
      print_result(r);
    }
  } catch (const rdmce::Error &e) {
    std::cerr << "error: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
