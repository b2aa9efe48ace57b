// bbtc -- drop-in for the reference's `bbtc` executable, counting on one B200.
//
// Same flags, defaults, checks and output lines as the reference's CUDA driver
// (argument parsing include/utils/utils.hpp:21-154, main src/bbtc.cu:15-90,
// timing fields include/utils/hooks.hpp:13-56).  Differences, forced by
// "one GPU" or added:
//   --ngpu       only 1 is served (the default "all devices" means 1); 0 (CPU
//                only) and > 1 print a message and exit like other bad input.
//   --nstream    accepted and checked; the persistent kernel uses one stream.
//   --border     tasks [0, b) run on the GPU only; the rest are shared with
//                CPU workers when there are any (bb_tc.cpp:142-252).
//   --cpu-workers (added) CPU worker threads beside the GPU: 0 (default) =
//                every task on the GPU; -1 = the reference's split, OpenMP
//                threads minus the --nstream GPU workers.
//   --copy-first the block CSR is device-resident from the layout build on, so
//                the "Copy tiles to device (s)" field measures a stream sync.
#include <omp.h>
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "bbtc.hpp"

extern "C" {
int bbtcio_read(const char* path, int* kind, void** handle);
int bbtcio_write_bbtc(const char* path, uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint64_t m);
int bbtcg_info(void* handle, uint32_t* n, uint64_t* m, uint64_t* m_raw);
int bbtcg_copy(void* handle, uint32_t* indptr, uint32_t* indices);
int bbtcg_free(void* handle);
int bbtcp_cuts(int kind, uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint32_t P, uint64_t seed,
               uint32_t* cuts);
}

namespace {

struct Parameters {
  std::string file_name = "-";
  std::string part_name = "pal";
  int n_gpu = 0;
  int n_stream = 4;
  int border = 0;
  int ncut = 32;
  int repeat = 5;
  int cpu_workers = 0;
  bool copy_first = false;
};

// Timed regions printed as "name : seconds" at exit (hooks.hpp:13-56).
std::vector<std::pair<std::string, std::string>> g_fields;
std::chrono::steady_clock::time_point g_start;
void RegionBegin() { g_start = std::chrono::steady_clock::now(); }
void RegionEnd(const std::string& name) {
  const double s =
      std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - g_start).count() /
      1e6;
  std::stringstream ss;
  ss << std::fixed << std::setprecision(4) << s;
  g_fields.emplace_back(name, ss.str());
}

std::string lower(const std::string& s) {
  std::string r;
  for (char c : s) r.push_back((char)std::tolower((unsigned char)c));
  return r;
}

void PrintUsage() {
  std::cout << "bbTC: A Block Based Triangle Counting Algorithm" << std::endl;
  std::cout << "syntax: bbtc --graph <path> [OPTION].. [--help]" << std::endl;
  std::cout << "Options:                                                           (Defaults:)" << std::endl;
  std::cout << "  --graph <path>        Path for the graph file.                   ()" << std::endl;
  std::cout << "                          Supported formats: edge lists, matrix" << std::endl;
  std::cout << "                          market files and binary CSR." << std::endl;
  std::cout << "  --partitioner <str>   Name of the partitioner algorithm.         (pal)" << std::endl;
  std::cout << "                          Algorithms: [uni | n1d | pal]" << std::endl;
  std::cout << "                          uni: uniform, checkerboard partitioning" << std::endl;
  std::cout << "                          n1d: Nicol's 1D Partitioning" << std::endl;
  std::cout << "                          rac: refine a cut partitioning" << std::endl;
  std::cout << "                          pal: probe a load partitioning" << std::endl;
  std::cout << "  --ncut <int>          Number of cuts                             (16)" << std::endl;
  std::cout << "  --ngpu <int>          Number of GPUs to use                      (all)" << std::endl;
  std::cout << "                          Note: this build counts on one GPU." << std::endl;
  std::cout << "  --nstream <int>       Number of streams per GPU                  (4)" << std::endl;
  std::cout << "                          Note: Cannot be 0." << std::endl;
  std::cout << "  --border <int>        Work queue border for GPUs                 (|T|/2)" << std::endl;
  std::cout << "                          Note: if set to -1, GPUs process all." << std::endl;
  std::cout << "  --cpu-workers <int>   CPU workers beside the GPU                 (0)" << std::endl;
  std::cout << "                          Note: -1 = threads minus GPU streams." << std::endl;
  std::cout << "  --copy-first          If set then copy graph to GPUs first       (false)" << std::endl;
  std::cout << "  --repeat <int>        Run bbTC algorithm '--repeat' times        (5)" << std::endl;
  std::cout << std::endl;
  std::cout << "Examples:" << std::endl;
  std::cout << "  bbtc --graph email-EuAll_adj.mtx --partitioner n1d --ncut 4" << std::endl;
  std::cout << "  bbtc --graph email-EuAll_adj.txt --ncut 4 --copy-first --border 4" << std::endl;
  std::cout << "  bbtc --graph email-EuAll_adj.el --border 4 --ngpu 1" << std::endl;
}

void CheckIntParams(const std::string& s, int p, int st = 0, int en = INT_MAX) {
  if (p <= st || p >= en) {
    std::cout << s << " has to be set in between: " << st << " < " << s << " < " << en << std::endl;
    PrintUsage();
    std::exit(0);
  }
}

bool FileExist(const std::string& name) {
  struct stat sb;
  return stat(name.c_str(), &sb) == 0;
}

int ToInt(const char* s) {
  char* end = nullptr;
  const long v = std::strtol(s, &end, 10);
  if (!s[0] || *end) {
    std::cout << "Wrong input" << std::endl;
    std::exit(0);
  }
  return (int)v;
}

void ParseArguments(Parameters& p, int argc, const char** argv, int devices) {
  if (argc < 3) {
    PrintUsage();
    std::exit(0);
  }
  p.n_gpu = devices;
  for (int i = 1; i < argc; i++) {
    const std::string a = lower(argv[i]);
    auto next = [&]() -> const char* {
      if (i + 1 >= argc) {
        std::cout << "Wrong input" << std::endl;
        std::exit(0);
      }
      return argv[++i];
    };
    if (a == "--graph") {
      p.file_name = next();
    } else if (a == "--ngpu") {
      const int t = ToInt(next());
      CheckIntParams("--ngpu", t, -1, devices + 1);
      p.n_gpu = t;
    } else if (a == "--nstream") {
      p.n_stream = ToInt(next());
      CheckIntParams("--nstream", p.n_stream);
    } else if (a == "--border") {
      p.border = ToInt(next());
      CheckIntParams("--border", p.border, -2);
    } else if (a == "--cpu-workers") {
      p.cpu_workers = ToInt(next());
      CheckIntParams("--cpu-workers", p.cpu_workers, -2);  // bounds are strict: -1 and up
    } else if (a == "--repeat") {
      p.repeat = ToInt(next());
      CheckIntParams("--repeat", p.repeat);
    } else if (a == "--copy-first") {
      p.copy_first = true;
    } else if (a == "--ncut") {
      p.ncut = ToInt(next());
      CheckIntParams("--ncut", p.ncut, 1, 65);
    } else if (a == "--partitioner") {
      p.part_name = next();
      if (p.part_name != "pal" && p.part_name != "n1d" && p.part_name != "rac" && p.part_name != "uni") {
        std::cout << "Wrong partitioning algorithm." << std::endl;
        PrintUsage();
        std::exit(0);
      }
    } else if (a == "--help") {
      PrintUsage();
      std::exit(0);
    } else {
      std::cout << "Wrong argument '" << argv[i] << "' given." << std::endl;
      PrintUsage();
      std::exit(0);
    }
  }
  if (!FileExist(p.file_name)) {
    std::cout << "Graph doesn't exist" << std::endl;
    PrintUsage();
    std::exit(0);
  }
}

}  // namespace

int main(int argc, const char** argv) {
  int devices = 0;
  {
    // the device count decides --ngpu's range, as in the reference (utils.hpp:93-95)
    bbtc_ctx* probe = nullptr;
    if (bbtc_ctx_create(0, &probe) == BBTC_OK) {
      devices = 1;
      bbtc_ctx_destroy(probe);
    }
  }
  Parameters params;
  ParseArguments(params, argc, argv, devices);
  if (devices == 0) {
    char buf[512];
    bbtc_last_error(buf, sizeof(buf));
    std::cout << "No usable B200 GPU: " << buf << std::endl;
    return 1;
  }
  if (params.n_gpu != 1) {
    std::cout << "--ngpu " << params.n_gpu << " is not served: this build counts on exactly one GPU." << std::endl;
    std::exit(0);
  }

  // graph: the .bbtc cache when present, else the text file (utils.hpp:168-170)
  std::string path = params.file_name;
  const bool cached = FileExist(path + ".bbtc");
  if (cached) path += ".bbtc";
  void* h = nullptr;
  int kind = 0;
  const int rc = bbtcio_read(path.c_str(), &kind, &h);
  if (rc != 0) {
    std::cout << "Unable to read the graph file '" << path << "' (" << rc << ")." << std::endl;
    return 1;
  }
  uint32_t n = 0;
  uint64_t m = 0;
  bbtcg_info(h, &n, &m, nullptr);
  std::vector<uint32_t> indptr((size_t)n + 1), indices(m);
  bbtcg_copy(h, indptr.data(), indices.data());
  bbtcg_free(h);
  std::cerr << "# Graph read.. N: " << n << ", NNZ: " << m << std::endl;
  if (kind != 2) {
    std::cerr << "# Saving binary CSR graph.." << std::endl;
    if (bbtcio_write_bbtc((params.file_name + ".bbtc").c_str(), n, indptr.data(), indices.data(), m) != 0)
      std::cerr << "# could not write " << params.file_name << ".bbtc" << std::endl;
  }

  try {
    bbtc::Context ctx(0);
    const uint32_t P = (uint32_t)params.ncut;
    // pal, the default
    const int pk = params.part_name == "uni" ? 0 : params.part_name == "n1d" ? 1 : params.part_name == "rac" ? 4 : 2;
    std::vector<uint32_t> cuts(P + 1);
    RegionBegin();
    bbtc::check(bbtcp_cuts(pk, n, indptr.data(), indices.data(), P, 1091467301ull, cuts.data()));
    bbtc::BlockCSR st(ctx, cuts, indptr, indices);
    RegionEnd("Partitioning and Layout construction (s)");

    auto t_list = bbtc::tasks::TaskList(P);
    bbtc::tasks::SortTasks(t_list, st);
    bbtc::BBTc bb(ctx, &st, t_list, P);
    bb.InitFlags();
    bb.SetNGPU(params.n_gpu);

    std::cout << "=====================================" << std::endl;
    std::cout << "Graph file: " << params.file_name << std::endl;
    std::cout << "Number of Vertices: " << st.GetNoOfVertices() << std::endl;
    std::cout << "Number of Edges: " << st.GetNoOfEdges() << std::endl;
    std::cout << "Number of Cuts: " << P << std::endl;
    std::cout << "Number of Tasks: " << t_list.size() << std::endl;
    std::cout << "Number of GPUs: " << bb.GetNGPU() << std::endl;
    std::cout << "Number of Workers: " << omp_get_max_threads() << std::endl;
    std::cout << "=====================================" << std::endl;

    if (params.border == -1 || params.border > (int)t_list.size())
      bb.Separator = (int)t_list.size();
    else if (params.border == -2)
      bb.Separator = (int)t_list.size() / 2;
    else
      bb.Separator = params.border;

    if (params.cpu_workers != 0) {
      const int k = params.cpu_workers > 0 ? params.cpu_workers
                                           : std::max(0, omp_get_max_threads() - params.n_stream * params.n_gpu);
      bb.SetCpuWorkers((uint32_t)k, indptr, indices);
    }

    RegionBegin();
    bb.PrepareGpu();
    RegionEnd("Cuda Initial Memory Allocations and Stream Creation");

    unsigned long long n_triangles = 0;
    for (int i = 0; i < params.repeat; i++) {
      bb.ResetFlags();
      if (params.copy_first) {
        RegionBegin();
        bb.CopyTilesToGpu();
        RegionEnd("Copy tiles to device (s)");
      }
      RegionBegin();
      n_triangles = bb.NoOfTriangles();
      RegionEnd("Triangle Counting Execution Time (s)");
    }
    std::cout << "Number of Triangles: " << n_triangles << std::endl;
    for (auto& f : g_fields) std::cout << f.first << " : " << f.second << std::endl;
    bb.CleanUp();
    st.CleanUp();
  } catch (const bbtc::Error& e) {
    std::cout << "bbtc error " << e.status() << ": " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
