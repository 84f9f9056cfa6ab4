// Benchmark driver for DiffusionB200 with the reference diffusion driver's
// command line (src/diffusion/main.cc:84-217): --nd N (2 or 3, default 3),
// --count N (100), --size N (256), --dump, --warmup, --help; the grid has
// nd sides of --size.  Two additions: --kernel {auto,generic,tb2,tb3,tb4}
// picks the B200 kernel (tb* in 3D only), and --dump-binary dumps a binary
// checkpoint instead of the text.  In the reference tree the same
// selection is one more branch of main.cc's variant chain, creating a
// DiffusionB200.
#include <assert.h>
#include <getopt.h>
#include <stdlib.h>
#include <string.h>

#include <iostream>
#include <vector>

#include "diffusion_b200.h"

namespace {

void Usage(const char* prog) {
  std::cerr << "Usage: " << prog << " [options]\n\n"
            << "Options\n"
            << "\t--nd N      Number of dimensions (default: 3)\n"
            << "\t--count N   Number of iterations (default: 100)\n"
            << "\t--size N    Size of each dimension (default: 256)\n"
            << "\t--dump      Dump the final data to file\n"
            << "\t--warmup    Enable warming-up runs\n"
            << "\t--dump-binary  Dump a binary checkpoint (.d3d) instead\n"
            << "\t--kernel K  auto | generic | tb2 | tb3 | tb4\n"
            << "\t--help      Display this help message\n";
}

}  // namespace

int main(int argc, char* argv[]) {
  int nd = 3, size = 256, count = 100, kernel = D3D_KERNEL_AUTO, depth = 1;
  bool dump = false, warmup = false, binary = false;
  static struct option opts[] = {
      {"nd", 1, 0, 0},     {"count", 1, 0, 0},       {"size", 1, 0, 0},
      {"dump", 0, 0, 0},   {"warmup", 0, 0, 0},      {"help", 0, 0, 0},
      {"kernel", 1, 0, 0}, {"dump-binary", 0, 0, 0}, {0, 0, 0, 0}};
  for (;;) {
    int idx = 0;
    const int c = getopt_long(argc, argv, "", opts, &idx);
    if (c == -1) break;
    if (c != 0) continue;  // unknown options are ignored, as in main.cc
    switch (idx) {
      case 0: nd = atoi(optarg); break;
      case 1: count = atoi(optarg); break;
      case 2: size = atoi(optarg); break;
      case 3: dump = true; break;
      case 4: warmup = true; break;
      case 5: Usage(argv[0]); return EXIT_SUCCESS;
      case 6:
        if (!strcmp(optarg, "generic")) {
          kernel = D3D_KERNEL_GENERIC;
        } else if (!strncmp(optarg, "tb", 2)) {
          kernel = D3D_KERNEL_TB;
          depth = atoi(optarg + 2);
        } else {
          kernel = D3D_KERNEL_AUTO;
        }
        break;
      case 7: dump = binary = true; break;
    }
  }
  assert(nd >= 2 && nd <= 3);
  std::vector<int> dims(nd, size);
  // A concrete object: the surface's base class has no virtual destructor.
  diffusion::DiffusionB200 bmk(nd, dims.data(), kernel, depth, binary);
  bmk.RunBenchmark(count, dump, warmup);
  return 0;
}
