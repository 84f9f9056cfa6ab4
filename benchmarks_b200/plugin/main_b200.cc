// Benchmark driver for Diffusion3DB200 with the reference driver's
// command line (src/diffusion3d/main.cc:84-126): --count N, --size N,
// --dump, --help; cubic grid of side --size (default 256), 100 steps.
// Two additions: --kernel {auto,generic,tb2,tb3,tb4} picks the B200 kernel,
// and --dump-binary dumps a binary checkpoint instead of the text.
// In the reference tree the same selection is one more branch of main.cc's
// variant chain: `#elif defined(CUDA_B200)` creating a Diffusion3DB200.
#include <getopt.h>
#include <stdlib.h>
#include <string.h>

#include <iostream>

#include "diffusion3d_b200.h"

namespace {

void Usage(const char* prog) {
  std::cerr << "Usage: " << prog << " [options]\n\n"
            << "Options\n"
            << "\t--count N   Number of iterations\n"
            << "\t--size N    Size of each dimension\n"
            << "\t--dump      Dump the final data to file\n"
            << "\t--dump-binary  Dump a binary checkpoint (.d3d) instead\n"
            << "\t--kernel K  auto | generic | tb2 | tb3 | tb4\n"
            << "\t--help      Display this help message\n";
}

}  // namespace

int main(int argc, char* argv[]) {
  int size = 256, count = 100, kernel = D3D_KERNEL_AUTO, depth = 1;
  bool dump = false, binary = false;
  static struct option opts[] = {{"count", 1, 0, 0},  {"size", 1, 0, 0},
                                 {"dump", 0, 0, 0},   {"help", 0, 0, 0},
                                 {"kernel", 1, 0, 0}, {"dump-binary", 0, 0, 0},
                                 {0, 0, 0, 0}};
  for (;;) {
    int idx = 0;
    const int c = getopt_long(argc, argv, "", opts, &idx);
    if (c == -1) break;
    if (c != 0) continue;  // unknown options are ignored, as in main.cc
    switch (idx) {
      case 0: count = atoi(optarg); break;
      case 1: size = atoi(optarg); break;
      case 2: dump = true; break;
      case 3: Usage(argv[0]); return EXIT_SUCCESS;
      case 4:
        if (!strcmp(optarg, "generic")) {
          kernel = D3D_KERNEL_GENERIC;
        } else if (!strncmp(optarg, "tb", 2)) {
          kernel = D3D_KERNEL_TB;
          depth = atoi(optarg + 2);
        } else {
          kernel = D3D_KERNEL_AUTO;
        }
        break;
      case 5: dump = binary = true; break;
    }
  }
  diffusion3d::Diffusion3D* bmk =
      new diffusion3d::Diffusion3DB200(size, size, size, kernel, depth,
                                       binary);
  bmk->RunBenchmark(count, dump);
  delete bmk;
  return 0;
}
