// Drop-in replacement of the reference's solver binary: `main_debug <model.json> <out_root>`
// (src/main.cu:58-76). Same two arguments, same output tree, exit code 1 on error.
// MFDM_DEVICE selects the CUDA device (default 0).
#include <cstdio>
#include <cstdlib>

#include "../../include/mfdm.h"

int main(int argc, char* argv[]) {
  if (argc != 3) {
    std::fprintf(stderr,
                 "usage: %s <model.json> <output_dir>\n"
                 "example: %s models/case/case.json output/case\n",
                 argv[0], argv[0]);
    return 1;
  }
  const char* dev = std::getenv("MFDM_DEVICE");
  const int rc = mfdm_run_cli(argv[1], argv[2], dev ? std::atoi(dev) : 0);
  if (rc != MFDM_OK) {
    std::fprintf(stderr, "error: %s\n", mfdm_last_error());
    return 1;
  }
  return 0;
}
