// Drop-in replacement of the reference's solver binary: `main_debug <model.json> <out_root>`
// (src/main.cu:58-76). Same two arguments, same output tree, exit code 1 on error.
// MFDM_DEVICE selects the CUDA device (default 0); MFDM_BATCH=1 runs every source
// of the JSON as one batch, each from rest (mfdm_run_cli_batch).
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
  const char* batch = std::getenv("MFDM_BATCH");
  const int device = dev ? std::atoi(dev) : 0;
  const int rc = (batch && batch[0] == '1') ? mfdm_run_cli_batch(argv[1], argv[2], device)
                                            : mfdm_run_cli(argv[1], argv[2], device);
  if (rc != MFDM_OK) {
    std::fprintf(stderr, "error: %s\n", mfdm_last_error());
    return 1;
  }
  return 0;
}
