// zsph_deltasph: the reference's deltasph program (single_gpu_sph_src/deltasph/
// main.cu) on this library.  Usage: zsph_deltasph [case.json] [--fused] [--simple]
// The case file defaults to ../input/input.json, as the reference's does; the
// initial particles are read from <input_path>/input.vtk and the outputs go to
// <output_path>/zsph<step>.vtk.  --fused runs one fused step per step instead
// of the reference's twelve launches; --simple runs the simple-SPH equations
// (the reference's simplesph program).  Optional case-file keys beyond the
// reference's: "equations", "eos", "snapshot_every" (snapshots of the state in
// output_path) and "resume" (continue from such a snapshot); the environment
// variable ZSPH_METRICS names a JSONL run log (see zsph_compat_run).
#include <cstdio>
#include <cstring>

#include "../include/zsph.h"

int main(int argc, char** argv) {
  const char* path = "../input/input.json";
  int mode = ZSPH_COMPAT_SEPARATE;
  for (int a = 1; a < argc; ++a) {
    if (std::strcmp(argv[a], "--fused") == 0) mode |= ZSPH_COMPAT_FUSED;
    else if (std::strcmp(argv[a], "--simple") == 0) mode |= ZSPH_COMPAT_SIMPLE;
    else path = argv[a];
  }
  int steps = 0;
  const int rc = zsph_compat_run(path, mode, &steps);
  if (rc != ZSPH_OK) {
    char msg[512];
    zsph_last_error(nullptr, msg, (int)sizeof msg);
    std::fprintf(stderr, "zsph_deltasph: %s (status %d, after %d steps)\n", msg, rc, steps);
    return 1;
  }
  std::printf("zsph_deltasph: %d steps of %s done\n", steps, path);
  return 0;
}
