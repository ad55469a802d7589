/* A plain C99 caller of include/zsph.h, for the CPU test of the boundary
 * (tests/test_c_abi_cpu.py): it proves that the header compiles as C, that
 * the library's entry points link with C linkage, and it reports the size of
 * every public struct as a C compiler lays it out, so that the Python mirror
 * of the structs can be checked against it.  With a case file argument it
 * runs the host-only set-up calls (read_json, set_cpu_param, set_gpu_param,
 * check_dt; no CUDA call) and prints the derived GPU parameters as hex. */
#include <stdio.h>
#include <string.h>

#include "zsph.h"

int main(int argc, char** argv) {
  printf("sizeof zsph_json_t %zu\n", sizeof(zsph_json_t));
  printf("sizeof zsph_cpu_param_t %zu\n", sizeof(zsph_cpu_param_t));
  printf("sizeof zsph_gpu_param_t %zu\n", sizeof(zsph_gpu_param_t));
  printf("sizeof zsph_ptc_t %zu\n", sizeof(zsph_ptc_t));
  printf("sizeof zsph_tmp_t %zu\n", sizeof(zsph_tmp_t));
  printf("sizeof zsph_learn_train_stats_t %zu\n", sizeof(zsph_learn_train_stats_t));
  printf("sizeof zsph_learn_run_stats_t %zu\n", sizeof(zsph_learn_run_stats_t));
  printf("sizeof zsph_tune_t %zu\n", sizeof(zsph_tune_t));
  printf("sizeof zsph_conservation_t %zu\n", sizeof(zsph_conservation_t));
  printf("sizeof zsph_rigid_t %zu\n", sizeof(zsph_rigid_t));
  printf("sizeof zsph_case_options_t %zu\n", sizeof(zsph_case_options_t));
  if (argc < 2) return 0;
  zsph_json_t j;
  zsph_cpu_param_t cp;
  zsph_gpu_param_t gp;
  char err[256];
  int rc = zsph_read_json(argv[1], &j, err, (int)sizeof err);
  if (rc != ZSPH_OK) {
    printf("read_json %d %s\n", rc, err);
    return 1;
  }
  rc = zsph_set_cpu_param(&cp, &j);
  printf("set_cpu_param %d\n", rc);
  float dt_max = 0.0f;
  printf("check_dt %d\n", zsph_check_dt(&cp, &dt_max));
  memset(&gp, 0, sizeof gp);
  rc = zsph_set_gpu_param(&gp, &cp);
  printf("set_gpu_param %d\n", rc);
  printf("grid_num %d\n", cp.grid_num);
  printf("gparam ");
  const unsigned char* b = (const unsigned char*)&gp;
  for (size_t k = 0; k < sizeof gp; ++k) printf("%02x", b[k]);
  printf("\n");
  return 0;
}
