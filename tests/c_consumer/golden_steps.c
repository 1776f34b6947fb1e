/* A plain C consumer of include/rigidfibers.h: reads an XcT fibers file
 * (count, then per fiber one line of position and one of orientation, the
 * format of the reference's src/parameters.cc:75-116), runs `steps` time
 * steps of the default configuration (tests/config.ini of the reference)
 * through rf_step, and prints the final positions then orientations, one
 * fiber per line.  Built and run by tests/test_c_consumer.py.
 *
 *   cc golden_steps.c -I include -L rigidfibers_b200 -lrigidfibers -o golden_steps
 *   ./golden_steps XcT_ref100.in 2 [gmres|bicgstab|direct]
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "rigidfibers.h"

static int fail(const char* what, int rc) {
  fprintf(stderr, "%s: %s: %s\n", what, rf_status_string(rc), rf_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 3) { fprintf(stderr, "usage: %s fibers.in steps [solver]\n", argv[0]); return 2; }
  FILE* f = fopen(argv[1], "r");
  int n = 0, steps = atoi(argv[2]);
  if (!f || fscanf(f, "%d", &n) != 1 || n < 1) { fprintf(stderr, "cannot read %s\n", argv[1]); return 2; }
  double* pos = malloc(sizeof(double) * 3 * n);
  double* ori = malloc(sizeof(double) * 3 * n);
  for (int i = 0; i < n; ++i) {
    double* p = pos + 3 * i;
    double* o = ori + 3 * i;
    if (fscanf(f, "%lf %lf %lf %lf %lf %lf", p, p + 1, p + 2, o, o + 1, o + 2) != 6) return 2;
  }
  fclose(f);
  rf_config cfg;
  rf_config_default(&cfg);
  if (argc > 3 && strcmp(argv[3], "bicgstab") == 0) cfg.solver = RF_SOLVER_BICGSTAB;
  if (argc > 3 && strcmp(argv[3], "direct") == 0) cfg.solver = RF_SOLVER_DIRECT;
  rf_handle* h = NULL;
  int rc = rf_create(&cfg, n, pos, ori, &h);
  if (rc != RF_OK) return fail("rf_create", rc);
  for (int t = 0; t < steps; ++t)
    if ((rc = rf_step(h, t)) != RF_OK) return fail("rf_step", rc);
  if ((rc = rf_get_state(h, pos, ori)) != RF_OK) return fail("rf_get_state", rc);
  for (int i = 0; i < n; ++i) printf("%.17g %.17g %.17g\n", pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  for (int i = 0; i < n; ++i) printf("%.17g %.17g %.17g\n", ori[3 * i], ori[3 * i + 1], ori[3 * i + 2]);
  rf_destroy(h);
  free(pos);
  free(ori);
  return 0;
}
