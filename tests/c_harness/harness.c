/*
 * A plain C caller of the library (no Python, no C++): the sequence a Fortran
 * or C driver runs -- create a solver from the equation and parameter files,
 * import a QuickSave directory, factorise, march, read the state back -- with
 * every return code checked.  Prints the step count, the relative change of
 * the state and the diagnostics.
 *
 * usage: harness <coral.equations> <coral.parameters.in> <QuickSave dir> <nsteps> <dt>
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "coral_b200.h"

#define CHECK(call)                                                                  \
  do {                                                                               \
    int rc_ = (call);                                                                \
    if (rc_ != CORAL_OK) {                                                           \
      fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, coral_last_error(h));      \
      return 1;                                                                      \
    }                                                                                \
  } while (0)

int main(int argc, char** argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: %s equations parameters quicksave_dir nsteps dt\n", argv[0]);
    return 2;
  }
  coral_handle* h = NULL;
  int rc = coral_create_from_files(argv[1], argv[2], NULL, 0, &h);
  if (rc != CORAL_OK) {
    fprintf(stderr, "coral_create_from_files failed (%d): %s\n", rc, coral_last_error(NULL));
    return 1;
  }
  const int nsteps = atoi(argv[4]);
  const double dt = atof(argv[5]);
  long long NXH, NYAA, T;
  CHECK(coral_query(h, CORAL_Q_NX, &NXH));
  NXH /= 2;
  CHECK(coral_query(h, CORAL_Q_NYAA, &NYAA));
  CHECK(coral_query(h, CORAL_Q_SYS_T + 0, &T));
  const size_t n = (size_t)(NXH * NYAA * T) * 2;
  double* f0 = (double*)malloc(n * sizeof(double));
  double* f1 = (double*)malloc(n * sizeof(double));
  if (!f0 || !f1) return 3;
  CHECK(coral_import_quicksave(h, argv[3], 1));
  CHECK(coral_get_field(h, 0, f0));
  CHECK(coral_factorize(h, dt));
  CHECK(coral_march(h, dt, nsteps));
  CHECK(coral_synchronize(h));
  CHECK(coral_get_field(h, 0, f1));
  double num = 0.0, den = 0.0;
  for (size_t i = 0; i < n; ++i) {
    num += (f1[i] - f0[i]) * (f1[i] - f0[i]);
    den += f0[i] * f0[i];
  }
  double diag[3];
  CHECK(coral_diagnostics(h, diag));
  printf("steps %d rel_change %.17e cfl_dt %.17e KE %.17e nonfinite %d\n", nsteps, sqrt(num / den), diag[0], diag[1],
         (int)diag[2]);
  free(f0);
  free(f1);
  coral_destroy(h);
  return 0;
}
