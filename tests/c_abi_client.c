/* A plain C99 client of the sp2b C ABI (include/sp2b.h, include/prg_sp2b.h), built and run
 * by tests/test_c_client.py.  It calls the host-side entry points only (no GPU) and prints
 * their results, one labelled line each, for the test to compare with the oracle. */
#include <stdio.h>
#include <stdlib.h>

#include "prg_sp2b.h"
#include "sp2b.h"

int main(void) {
  sp2b_opts o;
  int pp[100], imax = 0, i, nparts = 0, choice = -1, nms = 0;
  int part_ptr[16], nodes[100];
  int sgn[6] = {1, -1, 1, -1, -1, 1};
  double gg[1001], ee[1001], g2[1001], e2[1001];
  double buf[4] = {1.0, 2.0, 3.0, 4.0};
  float ms[4];
  bml_matrix_t* m;

  if (sp2b_opts_default(&o) != SP2B_OK) return 1;
  printf("opts %d %d %d\n", o.precision, o.mcweeny, o.device_ptrs);

  if (sp2b_sp2sequence(pp, &imax, -2.0, 3.0, 0.1, 0.5, 1e-12, 100) != SP2B_OK) return 2;
  printf("seq %d", imax);
  for (i = 0; i < imax; ++i) printf(" %d", pp[i]);
  printf("\n");

  if (sp2b_equal_partition(12, 100, &nparts, NULL, NULL) != SP2B_OK || nparts > 15) return 3;
  if (sp2b_equal_partition(12, 100, &nparts, part_ptr, nodes) != SP2B_OK) return 4;
  printf("parts %d", nparts);
  for (i = 0; i <= nparts; ++i) printf(" %d", part_ptr[i]);
  printf("\n");

  if (sp2b_sp2_entropy_function(-0.3, -2.0, 2.5, 6, sgn, gg, ee, 1001) != SP2B_OK) return 5;
  prg_sp2_entropy_function(-0.3, -2.0, 2.5, 6, sgn, g2, e2);
  if (sp2b_prg_last_status() != SP2B_OK) return 6;
  for (i = 0; i < 1001; ++i)
    if (gg[i] != g2[i] || ee[i] != e2[i]) return 7;
  printf("entropy %.17g %.17g %.17g\n", gg[1], gg[500], gg[1000]);

  if (sp2b_tune_set("c-client/key", 7) != SP2B_OK) return 8;
  if (sp2b_tune_get("c-client/key", &choice, ms, 4, &nms) != SP2B_OK) return 9;
  printf("tune %d %d %d\n", choice, nms, sp2b_tune_set("bad key", 1));

  m = sp2b_bml_wrap_dense(buf, 2);
  if (!m || sp2b_bml_n(m) != 2 || sp2b_bml_data(m) != buf) return 10;
  sp2b_bml_free(m);
  printf("bml ok\n");
  return 0;
}
