/* Host-side use of the schedule table through the plain C ABI (no device
 * needed): candidates, built-in rules, set/get by batch class, listing, and a
 * save/load round trip.  Prints "ok" and exits 0 on success. */
#include <stdio.h>
#include <string.h>

#include "rcwa_b200.h"

#define CHECK(cond)                                                   \
  do {                                                                \
    if (!(cond)) {                                                    \
      fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #cond); \
      return 1;                                                       \
    }                                                                 \
  } while (0)

int main(int argc, char** argv) {
  const char* path = argc > 1 ? argv[1] : "tuner_table.txt";
  rcwa_tuner* t = NULL;
  CHECK(rcwa_tuner_create(&t) == RCWA_OK && t);
  CHECK(rcwa_tuner_set_sms(t, 148) == RCWA_OK);
  int c[4];
  CHECK(rcwa_tuner_candidates(RCWA_TUNE_LU, 882, c) == 3 && c[0] == 0 && c[1] == 1 && c[2] == 2);
  CHECK(rcwa_tuner_candidates(RCWA_TUNE_LU, 200, c) == 2);
  CHECK(rcwa_tuner_candidates(RCWA_TUNE_SCHUR, 300, c) == 4 && c[3] == 192);
  CHECK(rcwa_tuner_candidates(7, 300, c) == -1);
  CHECK(rcwa_tuner_default(t, RCWA_TUNE_LU, 882, 148) == 2);
  CHECK(rcwa_tuner_default(t, RCWA_TUNE_LU, 200, 148) == 1);
  CHECK(rcwa_tuner_default(t, RCWA_TUNE_LU, 882, 600) == 0);
  CHECK(rcwa_tuner_set(t, RCWA_TUNE_SCHUR, 300, 20, 96) == RCWA_OK);
  CHECK(rcwa_tuner_set(t, RCWA_TUNE_LU, 882, 296, 0) == RCWA_OK);  /* 2 waves */
  CHECK(rcwa_tuner_set(t, RCWA_TUNE_LU, 882, 296, 5) == RCWA_ERR_INVALID);
  int choice = -2;
  CHECK(rcwa_tuner_get(t, RCWA_TUNE_LU, 882, 250, &choice) == RCWA_OK && choice == 0);
  CHECK(rcwa_tuner_get(t, RCWA_TUNE_LU, 882, 100, &choice) == RCWA_OK && choice == -1);
  CHECK(rcwa_tuner_count(t) == 2);
  int op, n, cls, ch, nc, cand[4];
  double ms[4];
  CHECK(rcwa_tuner_entry(t, 0, &op, &n, &cls, &ch, &nc, cand, ms) == RCWA_OK);
  CHECK(op == RCWA_TUNE_LU && n == 882 && cls == 2 && ch == 0 && nc == 3);
  CHECK(rcwa_tuner_entry(t, 2, &op, &n, &cls, &ch, &nc, cand, ms) == RCWA_ERR_INVALID);
  CHECK(rcwa_tuner_save(t, path) == RCWA_OK);
  rcwa_tuner* u = NULL;
  CHECK(rcwa_tuner_create(&u) == RCWA_OK);
  CHECK(rcwa_tuner_load(u, path) == RCWA_OK);
  CHECK(rcwa_tuner_count(u) == 2);
  CHECK(rcwa_tuner_get(u, RCWA_TUNE_SCHUR, 300, 20, &choice) == RCWA_OK && choice == 96);
  rcwa_tuner_destroy(u);
  rcwa_tuner_destroy(t);
  printf("ok\n");
  return 0;
}
