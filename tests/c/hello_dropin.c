/* A caller written the way the reference's own callers are (its Hello.c and
 * benchmark/small_SGEMM/LibShalom_sgemm.c): plain C, malloc'd HOST buffers,
 * the drop-in LibShalom_sgemm(NoTrans, Trans, ...) on an 80^3 problem with
 * inputs from srand48(seed); 2.0 * (float)drand48() - 1.0, A then B.  It
 * compiles against include/LibShalom.h alone and links the library.
 *
 * usage: hello_dropin <seed> <output file>   (C written as raw float32) */
#include <stdio.h>
#include <stdlib.h>

#include "LibShalom.h"

int main(int argc, char **argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s <seed> <output file>\n", argv[0]);
    return 2;
  }
  long M, N, K;
  M = N = K = 80;
  float *A = (float *)malloc(K * M * sizeof(float));
  float *B = (float *)malloc(K * N * sizeof(float));
  float *C = (float *)malloc(M * N * sizeof(float));
  if (!A || !B || !C) return 3;
  srand48(atol(argv[1]));
  for (long i = 0; i < M * K; ++i) A[i] = 2.0 * (float)drand48() - 1.0;
  for (long i = 0; i < N * K; ++i) B[i] = 2.0 * (float)drand48() - 1.0;
  /* warm-up and repeated calls, as the reference's caller does */
  for (int it = 0; it < 3; ++it) LibShalom_sgemm(NoTrans, Trans, C, A, B, M, N, K);
  int st = LibShalom_get_last_error();
  if (st != LIBSHALOM_SUCCESS) {
    fprintf(stderr, "LibShalom_sgemm: %s\n", LibShalom_error_string(st));
    return 4;
  }
  FILE *f = fopen(argv[2], "wb");
  if (!f || fwrite(C, sizeof(float), M * N, f) != (size_t)(M * N)) return 5;
  fclose(f);
  LibShalom_finalize();
  free(A);
  free(B);
  free(C);
  return 0;
}
