// ls_tune.cu -- shape-class tuning table of the GEMM schedulers.
//
// A shape class is (kind, b(M), b(N), b(K)) with b(x) the half-octave of x:
// 2 floor(log2 x) + (x >= 1.5 * 2^floor(log2 x)).  The table
// (ls_tune_table.inc) is written by libshalom_b200/autotune.py from CUDA-event
// timings of every candidate tile configuration and split-K factor on a B200;
// the library consults it before its cost model, and a class that is not in
// the table falls back to the model.
#include <algorithm>

#include "ls_common.cuh"
#include "ls_simt_launch.h"

namespace ls {

namespace {

struct TuneEntry {
  unsigned char kind, mb, nb, kb;
  signed char cfg;       // tile configuration (plain kinds), -1 = model
  unsigned char splits;  // split-K factor, 0 = model
};

const TuneEntry kTune[] = {
#include "ls_tune_table.inc"
    {255, 0, 0, 0, -1, 0},  // end
};

}  // namespace

int half_octave(long x) {
  if (x <= 1) return 0;
  const int e = 63 - __builtin_clzll((unsigned long long)x);
  const int half = e >= 1 && x >= (3L << (e - 1));
  return std::min(127, 2 * e + half);
}

bool tune_lookup(int kind, long M, long N, long K, int *cfg, int *splits) {
  const int mb = half_octave(M), nb = half_octave(N), kb = half_octave(K);
  for (const TuneEntry *t = kTune; t->kind != 255; ++t) {
    if (t->kind == kind && t->mb == mb && t->nb == nb && t->kb == kb) {
      *cfg = t->cfg;
      *splits = t->splits;
      return true;
    }
  }
  return false;
}

int tune_table_size() {
  int n = 0;
  for (const TuneEntry *t = kTune; t->kind != 255; ++t) ++n;
  return n;
}

}  // namespace ls
