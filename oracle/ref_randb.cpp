// Harness around the reference's random-boundary generator
// (lib/random-boundary/randomBound.h, included from the reference tree, not
// copied): reads n1 n2 n3 pad pctG seed and a float32 field from argv[1],
// applies RandomMY(field, 1, 0.2, dims, {pad, pad, pad}, pctG, seed) as
// randomB.x does (randomBound.cpp:40-42) and writes the field to argv[2].
// Built into oracle/_ref by build_ref.sh; test infrastructure only.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "randomBound.h"

int main(int argc, char** argv) {
  if (argc != 9) {
    std::fprintf(stderr, "usage: ref_randb in.f32 out.f32 n1 n2 n3 pad pctG seed\n");
    return 2;
  }
  const int n1 = std::atoi(argv[3]), n2 = std::atoi(argv[4]), n3 = std::atoi(argv[5]);
  const int pad = std::atoi(argv[6]);
  const float pct = (float)std::atof(argv[7]);
  const int seed = std::atoi(argv[8]);
  std::vector<float> f((size_t)n1 * n2 * n3);
  FILE* in = std::fopen(argv[1], "rb");
  if (!in || std::fread(f.data(), 4, f.size(), in) != f.size()) return 3;
  std::fclose(in);
  std::vector<int> dims = {n1, n2, n3};
  std::vector<int> thick = {pad, pad, pad};
  SEPMY::RandomMY(f.data(), 1, 0.2, dims, thick, pct, seed);
  FILE* out = std::fopen(argv[2], "wb");
  if (!out || std::fwrite(f.data(), 4, f.size(), out) != f.size()) return 4;
  std::fclose(out);
  return 0;
}
