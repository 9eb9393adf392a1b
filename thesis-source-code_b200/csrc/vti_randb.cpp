// Random-boundary generator: restatement of the reference's cluster random
// walk (lib/random-boundary/randomBound.h:48-396, RandomMY, as randomB.x calls
// it: randomBound.cpp:40-42). Host code.
//
// The pad cells (distance > 0 from the interior box) are partitioned into
// clusters grown by a random walk; every cluster gets one multiplier drawn
// from a window that depends on its seed cell's distance into the pad, and
// the field is multiplied cluster by cluster. The reference draws every
// random number from the C library's rand() after srand(seed); so does this
// code, in the same order, so the same C library gives the same boundary:
//   * a buffer of 50000 uniforms (1.0 * rand() / RAND_MAX) refilled when an
//     index runs past it (the refill thresholds differ by call site, :133,
//     :173, :383);
//   * seed cell of a cluster: round((nbound-1) * u) in float, moved to the
//     nearest unused cell at growing distance in the pad list (:362-389);
//   * growth: stop with probability 1 - pctG; otherwise pick the
//     round((size-1) * u)-th member of the cluster (ordered by pad index),
//     list the free neighbours among 26 (3D, weight 1) or 8 (2D, weights
//     e^-1 edge / e^-2 corner) directions, draw one by its cumulative weight
//     (first direction whose running sum reaches u * total), add it; a
//     member with no free neighbour leaves the growth set (:128-218);
//   * multipliers: cluster k (k < number of clusters; the last cluster keeps
//     1, as in the reference's loop bound :225) with pct = d_seed / max(pad):
//     pct == 0 gives 1; otherwise rand() draws r = (u - 0.5) * pct + base,
//     base = (1 - pct) * bval + pct * eval, until r lies in (eval/3, 1)
//     (eval < bval, velocity) or (1, 3 eval) (density) (:223-248).
// Deliberate differences: the seed distance of "cluster 0" (never a real
// cluster) is read by the reference from an uninitialised array element
// (:225, start[0]); it is taken as 0 here (what a fresh zero-filled
// allocation holds), which draws no random number for it. When the growth
// step's index runs one past the 50000-number buffer (:142 has no refill
// check) the reference reads beyond its buffer; this code reads 0 there.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <set>
#include <vector>

#include "vti_b200.h"

namespace {

struct Rng {
  static constexpr int kLen = 50000;
  // one guard element: the growth step reads u[i + 1] without a refill
  // check (randomBound.h:142); the reference then reads past its buffer
  std::vector<float> u = std::vector<float>(kLen + 1, 0.f);
  int i = 0;
  void refill() {
    for (int k = 0; k < kLen; ++k) u[k] = (float)((1. * rand()) / RAND_MAX);
    i = 0;
  }
};

struct Dir {
  int d1, d2, d3;
  float w;
};

std::vector<Dir> directions(bool three_d) {
  std::vector<Dir> v;
  if (three_d) {
    for (int a = -1; a <= 1; ++a)
      for (int b = -1; b <= 1; ++b)
        for (int c = -1; c <= 1; ++c)
          if (a || b || c) v.push_back({a, b, c, 1.f});
  } else {
    const float e1 = (float)std::exp(-1.), e2 = (float)std::exp(-2.);
    for (int a = -1; a <= 1; ++a)
      for (int b = -1; b <= 1; ++b)
        if (a || b) v.push_back({a, b, 0, (a && b) ? e2 : e1});
  }
  return v;
}

}  // namespace

extern "C" int vti_random_boundary(float* field, int n1, int n2, int n3, int pad, float pct_g,
                                   int seed, float bval, float eval) {
  if (!field || n1 < 1 || n2 < 1 || n3 < 1 || pad < 0) return VTI_ERR_ARG;
  const bool three_d = n3 > 1;
  const long long ncell = (long long)n1 * n2 * n3;
  const int t1 = pad, t2 = pad, t3 = three_d ? pad : 0;
  if (2 * t1 >= n1 || 2 * t2 >= n2 || (three_d && 2 * t3 >= n3)) return VTI_ERR_ARG;
  srand((unsigned)seed);
  const std::vector<Dir> dir = directions(three_d);
  const int ndir = (int)dir.size();
  // pad cells in grid order, their distance into the pad, cluster labels
  // (-1 interior, 0 free, k > 0 cluster k)
  std::vector<int> label(ncell);
  std::vector<long long> pad_cell;
  std::vector<float> dist;
  std::vector<long long> pad_index(ncell, -1);
  for (int i3 = 0; i3 < n3; ++i3) {
    const int c3 = std::min(std::max(std::min(std::max(i3, t3), n3 - t3 - 1), 0), n3 - 1);
    const float q3 = (float)((i3 - c3) * (i3 - c3));
    for (int i2 = 0; i2 < n2; ++i2) {
      const int c2 = std::min(std::max(i2, t2), n2 - t2 - 1);
      const float q2 = (float)((i2 - c2) * (i2 - c2));
      for (int i1 = 0; i1 < n1; ++i1) {
        const int c1 = std::min(std::max(i1, t1), n1 - t1 - 1);
        const float q1 = (float)((i1 - c1) * (i1 - c1));
        const long long g = ((long long)i3 * n2 + i2) * n1 + i1;
        const float dd = (float)std::sqrt(q1 + q2 + q3);
        if ((double)dd > 0.01) {
          label[g] = 0;
          pad_index[g] = (long long)pad_cell.size();
          pad_cell.push_back(g);
          dist.push_back(dd);
        } else {
          label[g] = -1;
        }
      }
    }
  }
  const long long nbound = (long long)pad_cell.size();
  if (nbound == 0) return VTI_OK;
  std::vector<char> used(nbound, 0);
  std::vector<int> search_rad(nbound, 1);
  std::vector<float> seed_dist(1, 0.f);  // index 0: never a cluster
  Rng rng;
  rng.refill();
  long long left = nbound;
  int nclust = 0;
  std::vector<int> free_dir(ndir);
  std::vector<float> cum(ndir);
  std::vector<char> tried(ndir);
  auto coords = [&](long long p, int& i1, int& i2, int& i3) {
    const long long g = pad_cell[p];
    i1 = (int)(g % n1);
    i2 = (int)((g / n1) % n2);
    i3 = (int)(g / ((long long)n1 * n2));
  };
  auto neighbour = [&](int i1, int i2, int i3, const Dir& d) -> long long {
    const int a = i1 + d.d1, b = i2 + d.d2, c = i3 + d.d3;
    if (a < 0 || b < 0 || c < 0 || a >= n1 || b >= n2 || c >= n3) return -1;
    return ((long long)c * n2 + b) * n1 + a;
  };
  while (left > 0) {
    // seed cell: a uniform pick, moved to the nearest unused pad index
    long long p = (long long)std::round((float)(nbound - 1) * rng.u[rng.i]);
    if (++rng.i >= Rng::kLen) rng.refill();
    if (used[p]) {
      for (int r = search_rad[p];; ++r) {
        const long long lo = std::max(p - r, 0LL), hi = std::min(p + r, nbound - 1);
        if (!used[lo]) {
          search_rad[p] = r - 1;
          p = lo;
          break;
        }
        if (!used[hi]) {
          search_rad[p] = r - 1;
          p = hi;
          break;
        }
      }
    }
    std::set<long long> members;  // growth set, ordered by pad index
    members.insert(p);
    used[p] = 1;
    ++nclust;
    label[pad_cell[p]] = nclust;
    seed_dist.push_back(dist[p]);
    --left;
    bool grow = true, reselect = false;
    while (grow && left > 0 && !members.empty()) {
      if (!reselect && rng.u[rng.i] > pct_g) {
        grow = false;
        if (++rng.i >= Rng::kLen - 10) rng.refill();
        continue;
      }
      reselect = false;
      ++rng.i;
      const int pick = (int)std::round((float)(members.size() - 1) * rng.u[rng.i]);
      auto it = members.begin();
      std::advance(it, pick);
      const long long q = *it;
      int i1, i2, i3;
      coords(q, i1, i2, i3);
      int nfree = 0;
      cum[0] = 0.f;
      for (int k = 0; k < ndir; ++k) {
        tried[k] = 1;
        const long long g = neighbour(i1, i2, i3, dir[k]);
        if (g >= 0 && label[g] == 0) {
          tried[k] = 0;
          free_dir[nfree] = k;
          cum[nfree] = cum[std::max(nfree - 1, 0)] + dir[k].w;
          ++nfree;
        }
      }
      if (nfree == 0) {
        reselect = true;
        members.erase(q);
        continue;
      }
      bool all_tried = false, searching = true;
      while (!all_tried && searching) {
        const float target = cum[nfree - 1] * rng.u[rng.i++];
        if (rng.i >= Rng::kLen) rng.refill();
        int j = 0;
        while (cum[j] < target) ++j;
        const int k = free_dir[j];
        if (!tried[k]) {
          tried[k] = 1;
          const long long g = neighbour(i1, i2, i3, dir[k]);
          if (g >= 0 && label[g] == 0) {
            label[g] = nclust;
            used[pad_index[g]] = 1;
            --left;
            searching = false;
            members.insert(pad_index[g]);
            // the walk continues from the new cell (its coordinates)
            coords(pad_index[g], i1, i2, i3);
          }
        }
        all_tried = true;
        for (int kk = 0; kk < ndir; ++kk)
          if (!tried[kk]) {
            all_tried = false;
            break;
          }
        if (all_tried && searching) grow = false;
      }
    }
  }
  // multipliers of clusters 0 .. nclust-1 (cluster nclust keeps 1)
  const float dmax = (float)std::max(std::max(t1, t2), t3);
  std::vector<float> mult(nclust + 1, 1.f);
  for (int k = 0; k < nclust; ++k) {
    const float pct = seed_dist[k] / dmax;
    const float base = (float)((1. - pct) * bval + pct * eval);
    if (pct == 0.f) {
      mult[k] = 1.f;
      continue;
    }
    for (;;) {
      float r = (float)rand() / (float)RAND_MAX;
      r = (float)((r - 0.5) * pct + base);
      if (eval > bval) {
        if (r > 1. && r < eval * 3) {
          mult[k] = r;
          break;
        }
      } else if (r > eval / 3. && r < 1.) {
        mult[k] = r;
        break;
      }
    }
  }
  for (long long g = 0; g < ncell; ++g)
    if (label[g] > 0) field[g] = field[g] * mult[label[g]];
  return VTI_OK;
}
