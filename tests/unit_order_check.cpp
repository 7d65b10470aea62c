// Checks unit_order (the matching's processing order, tr-spmm_b200/csrc/
// unit_order.h) against the C++ library's std::sort on the same comparator:
// identical permutations, ties included, on random and adversarial inputs.
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <random>
#include <vector>

#include "../tr-spmm_b200/csrc/unit_order.h"

int main() {
  std::mt19937 rng(12345);
  long cases = 0;
  for (int n : {0, 1, 2, 3, 15, 16, 17, 31, 33, 64, 100, 257, 1000, 4096, 20000}) {
    for (int keys : {1, 2, 3, 8, 33, 1000}) {
      for (int pattern = 0; pattern < 4; ++pattern) {
        std::vector<int> key(n);
        for (int i = 0; i < n; ++i) {
          switch (pattern) {
            case 0: key[i] = (int)(rng() % keys); break;          // random, many ties
            case 1: key[i] = i % keys; break;                     // sawtooth
            case 2: key[i] = (n - i) % keys; break;               // descending runs
            default: key[i] = (i * 7919) % (keys + 1); break;     // strided
          }
        }
        std::vector<int> a(n), b(n);
        std::iota(a.begin(), a.end(), 0);
        std::iota(b.begin(), b.end(), 0);
        std::sort(a.begin(), a.end(), [&](int x, int y) { return key[x] > key[y]; });
        trs::unit_order(b.data(), n, key.data());
        ++cases;
        if (a != b) {
          std::printf("MISMATCH n=%d keys=%d pattern=%d\n", n, keys, pattern);
          return 1;
        }
      }
    }
  }
  std::printf("ok %ld cases\n", cases);
  return 0;
}
