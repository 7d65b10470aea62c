// Processing order of the router's max-degree matching, shared by the host
// router and the device router.
//
// The reference orders the 2:4 units with std::sort on (degree desc, nnz
// desc) (TR-source/Block/block_online.cpp:360-363); on the complete
// compatibility graph every degree is equal and the order is "nnz desc" with
// ties left where the sort leaves them.  std::sort is not stable, so the
// tie order is whatever its algorithm produces, and the matching's pairs
// depend on it.  Both routers therefore run one restatement of that
// algorithm — introsort (D. Musser, "Introspective Sorting and Selection
// Algorithms", 1997) in the form the GNU C++ library's std::sort performs it:
// median-of-three pivot moved to the front, unguarded Hoare partition,
// recursion on the right part while looping on the left, ranges of at most
// 16 left for a final insertion sort, heapsort once 2*floor(log2 n)
// partitioning levels are used up — on the same input (0 .. n-1) with the
// same comparisons, so the host and the device produce the same order.
// The host router's equality with the reference's compiled router on tied
// inputs pins the restatement.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define TRS_HD __host__ __device__
#else
#define TRS_HD
#endif

namespace trs {
namespace unit_order_detail {

// a holds unit ids; before(x, y) = "x sorts before y" = key[x] > key[y]
struct Desc {
  const int* key;
  TRS_HD bool operator()(int x, int y) const { return key[x] > key[y]; }
};

TRS_HD inline void swap_at(int* a, int i, int j) {
  const int t = a[i];
  a[i] = a[j];
  a[j] = t;
}

// Sift the hole at `hole` down to a leaf along larger children, then let
// `value` rise from there (heap of len items, "larger" = sorts later).
TRS_HD inline void sift(int* a, int hole, int len, int value, const Desc& before) {
  const int top = hole;
  int child = hole;
  while (child < (len - 1) / 2) {
    child = 2 * (child + 1);
    if (before(a[child], a[child - 1])) --child;
    a[hole] = a[child];
    hole = child;
  }
  if ((len & 1) == 0 && child == (len - 2) / 2) {
    child = 2 * (child + 1);
    a[hole] = a[child - 1];
    hole = child - 1;
  }
  int parent = (hole - 1) / 2;
  while (hole > top && before(a[parent], value)) {
    a[hole] = a[parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  a[hole] = value;
}

TRS_HD inline void heap_sort(int* a, int len, const Desc& before) {
  if (len < 2) return;
  for (int parent = (len - 2) / 2;; --parent) {
    sift(a, parent, len, a[parent], before);
    if (parent == 0) break;
  }
  for (int last = len - 1; last > 0; --last) {
    const int value = a[last];
    a[last] = a[0];
    sift(a, 0, last, value, before);
  }
}

// a[lo .. hi) with a[lo - 1] (or a guard) bounding the walk on the left
TRS_HD inline void insert_unguarded(int* a, int i, const Desc& before) {
  const int v = a[i];
  int j = i - 1;
  while (before(v, a[j])) {
    a[j + 1] = a[j];
    --j;
  }
  a[j + 1] = v;
}

TRS_HD inline void insertion_sort(int* a, int lo, int hi, const Desc& before) {
  for (int i = lo + 1; i < hi; ++i) {
    if (before(a[i], a[lo])) {
      const int v = a[i];
      for (int j = i; j > lo; --j) a[j] = a[j - 1];
      a[lo] = v;
    } else {
      insert_unguarded(a, i, before);
    }
  }
}

TRS_HD inline int floor_log2(int n) {
  int k = 0;
  while (n > 1) { n >>= 1; ++k; }
  return k;
}

}  // namespace unit_order_detail

// Sorts a[0, n) (unit ids) by key descending, ties as described above.
TRS_HD inline void unit_order(int* a, int n, const int* key) {
  using namespace unit_order_detail;
  if (n <= 1) return;
  const Desc before{key};
  constexpr int kThreshold = 16;
  struct Range { int lo, hi, depth; };
  Range stack[64];          // each pushed range has a smaller depth than its parent
  int top = 0;
  stack[top++] = {0, n, 2 * floor_log2(n)};
  while (top > 0) {
    Range r = stack[--top];
    while (r.hi - r.lo > kThreshold) {
      if (r.depth == 0) {
        heap_sort(a + r.lo, r.hi - r.lo, before);
        break;
      }
      --r.depth;
      // median of (lo + 1, mid, hi - 1) to the front
      const int x = r.lo + 1, y = r.lo + (r.hi - r.lo) / 2, z = r.hi - 1;
      if (before(a[x], a[y])) {
        if (before(a[y], a[z])) swap_at(a, r.lo, y);
        else if (before(a[x], a[z])) swap_at(a, r.lo, z);
        else swap_at(a, r.lo, x);
      } else if (before(a[x], a[z])) {
        swap_at(a, r.lo, x);
      } else if (before(a[y], a[z])) {
        swap_at(a, r.lo, z);
      } else {
        swap_at(a, r.lo, y);
      }
      // unguarded partition of (lo, hi) around a[lo]
      int i = r.lo + 1, j = r.hi;
      for (;;) {
        while (before(a[i], a[r.lo])) ++i;
        --j;
        while (before(a[r.lo], a[j])) --j;
        if (!(i < j)) break;
        swap_at(a, i, j);
        ++i;
      }
      stack[top++] = {i, r.hi, r.depth};   // the right part, then loop on the left
      r.hi = i;
    }
  }
  if (n > kThreshold) {
    insertion_sort(a, 0, kThreshold, before);
    for (int i = kThreshold; i < n; ++i) insert_unguarded(a, i, before);
  } else {
    insertion_sort(a, 0, n, before);
  }
}

}  // namespace trs
