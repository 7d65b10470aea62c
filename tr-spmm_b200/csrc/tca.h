// TCA row clustering (the reference's optional row reorder,
// spmm/tr_csr_fp16/tr_tca_reorder.py:44-357): MinHash-LSH candidate pairs,
// exact Jaccard similarity, two levels of capped union-find clustering.
//
// The hash arithmetic below is shared by the host and the device code so
// that both produce the same signatures, band digests and therefore the same
// candidate pairs and row order.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#if defined(__CUDACC__)
#define TRS_HD __host__ __device__ __forceinline__
#else
#define TRS_HD inline
#endif

namespace trs {

constexpr int kTcaPerm = 128;          // MinHash permutations (the reference's num_perm)

// splitmix64 output function (Steele, Lea, Flood 2014): a bijective 64-bit mix.
TRS_HD uint64_t tca_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Coefficients of permutation i: h_i(x) = high 32 bits of (a_i * x + b_i)
// mod 2^64 (multiply-add-shift hashing, Dietzfelbinger 1996), a_i odd.
TRS_HD uint64_t tca_perm_a(uint64_t seed, int i) {
  return tca_mix64(seed + 0x9E3779B97F4A7C15ull * (uint64_t)(2 * i + 1)) | 1ull;
}
TRS_HD uint64_t tca_perm_b(uint64_t seed, int i) {
  return tca_mix64(seed + 0x9E3779B97F4A7C15ull * (uint64_t)(2 * i + 2));
}

// The key a column id is hashed from: the id spread over 32 bits first, so
// that consecutive ids do not give correlated minima under linear hashing.
TRS_HD uint32_t tca_key(int32_t col) { return (uint32_t)(tca_mix64((uint64_t)(uint32_t)col) >> 32); }

TRS_HD uint32_t tca_hash(uint64_t a, uint64_t b, uint32_t key) {
  return (uint32_t)((a * (uint64_t)key + b) >> 32);
}

// 64-bit digest of band j (signature values v[0..r)): rows whose digests
// agree in some band are candidate pairs.
TRS_HD uint64_t tca_band_digest(const uint32_t* v, int r, int j) {
  uint64_t d = tca_mix64(0x5BD1E9955BD1E995ull + (uint64_t)j);
  for (int i = 0; i < r; ++i) d = tca_mix64(d ^ ((uint64_t)v[i] + 0x9E3779B97F4A7C15ull));
  return d;
}

struct TcaParams {
  int32_t thres = 16;            // level-1 cluster cap (rows)
  int32_t cluster_thres = 128;   // level-2 cap (level-1 clusters)
  double lsh_threshold = 0.2;    // Jaccard threshold the LSH bands are tuned for
  uint64_t seed = 1;             // MinHash seed
  int64_t max_pairs = 1ll << 25; // refuse graphs with more candidate pairs
  int32_t device = 0;            // 1: signatures and Jaccard on the current GPU
};

struct TcaStats {
  int32_t bands = 0, rows_per_band = 0;
  int64_t pairs1 = 0, clusters1 = 0, pairs2 = 0, clusters2 = 0;
  double seconds[4] = {0, 0, 0, 0};   // sets + signatures, candidates, Jaccard, clustering
};

// LSH banding (b bands of r rows, b * r <= num_perm) minimising the equally
// weighted integrals of false-positive and false-negative probability
// around `threshold` (the banding analysis of Leskovec, Rajaraman and
// Ullman, Mining of Massive Datasets, ch. 3).
void tca_lsh_params(double threshold, int num_perm, int& bands, int& rows);

// Row order (new position -> old row) for the CSR pattern; any column order
// and duplicates are allowed (similarities are over column sets).
int tca_order(const int32_t* indptr, const int32_t* indices, int32_t n_rows, const TcaParams& p,
              std::vector<int32_t>& order, TcaStats& st, std::string& err);

// Device backends (tca_gpu.cu).  Lists are sorted, duplicate-free CSR rows.
int tca_signatures_gpu(const std::vector<int64_t>& ptr, const std::vector<int32_t>& col,
                       uint64_t seed, int bands, int rows, std::vector<uint32_t>& sig,
                       std::vector<uint64_t>& dig, std::string& err);
int tca_intersections_gpu(const std::vector<int64_t>& ptr, const std::vector<int32_t>& col,
                          const std::vector<int32_t>& pa, const std::vector<int32_t>& pb,
                          std::vector<int32_t>& inter, std::string& err);

}  // namespace trs
