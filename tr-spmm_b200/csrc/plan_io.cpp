// Plan files: a host plan (routing + layout, everything a device plan is
// uploaded from) written to disk once per graph, so later runs skip the
// router and the builder.
//
// Format (little-endian): the 8-byte tag "TRSPLAN1", a u32 version, the
// scalar fields, then each array as (u64 element count, raw elements) in a
// fixed order, then a 64-bit FNV-1a checksum of every preceding byte.
// Version 2 adds a block-layout flag after the scalar flags and the seven
// block arrays after the window arrays; version-1 files (window plans) still
// load.
// Loading checks the tag, the version, every count against the bytes left
// and the checksum, and refuses the file (with the reason) on any mismatch.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/trspmm.h"
#include "plan.h"

namespace trs {
namespace {

constexpr char kTag[8] = {'T', 'R', 'S', 'P', 'L', 'A', 'N', '1'};
constexpr uint32_t kVersion = 2;

struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  }
};

struct Writer {
  std::vector<uint8_t> buf;
  void raw(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    buf.insert(buf.end(), b, b + n);
  }
  template <class T> void put(T v) { raw(&v, sizeof(T)); }
  template <class T> void vec(const std::vector<T>& v) {
    put<uint64_t>(v.size());
    if (!v.empty()) raw(v.data(), v.size() * sizeof(T));
  }
};

struct Reader {
  const uint8_t* p;
  size_t left;
  bool ok = true;
  void raw(void* d, size_t n) {
    if (!ok || n > left) { ok = false; return; }
    std::memcpy(d, p, n);
    p += n;
    left -= n;
  }
  template <class T> T get() {
    T v{};
    raw(&v, sizeof(T));
    return v;
  }
  template <class T> void vec(std::vector<T>& v) {
    const uint64_t n = get<uint64_t>();
    if (!ok || n > left / sizeof(T)) { ok = false; return; }
    v.resize(n);
    if (n) raw(v.data(), n * sizeof(T));
  }
};

// Index ranges the kernels rely on: offsets monotone and consistent with
// the arrays they index, every column / row / entry / slot in range, the
// launch order a permutation of the windows.
bool contents_valid(const HostPlan& h) {
  const int64_t W = h.n_windows, rows = W * 16;
  const int64_t T = (int64_t)h.tile_col.size() / 16;
  if (h.n_rows < 0 || h.n_cols < 0 || h.n_rows > rows || (int64_t)h.tile_col.size() != T * 16 ||
      (int64_t)h.tile_a.size() != T * 256 || h.win_tile[0] != 0 || h.win_tile[W] != T)
    return false;
  for (int64_t w = 0; w < W; ++w)
    if (!(h.win_tile[w] <= h.win_split[w] && h.win_split[w] <= h.win_prom[w] &&
          h.win_prom[w] <= h.win_tile[w + 1]))
      return false;
  if (h.res_ptr[0] != 0 || h.res_ptr[rows] != (int64_t)h.res_col.size() ||
      h.res_edge.size() != h.res_col.size())
    return false;
  for (int64_t r = 0; r < rows; ++r)
    if (h.res_ptr[r] > h.res_ptr[r + 1]) return false;
  for (int32_t c : h.res_col)
    if (c < 0 || c >= h.n_cols) return false;
  for (int32_t c : h.tile_col)
    if (c < -1 || c >= h.n_cols) return false;
  std::vector<char> seen(W, 0);
  for (int32_t w : h.win_order) {
    if (w < 0 || w >= W || seen[w]) return false;
    seen[w] = 1;
  }
  for (int32_t o : h.row_out)
    if (o < -1 || o >= h.n_rows) return false;
  const int64_t n_edges = (int64_t)h.val_slot.size();
  const int64_t slots = T * 256 + (int64_t)h.res_col.size();
  for (int32_t e : h.res_edge)
    if (e < -1 || e >= n_edges) return false;
  const int64_t ents = (int64_t)h.ent_pos.size();
  for (int64_t e = 0; e < n_edges; ++e)
    if (h.val_slot[e] < -1 || h.val_slot[e] >= (h.block ? ents : slots) || h.edge_row[e] < -1 ||
        h.edge_row[e] >= rows)
      return false;
  if (!h.block)
    return h.blk_chunk.empty() && h.chunk_col.empty() && h.chunk_ent.empty() && ents == 0 &&
           h.ent_val.empty() && h.ent_src.empty() && h.blk_order.empty();
  // block layout: every offset monotone and in range, every position inside
  // a 128x16 FP16 tile, the launch order a permutation of the blocks
  const int64_t NB = (int64_t)h.blk_order.size();
  if (T != 0 || !h.res_col.empty() || W != NB * 8 || (int64_t)h.blk_chunk.size() != NB + 1 ||
      h.blk_chunk[0] != 0)
    return false;
  for (int64_t b = 0; b < NB; ++b)
    if (h.blk_chunk[b] > h.blk_chunk[b + 1] || (h.blk_chunk[b + 1] - h.blk_chunk[b]) % kChunkGroup)
      return false;
  const int64_t NC = h.blk_chunk[NB];
  if ((int64_t)h.chunk_col.size() != NC * kChunkCols || (int64_t)h.chunk_ent.size() != NC + 1 ||
      h.chunk_ent[0] != 0 || h.chunk_ent[NC] != ents || (int64_t)h.ent_val.size() != ents ||
      (int64_t)h.ent_src.size() != ents)
    return false;
  for (int64_t c = 0; c < NC; ++c)
    if (h.chunk_ent[c] > h.chunk_ent[c + 1]) return false;
  for (int32_t c : h.chunk_col)
    if (c < -1 || c >= h.n_cols) return false;
  for (uint16_t p : h.ent_pos)
    if ((p & 1) || p >= 4096) return false;
  for (int32_t e : h.ent_src)
    if (e < -1 || e >= n_edges) return false;
  std::vector<char> bseen(NB, 0);
  for (int32_t b : h.blk_order) {
    if (b < 0 || b >= NB || bseen[b]) return false;
    bseen[b] = 1;
  }
  return true;
}

}  // namespace

int save_host_plan(const HostPlan& hp, const char* path, std::string& err) {
  Writer w;
  w.raw(kTag, sizeof(kTag));
  w.put<uint32_t>(kVersion);
  w.put<int32_t>(hp.n_rows);
  w.put<int32_t>(hp.n_cols);
  w.put<int32_t>(hp.n_windows);
  w.put<uint8_t>(hp.row_scaled ? 1 : 0);
  w.put<uint8_t>(hp.reordered ? 1 : 0);
  w.put<uint8_t>(hp.block ? 1 : 0);
  w.put<int64_t>(hp.tc_tiles);
  w.put<int64_t>(hp.sptc_tiles);
  w.put<int64_t>(hp.prom_tiles);
  w.put<int64_t>(hp.nnz);
  w.vec(hp.win_tile);
  w.vec(hp.win_split);
  w.vec(hp.win_prom);
  w.vec(hp.tile_col);
  w.vec(hp.tile_a);
  w.vec(hp.res_ptr);
  w.vec(hp.res_col);
  w.vec(hp.res_val);
  w.vec(hp.res_edge);
  w.vec(hp.win_order);
  w.vec(hp.row_scale);
  w.vec(hp.row_out);
  w.vec(hp.val_slot);
  w.vec(hp.edge_row);
  w.vec(hp.blk_chunk);
  w.vec(hp.chunk_col);
  w.vec(hp.chunk_ent);
  w.vec(hp.ent_pos);
  w.vec(hp.ent_val);
  w.vec(hp.ent_src);
  w.vec(hp.blk_order);
  Fnv f;
  f.add(w.buf.data(), w.buf.size());
  w.put<uint64_t>(f.h);
  // write beside the target, then rename: readers never see a partial file
  const std::string tmp = std::string(path) + ".tmp";
  FILE* fp = std::fopen(tmp.c_str(), "wb");
  if (!fp) {
    err = "cannot open " + tmp + " for writing";
    return TR_ERR_ARG;
  }
  const size_t n = std::fwrite(w.buf.data(), 1, w.buf.size(), fp);
  const bool closed = std::fclose(fp) == 0;
  if (n != w.buf.size() || !closed) {
    std::remove(tmp.c_str());
    err = "short write to " + tmp;
    return TR_ERR_ARG;
  }
  if (std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    err = std::string("cannot rename the plan file into ") + path;
    return TR_ERR_ARG;
  }
  return TR_OK;
}

int load_host_plan(const char* path, HostPlan& hp, std::string& err) {
  FILE* fp = std::fopen(path, "rb");
  if (!fp) {
    err = std::string("cannot open plan file ") + path;
    return TR_ERR_ARG;
  }
  std::vector<uint8_t> buf;
  uint8_t chunk[1 << 16];
  for (size_t n; (n = std::fread(chunk, 1, sizeof(chunk), fp)) > 0;) buf.insert(buf.end(), chunk, chunk + n);
  std::fclose(fp);
  if (buf.size() < sizeof(kTag) + 4 + 8 || std::memcmp(buf.data(), kTag, sizeof(kTag)) != 0) {
    err = std::string("not a plan file: ") + path;
    return TR_ERR_ARG;
  }
  uint64_t stored = 0;
  std::memcpy(&stored, buf.data() + buf.size() - 8, 8);
  Fnv f;
  f.add(buf.data(), buf.size() - 8);
  if (f.h != stored) {
    err = std::string("plan file checksum mismatch (damaged or truncated): ") + path;
    return TR_ERR_ARG;
  }
  Reader r{buf.data() + sizeof(kTag), buf.size() - sizeof(kTag) - 8};
  const uint32_t version = r.get<uint32_t>();
  if (version != kVersion && version != 1) {
    err = "plan file version " + std::to_string(version) + " (this library reads version " +
          std::to_string(kVersion) + ")";
    return TR_ERR_UNSUPPORTED;
  }
  HostPlan h;
  h.n_rows = r.get<int32_t>();
  h.n_cols = r.get<int32_t>();
  h.n_windows = r.get<int32_t>();
  h.row_scaled = r.get<uint8_t>() != 0;
  h.reordered = r.get<uint8_t>() != 0;
  if (version >= 2) h.block = r.get<uint8_t>() != 0;
  h.tc_tiles = r.get<int64_t>();
  h.sptc_tiles = r.get<int64_t>();
  h.prom_tiles = r.get<int64_t>();
  h.nnz = r.get<int64_t>();
  r.vec(h.win_tile);
  r.vec(h.win_split);
  r.vec(h.win_prom);
  r.vec(h.tile_col);
  r.vec(h.tile_a);
  r.vec(h.res_ptr);
  r.vec(h.res_col);
  r.vec(h.res_val);
  r.vec(h.res_edge);
  r.vec(h.win_order);
  r.vec(h.row_scale);
  r.vec(h.row_out);
  r.vec(h.val_slot);
  r.vec(h.edge_row);
  if (version >= 2) {
    r.vec(h.blk_chunk);
    r.vec(h.chunk_col);
    r.vec(h.chunk_ent);
    r.vec(h.ent_pos);
    r.vec(h.ent_val);
    r.vec(h.ent_src);
    r.vec(h.blk_order);
  }
  const int64_t W = h.n_windows;
  const bool shapes = r.ok && r.left == 0 && W >= 0 && h.win_tile.size() == (size_t)W + 1 &&
                      h.win_split.size() == (size_t)W && h.win_prom.size() == (size_t)W &&
                      h.res_ptr.size() == (size_t)W * 16 + 1 && h.win_order.size() == (size_t)W &&
                      h.row_scale.size() == (size_t)W * 16 && h.row_out.size() == (size_t)W * 16 &&
                      h.res_col.size() == h.res_val.size() && h.val_slot.size() == h.edge_row.size();
  if (!shapes || !contents_valid(h)) {
    err = std::string("plan file has inconsistent arrays: ") + path;
    return TR_ERR_ARG;
  }
  hp = std::move(h);
  return TR_OK;
}

}  // namespace trs
