// The reference's on-disk trie format: load a trie the reference saved, or
// save one the reference can load.
//
// Reference: Trie<A,M>::save / load (storage_engine/src/Trie.cpp:15-75),
// ParMemoryBuffer::save / load (src/utils/ParMemoryBuffer.cpp:64-100),
// MemoryBuffer::save / load (src/utils/MemoryBuffer.cpp:104-172):
//   <dir>/ram/trieinfo.bin   bool annotated, A annotation, size_t num_rows,
//                            size_t num_columns, size_t num_buffers,
//                            size_t head size, size_t size[num_buffers]
//   <dir>/ram/data_head.bin, data_<i>.bin   "<size> <offset> " then size bytes
// The buffers hold TrieBlock<hybrid,M>s (trie/TrieBlock.hpp): a bool
// is_sparse, a Set<hybrid> header (trie/set/Set.hpp: u32 cardinality,
// u32 range = last value, size_t number_of_bytes, u8 type; 24 bytes), the
// set's bytes in its layout, then for the head one NextLevel
// {int buffer; size_t offset} per element (sparse) or per value 0..range
// (dense), common::is_sparse(cardinality, range) deciding (utils/common.hpp:60-66).
// The head block sits at offset 0 of the head buffer, which a reader built
// with NUM_THREADS threads finds at buffer index NUM_THREADS: a saved trie
// loads only into an engine with NUM_THREADS == num_buffers.
//
// Loading parses the files on the host into the sorted CSR and builds the
// device trie from it (index, reverse level, layouts by the given policy).
// Saving exports the CSR, lays every set out by hybrid::build's rule
// (layouts/hybrid.hpp:103-111: range bitset when dense, else uint), puts the
// child blocks of contiguous runs of head entries into the num_buffers
// thread buffers, and writes the head with its NextLevel array.
#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <vector>

#include "eh_internal.cuh"

namespace eh {

namespace {

constexpr int kSetHeader = 24;       // sizeof(Set<hybrid>)
constexpr int kBlockHeader = 1 + kSetHeader;
constexpr int kNextLevel = 16;       // sizeof(NextLevel)

bool sparse_block(uint64_t length, uint64_t range) {
  if (length > 2) return ((double)range / (double)length) > 128.0;
  return true;
}

std::vector<uint8_t> read_file(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  EH_REQUIRE(f != nullptr, EH_ERR_INVALID, "cannot open " + path);
  std::vector<uint8_t> b;
  uint8_t chunk[1 << 16];
  size_t n;
  while ((n = fread(chunk, 1, sizeof chunk, f)) > 0) b.insert(b.end(), chunk, chunk + n);
  fclose(f);
  return b;
}

// MemoryBuffer::load: "<size> <offset> " then size bytes
std::vector<uint8_t> read_buffer(const std::string& path) {
  std::vector<uint8_t> raw = read_file(path);
  size_t p = 0;
  auto num = [&](const char* what) {
    uint64_t v = 0;
    bool any = false;
    while (p < raw.size() && raw[p] >= '0' && raw[p] <= '9') {
      v = v * 10 + (raw[p++] - '0');
      any = true;
    }
    EH_REQUIRE(any && p < raw.size() && raw[p] == ' ', EH_ERR_INVALID, path + ": bad " + what);
    p++;
    return v;
  };
  const uint64_t size = num("size");
  (void)num("offset");
  EH_REQUIRE(raw.size() - p >= size, EH_ERR_INVALID, path + ": truncated");
  return std::vector<uint8_t>(raw.begin() + p, raw.begin() + p + size);
}

template <typename T>
T at(const std::vector<uint8_t>& b, uint64_t o) {
  EH_REQUIRE(o + sizeof(T) <= b.size(), EH_ERR_INVALID, "block outside its buffer");
  T v;
  memcpy(&v, b.data() + o, sizeof(T));
  return v;
}

struct SetHdr {
  uint32_t card, range;
  uint64_t nbytes;
  uint8_t type;
};

SetHdr set_header(const std::vector<uint8_t>& b, uint64_t block) {
  SetHdr h;
  h.card = at<uint32_t>(b, block + 1);
  h.range = at<uint32_t>(b, block + 5);
  h.nbytes = at<uint64_t>(b, block + 9);
  h.type = at<uint8_t>(b, block + 17);
  EH_REQUIRE(block + kBlockHeader + h.nbytes <= b.size(), EH_ERR_INVALID, "set bytes outside the buffer");
  return h;
}

// the values of the set of the block at `block`, appended to out
void decode_set(const std::vector<uint8_t>& b, uint64_t block, std::vector<uint32_t>& out) {
  const SetHdr h = set_header(b, block);
  const uint8_t* d = b.data() + block + kBlockHeader;
  const size_t before = out.size();
  if (!h.card) return;
  if (h.type == EH_LAYOUT_UINTEGER) {
    EH_REQUIRE(h.nbytes >= 4ull * h.card, EH_ERR_INVALID, "uint set shorter than its cardinality");
    const size_t o = out.size();
    out.resize(o + h.card);
    memcpy(out.data() + o, d, 4ull * h.card);
  } else if (h.type == EH_LAYOUT_RANGE_BITSET) {
    EH_REQUIRE(h.nbytes >= 8 && (h.nbytes - 8) % 12 == 0, EH_ERR_INVALID, "bad range bitset size");
    const uint64_t words = (h.nbytes - 8) / 12;
    uint64_t start;
    memcpy(&start, d, 8);
    for (uint64_t w = 0; w < words; w++) {
      uint64_t x;
      memcpy(&x, d + 8 + 8 * w, 8);
      while (x) {
        const int bit = __builtin_ctzll(x);
        out.push_back((uint32_t)((start + w) * 64 + bit));
        x &= x - 1;
      }
    }
  } else if (h.type == EH_LAYOUT_BLOCK_BITSET) {
    EH_REQUIRE(h.nbytes % 40 == 0, EH_ERR_INVALID, "bad block bitset size");
    for (uint64_t k = 0; k < h.nbytes / 40; k++) {
      uint32_t id;
      memcpy(&id, d + 40 * k, 4);
      for (int w = 0; w < 4; w++) {
        uint64_t x;
        memcpy(&x, d + 40 * k + 8 + 8 * w, 8);
        while (x) {
          const int bit = __builtin_ctzll(x);
          out.push_back(id * 256u + (uint32_t)(w * 64 + bit));
          x &= x - 1;
        }
      }
    }
  } else {
    throw Error{EH_ERR_INVALID, "unknown set type " + std::to_string(h.type)};
  }
  EH_REQUIRE(out.size() - before == h.card, EH_ERR_INVALID, "set cardinality does not match its bytes");
}

// hybrid::build of a sorted run: its bytes (range bitset when dense, uint otherwise)
void encode_set(const uint32_t* a, uint64_t n, std::vector<uint8_t>& out, uint8_t* type) {
  const uint64_t range = n > 1 ? (uint64_t)(a[n - 1] - a[0]) : 0;
  const bool bitset = !(n <= 2 || ((double)range / (double)n) > 128.0);
  if (!n) {
    *type = EH_LAYOUT_UINTEGER;
    return;
  }
  if (!bitset) {
    *type = EH_LAYOUT_UINTEGER;
    const size_t o = out.size();
    out.resize(o + 4 * n);
    memcpy(out.data() + o, a, 4 * n);
    return;
  }
  *type = EH_LAYOUT_RANGE_BITSET;
  const uint64_t start = a[0] >> 6, words = (a[n - 1] >> 6) - start + 1;
  const size_t o = out.size();
  out.resize(o + 8 + 12 * words, 0);
  memcpy(out.data() + o, &start, 8);
  uint8_t* W = out.data() + o + 8;
  uint8_t* R = W + 8 * words;
  uint64_t i = 0;
  for (uint64_t w = 0; w < words; w++) {
    const uint32_t rank = (uint32_t)i;  // elements before word w
    memcpy(R + 4 * w, &rank, 4);
    uint64_t x = 0;
    while (i < n && (a[i] >> 6) - start == w) x |= 1ull << (a[i++] & 63);
    memcpy(W + 8 * w, &x, 8);
  }
}

void append_block(std::vector<uint8_t>& buf, const uint32_t* a, uint64_t n) {
  const size_t h = buf.size();
  buf.resize(h + kBlockHeader, 0);
  uint8_t type = EH_LAYOUT_UINTEGER;
  encode_set(a, n, buf, &type);
  const uint32_t card = (uint32_t)n, last = n ? a[n - 1] : 0;
  const uint64_t nbytes = buf.size() - h - kBlockHeader;
  buf[h] = sparse_block(n, last) ? 1 : 0;
  memcpy(buf.data() + h + 1, &card, 4);
  memcpy(buf.data() + h + 5, &last, 4);
  memcpy(buf.data() + h + 9, &nbytes, 8);
  buf[h + 17] = type;
}

void write_buffer(const std::string& path, const std::vector<uint8_t>& b) {
  FILE* f = fopen(path.c_str(), "wb");
  EH_REQUIRE(f != nullptr, EH_ERR_INVALID, "cannot write " + path);
  fprintf(f, "%zu %zu ", b.size(), b.size());
  const bool ok = b.empty() || fwrite(b.data(), 1, b.size(), f) == b.size();
  EH_REQUIRE(fclose(f) == 0 && ok, EH_ERR_INVALID, "write failed: " + path);
}

}  // namespace

void trie_load_reference(eh_context* ctx, const char* dir, const eh_layout_config* cfg, eh_trie* t) {
  const std::string ram = std::string(dir) + "/ram/";
  const std::vector<uint8_t> info = read_file(ram + "trieinfo.bin");
  // sizeof(A) is 8 for void*, long, double and 4 for int, float: the file
  // length tells which
  int sa = -1;
  uint64_t nbuf = 0;
  for (int cand : {8, 4}) {
    if (info.size() < (size_t)(1 + cand + 32)) continue;
    const uint64_t n = at<uint64_t>(info, 1 + cand + 16);
    if (n < (1u << 20) && info.size() == 1 + cand + 32 + 8 * n) {
      sa = cand;
      nbuf = n;
      break;
    }
  }
  EH_REQUIRE(sa > 0, EH_ERR_INVALID, "unrecognised trieinfo.bin in " + ram);
  const uint64_t ncols = at<uint64_t>(info, 1 + sa + 8);
  EH_REQUIRE(ncols == 2, EH_ERR_UNSUPPORTED, "only two-level tries (binary relations) load");
  std::vector<std::vector<uint8_t>> bufs(nbuf + 1);
  for (uint64_t i = 0; i < nbuf; i++) bufs[i] = read_buffer(ram + "data_" + std::to_string(i) + ".bin");
  bufs[nbuf] = read_buffer(ram + "data_head.bin");
  const std::vector<uint8_t>& hb = bufs[nbuf];
  std::vector<uint32_t> head, vals;
  decode_set(hb, 0, head);
  const SetHdr hh = set_header(hb, 0);
  const bool dense = !sparse_block(hh.card, hh.range);
  const uint64_t next0 = kBlockHeader + hh.nbytes;
  std::vector<uint64_t> off(1, 0);
  std::vector<uint32_t> kept;
  kept.reserve(head.size());
  for (size_t i = 0; i < head.size(); i++) {
    const uint64_t e = dense ? head[i] : i;
    const int32_t bi = at<int32_t>(hb, next0 + kNextLevel * e);
    const uint64_t bo = at<uint64_t>(hb, next0 + kNextLevel * e + 8);
    if (bi < 0) continue;  // no child set: no row with this first value
    EH_REQUIRE((uint64_t)bi <= nbuf, EH_ERR_INVALID, "NextLevel names a missing buffer");
    const size_t before = vals.size();
    decode_set(bufs[bi], bo, vals);
    if (vals.size() == before) continue;
    kept.push_back(head[i]);
    off.push_back(vals.size());
  }
  EH_REQUIRE(vals.size() < (1ull << 32), EH_ERR_UNSUPPORTED, "tries hold fewer than 2^32 rows");
  cudaStream_t s = ctx->stream;
  t->ctx = ctx;
  t->n_head = (uint32_t)kept.size();
  t->rows = vals.size();
  t->head.alloc(t->n_head ? t->n_head : 1, s);
  t->off.alloc(t->n_head + 1, s);
  t->vals.alloc(t->rows ? t->rows : 1, s);
  uint32_t mx = 0;
  for (uint32_t v : kept) mx = std::max(mx, v);
  for (uint32_t v : vals) mx = std::max(mx, v);
  if (t->n_head) EH_CUDA(cudaMemcpyAsync(t->head.p, kept.data(), 4ull * t->n_head, cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(t->off.p, off.data(), 8ull * (t->n_head + 1), cudaMemcpyHostToDevice, s));
  if (t->rows) EH_CUDA(cudaMemcpyAsync(t->vals.p, vals.data(), 4ull * t->rows, cudaMemcpyHostToDevice, s));
  t->n_nodes = (t->n_head || t->rows) ? mx + 1 : 0;
  EH_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
  trie_build_from_csr(ctx, t);
  trie_layout(ctx, t, cfg);
}

void trie_save_reference(eh_context* ctx, const eh_trie* t, const char* dir, uint32_t num_threads) {
  EH_REQUIRE(num_threads >= 1 && num_threads <= 4096, EH_ERR_INVALID, "num_threads must be 1..4096");
  cudaStream_t s = ctx->stream;
  const uint32_t nh = t->n_head;
  std::vector<uint32_t> head(nh), vals(t->rows);
  std::vector<uint64_t> off(nh + 1);
  if (nh) EH_CUDA(cudaMemcpyAsync(head.data(), t->head.p, 4ull * nh, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaMemcpyAsync(off.data(), t->off.p, 8ull * (nh + 1), cudaMemcpyDeviceToHost, s));
  if (t->rows) EH_CUDA(cudaMemcpyAsync(vals.data(), t->vals.p, 4ull * t->rows, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  const uint64_t per = nh ? (nh + num_threads - 1) / num_threads : 0;
  std::vector<std::vector<uint8_t>> bufs(num_threads);
  std::vector<int32_t> where(nh);
  std::vector<uint64_t> at_off(nh);
  for (uint32_t i = 0; i < nh; i++) {
    const uint32_t b = (uint32_t)std::min<uint64_t>(i / per, num_threads - 1);
    where[i] = (int32_t)b;
    at_off[i] = bufs[b].size();
    append_block(bufs[b], vals.data() + off[i], off[i + 1] - off[i]);
    // MemoryBuffer::save writes its used length as an int (MemoryBuffer.cpp:108)
    EH_REQUIRE(bufs[b].size() < (1ull << 31), EH_ERR_UNSUPPORTED, "a buffer would exceed 2 GB: use more threads");
  }
  std::vector<uint8_t> hb;
  append_block(hb, head.data(), nh);
  const uint32_t last = nh ? head[nh - 1] : 0;
  const bool dense = !sparse_block(nh, last);
  const uint64_t n_next = dense ? (uint64_t)last + 1 : nh;
  const size_t next0 = hb.size();
  hb.resize(next0 + kNextLevel * n_next, 0);
  for (uint64_t e = 0; e < n_next; e++) {
    const int32_t none = -1;
    memcpy(hb.data() + next0 + kNextLevel * e, &none, 4);
  }
  for (uint32_t i = 0; i < nh; i++) {
    const uint64_t e = dense ? head[i] : i;
    memcpy(hb.data() + next0 + kNextLevel * e, &where[i], 4);
    memcpy(hb.data() + next0 + kNextLevel * e + 8, &at_off[i], 8);
  }
  EH_REQUIRE(hb.size() < (1ull << 31), EH_ERR_UNSUPPORTED, "head buffer would exceed 2 GB");
  const std::string ram = std::string(dir) + "/ram/";
  for (const std::string& d : {std::string(dir), ram})
    EH_REQUIRE(mkdir(d.c_str(), 0755) == 0 || errno == EEXIST, EH_ERR_INVALID, "cannot create " + d);
  write_buffer(ram + "data_head.bin", hb);
  for (uint32_t i = 0; i < num_threads; i++) write_buffer(ram + "data_" + std::to_string(i) + ".bin", bufs[i]);
  // trieinfo of a Trie<void*,ParMemoryBuffer>: not annotated
  std::vector<uint8_t> info(1 + 8 + 32 + 8ull * num_threads, 0);
  uint64_t v[4] = {t->rows, 2, num_threads, hb.size()};
  memcpy(info.data() + 9, v, 32);
  for (uint32_t i = 0; i < num_threads; i++) {
    const uint64_t sz = bufs[i].size();
    memcpy(info.data() + 41 + 8ull * i, &sz, 8);
  }
  FILE* f = fopen((ram + "trieinfo.bin").c_str(), "wb");
  EH_REQUIRE(f != nullptr, EH_ERR_INVALID, "cannot write " + ram + "trieinfo.bin");
  const bool ok = fwrite(info.data(), 1, info.size(), f) == info.size();
  EH_REQUIRE(fclose(f) == 0 && ok, EH_ERR_INVALID, "write failed: trieinfo.bin");
}

}  // namespace eh
