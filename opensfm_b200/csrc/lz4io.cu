// LZ4 frame compression and decompression on the host, for the depthmap
// files OpenSfM writes: `<image>.raw.npz` and `<image>.clean.npz` are an
// .npz archive wrapped in one LZ4 frame (opensfm/dataset.py:1080-1098
// compresses with lz4.frame.compress, and 1100-1112 decompresses).
//
// Written from the published format descriptions (LZ4 block format and LZ4
// frame format, and the xxHash32 specification):
//  - frame: magic 0x184D2204, descriptor (FLG, BD, optional content size
//    and dictionary id) with a one-byte header checksum = second byte of
//    xxHash32(descriptor); blocks of [4-byte LE size | data | optional
//    xxHash32]; the high bit of the size marks a stored (uncompressed)
//    block; a zero size ends the frame, then an optional xxHash32 of the
//    content.  Skippable frames (magic 0x184D2A5?) are skipped; frames may
//    be concatenated.
//  - block: sequences of [token | literal length bytes | literals |
//    2-byte LE offset | match length bytes]; lengths of 15 continue with
//    bytes added until one is below 255; matches are at least 4 bytes and
//    may overlap their output; the last sequence is literals only.
// The compressor is a greedy single-probe hash matcher; it writes
// independent blocks of up to 4 MB and stores a block uncompressed when
// compression does not shrink it.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "dense_b200.h"

namespace {

thread_local std::string g_io_error;
thread_local std::vector<uint8_t> g_last_out;
thread_local const void* g_last_src = nullptr;
thread_local int64_t g_last_n = -1;
thread_local uint32_t g_last_hash = 0;  // xxh32 of the cached input

dn_status io_fail(dn_status s, const char* m) {
  g_io_error = m;
  return s;
}

// ------------------------------------------------------------- xxHash32
constexpr uint32_t kP1 = 0x9E3779B1u, kP2 = 0x85EBCA77u, kP3 = 0xC2B2AE3Du, kP4 = 0x27D4EB2Fu,
                   kP5 = 0x165667B1u;

inline uint32_t rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
inline uint32_t rd32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
inline void wr32(uint8_t* p, uint32_t v) {
  p[0] = (uint8_t)v;
  p[1] = (uint8_t)(v >> 8);
  p[2] = (uint8_t)(v >> 16);
  p[3] = (uint8_t)(v >> 24);
}

uint32_t xxh32(const uint8_t* p, size_t n, uint32_t seed) {
  const uint8_t* end = p + n;
  uint32_t acc;
  if (n >= 16) {
    uint32_t v1 = seed + kP1 + kP2, v2 = seed + kP2, v3 = seed, v4 = seed - kP1;
    const uint8_t* lim = end - 16;
    do {
      v1 = rotl(v1 + rd32(p) * kP2, 13) * kP1;
      v2 = rotl(v2 + rd32(p + 4) * kP2, 13) * kP1;
      v3 = rotl(v3 + rd32(p + 8) * kP2, 13) * kP1;
      v4 = rotl(v4 + rd32(p + 12) * kP2, 13) * kP1;
      p += 16;
    } while (p <= lim);
    acc = rotl(v1, 1) + rotl(v2, 7) + rotl(v3, 12) + rotl(v4, 18);
  } else {
    acc = seed + kP5;
  }
  acc += (uint32_t)n;
  while (p + 4 <= end) {
    acc = rotl(acc + rd32(p) * kP3, 17) * kP4;
    p += 4;
  }
  while (p < end) {
    acc = rotl(acc + (uint32_t)(*p) * kP5, 11) * kP1;
    ++p;
  }
  acc ^= acc >> 15;
  acc *= kP2;
  acc ^= acc >> 13;
  acc *= kP3;
  acc ^= acc >> 16;
  return acc;
}

// ---------------------------------------------------------- LZ4 blocks
constexpr int kMinMatch = 4;
constexpr int kLastLiterals = 5;  // a block ends with at least 5 literals
constexpr int kMfLimit = 12;      // no match starts in the last 12 bytes
constexpr int kHashLog = 16;

inline void put_len(std::vector<uint8_t>& out, size_t len) {
  while (len >= 255) {
    out.push_back(255);
    len -= 255;
  }
  out.push_back((uint8_t)len);
}

void emit(std::vector<uint8_t>& out, const uint8_t* lit, size_t n_lit, size_t offset,
          size_t match_len) {
  const size_t ml = match_len ? match_len - kMinMatch : 0;
  out.push_back((uint8_t)(((n_lit >= 15 ? 15 : n_lit) << 4) | (match_len ? (ml >= 15 ? 15 : ml) : 0)));
  if (n_lit >= 15) put_len(out, n_lit - 15);
  out.insert(out.end(), lit, lit + n_lit);
  if (!match_len) return;
  out.push_back((uint8_t)offset);
  out.push_back((uint8_t)(offset >> 8));
  if (ml >= 15) put_len(out, ml - 15);
}

// Appends the compressed form of src[0, n) to out.
void compress_block(const uint8_t* src, size_t n, std::vector<uint8_t>& out) {
  std::vector<int64_t> table((size_t)1 << kHashLog, -1);
  size_t anchor = 0, pos = 0;
  if (n >= (size_t)kMfLimit + 1) {
    const size_t match_start_limit = n - kMfLimit;
    const size_t match_end_limit = n - kLastLiterals;
    while (pos < match_start_limit) {
      const uint32_t seq = rd32(src + pos);
      const uint32_t h = (seq * 2654435761u) >> (32 - kHashLog);
      const int64_t cand = table[h];
      table[h] = (int64_t)pos;
      if (cand >= 0 && pos - (size_t)cand <= 65535 && rd32(src + cand) == seq) {
        size_t ml = kMinMatch;
        while (pos + ml < match_end_limit && src[cand + ml] == src[pos + ml]) ++ml;
        emit(out, src + anchor, pos - anchor, pos - (size_t)cand, ml);
        pos += ml;
        anchor = pos;
      } else {
        ++pos;
      }
    }
  }
  emit(out, src + anchor, n - anchor, 0, 0);
}

// Decodes one block into out, whose tail from frame_start on is the earlier
// output of the frame (linked blocks may refer to it).  Returns false on a
// malformed block.
bool decompress_block(const uint8_t* p, size_t n, std::vector<uint8_t>& out, size_t frame_start,
                      size_t max_out) {
  const uint8_t* end = p + n;
  const size_t start = out.size();
  while (p < end) {
    const uint8_t token = *p++;
    size_t lit = token >> 4;
    if (lit == 15) {
      uint8_t b;
      do {
        if (p >= end) return false;
        b = *p++;
        lit += b;
      } while (b == 255);
    }
    if ((size_t)(end - p) < lit || out.size() - start + lit > max_out) return false;
    out.insert(out.end(), p, p + lit);
    p += lit;
    if (p == end) break;  // the last sequence has no match
    if (end - p < 2) return false;
    const size_t offset = (size_t)p[0] | ((size_t)p[1] << 8);
    p += 2;
    size_t ml = token & 15;
    if (ml == 15) {
      uint8_t b;
      do {
        if (p >= end) return false;
        b = *p++;
        ml += b;
      } while (b == 255);
    }
    ml += kMinMatch;
    if (offset == 0 || offset > out.size() - frame_start || out.size() - start + ml > max_out)
      return false;
    size_t from = out.size() - offset;
    for (size_t k = 0; k < ml; ++k) out.push_back(out[from + k]);  // may overlap
  }
  return true;
}

constexpr uint32_t kMagic = 0x184D2204u;
constexpr size_t kBlockMax = (size_t)4 << 20;  // BD code 7

dn_status decode_frames(const uint8_t* p, size_t n, std::vector<uint8_t>& out) {
  const uint8_t* end = p + n;
  out.clear();
  bool any = false;
  while (p < end) {
    if (end - p < 4) return io_fail(DN_INVALID_ARG, "truncated LZ4 frame");
    const uint32_t magic = rd32(p);
    p += 4;
    if ((magic & 0xFFFFFFF0u) == 0x184D2A50u) {  // skippable frame
      if (end - p < 4) return io_fail(DN_INVALID_ARG, "truncated skippable frame");
      const uint32_t len = rd32(p);
      p += 4;
      if ((size_t)(end - p) < len) return io_fail(DN_INVALID_ARG, "truncated skippable frame");
      p += len;
      continue;
    }
    if (magic != kMagic) return io_fail(DN_INVALID_ARG, "not an LZ4 frame (bad magic number)");
    const uint8_t* desc = p;
    if (end - p < 2) return io_fail(DN_INVALID_ARG, "truncated LZ4 frame descriptor");
    const uint8_t flg = p[0], bd = p[1];
    p += 2;
    if ((flg >> 6) != 1) return io_fail(DN_INVALID_ARG, "unsupported LZ4 frame version");
    const bool block_checksum = flg & 0x10, has_size = flg & 0x08, content_checksum = flg & 0x04;
    if (flg & 0x01) return io_fail(DN_INVALID_ARG, "LZ4 frames with a dictionary are not supported");
    const int bsid = (bd >> 4) & 7;
    if (bsid < 4) return io_fail(DN_INVALID_ARG, "invalid LZ4 block size code");
    const size_t block_max = (size_t)1 << (8 + 2 * bsid);
    uint64_t content_size = 0;
    if (has_size) {
      if (end - p < 8) return io_fail(DN_INVALID_ARG, "truncated LZ4 frame descriptor");
      content_size = (uint64_t)rd32(p) | ((uint64_t)rd32(p + 4) << 32);
      p += 8;
    }
    if (end - p < 1) return io_fail(DN_INVALID_ARG, "truncated LZ4 frame descriptor");
    const uint8_t hc = (uint8_t)(xxh32(desc, (size_t)(p - desc), 0) >> 8);
    if (*p++ != hc) return io_fail(DN_INVALID_ARG, "LZ4 frame header checksum mismatch");
    const size_t frame_start = out.size();
    for (;;) {
      if (end - p < 4) return io_fail(DN_INVALID_ARG, "truncated LZ4 block");
      const uint32_t bsize = rd32(p);
      p += 4;
      if (bsize == 0) break;
      const bool stored = bsize & 0x80000000u;
      const size_t len = bsize & 0x7FFFFFFFu;
      if (len > block_max || (size_t)(end - p) < len + (block_checksum ? 4 : 0))
        return io_fail(DN_INVALID_ARG, "truncated or oversized LZ4 block");
      if (block_checksum && xxh32(p, len, 0) != rd32(p + len))
        return io_fail(DN_INVALID_ARG, "LZ4 block checksum mismatch");
      if (stored) {
        out.insert(out.end(), p, p + len);
      } else if (!decompress_block(p, len, out, frame_start, block_max)) {
        return io_fail(DN_INVALID_ARG, "malformed LZ4 block");
      }
      p += len + (block_checksum ? 4 : 0);
    }
    if (content_checksum) {
      if (end - p < 4) return io_fail(DN_INVALID_ARG, "truncated LZ4 content checksum");
      if (xxh32(out.data() + frame_start, out.size() - frame_start, 0) != rd32(p))
        return io_fail(DN_INVALID_ARG, "LZ4 content checksum mismatch");
      p += 4;
    }
    if (has_size && content_size != out.size() - frame_start)
      return io_fail(DN_INVALID_ARG, "LZ4 content size mismatch");
    any = true;
  }
  if (!any) return io_fail(DN_INVALID_ARG, "no LZ4 frame");
  return DN_OK;
}

}  // namespace

extern "C" const char* dn_io_last_error(void) { return g_io_error.c_str(); }

extern "C" uint32_t dn_xxh32(const void* data, int64_t n, uint32_t seed) {
  return xxh32(static_cast<const uint8_t*>(data), (size_t)(n < 0 ? 0 : n), seed);
}

extern "C" int64_t dn_lz4f_compress_bound(int64_t n) {
  if (n < 0) return -1;
  const int64_t blocks = n / (int64_t)kBlockMax + 1;
  return 4 + 2 + 8 + 1 + blocks * 4 + n + 4;  // header, block sizes, stored data, end mark
}

extern "C" dn_status dn_lz4f_compress(const void* src, int64_t n, void* dst, int64_t capacity,
                                      int64_t* out_len) {
  if ((!src && n > 0) || n < 0 || !out_len) return io_fail(DN_INVALID_ARG, "NULL argument");
  const uint8_t* s = static_cast<const uint8_t*>(src);
  std::vector<uint8_t> out;
  out.reserve((size_t)n / 2 + 64);
  out.resize(4);
  wr32(out.data(), kMagic);
  // FLG: version 01, independent blocks, content size; BD: 4 MB blocks.
  const size_t desc = out.size();
  out.push_back(0x40 | 0x20 | 0x08);
  out.push_back(7 << 4);
  for (int k = 0; k < 8; ++k) out.push_back((uint8_t)((uint64_t)n >> (8 * k)));
  out.push_back((uint8_t)(xxh32(out.data() + desc, out.size() - desc, 0) >> 8));
  std::vector<uint8_t> blk;
  for (size_t off = 0; off < (size_t)n; off += kBlockMax) {
    const size_t len = std::min(kBlockMax, (size_t)n - off);
    blk.clear();
    compress_block(s + off, len, blk);
    const size_t at = out.size();
    out.resize(at + 4);
    if (blk.size() < len) {
      wr32(out.data() + at, (uint32_t)blk.size());
      out.insert(out.end(), blk.begin(), blk.end());
    } else {
      wr32(out.data() + at, (uint32_t)len | 0x80000000u);
      out.insert(out.end(), s + off, s + off + len);
    }
  }
  const size_t at = out.size();
  out.resize(at + 4);
  wr32(out.data() + at, 0);
  *out_len = (int64_t)out.size();
  if (!dst) return DN_OK;
  if (capacity < (int64_t)out.size()) return io_fail(DN_INVALID_ARG, "output buffer too small");
  memcpy(dst, out.data(), out.size());
  return DN_OK;
}

extern "C" dn_status dn_lz4f_decompress(const void* src, int64_t n, void* dst, int64_t capacity,
                                        int64_t* out_len) {
  if (!src || n <= 0 || !out_len) return io_fail(DN_INVALID_ARG, "NULL or empty input");
  // A size query keeps its decoded output for the fetch that follows; the
  // cache is reused only for the same pointer, length and input bytes (the
  // caller may have put another frame of the same length at that address).
  const uint32_t hash = xxh32(static_cast<const uint8_t*>(src), (size_t)n, 0);
  if (src != g_last_src || n != g_last_n || hash != g_last_hash) {
    g_last_src = nullptr;
    const dn_status st = decode_frames(static_cast<const uint8_t*>(src), (size_t)n, g_last_out);
    if (st != DN_OK) return st;
    g_last_src = src;
    g_last_n = n;
    g_last_hash = hash;
  }
  *out_len = (int64_t)g_last_out.size();
  if (!dst) return DN_OK;
  if (capacity < (int64_t)g_last_out.size())
    return io_fail(DN_INVALID_ARG, "output buffer too small");
  memcpy(dst, g_last_out.data(), g_last_out.size());
  g_last_src = nullptr;  // the result has been handed over
  g_last_out.clear();
  g_last_out.shrink_to_fit();
  return DN_OK;
}
