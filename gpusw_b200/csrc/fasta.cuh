// Native FASTA reader and encoder (host only, no CUDA calls): FASTA bytes -> residue codes
// through the scheme's 256-entry table, int32 offsets and record ids, in one pass.
//
// Semantics follow the reference package's reader and encoder (src/gpusw/encode.py:89-120
// read_fasta, :196-225 the encoding loop): lines are split at \n, \r\n or \r and stripped
// of spaces and tabs at both ends; empty lines are skipped; lines before the first header
// are ignored; a header line ">..." starts a record whose id is its first
// whitespace-separated word (or "seq<k>" for a bare ">", k = records so far); the record's
// sequence is its stripped lines joined; each byte maps through the table (case folding is
// part of the table); with unknown="error" the first byte that maps to the sentinel stops
// the parse and is reported with its record.
//
// Only plain ASCII text is taken: a byte >= 0x80 or one of \v \f \x1c-\x1f (characters
// that the reference's Unicode line splitting or stripping treats specially) returns
// GPUSW_ERR_UNSUPPORTED so that the caller runs its own reader, which reproduces the
// reference exactly for any text.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

struct gpusw_fasta {
  std::unique_ptr<uint8_t[]> codes;  // `ncodes` used (capacity: the input length)
  int64_t ncodes = 0;
  std::vector<int32_t> offsets{0};
  std::string ids;
  std::vector<int64_t> id_offsets{0};
  std::string err;
  int64_t bad_record = -1;  // unknown="error": record and byte of the first unknown symbol
  int bad_byte = -1;
};

namespace {

inline bool fasta_blank(uint8_t c) { return c == ' ' || c == '\t'; }
inline bool fasta_special(uint8_t c) { return c >= 0x80 || c == '\v' || c == '\f' || (c >= 0x1c && c <= 0x1f); }

// Returns GPUSW_OK, GPUSW_ERR_UNSUPPORTED (caller falls back), GPUSW_ERR_INVALID (unknown
// symbol, or more than 2^31 - 1 residues).
int fasta_parse(gpusw_fasta& f, const char* data, int64_t len, const uint8_t* lut, int sentinel,
                int unknown_error) {
  const uint8_t* p = reinterpret_cast<const uint8_t*>(data);
  {
    std::atomic<bool> special{false};
    parallel_ranges(len, [&](long long lo, long long hi) {
      bool sp = false;
      for (long long k = lo; k < hi; ++k) sp |= fasta_special(p[k]);
      if (sp) special = true;
    });
    if (special) return GPUSW_ERR_UNSUPPORTED;
  }
  // Pass 1 (sequential): lines, headers and ids; every sequence line becomes a segment
  // (source start, length) appended to the current record.
  struct Seg { int64_t src, n; };
  std::vector<Seg> segs;
  int64_t nout = 0;
  bool in_record = false;
  int64_t pos = 0;
  while (pos < len) {
    // one line: [pos, eol), then skip \r\n, \n or \r
    const uint8_t* nl = static_cast<const uint8_t*>(memchr(p + pos, '\n', (size_t)(len - pos)));
    int64_t eol = nl ? (int64_t)(nl - p) : len;
    const uint8_t* cr = static_cast<const uint8_t*>(memchr(p + pos, '\r', (size_t)(eol - pos)));
    int64_t next;
    if (cr) {
      eol = (int64_t)(cr - p);
      next = eol + 1;
      if (next < len && p[next] == '\n') ++next;
    } else {
      next = eol < len ? eol + 1 : len;
    }
    int64_t a = pos, b = eol;
    while (a < b && fasta_blank(p[a])) ++a;
    while (b > a && fasta_blank(p[b - 1])) --b;
    pos = next;
    if (a == b) continue;
    if (p[a] == '>') {
      if (in_record) f.offsets.push_back((int32_t)nout);
      int64_t s = a + 1;
      while (s < b && fasta_blank(p[s])) ++s;
      int64_t e = s;
      while (e < b && !fasta_blank(p[e])) ++e;
      if (b - a > 1) f.ids.append(reinterpret_cast<const char*>(p + s), (size_t)(e - s));
      else f.ids += "seq" + std::to_string(f.offsets.size() - 1);
      f.id_offsets.push_back((int64_t)f.ids.size());
      in_record = true;
      continue;
    }
    if (!in_record) continue;
    if (nout + (b - a) >= (int64_t)INT32_MAX) {
      f.err = "more than 2**31 - 1 residues in one sequence set";
      return GPUSW_ERR_INVALID;
    }
    segs.push_back({a, b - a});
    nout += b - a;
  }
  if (in_record) f.offsets.push_back((int32_t)nout);
  // Pass 2 (threaded over segments): table lookup into the output
  f.codes.reset(new uint8_t[(size_t)std::max<int64_t>(nout, 1)]);
  f.ncodes = nout;
  std::vector<int64_t> dst0(segs.size() + 1, 0);
  for (size_t k = 0; k < segs.size(); ++k) dst0[k + 1] = dst0[k] + segs[k].n;
  uint8_t* out = f.codes.get();
  parallel_ranges_min((long long)segs.size(), 1024, [&](long long lo, long long hi) {
    for (long long k = lo; k < hi; ++k) {
      const uint8_t* src = p + segs[(size_t)k].src;
      uint8_t* dst = out + dst0[(size_t)k];
      for (int64_t j = 0; j < segs[(size_t)k].n; ++j) dst[j] = lut[src[j]];
    }
  });
  if (unknown_error) {
    // the first code equal to the sentinel, in record order
    const uint8_t* hit = static_cast<const uint8_t*>(memchr(out, sentinel, (size_t)nout));
    if (hit) {
      const int64_t at = hit - out;
      const size_t r = (size_t)(std::upper_bound(f.offsets.begin(), f.offsets.end(), (int32_t)at) - f.offsets.begin()) - 1;
      const size_t sg = (size_t)(std::upper_bound(dst0.begin(), dst0.end(), at) - dst0.begin()) - 1;
      f.bad_record = (int64_t)r;
      f.bad_byte = p[segs[sg].src + (at - dst0[sg])];
      f.err = "out-of-alphabet symbol";
      return GPUSW_ERR_INVALID;
    }
  }
  return GPUSW_OK;
}

}  // namespace

extern "C" {

int gpusw_fasta_parse(const char* data, int64_t len, const uint8_t* lut, int32_t sentinel,
                      int unknown_error, gpusw_fasta** out) {
  if (!out) return GPUSW_ERR_INVALID;
  *out = nullptr;
  if ((!data && len > 0) || len < 0 || !lut || sentinel < 0 || sentinel > 255) return GPUSW_ERR_INVALID;
  gpusw_fasta* f = nullptr;
  try {
    f = new gpusw_fasta();
    const int rc = fasta_parse(*f, data, len, lut, sentinel, unknown_error);
    *out = f;
    return rc;
  } catch (const std::bad_alloc&) {
    delete f;
    return GPUSW_ERR_MEMORY;
  }
}

int32_t gpusw_fasta_count(const gpusw_fasta* f) { return f ? (int32_t)f->offsets.size() - 1 : 0; }
int64_t gpusw_fasta_residues(const gpusw_fasta* f) { return f ? f->ncodes : 0; }
const uint8_t* gpusw_fasta_codes(const gpusw_fasta* f) { return f ? f->codes.get() : nullptr; }
const int32_t* gpusw_fasta_offsets(const gpusw_fasta* f) { return f ? f->offsets.data() : nullptr; }
const char* gpusw_fasta_ids(const gpusw_fasta* f) { return f ? f->ids.data() : nullptr; }
const int64_t* gpusw_fasta_id_offsets(const gpusw_fasta* f) { return f ? f->id_offsets.data() : nullptr; }
const char* gpusw_fasta_error(const gpusw_fasta* f) { return f ? f->err.c_str() : ""; }
int64_t gpusw_fasta_bad_record(const gpusw_fasta* f) { return f ? f->bad_record : -1; }
int32_t gpusw_fasta_bad_byte(const gpusw_fasta* f) { return f ? f->bad_byte : -1; }
void gpusw_fasta_free(gpusw_fasta* f) { delete f; }

}  // extern "C"
