// Gotoh affine-gap scoring on sm_100a: the team wavefront core.
//
// Recurrence (same integers as the reference package's kernel, src/gpusw/kernel.py:56-158,
// and oracle, src/gpusw/reference.py:38-125): rows i run over the row sequence (the
// reference in a cross product), columns j over the column sequence (the query),
//   F(i,j) = max(H(i-1,j) + go, F(i-1,j) + ge)
//   E(i,j) = max(H(i,j-1) + go, E(i,j-1) + ge)
//   H(i,j) = max(H(i-1,j-1) + SUB[r_i][q_j], E, F)   (and >= 0 in local mode)
//
// Layout. A "team" of G lanes (G = 8, 16 or 32 consecutive lanes of one warp) scores one
// alignment task; lane L owns the W consecutive columns [L*W, L*W + W) of the current
// column pass and keeps their vertical state in registers. Row i reaches lane L at step
// t = i + L (anti-diagonal wavefront); the horizontal carry of each row travels one lane
// to the right per step through __shfl_up_sync, and so does the row's residue code.
//
// Packing. With P = 2 every 32-bit register holds two int16 cells of two different
// alignments (the column sequences c0, c1 of a pair against the same row sequence in a
// cross product, or two unrelated pairs), updated together by the DPX s16x2 instructions.
// With P = 1 a register holds one int32 cell (the int32 path and the overflow rerun).
//
// Algebra used to shorten the per-column dependency chain (exact over the integers):
//   HGO = H + go is stored instead of H, and the profile holds s' = s - go, so that
//   X(i,j)   = max(HGO(i-1,j-1) + s', F(i,j) [, 0 in local mode])    (= max(Hdiag+s, F))
//   E(i,j)   = max(E(i,j-1) + max(ge, go), X(i,j-1) + go)             (H = max(X, E))
//   HGO(i,j) = max(E(i,j) + go, X(i,j) + go)
// so the only serial dependency along a row is one add-max per column (the E chain).
// Cost per cell register: F, X, X+go, E, HGO = 5 int16x2 ops, plus 1/2 op for the
// running maximum (3-input max over two columns).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gsw {

constexpr int kModeLocal = 0, kModeGlobal = 1, kModeSemi = 2;

// Per-call scheme constants shared by every kernel.
struct SchemeDev {
  int mode;       // kModeLocal / kModeGlobal / kModeSemi
  int free_q;     // semiglobal: free end gaps in the query (column sequence)
  int free_r;     // semiglobal: free end gaps in the reference (row sequence)
  int go, ge;     // gap open / extend (<= 0)
  int ges;        // max(ge, go): E extension cost once H = max(X, E) is folded in
  int ns;         // side of the substitution table (alphabet + sentinel)
  int pad_code;   // profile row used for padded rows (= ns)
  int s_pad;      // substitution score of padded cells (<= 0)
  int ovf_limit;  // int16 runs: a score above this may have wrapped -> rescore in int32
  int neg_e0, neg_f, neg_low;  // per-width sentinels (see make_scheme on the host)
};

// -------------------------------------------------------------------------------------
// Lane arithmetic: P = 2 -> two int16 cells per register (DPX s16x2), P = 1 -> int32.
template <int P> struct V;
template <> struct V<2> {
  static __device__ __forceinline__ uint32_t addmax(uint32_t a, uint32_t b, uint32_t c) {
    return __viaddmax_s16x2(a, b, c);
  }
  static __device__ __forceinline__ uint32_t addmax_relu(uint32_t a, uint32_t b, uint32_t c) {
    return __viaddmax_s16x2_relu(a, b, c);
  }
  static __device__ __forceinline__ uint32_t max3(uint32_t a, uint32_t b, uint32_t c) {
    return __vimax3_s16x2(a, b, c);
  }
  static __device__ __forceinline__ uint32_t max2(uint32_t a, uint32_t b) { return __vmaxs2(a, b); }
  static __device__ __forceinline__ uint32_t add(uint32_t a, uint32_t b) { return __vadd2(a, b); }
  static __device__ __forceinline__ uint32_t splat(int v) { return (uint32_t)(v & 0xFFFF) * 0x10001u; }
  static __device__ __forceinline__ uint32_t pack(int lo, int hi) {
    return (uint32_t)(lo & 0xFFFF) | ((uint32_t)(hi & 0xFFFF) << 16);
  }
  static __device__ __forceinline__ int get(uint32_t w, int h) { return (int)(int16_t)(w >> (16 * h)); }
  static __device__ __forceinline__ uint32_t half_mask(int h) { return h ? 0xFFFF0000u : 0x0000FFFFu; }
};
template <> struct V<1> {
  static __device__ __forceinline__ uint32_t addmax(uint32_t a, uint32_t b, uint32_t c) {
    return (uint32_t)__viaddmax_s32((int)a, (int)b, (int)c);
  }
  static __device__ __forceinline__ uint32_t addmax_relu(uint32_t a, uint32_t b, uint32_t c) {
    return (uint32_t)__viaddmax_s32_relu((int)a, (int)b, (int)c);
  }
  static __device__ __forceinline__ uint32_t max3(uint32_t a, uint32_t b, uint32_t c) {
    return (uint32_t)__vimax3_s32((int)a, (int)b, (int)c);
  }
  static __device__ __forceinline__ uint32_t max2(uint32_t a, uint32_t b) { return (uint32_t)max((int)a, (int)b); }
  static __device__ __forceinline__ uint32_t add(uint32_t a, uint32_t b) { return a + b; }
  static __device__ __forceinline__ uint32_t splat(int v) { return (uint32_t)v; }
  static __device__ __forceinline__ uint32_t pack(int lo, int) { return (uint32_t)lo; }
  static __device__ __forceinline__ int get(uint32_t w, int) { return (int)w; }
  static __device__ __forceinline__ uint32_t half_mask(int) { return 0xFFFFFFFFu; }
};

// H(0, j) / H(i, 0) boundary value of a DP edge of length k (k >= 0).
__device__ __forceinline__ int edge_value(const SchemeDev& S, bool free_edge, int k) {
  if (k == 0 || S.mode == kModeLocal || (S.mode == kModeSemi && free_edge)) return 0;
  return S.go + (k - 1) * S.ge;
}

// Score of a pair with an empty side (src/gpusw/reference.py:48-54).
__device__ __forceinline__ int empty_score(const SchemeDev& S, int n, int m) {
  if (S.mode == kModeLocal || (n == 0 && m == 0)) return 0;
  if (n == 0) return (S.mode == kModeSemi && S.free_q) ? 0 : S.go + (m - 1) * S.ge;
  return (S.mode == kModeSemi && S.free_r) ? 0 : S.go + (n - 1) * S.ge;
}

// Packed residue codes: sequence words start 16-byte aligned; code c of a sequence sits
// in word c / per at bit (c % per) * bits.
// Code r of a packed sequence starting at word pointer w (per codes per word): shifts for
// per = 4, 8, 16 and a multiply-high for per = 6 instead of an integer division.
__device__ __forceinline__ uint32_t packed_row_code(const uint32_t* w, int r, int bits, int per) {
  unsigned q, rem;
  if (per == 6) {
    q = __umulhi((unsigned)r, 0xAAAAAAABu) >> 2;  // r / 6 for every 32-bit r
    rem = (unsigned)r - q * 6u;
  } else {
    const int sh = __ffs(per) - 1;                 // per = 4, 8 or 16
    q = (unsigned)r >> sh;
    rem = (unsigned)r & (unsigned)(per - 1);
  }
  return (__ldg(w + q) >> (rem * (unsigned)bits)) & ((1u << bits) - 1u);
}

struct Packed {
  const uint32_t* words;
  const long long* woff;  // first word of each sequence
  const int* len;
  int bits, per;
  __device__ __forceinline__ int code(int seq, int c) const {
    uint32_t w = __ldg(words + woff[seq] + c / per);
    return (int)((w >> ((c % per) * bits)) & ((1u << bits) - 1u));
  }
  // The same code without an integer division (the per-team profile builders of the pairs
  // kernel, where the decode is a visible share of a short alignment's work).
  __device__ __forceinline__ int code_fast(int seq, int c) const {
    return (int)packed_row_code(words + woff[seq], c, bits, per);
  }
};

// A sequence set as the reference package encodes it (one code byte per residue,
// int32 offsets of n + 1 entries), read in place from caller-owned device memory.
struct ByteSeqs {
  const uint8_t* codes;
  const int* off;
  int n;
  __device__ __forceinline__ int length(int s) const { return off[s + 1] - off[s]; }
  __device__ __forceinline__ int code(int s, int c) const { return (int)__ldg(codes + off[s] + c); }
};

// Residue code for the per-team profile builders: packed sets decode without a division.
__device__ __forceinline__ int seq_code(const Packed& s, int seq, int c) { return s.code_fast(seq, c); }
__device__ __forceinline__ int seq_code(const ByteSeqs& s, int seq, int c) { return s.code(seq, c); }

// Lane 0's code feed for a byte-coded row: the team_pass call passes the row's first
// byte through its word-pointer parameter; one byte per step, the pad code past the end.
struct RowFeed8 {
  const uint8_t* p;
  int m, pad;
  __device__ __forceinline__ void init(const uint32_t* w, int, int, int m_, int pad_) {
    p = reinterpret_cast<const uint8_t*>(w);
    m = m_;
    pad = pad_;
  }
  __device__ __forceinline__ int next(int t) const { return t < m ? (int)__ldg(p + t) : pad; }
};

// Lane 0's code feed for one row sequence: one packed word per `per` steps.
struct RowFeed {
  const uint32_t* ptr;
  uint32_t cur;
  int pos, bits, per, m, pad;
  uint32_t mask;
  __device__ __forceinline__ void init(const uint32_t* p, int bits_, int per_, int m_, int pad_) {
    ptr = p; bits = bits_; per = per_; m = m_; pad = pad_; pos = 0;
    mask = (1u << bits_) - 1u;
    cur = m_ > 0 ? __ldg(p) : 0u;
  }
  // Code of row t (t = 0, 1, 2, ... called once per step); pad once past the end.
  __device__ __forceinline__ int next(int t) {
    int c = (int)(cur & mask);
    cur >>= bits;
    if (++pos == per) {
      pos = 0;
      ++ptr;
      cur = (t + 1 < m) ? __ldg(ptr) : 0u;
    }
    return t < m ? c : pad;
  }
};

// Per-lane accumulators of one task, merged over the column passes of the task.
struct Acc {
  int bi = 0x7FFFFFFF, bj = 0x7FFFFFFF;  // LOCATE: first cell (row-major) holding `best`
  uint32_t best;    // running max of HGO (local score / int16 overflow guard)
  uint32_t endrow;  // max over the last row of HGO at real columns   (non-local)
  uint32_t corner;  // HGO at (m, n)                                   (non-local)
  uint32_t endcol;  // max over rows of HGO at column n                 (non-local, free_q)
};

// One column pass of one team task.
//
// prof      : shared-memory profile, row a at prof + a * pstride; uint4 slot k4*G + lane
//             holds the 4 consecutive columns L*W + 4*k4 .. +3 of this pass (lo/hi halves
//             are the two packed alignments when P = 2).
// prof_hi   : second profile for PAIRS (the hi half scores against its own row codes).
// rows      : row sequence(s); rows[1] is used only for PAIRS.
// m0, m1    : row lengths (cross product: m1 == m0).
// n0, n1    : full column lengths of the two halves.
// col0      : first column (0-based) of this pass.
// bnd       : boundary column (E, X+go) at column col0-1 for each row, read by lane 0 when
//             has_prev, written by lane G-1 when has_next (in place: row i is read at step
//             i and written at step i + G - 1).
//
// LEFTPAD (semiglobal with both ends free only): every column sequence is right-aligned to
// the last column of the last pass; the columns in front of it score 0 against every
// residue, which reproduces the free column-0 boundary exactly (H stays 0, E enters the
// first real column at go). The query's last column is then register W-1 of lane G-1 in
// the last pass, so the end-column maximum costs one op per step instead of one per cell,
// and the end row needs no column mask (the dummy columns hold 0, which the result takes
// as a floor anyway).
//
// LOCATE (P = 1, local): instead of the 3-input running max, keep the first cell in
// row-major order (reference row, then query column) that holds the maximum; across column
// passes an equal value replaces the stored cell only if it comes earlier in that order.
template <int G, int W, int P, bool LOCAL, bool PAIRS, bool LEFTPAD = false, class Feed = RowFeed,
          bool LOCATE = false>
__device__ __forceinline__ void team_pass(const SchemeDev& S, const uint4* __restrict__ prof,
                                          int pstride, const uint32_t* row_w0,
                                          const uint32_t* row_w1, int row_bits, int row_per,
                                          int m0, int m1, int n0, int n1, int col0,
                                          uint2* bnd, bool has_prev, bool has_next, int lane,
                                          unsigned wmask, Acc& acc, bool last_pass = true) {
  using Ops = V<P>;
  static_assert(W % 4 == 0, "W must be a multiple of 4");
  const uint32_t GO = Ops::splat(S.go), GE = Ops::splat(S.ge), GES = Ops::splat(S.ges);
  const uint32_t NEGF = Ops::splat(S.neg_f), NEGE0 = Ops::splat(S.neg_e0);
  const uint32_t NEGLOW = Ops::splat(S.neg_low);
  const int mrows = PAIRS ? max(m0, m1) : m0;
  const bool track_endcol = !LOCAL && S.mode == kModeSemi && S.free_q;
  const bool ladder_row0 = !(S.mode == kModeLocal || (S.mode == kModeSemi && S.free_r));
  const bool ladder_col0 = !(S.mode == kModeLocal || (S.mode == kModeSemi && S.free_q));

  // Vertical state of my W columns: HGO(0, j) and F(0, j) = -inf.
  uint32_t HGO[W], F[W], CM[W];
  const int jbase = col0 + lane * W;  // 0-based column of my register 0
#pragma unroll
  for (int k = 0; k < W; ++k) {
    int h0 = ladder_row0 ? edge_value(S, false, jbase + k + 1) : 0;
    HGO[k] = Ops::splat(h0 + S.go);
    F[k] = NEGF;
    CM[k] = NEGLOW;
  }
  // HGO of the column left of my strip at the current row (diag of the next row).
  uint32_t hgo_left = Ops::splat((ladder_row0 ? edge_value(S, false, jbase) : 0) + S.go);
  // Outputs of my last column for the lane to the right.
  uint32_t e_out = NEGE0, x_out = GO;
  int code = S.pad_code;
  // Lane 0 column-0 boundary: X(i,0) + go = H(i,0) + go for i >= 1.
  uint32_t xb = Ops::splat((ladder_col0 ? S.go : 0) + S.go);
  const uint32_t xb_step = ladder_col0 ? GE : 0u;

  Feed f0, f1;
  f0.init(row_w0, row_bits, row_per, m0, S.pad_code);
  if (PAIRS) f1.init(row_w1, row_bits, row_per, m1, S.pad_code);

  const int nsteps = mrows + G - 1;
  for (int t = 0; t < nsteps; ++t) {
    // Values the left lane produced in the previous step (row t - lane).
    uint32_t e_in = __shfl_up_sync(wmask, e_out, 1, G);
    uint32_t x_in = __shfl_up_sync(wmask, x_out, 1, G);
    int c_in = __shfl_up_sync(wmask, code, 1, G);
    int feed = f0.next(t);
    if (PAIRS) feed |= f1.next(t) << 16;
    const int i = t - lane;  // my row (0-based)
    if (lane == 0) {
      code = feed;
      if (has_prev) {
        uint2 b = (i < mrows) ? bnd[i] : make_uint2(NEGE0, GO);
        e_in = b.x;
        x_in = b.y;
      } else {
        e_in = NEGE0;
        x_in = xb;
      }
    } else {
      code = c_in;
    }
    xb = Ops::add(xb, xb_step);
    if (i < 0 || i >= mrows) continue;

    const uint4* pr0 = prof + (PAIRS ? (code & 0xFFFF) : code) * pstride + lane;
    const uint4* pr1 = prof + (PAIRS ? (code >> 16) : code) * pstride + lane;
    // Columns in chunks of CH: F, X and X + go (independent across columns), then the
    // E chain (one add-max per column) and the new HGO. Chunking bounds live registers.
    constexpr int CH = (W % 16 == 0) ? 16 : ((W % 8 == 0) ? 8 : 4);
    static_assert(W % CH == 0, "column chunks must tile W");
    uint32_t diag = hgo_left;
    uint32_t e = Ops::addmax(e_in, GES, x_in);
    hgo_left = Ops::addmax(e_in, GO, x_in);
    uint32_t xlast = 0;
#pragma unroll
    for (int c0 = 0; c0 < W; c0 += CH) {
      // Substitution scores s' = s - go of this chunk's columns for the row's code(s).
      uint32_t sp[CH];
#pragma unroll
      for (int k4 = 0; k4 < CH / 4; ++k4) {
        const int slot = (c0 / 4 + k4) * G;
        const uint4 a = pr0[slot];
        if (PAIRS) {
          const uint4 b = pr1[slot];
          // low half from a, high half from b: one byte permute per register
          sp[4 * k4 + 0] = __byte_perm(a.x, b.x, 0x7610);
          sp[4 * k4 + 1] = __byte_perm(a.y, b.y, 0x7610);
          sp[4 * k4 + 2] = __byte_perm(a.z, b.z, 0x7610);
          sp[4 * k4 + 3] = __byte_perm(a.w, b.w, 0x7610);
        } else {
          sp[4 * k4 + 0] = a.x;
          sp[4 * k4 + 1] = a.y;
          sp[4 * k4 + 2] = a.z;
          sp[4 * k4 + 3] = a.w;
        }
      }
      uint32_t XG[CH];
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        uint32_t f = Ops::addmax(F[c0 + k], GE, HGO[c0 + k]);
        F[c0 + k] = f;
        uint32_t x = LOCAL ? Ops::addmax_relu(diag, sp[k], f) : Ops::addmax(diag, sp[k], f);
        diag = HGO[c0 + k];
        XG[k] = Ops::add(x, GO);
      }
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        HGO[c0 + k] = Ops::addmax(e, GO, XG[k]);
        if (c0 + k + 1 < W) e = Ops::addmax(e, GES, XG[k]);
      }
      xlast = XG[CH - 1];
    }
    e_out = e;
    x_out = xlast;
    if (LOCATE) {
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const int v = (int)HGO[k], b = (int)acc.best, j = jbase + k;
        if (j < n0 && (v > b || (v == b && (i < acc.bi || (i == acc.bi && j < acc.bj))))) {
          acc.best = (uint32_t)v;
          acc.bi = i;
          acc.bj = j;
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k + 1 < W; k += 2) acc.best = Ops::max3(acc.best, HGO[k], HGO[k + 1]);
    }
    if (has_next && lane == G - 1) bnd[i] = make_uint2(e_out, x_out);

    if (LEFTPAD) {
      // end column = register W-1 of lane G-1 in the last pass; rows past a half's end
      // are masked out; the end row is taken over all columns.
      if (last_pass && lane == G - 1) {
        const uint32_t keep = (i < m0 ? Ops::half_mask(0) : 0u) | (i < m1 ? Ops::half_mask(1) : 0u);
        acc.endcol = Ops::max2(acc.endcol, (HGO[W - 1] & keep) | (NEGLOW & ~keep));
      }
#pragma unroll
      for (int h = 0; h < P; ++h) {
        if (i == (h ? m1 : m0) - 1) {
          const uint32_t hm = Ops::half_mask(h);
          uint32_t v = acc.endrow;
#pragma unroll
          for (int k = 0; k < W; ++k) v = Ops::max2(v, HGO[k]);
          acc.endrow = (acc.endrow & ~hm) | (v & hm);
        }
      }
    } else if (!LOCAL) {
      if (track_endcol) {
        if (PAIRS && m0 != m1) {
          // Rows past a half's end must not count towards that half's last column.
          uint32_t keep = (i < m0 ? Ops::half_mask(0) : 0u) | (i < m1 ? Ops::half_mask(1) : 0u);
#pragma unroll
          for (int k = 0; k < W; ++k) CM[k] = Ops::max2(CM[k], (HGO[k] & keep) | (NEGLOW & ~keep));
        } else {
#pragma unroll
          for (int k = 0; k < W; ++k) CM[k] = Ops::max2(CM[k], HGO[k]);
        }
      }
      // Last row of a half: the end row and the corner.
#pragma unroll
      for (int h = 0; h < P; ++h) {
        const int mh = h ? m1 : m0;
        const int nh = h ? n1 : n0;
        if (i == mh - 1) {
          const uint32_t hm = Ops::half_mask(h);
#pragma unroll
          for (int k = 0; k < W; ++k) {
            const int j = jbase + k;  // 0-based column
            if (j < nh) {
              uint32_t v = Ops::max2(acc.endrow, HGO[k]);
              acc.endrow = (acc.endrow & ~hm) | (v & hm);
            }
            if (j == nh - 1) acc.corner = (acc.corner & ~hm) | (HGO[k] & hm);
          }
        }
      }
    }
  }
  if (!LEFTPAD && track_endcol) {
#pragma unroll
    for (int h = 0; h < P; ++h) {
      const int nh = h ? n1 : n0;
      const uint32_t hm = Ops::half_mask(h);
#pragma unroll
      for (int k = 0; k < W; ++k)
        if (jbase + k == nh - 1) acc.endcol = (acc.endcol & ~hm) | (CM[k] & hm);
    }
  }
}

// Lane-local profile fill: lane `lane` writes exactly the slots it reads in team_pass
// (its W columns of the pass, every code row plus the pad row), so no synchronisation
// with other lanes is needed. `sub` may point to shared memory. pad0/pad1 shift the
// halves' columns right (LEFTPAD); positions left of a sequence score 0, positions past
// its end score s_pad.
template <int G, int W, int P, class Seqs = Packed>
__device__ __forceinline__ void build_profile_lane(const SchemeDev& S, const int* sub,
                                                   const Seqs& cols, int c0, int n0, int pad0,
                                                   int c1, int n1, int pad1, int col0,
                                                   uint4* prof, int pstride, int lane) {
  const int pad_s = S.s_pad - S.go, zero_s = -S.go;
  int code[2][W];
#pragma unroll
  for (int h = 0; h < P; ++h) {
    const int c = h ? c1 : c0, n = h ? n1 : n0, pd = h ? pad1 : pad0;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const int j = col0 + lane * W + k - pd;  // real column, or < 0 (dummy) / >= n (past end)
      code[h][k] = (c >= 0 && j >= 0 && j < n) ? seq_code(cols, c, j) : (j < 0 ? -1 : -2);
    }
  }
  for (int a = 0; a <= S.ns; ++a) {
    uint4* row = prof + a * pstride + lane;
#pragma unroll
    for (int k4 = 0; k4 < W / 4; ++k4) {
      uint32_t v[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        int hv[2] = {pad_s, pad_s};
#pragma unroll
        for (int h = 0; h < P; ++h) {
          const int cd = code[h][4 * k4 + e];
          hv[h] = cd >= 0 ? (a < S.ns ? sub[a * S.ns + cd] - S.go : pad_s)
                          : (cd == -1 ? (a < S.ns ? zero_s : pad_s) : pad_s);
        }
        v[e] = V<P>::pack(hv[0], hv[1]);
      }
      row[k4 * G] = make_uint4(v[0], v[1], v[2], v[3]);
    }
  }
}

// Int8 form of build_profile_lane for two halves (P = 2, used when every profile value fits
// in a signed byte): half h's values go to its own table profH, four columns per 32-bit
// slot k4 * G + lane of each code row (pstride8 slots per row). The values come from `ext`,
// the per-block table of every (column class, row code) byte (see pairs_ext_stride): for
// each group of four columns and four row codes, four 32-bit loads and a 4 x 4 byte
// transpose (eight byte permutes) give the four row words.
template <int G, int W, class Seqs = Packed>
__device__ __forceinline__ void build_profile_lane8(const SchemeDev& S, const uint32_t* ext,
                                                    const Seqs& cols, int c0, int n0, int pad0,
                                                    int c1, int n1, int pad1, int col0,
                                                    uint32_t* prof0, uint32_t* prof1,
                                                    int pstride8, int lane) {
  const int rw = ((S.ns + 1 + 3) & ~3) / 4;  // 32-bit words per column class
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int c = h ? c1 : c0, n = h ? n1 : n0, pd = h ? pad1 : pad0;
    uint32_t* prof = h ? prof1 : prof0;
    int cls[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const int j = col0 + lane * W + k - pd;  // real column, or < 0 (dummy) / >= n (past end)
      cls[k] = (c >= 0 && j >= 0 && j < n) ? seq_code(cols, c, j) : (j < 0 ? S.ns : S.ns + 1);
      cls[k] *= rw;
    }
    for (int rg = 0; rg < rw; ++rg) {
      uint32_t* row = prof + (4 * rg) * pstride8 + lane;
#pragma unroll
      for (int g = 0; g < W / 4; ++g) {
        const uint32_t w0 = ext[cls[4 * g] + rg], w1 = ext[cls[4 * g + 1] + rg];
        const uint32_t w2 = ext[cls[4 * g + 2] + rg], w3 = ext[cls[4 * g + 3] + rg];
        const uint32_t t0 = __byte_perm(w0, w1, 0x5140), t1 = __byte_perm(w0, w1, 0x7362);
        const uint32_t t2 = __byte_perm(w2, w3, 0x5140), t3 = __byte_perm(w2, w3, 0x7362);
        // row 4 rg + r, columns 4 g .. 4 g + 3
        row[g * G] = __byte_perm(t0, t2, 0x5410);
        if (4 * rg + 1 <= S.ns) row[pstride8 + g * G] = __byte_perm(t0, t2, 0x7632);
        if (4 * rg + 2 <= S.ns) row[2 * pstride8 + g * G] = __byte_perm(t1, t3, 0x5410);
        if (4 * rg + 3 <= S.ns) row[3 * pstride8 + g * G] = __byte_perm(t1, t3, 0x7632);
      }
    }
  }
}

// Register e (0..3) of a 4-column group from the int8 tables: byte e of a (half 0) and of b
// (half 1), each sign-extended to 16 bits, as one s16x2 word (one prmt with sign replication:
// a selector nibble with bit 3 set yields the sign of the byte it names).
template <int E>
__device__ __forceinline__ uint32_t sx16x2(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b),
      "n"(E | ((8 | E) << 4) | ((4 + E) << 8) | ((12 + E) << 12)));
  return d;
}

// Max-reduce an accumulator word over the G lanes of a team.
template <int G, int P>
__device__ __forceinline__ uint32_t team_max(uint32_t v, unsigned wmask) {
#pragma unroll
  for (int off = G / 2; off > 0; off >>= 1) v = V<P>::max2(v, __shfl_xor_sync(wmask, v, off, G));
  return v;
}

// LOCATE reduction (int32): best value first, then the earliest (row, column).
template <int G>
__device__ __forceinline__ void team_argmax(Acc& a, unsigned wmask) {
#pragma unroll
  for (int off = G / 2; off > 0; off >>= 1) {
    const int ov = (int)__shfl_xor_sync(wmask, a.best, off, G);
    const int oi = __shfl_xor_sync(wmask, a.bi, off, G);
    const int oj = __shfl_xor_sync(wmask, a.bj, off, G);
    const int v = (int)a.best;
    if (ov > v || (ov == v && (oi < a.bi || (oi == a.bi && oj < a.bj)))) {
      a.best = (uint32_t)ov;
      a.bi = oi;
      a.bj = oj;
    }
  }
}

// -------------------------------------------------------------------------------------
// Explicit-pair column pass with a branch-free steady state (pairs kernel).
//
// Same recurrence, layout and packing as team_pass with PAIRS = true, restructured for the
// read/window shapes where a team's per-row bookkeeping otherwise costs as much as its
// cells:
//  * Row codes come from a per-team ring in shared memory that already holds, for each row,
//    the profile offsets of both halves (a half past its own end gets the pad row). Every
//    lane reads the entry of its own row, so codes are neither shuffled nor decoded per
//    step; the team refills half of the ring every kRingHalf steps.
//  * Steps run in three stretches: the first G-1 (lanes still entering) and the rows from
//    min(m0, m1) - 1 on (lanes leaving, last-row bookkeeping) take the checked path; in
//    between every lane holds a real row of both halves, so the step has no branch.
//  * The end column (LEFTPAD) is a per-lane running max merged by lane G-1 at the end.
//  * The multi-pass boundary column is prefetched one row ahead by lane 0.
// Not covered (team_pass is used instead): LOCATE, and the non-left-padded semiglobal mode
// with free query ends, whose end column needs a mask per cell.
constexpr int kRing = 128, kRingHalf = kRing / 2;

template <int G, int W, int P, bool LOCAL, bool LEFTPAD, bool P8>
struct FastPass {
  using Ops = V<P>;
  const SchemeDev& S;
  const uint4* prof_lane;  // profile row 0, my slot
  const uint32_t* p8_lane0;  // P8: half 0's int8 table, row 0, my slot
  const uint32_t* p8_lane1;  // P8: half 1's int8 table
  uint32_t* ring;
  const uint32_t *w0, *w1;
  int bits, per, pstride;
  int m0, m1, mrows, n0, n1, jbase, lane;
  unsigned wmask;
  bool is_l0, is_last;
  uint2* bnd;
  uint32_t GO, GE, GES, NEGE0, NEGLOW, xb_step;
  uint32_t HGO[W], F[W];
  uint32_t hgo_left, e_out, x_out, xb, ec;
  uint2 nb;  // lane 0, multi-pass: boundary of its next row

  __device__ __forceinline__ FastPass(const SchemeDev& S_) : S(S_) {}

  // ring entries of rows [r0, r1) (clipped to [0, mrows)), lane-strided
  __device__ __forceinline__ void fill(int r0, int r1) {
    r0 = max(r0, 0);
    r1 = min(r1, mrows);
    const uint32_t pad = (uint32_t)(S.pad_code * pstride);
    for (int r = r0 + lane; r < r1; r += G) {
      uint32_t a = pad, b = pad;
      if (r < m0) a = packed_row_code(w0, r, bits, per) * (uint32_t)pstride;
      if (P == 2 && r < m1) b = packed_row_code(w1, r, bits, per) * (uint32_t)pstride;
      ring[r & (kRing - 1)] = a | (b << 16);
    }
  }

  __device__ __forceinline__ void maybe_refill(int t) {
    if (t > 0 && (t & (kRingHalf - 1)) == 0) {
      __syncwarp(wmask);
      fill(t + kRingHalf + 1 - G, t + kRing + 1 - G);
      __syncwarp(wmask);
    }
  }

  template <bool CHECKED, bool HP, bool HN, bool TRACK>
  __device__ __forceinline__ void step(int t, Acc& acc) {
    uint32_t e_in = __shfl_up_sync(wmask, e_out, 1, G);
    uint32_t x_in = __shfl_up_sync(wmask, x_out, 1, G);
    const int i = t - lane;  // my row (0-based)
    if (HP) {
      e_in = is_l0 ? nb.x : e_in;
      x_in = is_l0 ? nb.y : x_in;
      const int ni = t + 1;  // lane 0's next row
      if (is_l0) nb = ni < mrows ? bnd[ni] : make_uint2(NEGE0, GO);
    } else {
      e_in = is_l0 ? NEGE0 : e_in;
      x_in = is_l0 ? xb : x_in;
    }
    xb = Ops::add(xb, xb_step);
    if (CHECKED && (unsigned)i >= (unsigned)mrows) return;

    const uint32_t pc = ring[i & (kRing - 1)];
    const uint4* pr0 = prof_lane + (pc & 0xFFFFu);
    const uint4* pr1 = prof_lane + (pc >> 16);
    const uint32_t* q0 = p8_lane0 + (pc & 0xFFFFu);
    const uint32_t* q1 = p8_lane1 + (pc >> 16);
    constexpr int CH = (W % 16 == 0) ? 16 : ((W % 8 == 0) ? 8 : 4);
    static_assert(W % CH == 0, "column chunks must tile W");
    uint32_t diag = hgo_left;
    uint32_t e = Ops::addmax(e_in, GES, x_in);
    hgo_left = Ops::addmax(e_in, GO, x_in);
    uint32_t xlast = 0;
#pragma unroll
    for (int c0 = 0; c0 < W; c0 += CH) {
      uint32_t sp[CH];
#pragma unroll
      for (int k4 = 0; k4 < CH / 4; ++k4) {
        const int slot = (c0 / 4 + k4) * G;
        if (P8) {
          const uint32_t a = q0[slot], b = q1[slot];
          sp[4 * k4 + 0] = sx16x2<0>(a, b);
          sp[4 * k4 + 1] = sx16x2<1>(a, b);
          sp[4 * k4 + 2] = sx16x2<2>(a, b);
          sp[4 * k4 + 3] = sx16x2<3>(a, b);
          continue;
        }
        const uint4 a = pr0[slot];
        if (P == 2) {
          const uint4 b = pr1[slot];
          // low half from a, high half from b: one byte permute per register
          sp[4 * k4 + 0] = __byte_perm(a.x, b.x, 0x7610);
          sp[4 * k4 + 1] = __byte_perm(a.y, b.y, 0x7610);
          sp[4 * k4 + 2] = __byte_perm(a.z, b.z, 0x7610);
          sp[4 * k4 + 3] = __byte_perm(a.w, b.w, 0x7610);
        } else {
          sp[4 * k4 + 0] = a.x;
          sp[4 * k4 + 1] = a.y;
          sp[4 * k4 + 2] = a.z;
          sp[4 * k4 + 3] = a.w;
        }
      }
      uint32_t XG[CH];
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        uint32_t f = Ops::addmax(F[c0 + k], GE, HGO[c0 + k]);
        F[c0 + k] = f;
        uint32_t x = LOCAL ? Ops::addmax_relu(diag, sp[k], f) : Ops::addmax(diag, sp[k], f);
        diag = HGO[c0 + k];
        XG[k] = Ops::add(x, GO);
      }
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        HGO[c0 + k] = Ops::addmax(e, GO, XG[k]);
        if (c0 + k + 1 < W) e = Ops::addmax(e, GES, XG[k]);
      }
      xlast = XG[CH - 1];
    }
    e_out = e;
    x_out = xlast;
    if (TRACK) {
#pragma unroll
      for (int k = 0; k + 1 < W; k += 2) acc.best = Ops::max3(acc.best, HGO[k], HGO[k + 1]);
    }
    if (HN && is_last) bnd[i] = make_uint2(e_out, x_out);

    if (LEFTPAD) {
      if (CHECKED) {
        const uint32_t keep = (i < m0 ? Ops::half_mask(0) : 0u) | (i < m1 ? Ops::half_mask(1) : 0u);
        ec = Ops::max2(ec, (HGO[W - 1] & keep) | (NEGLOW & ~keep));
#pragma unroll
        for (int h = 0; h < P; ++h) {
          if (i == (h ? m1 : m0) - 1) {
            const uint32_t hm = Ops::half_mask(h);
            uint32_t v = acc.endrow;
#pragma unroll
            for (int k = 0; k < W; ++k) v = Ops::max2(v, HGO[k]);
            acc.endrow = (acc.endrow & ~hm) | (v & hm);
          }
        }
      } else {
        ec = Ops::max2(ec, HGO[W - 1]);
      }
    } else if (!LOCAL && CHECKED) {
      // last row of a half: the end row and the corner
#pragma unroll
      for (int h = 0; h < P; ++h) {
        const int mh = h ? m1 : m0;
        const int nh = h ? n1 : n0;
        if (i == mh - 1) {
          const uint32_t hm = Ops::half_mask(h);
#pragma unroll
          for (int k = 0; k < W; ++k) {
            const int j = jbase + k;
            if (j < nh) {
              uint32_t v = Ops::max2(acc.endrow, HGO[k]);
              acc.endrow = (acc.endrow & ~hm) | (v & hm);
            }
            if (j == nh - 1) acc.corner = (acc.corner & ~hm) | (HGO[k] & hm);
          }
        }
      }
    }
  }

  template <bool HP, bool HN, bool TRACK>
  __device__ __forceinline__ void run(Acc& acc) {
    const int mmin = P == 2 ? min(m0, m1) : m0;
    const int nsteps = mrows + G - 1;
    const int s0 = min(G - 1, nsteps), s1 = max(s0, mmin - 1);
    int t = 0;
    for (; t < s0; ++t) {
      maybe_refill(t);
      step<true, HP, HN, TRACK>(t, acc);
    }
    while (t < s1) {
      maybe_refill(t);
      const int te = min(s1, (t | (kRingHalf - 1)) + 1);
#pragma unroll 1
      for (; t < te; ++t) step<false, HP, HN, TRACK>(t, acc);
    }
    for (; t < nsteps; ++t) {
      maybe_refill(t);
      step<true, HP, HN, TRACK>(t, acc);
    }
  }
};

// P8 (P = 2): the profile is the pair of int8 tables at prof8 (half 0) and prof8 +
// (ns + 1) * pstride (half 1), pstride counting 32-bit slots; prof is unused.
template <int G, int W, int P, bool LOCAL, bool LEFTPAD, bool P8 = false>
__device__ __forceinline__ void team_pass_fast(const SchemeDev& S, const uint4* __restrict__ prof,
                                               const uint32_t* prof8,
                                               int pstride, uint32_t* ring,
                                               const uint32_t* row_w0, const uint32_t* row_w1,
                                               int row_bits, int row_per, int m0, int m1, int n0,
                                               int n1, int col0, uint2* bnd, bool has_prev,
                                               bool has_next, int lane, unsigned wmask, Acc& acc,
                                               bool last_pass) {
  using Ops = V<P>;
  static_assert(W % 4 == 0, "W must be a multiple of 4");
  static_assert(!P8 || P == 2, "int8 tables hold two halves");
  FastPass<G, W, P, LOCAL, LEFTPAD, P8> fp(S);
  fp.prof_lane = prof + lane;
  fp.p8_lane0 = prof8 + lane;
  fp.p8_lane1 = prof8 + (S.ns + 1) * pstride + lane;
  fp.ring = ring;
  fp.w0 = row_w0;
  fp.w1 = P == 2 ? row_w1 : row_w0;
  fp.bits = row_bits;
  fp.per = row_per;
  fp.pstride = pstride;
  fp.m0 = m0;
  fp.m1 = P == 2 ? m1 : m0;
  fp.mrows = P == 2 ? max(m0, m1) : m0;
  fp.n0 = n0;
  fp.n1 = n1;
  fp.lane = lane;
  fp.wmask = wmask;
  fp.is_l0 = lane == 0;
  fp.is_last = lane == G - 1;
  fp.bnd = bnd;
  fp.GO = Ops::splat(S.go);
  fp.GE = Ops::splat(S.ge);
  fp.GES = Ops::splat(S.ges);
  fp.NEGE0 = Ops::splat(S.neg_e0);
  fp.NEGLOW = Ops::splat(S.neg_low);
  const bool ladder_row0 = !(S.mode == kModeLocal || (S.mode == kModeSemi && S.free_r));
  const bool ladder_col0 = !(S.mode == kModeLocal || (S.mode == kModeSemi && S.free_q));
  fp.jbase = col0 + lane * W;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const int h0 = ladder_row0 ? edge_value(S, false, fp.jbase + k + 1) : 0;
    fp.HGO[k] = Ops::splat(h0 + S.go);
    fp.F[k] = Ops::splat(S.neg_f);
  }
  fp.hgo_left = Ops::splat((ladder_row0 ? edge_value(S, false, fp.jbase) : 0) + S.go);
  fp.e_out = fp.NEGE0;
  fp.x_out = fp.GO;
  fp.xb = Ops::splat((ladder_col0 ? S.go : 0) + S.go);
  fp.xb_step = ladder_col0 ? fp.GE : 0u;
  fp.ec = fp.NEGLOW;
  fp.nb = make_uint2(fp.NEGE0, fp.GO);
  if (has_prev && lane == 0 && fp.mrows > 0) fp.nb = bnd[0];
  __syncwarp(wmask);
  fp.fill(0, kRing + 1 - G);
  __syncwarp(wmask);
  // The running maximum is the local score, and in int16 the overflow guard; it is skipped
  // where no cell can exceed the guard: outside local mode every H is at most
  // min(n, m) * max(substitution score), since boundaries and gaps only subtract.
  const int max_sub = 32767 - S.ovf_limit;
  const bool track = LOCAL || (P == 2 && (long long)min(max(n0, n1), fp.mrows) * max_sub > S.ovf_limit);
  if (track) {
    if (has_prev) {
      if (has_next) fp.template run<true, true, true>(acc);
      else fp.template run<true, false, true>(acc);
    } else {
      if (has_next) fp.template run<false, true, true>(acc);
      else fp.template run<false, false, true>(acc);
    }
  } else {
    if (has_prev) {
      if (has_next) fp.template run<true, true, false>(acc);
      else fp.template run<true, false, false>(acc);
    } else {
      if (has_next) fp.template run<false, true, false>(acc);
      else fp.template run<false, false, false>(acc);
    }
  }
  if (LEFTPAD && last_pass && lane == G - 1) acc.endcol = Ops::max2(acc.endcol, fp.ec);
}

// Final score of half h from the team-reduced accumulators (HGO units: subtract go).
template <int P>
__device__ __forceinline__ int finish_score_leftpad(const SchemeDev& S, const Acc& a, int h, bool* overflow) {
  const int best = V<P>::get(a.best, h) - S.go;
  if (P == 2) *overflow = best > S.ovf_limit;
  const int ec = V<P>::get(a.endcol, h) - S.go, er = V<P>::get(a.endrow, h) - S.go;
  return max(max(ec, er), 0);
}

template <int P>
__device__ __forceinline__ int finish_score(const SchemeDev& S, const Acc& a, int h, bool* overflow) {
  const int best = V<P>::get(a.best, h) - S.go;
  if (P == 2) *overflow = best > S.ovf_limit;
  if (S.mode == kModeLocal) return best;
  const int corner = V<P>::get(a.corner, h) - S.go;
  if (S.mode == kModeGlobal) return corner;
  int res = corner;
  if (S.free_q) res = max(res, V<P>::get(a.endcol, h) - S.go);
  if (S.free_r) res = max(res, V<P>::get(a.endrow, h) - S.go);
  if (S.free_q && S.free_r) res = max(res, 0);
  return res;
}

}  // namespace gsw

namespace gsw {

// Stream bytes: one residue code per byte, bit 7 set on the last row of a sequence;
// kStreamPad pads both ends of every team stream (and stands for "no row").
constexpr int kStreamPadLen = 32;

// Local mode, one column pass over a *stream* of row sequences. The team's rows are
// concatenated; lane L works on stream row g = t - L at step t, reads its own code byte,
// and when a row carries the last-row flag it folds its running max into the sequence's
// partial slot and resets its column state, so the next sequence starts with the row-0
// boundary while lanes to its right still finish the previous one. The skew of G - 1
// steps is paid once per stream instead of once per sequence.
//
// Rows before a lane's first row and after the stream's end read the pad code, whose
// profile row scores every column at s_pad <= 0: from the row-0 state such a row leaves
// H = 0 and F = go, which scores the next real row exactly like F = -inf, so no
// per-step bounds checks are needed.
//
// codes    : stream bytes, codes[-G .. total + G) addressable (pads on both sides).
// part     : shared, part[slot * G + lane] = running max (HGO units) of sequence `slot`;
//            max-merged across column passes.
// bnd      : multi-pass boundary (E, X + go) per stream row, addressable from -G.
template <int G, int W, int P>
__device__ __forceinline__ void team_stream_local(const SchemeDev& S, const uint4* __restrict__ prof,
                                                  int pstride, const int8_t* __restrict__ codes,
                                                  int total, uint2* bnd, bool has_prev,
                                                  bool has_next, int lane, unsigned wmask,
                                                  uint32_t* part) {
  using Ops = V<P>;
  const uint32_t GO = Ops::splat(S.go), GE = Ops::splat(S.ge), GES = Ops::splat(S.ges);
  const uint32_t NEGF = Ops::splat(S.neg_f), NEGE0 = Ops::splat(S.neg_e0);
  uint32_t HGO[W], F[W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    HGO[k] = GO;
    F[k] = NEGF;
  }
  uint32_t hgo_left = GO, best = GO;
  uint32_t e_out = NEGE0, x_out = GO;
  int slot = 0;
  const int8_t* cp = codes - lane;
  int8_t cb_next = cp[0];
  const int nsteps = total + G - 1;
  for (int t = 0; t < nsteps; ++t) {
    const int8_t cb = cb_next;
    cb_next = cp[t + 1];
    uint32_t e_in = __shfl_up_sync(wmask, e_out, 1, G);
    uint32_t x_in = __shfl_up_sync(wmask, x_out, 1, G);
    if (has_prev) {  // uniform across the team
      if (lane == 0) {
        const uint2 b = bnd[t];
        e_in = b.x;
        x_in = b.y;
      }
    } else {  // lane 0's row-0 boundary by selection, no divergent branch
      e_in = lane == 0 ? NEGE0 : e_in;
      x_in = lane == 0 ? GO : x_in;
    }
    const int code = cb & 0x7F;
    const uint4* pr = prof + code * pstride + lane;
    constexpr int CH = (W % 16 == 0) ? 16 : ((W % 8 == 0) ? 8 : 4);
    static_assert(W % CH == 0, "column chunks must tile W");
    uint32_t diag = hgo_left;
    uint32_t e = Ops::addmax(e_in, GES, x_in);
    hgo_left = Ops::addmax(e_in, GO, x_in);
    uint32_t xlast = 0;
#pragma unroll
    for (int c0 = 0; c0 < W; c0 += CH) {
      uint32_t sp[CH];
#pragma unroll
      for (int k4 = 0; k4 < CH / 4; ++k4) {
        const uint4 a = pr[(c0 / 4 + k4) * G];
        sp[4 * k4 + 0] = a.x;
        sp[4 * k4 + 1] = a.y;
        sp[4 * k4 + 2] = a.z;
        sp[4 * k4 + 3] = a.w;
      }
      uint32_t XG[CH];
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const uint32_t f = Ops::addmax(F[c0 + k], GE, HGO[c0 + k]);
        F[c0 + k] = f;
        const uint32_t x = Ops::addmax_relu(diag, sp[k], f);
        diag = HGO[c0 + k];
        XG[k] = Ops::add(x, GO);
      }
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        HGO[c0 + k] = Ops::addmax(e, GO, XG[k]);
        if (c0 + k + 1 < W) e = Ops::addmax(e, GES, XG[k]);
      }
      xlast = XG[CH - 1];
    }
    e_out = e;
    x_out = xlast;
#pragma unroll
    for (int k = 0; k + 1 < W; k += 2) best = Ops::max3(best, HGO[k], HGO[k + 1]);
    if (has_next && lane == G - 1) bnd[t - (G - 1)] = make_uint2(e_out, x_out);
    if (cb < 0) {  // last row of a sequence: fold the partial max, reset to row 0
      uint32_t* ps = part + slot * G + lane;
      *ps = Ops::max2(*ps, best);
      ++slot;
      best = GO;
      hgo_left = GO;
#pragma unroll
      for (int k = 0; k < W; ++k) {
        HGO[k] = GO;
        F[k] = NEGF;
      }
    }
  }
}

}  // namespace gsw
