// Kernels of the scoring engine: the cross-product kernel (one column pair per CTA work
// item, profile shared by the CTA), the pairs kernel (one pair of pairs per team, any
// length through column passes), the per-query top-k and the residue packer.
#pragma once
#include "dp_core.cuh"

namespace gsw {

// A scored cell the int16 run could not represent; rescored by the int32 pairs kernel.
struct Ovf {
  int q, r;          // column (query) and row (reference) sequence
  long long pos;     // output position
};

__device__ __forceinline__ void push_overflow(Ovf* list, int* count, int cap, int q, int r,
                                              long long pos) {
  int slot = atomicAdd(count, 1);
  if (slot < cap) list[slot] = Ovf{q, r, pos};
}

// Fill the profile of one column pass: nprow rows (codes 0..ns-1 plus the pad row),
// uint4 slot u = k4 * G + L of row a holds columns L*W + 4*k4 .. +3 (pass-relative),
// s' = SUB[a][code] - go, or s_pad - go past a column's end / on the pad row.
// Threads [tid0, tid0 + nthreads) of the caller cooperate.
template <int G, int W, int P>
__device__ __forceinline__ void build_profile(const SchemeDev& S, const int* __restrict__ sub,
                                              const Packed& cols, int c0, int n0, int c1,
                                              int n1, int col0, uint4* prof, int pstride,
                                              int tid, int nthreads) {
  constexpr int SLOTS = G * W / 4;
  const int nprow = S.ns + 1;
  const int pad = S.s_pad - S.go;
  for (int idx = tid; idx < nprow * SLOTS; idx += nthreads) {
    const int a = idx / SLOTS, u = idx - a * SLOTS;
    const int L = u % G, k4 = u / G;
    const int jb = col0 + L * W + 4 * k4;
    uint32_t v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int j = jb + e;
      int lo = pad, hi = pad;
      if (a < S.ns) {
        if (c0 >= 0 && j < n0) lo = __ldg(sub + a * S.ns + cols.code(c0, j)) - S.go;
        if (P == 2 && c1 >= 0 && j < n1) hi = __ldg(sub + a * S.ns + cols.code(c1, j)) - S.go;
      }
      v[e] = V<P>::pack(lo, hi);
    }
    prof[a * pstride + u] = make_uint4(v[0], v[1], v[2], v[3]);
  }
}

template <int P>
__device__ __forceinline__ Acc init_acc(const SchemeDev& S) {
  Acc a;
  a.best = V<P>::splat(S.mode == kModeLocal ? S.go : S.neg_low);
  a.endrow = a.corner = a.endcol = V<P>::splat(S.neg_low);
  return a;
}

template <int G, int P>
__device__ __forceinline__ Acc reduce_acc(const SchemeDev& S, Acc a, unsigned wmask) {
  a.best = team_max<G, P>(a.best, wmask);
  if (S.mode != kModeLocal) {
    a.endrow = team_max<G, P>(a.endrow, wmask);
    a.corner = team_max<G, P>(a.corner, wmask);
    a.endcol = team_max<G, P>(a.endcol, wmask);
  }
  return a;
}

// -------------------------------------------------------------------------------------
// Pairs: work item = P alignments (one per register half), each with its own column and
// row sequence. The team builds its own profile for every column pass; passes hand the
// boundary column over through a per-team scratch strip in global memory.
struct PairsParams {
  SchemeDev S;
  const int* sub;
  Packed cols, rows;
  // Item sources (exactly one is used):
  //  explicit: alignment a of item t is order[t * P + a] -> (qi, rj, pos = index)
  //  overflow: alignment t is ovf[t] (P == 1), n_items = min(*ovf_count, ovf_cap)
  //  cross:    item t = (pair t / n_rows, row_perm[t % n_rows]) with pairs/pair_out
  const int* qi;
  const int* rj;
  const int* order;
  long long n_align;         // explicit mode: number of alignments
  const Ovf* ovf_in;
  const int* ovf_in_count;
  int ovf_in_cap;
  int* ovf_flag;             // overflow mode: max of the input counts seen in a call
  const int2* pairs;
  const int2* pair_out;
  const int* row_perm;
  int n_rows;
  long long out_ld;
  long long n_items;         // explicit / cross
  int item_mode;             // 0 explicit, 1 overflow, 2 cross
  unsigned long long* queue; // work counter, zero at launch
  int* out;
  uint2* bnd;                // per-team boundary strips
  int bnd_cap;               // rows per strip
  Ovf* ovf;                  // int16 overflow output
  int* ovf_count;
  int ovf_cap;
  int* out_i;                // LOCATE: row (reference) index of the best cell, or -1
  int* out_j;                // LOCATE: column (query) index of the best cell, or -1
};

template <int P>
struct PairItem {
  int q[P], r[P];
  long long pos[P];
  bool valid[P];
};

template <int P>
__device__ __forceinline__ PairItem<P> decode_item(const PairsParams& p, long long t) {
  PairItem<P> it;
#pragma unroll
  for (int a = 0; a < P; ++a) {
    it.valid[a] = false;
    it.q[a] = it.r[a] = -1;
    it.pos[a] = -1;
    if (p.item_mode == 0) {
      const long long k = t * P + a;
      if (k < p.n_align) {
        const int idx = p.order ? p.order[k] : (int)k;
        it.q[a] = p.qi[idx];
        it.r[a] = p.rj[idx];
        it.pos[a] = idx;
        it.valid[a] = true;
      }
    } else if (p.item_mode == 1) {
      const Ovf o = p.ovf_in[t];
      it.q[a] = o.q;
      it.r[a] = o.r;
      it.pos[a] = o.pos;
      it.valid[a] = true;
    } else {
      const int pi = (int)(t / p.n_rows);
      const int rs = p.row_perm[t % p.n_rows];
      const int2 pr = p.pairs[pi], po = p.pair_out[pi];
      const int c = a ? pr.y : pr.x;
      if (c >= 0) {
        it.q[a] = c;
        it.r[a] = rs;
        it.pos[a] = (long long)(a ? po.y : po.x) * p.out_ld + rs;
        it.valid[a] = true;
      }
    }
  }
  return it;
}

constexpr int kSubSmemMax = 64;  // substitution tables up to 64 x 64 are staged in shared memory

// Dynamic shared memory of the pairs kernel: the substitution table (when ns <= 64, in
// whole uint4) followed by one profile per team.
__host__ __device__ __forceinline__ int pairs_sub_uint4(int ns) {
  return ns <= kSubSmemMax ? (ns * ns + 3) / 4 : 0;
}

// P8: after the substitution table, the int8 profile value of every (column class, row
// code) -- classes 0..ns-1 are residue codes, ns a dummy column left of a left-padded
// sequence, ns+1 a column past a sequence's end -- as `pairs_ext_stride(ns)` bytes per class
// (the ns + 1 row codes, padded to whole 32-bit words), so that a lane fetches four row
// values of a column with one 32-bit load.
__host__ __device__ __forceinline__ int pairs_ext_stride(int ns) { return (ns + 1 + 3) & ~3; }
__host__ __device__ __forceinline__ int pairs_ext_uint4(int ns) {
  return ((ns + 2) * pairs_ext_stride(ns) + 15) / 16;
}

// At most 256 threads per block; one resident block is enough for the register budget, so
// the compiler keeps every W-column state in registers (no spills in any instantiation).
//
// P8 (P = 2, the branch-free pass only): the query profile is held as two int8 tables, half
// the shared memory of the s16x2 table, and registers are capped at 128 (two 256-thread
// blocks), so that more teams stay resident per SM.
template <int G, int W, int P, bool LOCAL, bool LEFTPAD, bool LOCATE = false, bool P8 = false>
__global__ void __launch_bounds__(256, P8 ? 2 : 1) pairs_kernel(const PairsParams p) {
  extern __shared__ uint4 smem_prof[];
  constexpr int SLOTS = G * W / 4;
  const int pstride = (SLOTS + 7) & ~7;
  const int team = threadIdx.x / G, lane = threadIdx.x % G, nteams = blockDim.x / G;
  const unsigned wmask = (G == 32) ? 0xFFFFFFFFu
                                   : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
  const int ns = p.S.ns;
  const int sub_u4 = pairs_sub_uint4(ns);
  const int ext_u4 = P8 ? pairs_ext_uint4(ns) : 0;
  const int* sub = p.sub;
  if (sub_u4 > 0) {
    int* s_sub = reinterpret_cast<int*>(smem_prof);
    for (int i = threadIdx.x; i < ns * ns; i += blockDim.x) s_sub[i] = p.sub[i];
    sub = s_sub;
  }
  const uint32_t* ext = reinterpret_cast<const uint32_t*>(smem_prof + sub_u4);
  if (P8) {
    uint8_t* e8 = reinterpret_cast<uint8_t*>(smem_prof + sub_u4);
    const int stride = pairs_ext_stride(ns), pad_s = p.S.s_pad - p.S.go, zero_s = -p.S.go;
    for (int i = threadIdx.x; i < (ns + 2) * stride; i += blockDim.x) {
      const int cls = i / stride, a = i % stride;
      int v = pad_s;
      if (a < ns && cls < ns) v = p.sub[a * ns + cls] - p.S.go;
      else if (a < ns && cls == ns) v = zero_s;
      e8[i] = (uint8_t)(v & 0xFF);
    }
  }
  if (sub_u4 > 0 || P8) __syncthreads();
  // per team: its profile (s16x2 table, or the two int8 tables), then its row-code ring
  const size_t team_u4 = (P8 ? (size_t)(ns + 1) * pstride / 2 : (size_t)(ns + 1) * pstride) + kRing / 4;
  uint4* prof = smem_prof + sub_u4 + ext_u4 + (size_t)team * team_u4;
  uint32_t* prof8 = reinterpret_cast<uint32_t*>(prof);
  uint32_t* ring = reinterpret_cast<uint32_t*>(prof + team_u4 - kRing / 4);
  uint2* bnd = p.bnd ? p.bnd + ((size_t)blockIdx.x * nteams + team) * p.bnd_cap : nullptr;
  // the branch-free pass covers every mode but the unpadded free-query-end semiglobal one
  const bool fast = LOCAL || LEFTPAD || !(p.S.mode == kModeSemi && p.S.free_q);
  long long n_items = p.n_items;
  if (p.item_mode == 1) {
    n_items = min(*p.ovf_in_count, p.ovf_in_cap);
    if (blockIdx.x == 0 && threadIdx.x == 0 && p.ovf_flag) atomicMax(p.ovf_flag, *p.ovf_in_count);
  }
  // The next work item is taken from the queue and decoded (order -> pair indices) at the
  // top of the current one, so that chain of dependent global loads completes while this item
  // is scored instead of stalling the team between items (10^6 read/window pairs: +6.5 %).
  unsigned long long tq = 0;
  if (lane == 0) tq = atomicAdd(p.queue, 1ull);
  long long t_next = (long long)__shfl_sync(wmask, tq, 0, G);
  PairItem<P> it_next{};
  if (t_next < n_items) it_next = decode_item<P>(p, t_next);
  for (;;) {
    const long long t = t_next;
    if (t >= n_items) break;
    const PairItem<P> it = it_next;
    if (lane == 0) tq = atomicAdd(p.queue, 1ull);
    t_next = (long long)__shfl_sync(wmask, tq, 0, G);
    if (t_next < n_items) it_next = decode_item<P>(p, t_next);
    int n[P], m[P];
#pragma unroll
    for (int a = 0; a < P; ++a) {
      n[a] = it.valid[a] ? p.cols.len[it.q[a]] : 0;
      m[a] = it.valid[a] ? p.rows.len[it.r[a]] : 0;
    }
    const int n0 = n[0], m0 = m[0];
    const int n1 = P == 2 ? n[1] : 0, m1 = P == 2 ? m[1] : 0;
    const int ncols = max(n0, n1), mrows = max(m0, m1);
    Acc acc = init_acc<P>(p.S);
    if (ncols > 0 && mrows > 0) {
      const int npass = (ncols + G * W - 1) / (G * W);
      const int span = npass * G * W;
      const int pad0 = LEFTPAD ? span - n0 : 0, pad1 = LEFTPAD ? span - n1 : 0;
      const uint32_t* w0 = p.rows.words + p.rows.woff[max(it.r[0], 0)];
      const uint32_t* w1 = (P == 2 && it.r[P - 1] >= 0) ? p.rows.words + p.rows.woff[it.r[P - 1]] : w0;
      for (int ps = 0; ps < npass; ++ps) {
        if constexpr (P8) {
          build_profile_lane8<G, W>(p.S, ext, p.cols, it.valid[0] ? it.q[0] : -1, n0, pad0,
                                    it.valid[P - 1] ? it.q[P - 1] : -1, n1, pad1, ps * G * W,
                                    prof8, prof8 + (ns + 1) * pstride, pstride, lane);
          team_pass_fast<G, W, P, LOCAL, LEFTPAD, true>(p.S, prof, prof8, pstride, ring, w0, w1,
                                                        p.rows.bits, p.rows.per, m0, m1,
                                                        LEFTPAD ? span : n0, LEFTPAD ? span : n1,
                                                        ps * G * W, bnd, ps > 0, ps + 1 < npass,
                                                        lane, wmask, acc, ps + 1 == npass);
          __syncwarp(wmask);
          continue;
        }
        build_profile_lane<G, W, P>(p.S, sub, p.cols, it.valid[0] ? it.q[0] : -1, n0, pad0,
                                    (P == 2 && it.valid[P - 1]) ? it.q[P - 1] : -1, n1, pad1,
                                    ps * G * W, prof, pstride, lane);
        if constexpr (!LOCATE) {
          if (fast) {
            team_pass_fast<G, W, P, LOCAL, LEFTPAD>(p.S, prof, prof8, pstride, ring, w0, w1, p.rows.bits,
                                                    p.rows.per, m0, P == 2 ? m1 : m0,
                                                    LEFTPAD ? span : n0, LEFTPAD ? span : n1,
                                                    ps * G * W, bnd, ps > 0, ps + 1 < npass, lane,
                                                    wmask, acc, ps + 1 == npass);
            __syncwarp(wmask);
            continue;
          }
        }
        team_pass<G, W, P, LOCAL, true, LEFTPAD, RowFeed, LOCATE>(p.S, prof, pstride, w0, w1, p.rows.bits,
                                                 p.rows.per, m0, P == 2 ? m1 : m0,
                                                 LEFTPAD ? span : n0, LEFTPAD ? span : n1,
                                                 ps * G * W, bnd, ps > 0, ps + 1 < npass, lane,
                                                 wmask, acc, ps + 1 == npass);
        __syncwarp(wmask);
      }
      if (LOCATE) team_argmax<G>(acc, wmask);
      else acc = reduce_acc<G, P>(p.S, acc, wmask);
    }
    if (LOCATE) {  // P == 1: the maximum over all cells and its first cell, row-major
      if (lane == 0 && it.valid[0]) {
        const bool cells = n[0] > 0 && m[0] > 0;
        const int best = cells ? (int)acc.best - p.S.go : 0;
        const bool hit = cells && (!LOCAL || best > 0);
        p.out[it.pos[0]] = best;
        p.out_i[it.pos[0]] = hit ? acc.bi : -1;
        p.out_j[it.pos[0]] = hit ? acc.bj : -1;
      }
      continue;
    }
    if (lane == 0) {
#pragma unroll
      for (int a = 0; a < P; ++a) {
        if (!it.valid[a]) continue;
        bool ovf = false;
        int score;
        if (n[a] == 0 || m[a] == 0) score = empty_score(p.S, n[a], m[a]);
        else if (LEFTPAD) score = finish_score_leftpad<P>(p.S, acc, a, &ovf);
        else score = finish_score<P>(p.S, acc, a, &ovf);
        if (P == 2 && ovf && n[a] > 0 && m[a] > 0) {
          push_overflow(p.ovf, p.ovf_count, p.ovf_cap, it.q[a], it.r[a], it.pos[a]);
          score = INT_MIN;
        }
        p.out[it.pos[a]] = score;
      }
    }
  }
}

// -------------------------------------------------------------------------------------
// Per-row top-k of an int32 score matrix in the order (score descending, index ascending):
// key = (score with its sign bit flipped) << 32 | ~index, so a larger key ranks first and
// no two keys tie. Each round keeps, per thread, the best 32 keys below the previous
// round's last key, then merges them warp by warp; ceil(k / 32) rounds.
constexpr int kTopkPer = 32;

__device__ __forceinline__ unsigned long long topk_key(int score, int idx) {
  return ((unsigned long long)((unsigned)score ^ 0x80000000u) << 32) | (unsigned)(~idx);
}

__global__ void __launch_bounds__(256) topk_kernel(const int* __restrict__ scores, long long ld,
                                                   int ncols, int k, int* out_idx,
                                                   int* out_score, long long out_ld) {
  __shared__ unsigned long long s_keys[8][kTopkPer];
  __shared__ unsigned long long s_last;
  const int row = blockIdx.x;
  const int* srow = scores + (long long)row * ld;
  const int warp = threadIdx.x / 32, ln = threadIdx.x % 32, nw = blockDim.x / 32;
  const int kk = min(k, ncols);
  unsigned long long bound = ~0ull;  // keys must be strictly below this
  int done = 0;
  while (done < kk) {
    const int want = min(kTopkPer, kk - done);
    unsigned long long lst[kTopkPer];
#pragma unroll
    for (int s = 0; s < kTopkPer; ++s) lst[s] = 0ull;
    for (int j = threadIdx.x; j < ncols; j += blockDim.x) {
      const unsigned long long key = topk_key(srow[j], j);
      if (key >= bound || key <= lst[kTopkPer - 1]) continue;
      // insert into the descending list
      unsigned long long cur = key;
#pragma unroll
      for (int s = 0; s < kTopkPer; ++s) {
        const unsigned long long hi = cur > lst[s] ? cur : lst[s];
        cur = cur > lst[s] ? lst[s] : cur;
        lst[s] = hi;
      }
    }
    // warp merge: `want` rounds of arg-max over the lanes' list heads
    int head = 0;
    for (int s = 0; s < want; ++s) {
      unsigned long long mine = head < kTopkPer ? lst[0] : 0ull;
      unsigned long long best = mine;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, best, off);
        best = o > best ? o : best;
      }
      if (ln == 0) s_keys[warp][s] = best;
      if (best != 0ull && mine == best) {  // pop my head
#pragma unroll
        for (int q = 0; q + 1 < kTopkPer; ++q) lst[q] = lst[q + 1];
        lst[kTopkPer - 1] = 0ull;
        ++head;
      }
    }
    __syncthreads();
    // block merge by warp 0 over the nw sorted lists
    if (warp == 0) {
      int pos = 0;  // my list is s_keys[ln] for ln < nw
      for (int s = 0; s < want; ++s) {
        unsigned long long mine = (ln < nw && pos < want) ? s_keys[ln][pos] : 0ull;
        unsigned long long best = mine;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, best, off);
          best = o > best ? o : best;
        }
        if (best != 0ull && mine == best) ++pos;
        if (ln == 0) {
          const int idx = (int)(~(unsigned)(best & 0xFFFFFFFFull));
          const int sc = (int)((unsigned)(best >> 32) ^ 0x80000000u);
          out_idx[(long long)row * out_ld + done + s] = idx;
          out_score[(long long)row * out_ld + done + s] = sc;
          if (s == want - 1) s_last = best;
        }
      }
    }
    __syncthreads();
    bound = s_last;
    done += want;
    __syncthreads();
  }
}


// Per-row top-k for k <= 32 by threshold and filter, one CTA (256 threads) per row:
//  1. each thread takes the largest score of its strided part of the row; the k-th largest of
//     these 256 maxima, T, is a lower bound of the row's k-th score (the k threads holding
//     the larger maxima hold k distinct scores >= T);
//  2. a second pass over the row (now mostly in L2) appends every (score >= T, index) to a
//     shared candidate list -- it holds the whole top-k, since every top-k score is >= T;
//  3. the candidates are ranked by (score desc, index asc), each by counting the candidates
//     that beat it, and the first k written.
// A row with more than kTopkCand candidates (massive ties at T) falls back to k rounds of
// block-wide arg-max over the whole row. Same keys, same order as topk_kernel.
constexpr int kTopkCand = 2048;

__device__ __forceinline__ int topk_kth_of_block(int v, int k, int* s_tmp) {
  // k-th largest of the 256 values v (one per thread): each thread counts how many values
  // beat its own (ties broken by thread index) and the one with rank k - 1 publishes it
  const int t = threadIdx.x;
  s_tmp[t] = v;
  __syncthreads();
  int rank = 0;
  for (int i = 0; i < 256; ++i) {
    const int o = s_tmp[i];
    rank += (o > v) || (o == v && i < t);
  }
  __syncthreads();
  if (rank == k - 1) s_tmp[256] = v;
  __syncthreads();
  return s_tmp[256];
}

__global__ void __launch_bounds__(256) topk_filter_kernel(const int* __restrict__ scores, long long ld,
                                                          int ncols, int k, int* out_idx,
                                                          int* out_score, long long out_ld) {
  __shared__ int s_tmp[257];
  __shared__ int s_n;
  __shared__ int s_sc[kTopkCand];
  __shared__ int s_ix[kTopkCand];
  const int row = blockIdx.x;
  const int* srow = scores + (long long)row * ld;
  const int kk = min(k, ncols);
  const bool vec = (ld & 3) == 0;
  const int n4 = vec ? ncols / 4 : 0;
  // pass 1: per-thread maximum
  int m = INT_MIN;
  for (int q = threadIdx.x; q < n4; q += 256) {
    const int4 x = __ldg(reinterpret_cast<const int4*>(srow) + q);
    m = max(m, max(max(x.x, x.y), max(x.z, x.w)));
  }
  for (int j = 4 * n4 + threadIdx.x; j < ncols; j += 256) m = max(m, __ldg(srow + j));
  // threads without elements hold INT_MIN, which never raises T above a real score
  const int T = topk_kth_of_block(m, min(kk, 256), s_tmp);
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  // pass 2: candidates >= T
  auto add = [&](int sc, int j) {
    if (sc < T) return;
    const int p = atomicAdd(&s_n, 1);
    if (p < kTopkCand) {
      s_sc[p] = sc;
      s_ix[p] = j;
    }
  };
  for (int q = threadIdx.x; q < n4; q += 256) {
    const int4 x = __ldg(reinterpret_cast<const int4*>(srow) + q);
    if (max(max(x.x, x.y), max(x.z, x.w)) < T) continue;
    add(x.x, 4 * q);
    add(x.y, 4 * q + 1);
    add(x.z, 4 * q + 2);
    add(x.w, 4 * q + 3);
  }
  for (int j = 4 * n4 + threadIdx.x; j < ncols; j += 256) add(__ldg(srow + j), j);
  __syncthreads();
  const int nc = s_n;
  if (nc <= kTopkCand) {
    // 3: rank every candidate among the candidates; ranks < kk are the output positions
    for (int c = threadIdx.x; c < nc; c += 256) {
      const int sc = s_sc[c], ix = s_ix[c];
      int rank = 0;
      for (int o = 0; o < nc && rank < kk; ++o) {
        const int so = s_sc[o];
        rank += (so > sc) || (so == sc && s_ix[o] < ix);
      }
      if (rank < kk) {
        out_idx[(long long)row * out_ld + rank] = ix;
        out_score[(long long)row * out_ld + rank] = sc;
      }
    }
    return;
  }
  // too many ties at T: kk rounds of block-wide arg-max over the row, each below the last
  // round's key (few registers; only rows with massive ties come here)
  unsigned long long bound = ~0ull;
  for (int s = 0; s < kk; ++s) {
    unsigned long long best = 0ull;
    for (int j = threadIdx.x; j < ncols; j += 256) {
      const unsigned long long key = topk_key(__ldg(srow + j), j);
      if (key < bound && key > best) best = key;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, best, off);
      best = o > best ? o : best;
    }
    __shared__ unsigned long long s_best[8];
    if ((threadIdx.x & 31) == 0) s_best[threadIdx.x / 32] = best;
    __syncthreads();
    best = s_best[0];
#pragma unroll
    for (int w = 1; w < 8; ++w) best = s_best[w] > best ? s_best[w] : best;
    if (threadIdx.x == 0) {
      out_idx[(long long)row * out_ld + s] = (int)(~(unsigned)(best & 0xFFFFFFFFull));
      out_score[(long long)row * out_ld + s] = (int)((unsigned)(best >> 32) ^ 0x80000000u);
    }
    bound = best;
    __syncthreads();
  }
}

// -------------------------------------------------------------------------------------
// Local-mode cross product over row *streams*: rows (sorted longest first) are grouped
// in streams of kStreamRows; a work item is (column pair, chunk of nteams streams); each
// team of the CTA scores one stream for every column pass of the pair.
constexpr int kStreamRows = 8;

struct StreamParams {
  SchemeDev S;
  const int* sub;
  Packed cols;
  const int* row_len;         // length of each reference
  const int* row_perm;        // stream order of the references (stream s = rows s*8 .. s*8+7)
  int n_rows;
  const int8_t* stream;       // stream bytes
  const long long* stream_off;  // first code byte of each stream
  const int* stream_total;    // rows (residues) in each stream
  int n_streams;
  const int2* pairs;
  const int2* pair_out;
  const int2* items;          // (pair, chunk)
  int n_items;
  int* queue;
  int* out;
  long long out_ld;
  Ovf* ovf;
  int* ovf_count;
  int ovf_cap;
  uint2* bnd;                 // multi-pass boundary strips, one per (CTA, team)
  long long bnd_strip;        // entries per strip (max stream total + 2 pads)
};

// One work item of the streaming kernel: (column pair, chunk of nteams streams), every column
// pass of the pair scored by the CTA's teams, one stream each, and the stream's scores written.
// bnd_teams: boundary strips reserved per CTA (the CTA's teams, or the most any shape has).
template <int G, int W, int P>
__device__ __forceinline__ void stream_item(const StreamParams& p, const int2 item, uint4* smem_prof,
                                            uint32_t* s_part, int bnd_teams) {
  constexpr int SLOTS = G * W / 4;
  const int pstride = (SLOTS + 7) & ~7;
  const int team = threadIdx.x / G, lane = threadIdx.x % G, nteams = blockDim.x / G;
  const unsigned wmask = (G == 32) ? 0xFFFFFFFFu
                                   : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
  uint32_t* part = s_part + team * kStreamRows * G;
  uint2* bnd = p.bnd ? p.bnd + ((long long)blockIdx.x * bnd_teams + team) * p.bnd_strip + kStreamPadLen
                     : nullptr;
  const uint32_t GO = V<P>::splat(p.S.go);
  const int2 pr = p.pairs[item.x], po = p.pair_out[item.x];
  const int n0 = pr.x >= 0 ? p.cols.len[pr.x] : 0;
  const int n1 = (P == 2 && pr.y >= 0) ? p.cols.len[pr.y] : 0;
  const int ncols = max(max(n0, n1), 1);
  const int npass = (ncols + G * W - 1) / (G * W);
  const int s = item.y * nteams + team;
  const bool have = s < p.n_streams;
  const int total = have ? p.stream_total[s] : 0;
#pragma unroll
  for (int q = 0; q < kStreamRows; ++q) part[q * G + lane] = GO;
  for (int ps = 0; ps < npass; ++ps) {
    __syncthreads();
    build_profile<G, W, P>(p.S, p.sub, p.cols, pr.x, n0, P == 2 ? pr.y : -1, n1, ps * G * W,
                           smem_prof, pstride, threadIdx.x, blockDim.x);
    __syncthreads();
    if (total > 0)
      team_stream_local<G, W, P>(p.S, smem_prof, pstride, p.stream + p.stream_off[s], total, bnd,
                                 ps > 0, ps + 1 < npass, lane, wmask, part);
  }
  __syncwarp(wmask);
  // lane j < kStreamRows writes the scores of the stream's j-th reference
  if (have && lane < kStreamRows) {
    const int pos = s * kStreamRows + lane;
    if (pos < p.n_rows) {
      const int rs = p.row_perm[pos];
      const int m = p.row_len[rs];
      int slot = 0;
      for (int j = 0; j < lane; ++j)
        if (p.row_len[p.row_perm[s * kStreamRows + j]] > 0) ++slot;
      uint32_t best = GO;
      if (m > 0)
        for (int l = 0; l < G; ++l) best = V<P>::max2(best, part[slot * G + l]);
#pragma unroll
      for (int h = 0; h < P; ++h) {
        const int c = h ? pr.y : pr.x;
        if (c < 0) continue;
        const int nh = h ? n1 : n0;
        const long long opos = (long long)(h ? po.y : po.x) * p.out_ld + rs;
        int score;
        if (m == 0 || nh == 0) {
          score = 0;  // local mode: an empty side scores 0
        } else {
          score = V<P>::get(best, h) - p.S.go;
          if (P == 2 && score > p.S.ovf_limit) {
            push_overflow(p.ovf, p.ovf_count, p.ovf_cap, c, rs, opos);
            score = INT_MIN;
          }
        }
        p.out[opos] = score;
      }
    }
  }
  __syncthreads();
}

// One shape per launch: persistent CTAs take items (pair, chunk) from the launch's queue.
// It keeps its own copy of the item body (stream_item is the same work): calling stream_item
// here changed the register allocation and measured 5.6 % slower on the 16S step (2,434 vs
// 2,304 ms).
template <int G, int W, int P>
__global__ void __launch_bounds__(256) cross_stream_kernel(const StreamParams p) {
  extern __shared__ uint4 smem_prof[];
  __shared__ int s_item;
  __shared__ uint32_t s_part[256 * kStreamRows];
  constexpr int SLOTS = G * W / 4;
  const int pstride = (SLOTS + 7) & ~7;
  const int team = threadIdx.x / G, lane = threadIdx.x % G, nteams = blockDim.x / G;
  const unsigned wmask = (G == 32) ? 0xFFFFFFFFu
                                   : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
  uint32_t* part = s_part + team * kStreamRows * G;
  uint2* bnd = p.bnd ? p.bnd + ((long long)blockIdx.x * nteams + team) * p.bnd_strip + kStreamPadLen
                     : nullptr;
  const uint32_t GO = V<P>::splat(p.S.go);
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(p.queue, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= p.n_items) break;
    const int2 item = p.items[it];
    const int2 pr = p.pairs[item.x], po = p.pair_out[item.x];
    const int n0 = pr.x >= 0 ? p.cols.len[pr.x] : 0;
    const int n1 = (P == 2 && pr.y >= 0) ? p.cols.len[pr.y] : 0;
    const int ncols = max(max(n0, n1), 1);
    const int npass = (ncols + G * W - 1) / (G * W);
    const int s = item.y * nteams + team;
    const bool have = s < p.n_streams;
    const int total = have ? p.stream_total[s] : 0;
#pragma unroll
    for (int q = 0; q < kStreamRows; ++q) part[q * G + lane] = GO;
    for (int ps = 0; ps < npass; ++ps) {
      __syncthreads();
      build_profile<G, W, P>(p.S, p.sub, p.cols, pr.x, n0, P == 2 ? pr.y : -1, n1, ps * G * W,
                             smem_prof, pstride, threadIdx.x, blockDim.x);
      __syncthreads();
      if (total > 0)
        team_stream_local<G, W, P>(p.S, smem_prof, pstride, p.stream + p.stream_off[s], total, bnd,
                                   ps > 0, ps + 1 < npass, lane, wmask, part);
    }
    __syncwarp(wmask);
    // lane j < kStreamRows writes the scores of the stream's j-th reference
    if (have && lane < kStreamRows) {
      const int pos = s * kStreamRows + lane;
      if (pos < p.n_rows) {
        const int rs = p.row_perm[pos];
        const int m = p.row_len[rs];
        int slot = 0;
        for (int j = 0; j < lane; ++j)
          if (p.row_len[p.row_perm[s * kStreamRows + j]] > 0) ++slot;
        uint32_t best = GO;
        if (m > 0)
          for (int l = 0; l < G; ++l) best = V<P>::max2(best, part[slot * G + l]);
#pragma unroll
        for (int h = 0; h < P; ++h) {
          const int c = h ? pr.y : pr.x;
          if (c < 0) continue;
          const int nh = h ? n1 : n0;
          const long long opos = (long long)(h ? po.y : po.x) * p.out_ld + rs;
          int score;
          if (m == 0 || nh == 0) {
            score = 0;  // local mode: an empty side scores 0
          } else {
            score = V<P>::get(best, h) - p.S.go;
            if (P == 2 && score > p.S.ovf_limit) {
              push_overflow(p.ovf, p.ovf_count, p.ovf_cap, c, rs, opos);
              score = INT_MIN;
            }
          }
          p.out[opos] = score;
        }
      }
    }
    __syncthreads();
  }
}

// The streaming kernel's shapes, by index: (index, G, W). The host's shape table and its
// per-shape launches are generated from the same list.
#define GSW_STREAM_SHAPES(X)                                                              \
  X(0, 8, 4) X(1, 8, 8) X(2, 8, 12) X(3, 8, 16) X(4, 8, 24) X(5, 8, 32) X(6, 16, 16)     \
  X(7, 16, 20) X(8, 16, 24) X(9, 16, 32) X(10, 32, 16) X(11, 32, 20) X(12, 32, 24)         \
  X(13, 32, 32) X(14, 8, 20) X(15, 8, 28) X(16, 16, 28) X(17, 32, 28)

// Every shape in one launch (a length-scheduled call): one queue of items across shapes,
// ordered by the host longest first; item.y = chunk | shape << 24. Each CTA switches its team
// layout to the item's shape; the dynamic shared memory holds the largest profile of the call,
// and boundary strips are reserved for 32 teams per CTA (the most any shape has).
template <int P>
__global__ void __launch_bounds__(256) cross_stream_multi_kernel(const StreamParams p) {
  extern __shared__ uint4 smem_prof[];
  __shared__ int s_item;
  __shared__ uint32_t s_part[256 * kStreamRows];
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(p.queue, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= p.n_items) break;
    const int2 raw = p.items[it];
    const int2 item = make_int2(raw.x, raw.y & 0xFFFFFF);
    switch ((unsigned)raw.y >> 24) {
#define GSW_MULTI_CASE(IDX, G_, W_) \
  case IDX: stream_item<G_, W_, P>(p, item, smem_prof, s_part, 32); break;
      GSW_STREAM_SHAPES(GSW_MULTI_CASE)
#undef GSW_MULTI_CASE
      default: break;
    }
  }
}

// Unpack the packed references, in stream order, into stream bytes (bit 7 = last row of
// the reference). One warp per reference; pads are pre-filled by the caller.
__global__ void build_stream_kernel(const Packed rows, const int* __restrict__ order, int n,
                                    const long long* __restrict__ dst, int8_t* __restrict__ out) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) / 32, ln = threadIdx.x % 32;
  if (w >= n) return;
  const int r = order[w];
  const int m = rows.len[r];
  int8_t* o = out + dst[w];
  for (int c = ln; c < m; c += 32) o[c] = (int8_t)(rows.code(r, c) | (c == m - 1 ? 0x80 : 0));
}

// -------------------------------------------------------------------------------------
// Pairs scored from caller-owned device memory with no allocation by the library: the
// reference package's byte codes and int32 offsets are read in place, scoring is int32
// (one alignment per lane, so no int16 overflow list is needed), and the work counter,
// the error word and the boundary strips live in a scratch area whose address the host
// passes in. Indices, lengths and codes are checked here, before any code is used as a
// table row: a bad pair is recorded in the error word and skipped, its output left
// untouched.
struct NoAllocParams {
  SchemeDev S;
  const int* sub;              // ns x ns substitution table in the scratch area
  ByteSeqs cols, rows;
  const int* qi;
  const int* rj;
  int n;
  int* out;
  unsigned long long* queue;   // scratch: work counter (zeroed by the host per call)
  int* err;                    // scratch: [0] = 1 bad index, 2 row longer than a strip,
                               // 3 code >= ns or decreasing offsets; [1] = pair
  uint2* bnd;                  // scratch: boundary strips, one per team
  int bnd_cap;                 // rows per strip (0: single-pass only)
  int max_len;                 // the caller's bound on every sequence length
};

// True on every lane of the team when some code of sequence s is >= ns.
template <int G>
__device__ __forceinline__ bool team_has_bad_code(const ByteSeqs& seqs, int s, int len, int ns,
                                                  int lane, unsigned wmask) {
  const uint8_t* c = seqs.codes + seqs.off[s];
  bool bad = false;
  for (int i = lane; i < len; i += G) bad |= (int)__ldg(c + i) >= ns;
  return __any_sync(wmask, bad) != 0;
}

template <int G, int W, bool LOCAL, bool LEFTPAD>
__global__ void __launch_bounds__(256) pairs_noalloc_kernel(const NoAllocParams p) {
  extern __shared__ uint4 smem_prof[];
  __shared__ int s_sub[kSubSmemMax * kSubSmemMax];
  constexpr int SLOTS = G * W / 4;
  const int pstride = (SLOTS + 7) & ~7;
  const int team = threadIdx.x / G, lane = threadIdx.x % G, nteams = blockDim.x / G;
  const unsigned wmask = (G == 32) ? 0xFFFFFFFFu
                                   : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
  const int ns = p.S.ns;
  for (int i = threadIdx.x; i < ns * ns; i += blockDim.x) s_sub[i] = p.sub[i];
  __syncthreads();
  uint4* prof = smem_prof + (size_t)team * (ns + 1) * pstride;
  uint2* bnd = p.bnd ? p.bnd + ((size_t)blockIdx.x * nteams + team) * p.bnd_cap : nullptr;
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(p.queue, 1ull);
    t = __shfl_sync(wmask, t, 0, G);
    if ((long long)t >= p.n) break;
    const int k = (int)t;
    const int q = p.qi[k], r = p.rj[k];
    if (q < 0 || q >= p.cols.n || r < 0 || r >= p.rows.n) {
      if (lane == 0 && atomicCAS(p.err, 0, 1) == 0) p.err[1] = k;
      continue;
    }
    const int n0 = p.cols.length(q), m0 = p.rows.length(r);
    if (n0 < 0 || m0 < 0) {
      if (lane == 0 && atomicCAS(p.err, 0, 3) == 0) p.err[1] = k;
      continue;
    }
    if (n0 > p.max_len || m0 > p.max_len) {
      if (lane == 0 && atomicCAS(p.err, 0, 2) == 0) p.err[1] = k;
      continue;
    }
    // a code >= ns would index past the profile and the table: check both before use
    if (team_has_bad_code<G>(p.cols, q, n0, ns, lane, wmask) ||
        team_has_bad_code<G>(p.rows, r, m0, ns, lane, wmask)) {
      if (lane == 0 && atomicCAS(p.err, 0, 3) == 0) p.err[1] = k;
      continue;
    }
    Acc acc = init_acc<1>(p.S);
    if (n0 > 0 && m0 > 0) {
      const int npass = (n0 + G * W - 1) / (G * W);
      if (npass > 1 && (bnd == nullptr || m0 > p.bnd_cap)) {
        if (lane == 0 && atomicCAS(p.err, 0, 2) == 0) p.err[1] = k;
        continue;
      }
      const int span = npass * G * W;
      const int pad0 = LEFTPAD ? span - n0 : 0;
      const uint32_t* w0 = reinterpret_cast<const uint32_t*>(p.rows.codes + p.rows.off[r]);
      for (int ps = 0; ps < npass; ++ps) {
        build_profile_lane<G, W, 1, ByteSeqs>(p.S, s_sub, p.cols, q, n0, pad0, -1, 0, 0,
                                              ps * G * W, prof, pstride, lane);
        team_pass<G, W, 1, LOCAL, true, LEFTPAD, RowFeed8>(
            p.S, prof, pstride, w0, w0, 0, 0, m0, m0, LEFTPAD ? span : n0, LEFTPAD ? span : 0,
            ps * G * W, bnd, ps > 0, ps + 1 < npass, lane, wmask, acc, ps + 1 == npass);
        __syncwarp(wmask);
      }
      acc = reduce_acc<G, 1>(p.S, acc, wmask);
    }
    if (lane == 0) {
      bool ovf = false;
      int score;
      if (n0 == 0 || m0 == 0) score = empty_score(p.S, n0, m0);
      else if (LEFTPAD) score = finish_score_leftpad<1>(p.S, acc, 0, &ovf);
      else score = finish_score<1>(p.S, acc, 0, &ovf);
      p.out[k] = score;
    }
  }
}

// -------------------------------------------------------------------------------------
// Inter-sequence pairs kernel: one thread scores two alignments from start to end, as the
// low and high int16 halves of every register -- no team, no shuffles, no wavefront skew.
//
// Columns (query) are scored in strips of up to W held in registers: per column its H + go
// (HGO), its F and a byte-permute selector. The substitution value of a cell is one `prmt`:
// the row's table word of each half (four int8 values s - go, one per column code 0..3, from
// a shared table of ns + 1 words: entry ns is the pad row, 0) indexed by the column's
// selector, whose nibbles pick byte q of the low half's word and byte 4 + q of the high
// half's, each followed by its sign byte. A cell then costs the byte permute, three DPX ops
// (E and F add-max, H max3) and two vadd2 (H + s and H + go). Past a query's end the
// selector nibbles are 8 (the sign of byte 0: s' = 0 or -1, so s <= go <= 0); past a
// reference's end the row uses the pad entry (s' = 0).
//
// A strip boundary -- (HGO, E) of the strip's last column for every row -- goes through a
// per-thread column of `bnd`, entry (row * stride), overwritten in place by the next strip.
//
// Applies when the query set holds only codes 0..3 (2-bit packed) and every s - go of those
// columns fits a signed byte. Both alignments of a thread have the same query length unless
// the scheme is local (ends past a query only lower a local score); references may differ.
// Results follow the reference's recurrence (src/gpusw/reference.py:58-125) exactly as the
// team kernels do: HGO units, captures of the corner, the last column (free query end) and
// the last row (free reference end) per half.
struct InterParams {
  SchemeDev S;
  const int* sub;
  Packed cols, rows;
  const int* qi;
  const int* rj;
  const int2* items;          // (alignment a, alignment b or -1), longest first
  long long n_items;
  unsigned long long* queue;  // items taken 32 at a time per warp, zero at launch
  uint2* bnd;                 // boundary columns, bnd[row * stride + thread]
  long long stride;           // threads of the launch
  int* out;
  Ovf* ovf;
  int* ovf_count;
  int ovf_cap;
};

constexpr int kInterW = 32;       // columns per strip
constexpr int kInterTabMax = 65;  // row table words (ns + 1 <= 65)
constexpr int kInterBlock = 192;  // threads per block: two blocks per SM at up to 170 registers

struct InterItem {
  int n, na, nb, ma, mb, M;
  uint32_t qa, qb;  // first packed word of each query (the host keeps word counts below 2^32)
  uint32_t ra, rb;  // first packed word of each reference
  Acc acc;
};

__device__ __forceinline__ uint32_t prmt_sel(uint32_t lo, uint32_t hi, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(lo), "r"(hi), "r"(sel));
  return d;
}

// One strip of WL4 columns starting at column s0 (0-based; s0 % 16 == 0). dd = WL4 - (real
// columns of the last strip), 0..3, so the query's last column is register WL4 - 1 - dd.
template <int WL4, bool FIRST, bool LAST, bool LOCAL, bool TRACK>
__device__ __forceinline__ void inter_strip(const InterParams& p, const uint32_t* s_tab, uint4* s_q,
                                            InterItem& it, int s0, int dd, uint2* bnd) {
  const SchemeDev& S = p.S;
  const uint32_t GO = V<2>::splat(S.go), GE = V<2>::splat(S.ge), NEGF = V<2>::splat(S.neg_f);
  // column selectors from the 2-bit codes of both queries (two words cover 32 columns), kept
  // in the thread's shared-memory column s_q[g * blockDim.x] (four per uint4) to leave the
  // registers to the strip's HGO and F
  {
    uint32_t Q[WL4];
    const int w0 = s0 >> 4;
    const uint32_t* qw = p.cols.words;
    const uint32_t a0 = it.na > s0 ? __ldg(qw + it.qa + w0) : 0u;
    const uint32_t a1 = (WL4 > 16 && it.na > s0 + 16) ? __ldg(qw + it.qa + w0 + 1) : 0u;
    const uint32_t b0 = it.nb > s0 ? __ldg(qw + it.qb + w0) : 0u;
    const uint32_t b1 = (WL4 > 16 && it.nb > s0 + 16) ? __ldg(qw + it.qb + w0 + 1) : 0u;
#pragma unroll
    for (int k = 0; k < WL4; ++k) {
      const uint32_t ca = ((k < 16 ? a0 >> (2 * k) : a1 >> (2 * (k - 16))) & 3u);
      const uint32_t cb = ((k < 16 ? b0 >> (2 * k) : b1 >> (2 * (k - 16))) & 3u);
      const uint32_t qa = s0 + k < it.na ? ca * 0x11u + 0x80u : 0x88u;
      const uint32_t qb = s0 + k < it.nb ? (cb * 0x11u + 0xC4u) << 8 : 0x8800u;
      Q[k] = qa | qb;
    }
#pragma unroll
    for (int g = 0; g < WL4 / 4; ++g)
      s_q[g * blockDim.x] = make_uint4(Q[4 * g], Q[4 * g + 1], Q[4 * g + 2], Q[4 * g + 3]);
  }
  // row 0: the top boundary H(0, j), F = -inf
  uint32_t Hgo[WL4], F[WL4];
#pragma unroll
  for (int k = 0; k < WL4; ++k) {
    Hgo[k] = V<2>::splat(edge_value(S, S.free_r, s0 + k + 1) + S.go);
    F[k] = NEGF;
  }
  uint32_t dleft = V<2>::splat(edge_value(S, S.free_r, s0) + S.go);  // HGO(i - 1, s0)
  // left boundary of the first strip: H(i, 0) = 0 or the gap ladder, E = -inf
  const bool ladder = !(S.mode == kModeLocal || (S.mode == kModeSemi && S.free_q));
  uint32_t lad = V<2>::splat(ladder ? 2 * S.go : S.go);  // HGO(1, 0)
  // row codes: one packed word per `per` rows for each half; the table words of the next row
  // are fetched while the current row is scored
  const int rbits = p.rows.bits, rper = p.rows.per;
  const uint32_t rmask = (1u << rbits) - 1u;
  const uint32_t* rw = p.rows.words;
  uint32_t wa = it.ma > 0 ? __ldg(rw + it.ra) : 0u, wb = it.mb > 0 ? __ldg(rw + it.rb) : 0u;
  int rpos = 0;
  uint32_t rwa = it.ra, rwb = it.rb;  // word offsets of the current row words
  auto row_tab = [&](int i, uint32_t& ta, uint32_t& tb) {  // table words of row i, then advance
    ta = s_tab[i < it.ma ? (int)(wa & rmask) : S.ns];
    tb = s_tab[i < it.mb ? (int)(wb & rmask) : S.ns];
    wa >>= rbits;
    wb >>= rbits;
    if (++rpos == rper) {
      rpos = 0;
      ++rwa;
      ++rwb;
      wa = i + 1 < it.ma ? __ldg(rw + rwa) : 0u;
      wb = i + 1 < it.mb ? __ldg(rw + rwb) : 0u;
    }
  };
  uint32_t TA = 0, TB = 0;
  if (it.M > 0) row_tab(0, TA, TB);
  uint2* bp = bnd;  // this row's boundary entry
  uint2 nb = make_uint2(0u, 0u);
  if (!FIRST) nb = *bp;
  const uint32_t v_neg = V<2>::splat(S.neg_low);
  const uint32_t GEL = ladder ? GE : 0u;
  // the cells of row i from the row's table words (ta, tb) and left boundary (hl, e)
  auto cells = [&](uint32_t ta, uint32_t tb, uint32_t hl, uint32_t& e) {
    uint32_t d = dleft, hgo_l = hl;
    dleft = hl;
#pragma unroll
    for (int k = 0; k < WL4; ++k) {
      const uint4 q4 = s_q[(k >> 2) * blockDim.x];
      const uint32_t qk = (k & 3) == 0 ? q4.x : (k & 3) == 1 ? q4.y : (k & 3) == 2 ? q4.z : q4.w;
      const uint32_t ds = __vadd2(d, prmt_sel(ta, tb, qk));
      e = __viaddmax_s16x2(e, GE, hgo_l);
      const uint32_t f = __viaddmax_s16x2(F[k], GE, Hgo[k]);
      const uint32_t h = LOCAL ? __vimax3_s16x2_relu(ds, e, f) : __vimax3_s16x2(ds, e, f);
      d = Hgo[k];
      F[k] = f;
      Hgo[k] = __vadd2(h, GO);
      hgo_l = Hgo[k];
      if (TRACK && (k & 1)) it.acc.best = __vimax3_s16x2(it.acc.best, Hgo[k - 1], Hgo[k]);
    }
  };
  auto last_col = [&]() {  // HGO at the query's last column (the last strip only)
    return dd == 0 ? Hgo[WL4 - 1] : dd == 1 ? Hgo[WL4 - 2] : dd == 2 ? Hgo[WL4 - 3] : Hgo[WL4 - 4];
  };
  // Rows before the first capture row, where both halves are live: no branch between rows
  // (the next row words and boundary entry are loaded unconditionally -- the word after a
  // sequence lies in the set's slack or its neighbour, the boundary column holds max m rows),
  // so two rows unrolled give the scheduler two chains of dependent cell updates.
  const int mfast = max(0, min(it.ma, it.mb) - 1);
  int i = 0;
#pragma unroll 2
  for (; i < mfast; ++i) {
    const uint32_t ta = TA, tb = TB;
    TA = s_tab[wa & rmask];  // row i + 1 < min(ma, mb): both halves real
    TB = s_tab[wb & rmask];
    wa >>= rbits;
    wb >>= rbits;
    const bool rl = ++rpos == rper;
    rpos = rl ? 0 : rpos;
    rwa += rl;
    rwb += rl;
    const uint32_t la = __ldg(rw + rwa), lb = __ldg(rw + rwb);
    wa = rl ? la : wa;
    wb = rl ? lb : wb;
    uint32_t hl, e;
    if (FIRST) {
      hl = lad;
      e = NEGF;
      lad = __vadd2(lad, GEL);
    } else {
      hl = nb.x;
      e = nb.y;
      nb = bp[p.stride];
    }
    cells(ta, tb, hl, e);
    if (!LAST) *bp = make_uint2(Hgo[WL4 - 1], e);
    bp += p.stride;
    if (!LOCAL && LAST) it.acc.endcol = __vmaxs2(it.acc.endcol, last_col());
  }
  for (; i < it.M; ++i) {
    const uint32_t ta = TA, tb = TB;
    if (i + 1 < it.M) row_tab(i + 1, TA, TB);
    uint32_t hl, e;
    if (FIRST) {
      hl = lad;
      e = NEGF;
      lad = __vadd2(lad, GEL);
    } else {
      hl = nb.x;
      e = nb.y;
      if (i + 1 < it.M) nb = bp[p.stride];
    }
    cells(ta, tb, hl, e);
    if (!LAST) *bp = make_uint2(Hgo[WL4 - 1], e);
    bp += p.stride;
    if (!LOCAL) {
      if (LAST) {  // H(i, n) of the rows each half has (used for a free query end)
        const uint32_t live = (i < it.ma ? 0x0000FFFFu : 0u) | (i < it.mb ? 0xFFFF0000u : 0u);
        it.acc.endcol = __vmaxs2(it.acc.endcol, (last_col() & live) | (v_neg & ~live));
      }
      if (i == it.ma - 1 || i == it.mb - 1) {  // a half's last row: corner and last-row maximum
        const uint32_t half = (i == it.ma - 1 ? 0x0000FFFFu : 0u) | (i == it.mb - 1 ? 0xFFFF0000u : 0u);
        uint32_t rmax = v_neg;
#pragma unroll
        for (int k = 0; k < WL4; ++k)
          if (!LAST || k < WL4 - 4 || k < WL4 - dd) rmax = __vmaxs2(rmax, Hgo[k]);
        it.acc.endrow = __vmaxs2(it.acc.endrow, (rmax & half) | (v_neg & ~half));
        if (LAST) it.acc.corner = (last_col() & half) | (it.acc.corner & ~half);
      }
    }
  }
}

template <bool FIRST, bool LOCAL, bool TRACK>
__device__ __forceinline__ void inter_last_strip(const InterParams& p, const uint32_t* s_tab, uint4* s_q,
                                                 InterItem& it, int s0, uint2* bnd) {
  const int wl = it.n - s0, wl4 = (wl + 3) & ~3, dd = wl4 - wl;
  switch (wl4 >> 2) {
    case 1: inter_strip<4, FIRST, true, LOCAL, TRACK>(p, s_tab, s_q, it, s0, dd, bnd); break;
    case 2: inter_strip<8, FIRST, true, LOCAL, TRACK>(p, s_tab, s_q, it, s0, dd, bnd); break;
    case 3: inter_strip<12, FIRST, true, LOCAL, TRACK>(p, s_tab, s_q, it, s0, dd, bnd); break;
    case 4: inter_strip<16, FIRST, true, LOCAL, TRACK>(p, s_tab, s_q, it, s0, dd, bnd); break;
    case 5: inter_strip<20, FIRST, true, LOCAL, TRACK>(p, s_tab, s_q, it, s0, dd, bnd); break;
    case 6: inter_strip<24, FIRST, true, LOCAL, TRACK>(p, s_tab, s_q, it, s0, dd, bnd); break;
    case 7: inter_strip<28, FIRST, true, LOCAL, TRACK>(p, s_tab, s_q, it, s0, dd, bnd); break;
    default: inter_strip<32, FIRST, true, LOCAL, TRACK>(p, s_tab, s_q, it, s0, dd, bnd); break;
  }
}

// Persistent: each warp takes 32 consecutive items per queue step (one per lane); the host
// orders items by query length then reference length, longest first, so a warp's lanes run
// strips of the same widths over similar row counts.
//
// 192-thread blocks: the strip's HGO and F (64 registers), two rows in flight and the row
// state take 160-170 registers, spill-free only under a cap above 128; at 256 threads (cap
// 128) the kernel spilled and ran 0-13 % slower.
template <bool LOCAL, bool TRACK>
__global__ void __launch_bounds__(kInterBlock, 2) pairs_inter_kernel(const InterParams p) {
  static_assert(kInterW == 32, "two packed query words per strip");
  __shared__ uint32_t s_tab[kInterTabMax];
  __shared__ uint4 s_qsel[kInterW / 4 * kInterBlock];
  uint4* s_q = s_qsel + threadIdx.x;
  const SchemeDev& S = p.S;
  for (int r = threadIdx.x; r <= S.ns; r += blockDim.x) {
    uint32_t w = 0;
    if (r < S.ns)
      for (int c = 0; c < 4 && c < S.ns; ++c) w |= (uint32_t)((p.sub[r * S.ns + c] - S.go) & 0xFF) << (8 * c);
    s_tab[r] = w;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  uint2* bnd = p.bnd ? p.bnd + (long long)blockIdx.x * blockDim.x + threadIdx.x : nullptr;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(p.queue, 32ull);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if ((long long)base >= p.n_items) break;
    const long long t = (long long)base + lane;
    if (t >= p.n_items) continue;
    const int2 ab = p.items[t];
    const int a = ab.x, b = ab.y >= 0 ? ab.y : ab.x;
    InterItem it;
    const int qa = p.qi[a], ra = p.rj[a], qb = p.qi[b], rb = p.rj[b];
    it.na = p.cols.len[qa];
    it.nb = p.cols.len[qb];
    it.ma = p.rows.len[ra];
    it.mb = p.rows.len[rb];
    it.n = max(it.na, it.nb);
    it.M = max(it.ma, it.mb);
    it.qa = (uint32_t)p.cols.woff[qa];
    it.qb = (uint32_t)p.cols.woff[qb];
    it.ra = (uint32_t)p.rows.woff[ra];
    it.rb = (uint32_t)p.rows.woff[rb];
    it.acc = init_acc<2>(S);
    if (it.n > 0 && it.M > 0) {
      const int nstrip = (it.n + kInterW - 1) / kInterW;
      if (nstrip == 1) {
        inter_last_strip<true, LOCAL, TRACK>(p, s_tab, s_q, it, 0, bnd);
      } else {
        inter_strip<kInterW, true, false, LOCAL, TRACK>(p, s_tab, s_q, it, 0, 0, bnd);
        for (int sx = 1; sx + 1 < nstrip; ++sx)
          inter_strip<kInterW, false, false, LOCAL, TRACK>(p, s_tab, s_q, it, sx * kInterW, 0, bnd);
        inter_last_strip<false, LOCAL, TRACK>(p, s_tab, s_q, it, (nstrip - 1) * kInterW, bnd);
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h == 1 && ab.y < 0) continue;
      const int nh = h ? it.nb : it.na, mh = h ? it.mb : it.ma;
      bool ovf = false;
      int score;
      if (nh == 0 || mh == 0) score = empty_score(S, nh, mh);
      else score = finish_score<2>(S, it.acc, h, &ovf);
      const int al = h ? ab.y : a;
      if (ovf && nh > 0 && mh > 0) {
        push_overflow(p.ovf, p.ovf_count, p.ovf_cap, h ? qb : qa, h ? rb : ra, al);
        score = INT_MIN;
      }
      p.out[al] = score;
    }
  }
}

}  // namespace gsw
