// Host side of the scoring engine: context, resident sequence sets, the length-binned
// launch planner, the int16 -> int32 overflow rescoring and the C ABI of
// include/gpusw_b200.h.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <climits>
#include <condition_variable>
#include <functional>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gpusw_b200.h"
#include "kernels.cuh"

#if defined(__x86_64__) && !defined(__CUDA_ARCH__)
#include <immintrin.h>
#define GSW_X86_PACK 1
#endif

namespace {

using gsw::SchemeDev;

struct Error {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const std::string& msg) { throw Error{code, msg}; }

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      fail(e_ == cudaErrorMemoryAllocation ? GPUSW_ERR_MEMORY : GPUSW_ERR_CUDA,           \
           std::string(#call) + ": " + cudaGetErrorString(e_));                           \
  } while (0)

// Grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int64_t* held = nullptr;
  void* get(size_t need) {
    if (need > bytes) {
      if (p) {
        cudaFree(p);
        if (held) *held -= (int64_t)bytes;
      }
      p = nullptr;
      bytes = 0;
      size_t want = std::max(need, bytes * 2);
      CK(cudaMalloc(&p, want));
      bytes = want;
      if (held) *held += (int64_t)bytes;
    }
    return p;
  }
  template <class T> T* as(size_t n) { return static_cast<T*>(get(std::max<size_t>(1, n) * sizeof(T))); }
  void release() {
    if (p) cudaFree(p);
    if (held && bytes) *held -= (int64_t)bytes;
    p = nullptr;
    bytes = 0;
  }
};

// Allocator whose resize() leaves elements uninitialised, so the pages of a large host
// array are first touched by the threaded loop that fills it rather than by one thread
// zeroing it (for 10^6 sequences that zeroing alone took 1-2 ms per set upload).
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
  template <class U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};

struct Db {
  int n = 0;
  int bits = 2, per = 16, max_code = 0, max_len = 0;
  std::vector<int, NoInitAlloc<int>> len;         // filled by threaded loops in db_upload
  std::vector<long long, NoInitAlloc<long long>> woff;
  std::vector<int> perm_desc;  // sequences by length, longest first (stable)
  void* base = nullptr;        // one allocation: words, then woff_d, then len_d
  uint32_t* words = nullptr;
  long long* woff_d = nullptr;
  int* len_d = nullptr;
  bool order_ready = false;    // perm_desc / perm_d / ident_d built (on first use as rows)
  void* order_base = nullptr;  // one allocation: perm_d, then ident_d
  int* perm_d = nullptr;
  int* ident_d = nullptr;      // identity order (plain form)
  int64_t bytes = 0;
  // stream buffers (bytes + per-stream offsets/totals), keyed by (plain order, pad code)
  struct Stream {
    int8_t* bytes = nullptr;
    long long* off = nullptr;
    int* total = nullptr;
    std::vector<int> total_h;  // host copy of the totals (item costs of a multi-shape launch)
    int n_streams = 0, max_total = 0;
    int64_t nbytes = 0;
  };
  std::vector<std::pair<std::pair<int, int>, Stream>> streams;
  gsw::Packed packed() const {
    gsw::Packed p;
    p.words = words;
    p.woff = woff_d;
    p.len = len_d;
    p.bits = bits;
    p.per = per;
    return p;
  }
};

struct HostScheme {
  int mode = 0, go = 0, ge = 0, free_q = 0, free_r = 0, ns = 0;
  int max_sub = 0, min_sub = 0;
  std::vector<int> sub;
};

// Kernel shapes compiled: team size G and columns per lane W.
struct Shape {
  int G, W;
  int cap() const { return G * W; }
};
// Pairs kernel shapes (explicit pairs, and the cross products of non-local schemes).
const Shape kPairShapes[] = {{8, 8},  {8, 12},  {8, 16},  {8, 20},
                             {8, 24}, {16, 16}, {16, 24}, {32, 16}};
// Local-mode streaming kernel shapes (columns per pass = G * W).
// The last four fill the 160 / 224 / 448 / 896-column gaps of the first fourteen (for
// uneven lengths the planner otherwise pads a query up to the next cap).
const Shape kStreamShapes[] = {{8, 4},   {8, 8},   {8, 12},  {8, 16},  {8, 24},
                               {8, 32},  {16, 16}, {16, 20}, {16, 24}, {16, 32},
                               {32, 16}, {32, 20}, {32, 24}, {32, 32}, {8, 20},
                               {8, 28},  {16, 28}, {32, 28}};
constexpr int kNumStream = sizeof(kStreamShapes) / sizeof(Shape);
constexpr int kNumPair = sizeof(kPairShapes) / sizeof(Shape);
constexpr size_t kSmemCap = 200 * 1024;
constexpr int kOvfCap = 1 << 20;

int pstride_of(const Shape& s) { return ((s.G * s.W / 4) + 7) & ~7; }
size_t profile_bytes(const Shape& s, int ns) { return (size_t)(ns + 1) * pstride_of(s) * 16; }

// Everything one launch sequence touches on the device, plus its stage-timing events.
// The context owns one set for uncached calls; every cached plan owns its own, because a
// captured CUDA graph keeps the raw pointers.
struct Bufs {
  DevBuf meta, queue, ovf, ovf_count, ovf_flag, bnd, out, idx, sc;
  long long inter_items = 0;  // items of the inter-sequence pairs kernel in this launch sequence
  std::vector<cudaEvent_t> pool;
  int pool_used = 0;
  std::vector<std::pair<int, int>> score_marks, topk_marks;
  bool capturing = false;  // recording a graph: no host copies, events as graph nodes
  void set_held(int64_t* h) {
    for (DevBuf* b : {&meta, &queue, &ovf, &ovf_count, &ovf_flag, &bnd, &out, &idx, &sc}) b->held = h;
  }
  void release() {
    for (DevBuf* b : {&meta, &queue, &ovf, &ovf_count, &ovf_flag, &bnd, &out, &idx, &sc}) b->release();
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
    pool.clear();
  }
  void reset_marks() {
    pool_used = 0;
    score_marks.clear();
    topk_marks.clear();
  }
};

// A cached launch plan: the same call (same sets, scheme, width, options and index
// arrays) replays its CUDA graph instead of planning and launching again.
struct Plan {
  std::vector<long long> key;
  Bufs B;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long last_use = 0;
  long long launches = 0;
  ~Plan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    B.release();
  }
};

}  // namespace

constexpr int kAuxStreams = 3;  // extra streams a call's shape launches fan out to

struct gpusw_ctx {
  int device = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t aux[kAuxStreams] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[kAuxStreams] = {};
  std::string err;
  bool has_scheme = false;
  HostScheme sch;
  int* sub_d = nullptr;
  std::unordered_map<int, std::unique_ptr<Db>> dbs;
  int next_db = 1;
  int plain = 0;
  int64_t mem_budget = 4ll << 30;
  int64_t held = 0;
  Bufs shared;
  DevBuf flush;
  uint32_t* pinned = nullptr;  // host staging for set uploads (page-locked, grow-only)
  size_t pinned_words = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  Bufs* last_bufs = nullptr;  // the set whose stage marks the last call used
  std::vector<std::unique_ptr<Plan>> plans;
  std::vector<std::vector<long long>> seen_keys;  // cacheable keys run once, not yet recorded
  unsigned long long use_clock = 0;
  long long scheme_version = 0;
  // gpusw_score_pairs_zip: three pipeline slots (page-locked staging, device image, buffers,
  // completion event); slot 0 runs on `stream`, slots 1 and 2 on aux[0] and aux[1]
  struct ZipSlot {
    char* pinned = nullptr;
    size_t pinned_bytes = 0;
    int32_t* pinned_out = nullptr;
    size_t pinned_out_n = 0;
    DevBuf image;
    Bufs B;
    cudaEvent_t done = nullptr;
    cudaEvent_t tev[4] = {};  // GPUSW_TRACE=1: before/after the image copy, after the kernels and the result copy
  } zip[3];
  DevBuf zip_iota;  // 0, 1, 2, ... (the pair index arrays of a chunk)
  long long zip_iota_n = 0;
  int graphs = 1;              // replay cached plans as CUDA graphs
  int autotune = 1;            // tune stream shapes on first use
  int stream_multi = 0;        // a batched call's streaming shapes in one launch (else one per shape)
  int inter = 1;               // short explicit int16 pairs through the inter-sequence kernel where it pays
  std::vector<std::pair<std::pair<int, int>, std::vector<double>>> tune;  // (ns, P) -> us/row-pass
  gpusw_stats st{};
};

namespace {

thread_local std::string g_create_error;

void set_device(gpusw_ctx* c) { CK(cudaSetDevice(c->device)); }

// ---------------------------------------------------------------------------- scheme
SchemeDev make_scheme(const HostScheme& h, int P) {
  SchemeDev S;
  S.mode = h.mode;
  S.free_q = h.free_q;
  S.free_r = h.free_r;
  S.go = h.go;
  S.ge = h.ge;
  S.ges = std::max(h.ge, h.go);
  S.ns = h.ns;
  S.pad_code = h.ns;
  S.s_pad = std::min(0, h.min_sub);
  const long long lo = P == 2 ? -32768ll : (long long)INT_MIN;
  S.neg_low = (int)lo;
  S.neg_f = (int)(lo - h.ge);
  S.neg_e0 = (int)(lo - h.go);
  S.ovf_limit = P == 2 ? 32767 - std::max(0, h.max_sub) : INT_MAX;
  return S;
}

// Can every value of a DP of at most max_n columns and max_m rows be held in the width?
// For int16 only the lower side is checked here; the upper side is caught at run time.
bool width_ok(const HostScheme& h, int P, long long max_n, long long max_m) {
  const long long lo = P == 2 ? -32768ll : (long long)INT_MIN;
  const long long hi = P == 2 ? 32767ll : (long long)INT_MAX;
  const long long g = std::min(h.go, h.ge);
  const long long smin = std::min(0, h.min_sub);
  const long long ges = std::max(h.ge, h.go);
  const long long hmin = h.mode == gsw::kModeLocal ? 0 : (max_n + max_m) * g;
  const long long lmin = hmin + 2 * g + smin;
  if (lmin < lo + (ges - h.go)) return false;
  if ((long long)h.max_sub - h.go > hi || smin - h.go < lo) return false;
  if (P == 1) {
    const long long hmax = std::min(max_n, max_m) * (long long)std::max(0, h.max_sub);
    if (hmax + std::max(0, h.max_sub) > hi) return false;
  }
  return true;
}

// Host phase timing, printed to stderr when the environment sets GPUSW_TRACE=1. Diagnostics
// only: every phase runs the same with or without it.
struct HostTrace {
  using clk = std::chrono::steady_clock;
  const char* call;
  bool on;
  clk::time_point last;
  explicit HostTrace(const char* name) : call(name), on(enabled()), last(clk::now()) {}
  static bool enabled() {
    static const bool e = [] { const char* v = std::getenv("GPUSW_TRACE"); return v && v[0] == '1'; }();
    return e;
  }
  void lap(const char* phase) {
    if (!on) return;
    const auto now = clk::now();
    std::fprintf(stderr, "[gpusw] %s %s %.3f ms\n", call, phase,
                 std::chrono::duration<double, std::milli>(now - last).count());
    last = now;
  }
};

// ------------------------------------------------------------------------- sequences
int host_threads() { return (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency())); }

// Persistent fork-join workers for the host-side passes (packing, scans, planning), so a call
// does not pay thread creation. One job at a time; a caller that finds the pool busy (another
// context's thread) spawns its own threads instead. Workers are never joined: they sleep on
// the condition variable until the process ends.
class HostPool {
 public:
  static HostPool& get() {
    static HostPool* p = new HostPool();
    return *p;
  }
  // Runs job(t) for t in [0, nt); job(0) on the calling thread. False if the pool is busy.
  bool run(int nt, const std::function<void(int)>& job) {
    std::unique_lock<std::mutex> busy(run_mu_, std::try_to_lock);
    if (!busy.owns_lock()) return false;
    {
      std::lock_guard<std::mutex> g(mu_);
      while ((int)workers_.size() < nt - 1) {
        const int id = (int)workers_.size();
        workers_.emplace_back([this, id] { loop(id); });
        workers_.back().detach();
      }
      job_ = &job;
      active_ = nt - 1;
      pending_ = nt - 1;
      pending_atomic_.store(pending_, std::memory_order_release);
      ++gen_;
    }
    gen_seen_.store(gen_, std::memory_order_release);
    cv_.notify_all();
    job(0);
    // the workers finish within microseconds of each other: spin briefly before sleeping
    for (int spin = 0; spin < kSpin && pending_atomic_.load(std::memory_order_acquire) != 0; ++spin) cpu_relax();
    std::unique_lock<std::mutex> g(mu_);
    done_.wait(g, [&] { return pending_ == 0; });
    job_ = nullptr;
    return true;
  }

 private:
  // Spin iterations (a pause each, ~100 microseconds in all) before a worker or the caller
  // sleeps on its condition variable: a pipelined call runs several short parallel passes in
  // a row, and a futex wake-up of every worker costs as much as a pass.
  static constexpr int kSpin = 20000;
  static void cpu_relax() {
#if defined(__x86_64__) && !defined(__CUDA_ARCH__)
    _mm_pause();
#endif
  }
  void loop(int id) {
    unsigned long long seen = 0;
    for (;;) {
      for (int spin = 0; spin < kSpin && gen_seen_.load(std::memory_order_acquire) == seen; ++spin) cpu_relax();
      const std::function<void(int)>* job;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return gen_ != seen; });
        seen = gen_;
        if (id >= active_) continue;
        job = job_;
      }
      (*job)(id + 1);
      std::lock_guard<std::mutex> g(mu_);
      pending_atomic_.store(--pending_, std::memory_order_release);
      if (pending_ == 0) done_.notify_all();
    }
  }
  std::mutex run_mu_, mu_;
  std::condition_variable cv_, done_;
  std::vector<std::thread> workers_;
  const std::function<void(int)>* job_ = nullptr;
  int active_ = 0, pending_ = 0;
  unsigned long long gen_ = 0;
  std::atomic<unsigned long long> gen_seen_{0};  // gen_, readable without the mutex
  std::atomic<int> pending_atomic_{0};            // pending_, readable without the mutex
};

// Run f(begin, end) over [0, n) split into contiguous ranges on the host's cores (one range
// when n is below `min_n`). The split depends only on n and the core count.
template <class F>
void parallel_ranges_min(long long n, long long min_n, F&& f) {
  const int nt = n < min_n ? 1 : (int)std::min<long long>(host_threads(), n);
  if (nt == 1) {
    f(0ll, n);
    return;
  }
  const std::function<void(int)> job = [&](int t) { f(n * t / nt, n * (t + 1) / nt); };
  if (HostPool::get().run(nt, job)) return;
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) th.emplace_back([&, t] { job(t); });
  for (auto& x : th) x.join();
}

template <class F>
void parallel_ranges(long long n, F&& f) {
  parallel_ranges_min(n, 1 << 16, std::forward<F>(f));
}

// Eight 2-bit codes, one per byte of x (byte e = code e), folded into 16 bits (code e at
// bits 2e..2e+1): neighbouring fields are merged pairwise three times.
inline uint32_t fold2(uint64_t x) {
  x = (x | (x >> 6)) & 0x000F000F000F000Full;
  x = (x | (x >> 12)) & 0x000000FF000000FFull;
  return (uint32_t)((x | (x >> 24)) & 0xFFFFull);
}
// Eight 4-bit codes, one per byte, folded into 32 bits (code e at bits 4e..4e+3).
inline uint32_t fold4(uint64_t x) {
  x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
  x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
  return (uint32_t)(x | (x >> 16));
}

#if GSW_X86_PACK
// SSSE3 packing of sequences [s0, s1) at 2 or 4 bits (the same words as the scalar fold2 /
// fold4 path, checked bit-exact): 16 code bytes become one word at 2 bits (b0 + 4 b1 per byte
// pair by a multiply-add, 16 x that per pair of pairs by a second one, then the low byte of
// each 32-bit lane) or two words at 4 bits (b0 + 16 b1 per byte pair, narrowed to bytes). A
// sequence's last partial block is read by one 16-byte load ending at its last code and moved
// down by a byte shuffle (shorter sequences copy it to a zeroed buffer), so no load leaves the
// sequence. The OR of every code byte goes to *or_out.
__attribute__((target("ssse3"))) inline void fold16_ssse3(__m128i v, int bits, uint32_t* dst) {
  if (bits == 2) {
    const __m128i t = _mm_madd_epi16(_mm_maddubs_epi16(v, _mm_set1_epi16(0x0401)), _mm_set1_epi32(0x00100001));
    const __m128i lanes = _mm_setr_epi8(0, 4, 8, 12, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1);
    dst[0] = (uint32_t)_mm_cvtsi128_si32(_mm_shuffle_epi8(t, lanes));
  } else {
    const __m128i t = _mm_maddubs_epi16(v, _mm_set1_epi16(0x1001));
    const uint64_t x = (uint64_t)_mm_cvtsi128_si64(_mm_packus_epi16(t, t));
    memcpy(dst, &x, 8);
  }
}

__attribute__((target("ssse3"))) void pack_range_ssse3(const uint8_t* codes, const int32_t* offs,
                                                       const int* len_of, const long long* woff,
                                                       int bits, uint32_t* words, int s0, int s1,
                                                       uint8_t* or_out) {
  const int per = 32 / bits;
  const __m128i iota = _mm_setr_epi8(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
  __m128i acc = _mm_setzero_si128();
  const int wpb = 16 / per;  // words per 16-code block: 1 at 2 bits, 2 at 4 bits
  for (int s = s0; s < s1; ++s) {
    const uint8_t* src = codes + offs[s];
    const int len = len_of[s];
    uint32_t* dst = words + woff[s];
    const long long nw = (((long long)len + per - 1) / per + 3) & ~3ll;
    const int full = len / 16, tail = len % 16;
    for (int b = 0; b < full; ++b) {
      const __m128i v = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + 16 * b));
      acc = _mm_or_si128(acc, v);
      fold16_ssse3(v, bits, dst + (long long)b * wpb);
    }
    long long w = (long long)full * wpb;
    if (tail) {
      __m128i v;
      if (len >= 16) {  // bytes [len - 16, len): shift down by 16 - tail, zero the top
        const __m128i x = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + len - 16));
        const __m128i idx = _mm_add_epi8(iota, _mm_set1_epi8((char)(16 - tail)));
        const __m128i keep = _mm_cmplt_epi8(iota, _mm_set1_epi8((char)tail));
        v = _mm_and_si128(_mm_shuffle_epi8(x, idx), keep);
      } else {
        alignas(16) uint8_t t[16] = {};
        memcpy(t, src, (size_t)tail);
        v = _mm_load_si128(reinterpret_cast<const __m128i*>(t));
      }
      acc = _mm_or_si128(acc, v);
      fold16_ssse3(v, bits, dst + w);
      w += wpb;
    }
    for (; w < nw; ++w) dst[w] = 0u;
  }
  alignas(16) uint8_t b[16];
  _mm_store_si128(reinterpret_cast<__m128i*>(b), acc);
  uint8_t o = 0;
  for (int i = 0; i < 16; ++i) o |= b[i];
  *or_out = o;
}

bool host_has_ssse3() {
  static const bool v = __builtin_cpu_supports("ssse3");
  return v;
}
#endif

// Pack sequences [s0, s1) into words (each sequence's words including its alignment
// padding, so the destination needs no prior zeroing). With or_out, the OR of every code
// byte packed is stored there: it has a bit at or above `bits` exactly when some code does
// not fit the width (the words are then wrong and the caller packs again, wider).
void pack_range(const uint8_t* codes, const int32_t* offs, const Db& d, uint32_t* words, int s0, int s1,
                uint8_t* or_out = nullptr) {
  uint8_t orv = 0;
#if GSW_X86_PACK
  if ((d.bits == 2 || d.bits == 4) && host_has_ssse3()) {
    pack_range_ssse3(codes, offs, d.len.data(), d.woff.data(), d.bits, words, s0, s1, &orv);
    if (or_out) *or_out = orv;
    return;
  }
#endif
  for (int s = s0; s < s1; ++s) {
    const uint8_t* src = codes + offs[s];
    const int len = d.len[s];
    uint32_t* dst = words + d.woff[s];
    // every sequence holds exactly this many words (data + 16-byte alignment), so a range
    // never reads the word offset of a sequence outside it (another thread may be writing it)
    const long long nw = (((long long)len + d.per - 1) / d.per + 3) & ~3ll;
    long long w = 0;
    int c = 0;
    // Whole words of 2-, 4- and 8-bit codes: gather 8 code bytes per 64-bit load and fold
    // neighbouring fields together (codes are below 2^bits, so no masking of the input).
    if (d.bits == 2) {
      uint64_t o = 0;
      for (; c + 16 <= len; c += 16, ++w) {
        uint64_t a, b;
        memcpy(&a, src + c, 8);
        memcpy(&b, src + c + 8, 8);
        o |= a | b;
        dst[w] = fold2(a) | (fold2(b) << 16);
      }
      for (int i = 0; i < 8; ++i) orv |= (uint8_t)(o >> (8 * i));
    } else if (d.bits == 4) {
      uint64_t o = 0;
      for (; c + 8 <= len; c += 8, ++w) {
        uint64_t a;
        memcpy(&a, src + c, 8);
        o |= a;
        dst[w] = fold4(a);
      }
      for (int i = 0; i < 8; ++i) orv |= (uint8_t)(o >> (8 * i));
    } else if (d.bits == 8) {
      for (; c + 4 <= len; c += 4, ++w) memcpy(dst + w, src + c, 4);
    }
    for (; w < nw; ++w) {
      uint32_t v = 0;
      for (int e = 0; e < d.per && c < len; ++e, ++c) {
        orv |= src[c];
        v |= (uint32_t)src[c] << (e * d.bits);
      }
      dst[w] = v;
    }
  }
  if (or_out) *or_out = orv;
}

Db& get_db(gpusw_ctx* c, int32_t h) {
  auto it = c->dbs.find(h);
  if (it == c->dbs.end()) fail(GPUSW_ERR_NOT_FOUND, "unknown sequence-set handle " + std::to_string(h));
  return *it->second;
}

void require_scheme(gpusw_ctx* c, const Db& a, const Db& b) {
  if (!c->has_scheme) fail(GPUSW_ERR_SCHEME, "no scheme set (call gpusw_set_scheme first)");
  if (a.max_code >= c->sch.ns || b.max_code >= c->sch.ns)
    fail(GPUSW_ERR_INVALID, "sequence codes exceed the scheme's substitution table");
}

// -------------------------------------------------------------------------- launches
// Where one launch goes. Launches of a call that may run concurrently (run_group) get a
// stream each and disjoint boundary strips, sized by a first pass that launches nothing.
struct LaunchCfg {
  cudaStream_t st = nullptr;  // nullptr: the context stream
  long long bnd_off = -1;     // >= 0: boundary strips at B.bnd + bnd_off (sized beforehand)
  size_t* need = nullptr;     // sizing pass: store the strip entries needed, launch nothing
};

// Teams per CTA of the pairs kernel: each team holds its own profile.
int pair_teams(const Shape& s, int ns) {
  const int t = (int)std::min<size_t>(256 / s.G, kSmemCap / profile_bytes(s, ns));
  return std::max(1, t);
}

template <int G, int W, int P, bool L, bool LP, bool LOC = false, bool P8 = false>
void launch_pairs_t(gpusw_ctx* c, Bufs& B, gsw::PairsParams prm, int /*teams_hint*/, long long max_rows,
                    bool multipass, const LaunchCfg& lc = LaunchCfg()) {
  auto k = gsw::pairs_kernel<G, W, P, L, LP, LOC, P8>;
  const Shape s{G, W};
  const size_t sub_bytes = (size_t)(gsw::pairs_sub_uint4(prm.S.ns) + (P8 ? gsw::pairs_ext_uint4(prm.S.ns) : 0)) * 16;
  // per team: the profile (s16x2, or two int8 tables of one byte per column) + row-code ring
  const size_t prof = (P8 ? profile_bytes(s, prm.S.ns) / 2 : profile_bytes(s, prm.S.ns)) +
                      gsw::kRing * sizeof(uint32_t);
  static int configured_dev = -1;
  static size_t configured_smem = 0;
  const size_t max_smem = 227 * 1024;
  if (configured_dev != c->device) {
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
    configured_smem = max_smem;
    configured_dev = c->device;
  }
  // teams per block: the count that keeps the most warps resident (ties: larger blocks),
  // within the kernel's own thread limit
  static int max_threads = 0;
  if (!max_threads) {
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, k));
    max_threads = std::min(256, fa.maxThreadsPerBlock);
  }
  int teams = 1, best_warps = -1, bps_best = 1;
  for (int t = 1; t * G <= max_threads; t *= 2) {
    const size_t smem = sub_bytes + prof * t;
    if (smem > max_smem) break;
    int bps = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, G * t, smem));
    const int warps = bps * G * t / 32;
    if (bps > 0 && warps >= best_warps) {
      best_warps = warps;
      teams = t;
      bps_best = bps;
    }
  }
  const size_t smem = sub_bytes + prof * teams;
  long long grid = (long long)c->sms * std::max(1, bps_best);
  const long long team_items = prm.item_mode == 1 ? kOvfCap : prm.n_items;
  grid = std::max(1ll, std::min(grid, (team_items + teams - 1) / teams));
  const size_t need = multipass ? (size_t)grid * teams * (size_t)std::max(1ll, max_rows) : 0;
  if (lc.need) {
    *lc.need = need;
    return;
  }
  if (multipass) {
    prm.bnd = lc.bnd_off >= 0 ? static_cast<uint2*>(B.bnd.p) + lc.bnd_off : B.bnd.as<uint2>(need);
    prm.bnd_cap = (int)std::max(1ll, max_rows);
  } else {
    prm.bnd = nullptr;
    prm.bnd_cap = 0;
  }
  k<<<(int)grid, G * teams, smem, lc.st ? lc.st : c->stream>>>(prm);
  CK(cudaGetLastError());
  c->st.last_launches++;
}

template <int P, bool L, bool LP, bool P8 = false>
void launch_pairs_shape(gpusw_ctx* c, Bufs& B, int shape, const gsw::PairsParams& prm, int teams, long long max_rows, bool mp,
                        const LaunchCfg& lc) {
  switch (shape) {
    case 0: launch_pairs_t<8, 8, P, L, LP, false, P8>(c, B, prm, teams, max_rows, mp, lc); break;
    case 1: launch_pairs_t<8, 12, P, L, LP, false, P8>(c, B, prm, teams, max_rows, mp, lc); break;
    case 2: launch_pairs_t<8, 16, P, L, LP, false, P8>(c, B, prm, teams, max_rows, mp, lc); break;
    case 3: launch_pairs_t<8, 20, P, L, LP, false, P8>(c, B, prm, teams, max_rows, mp, lc); break;
    case 4: launch_pairs_t<8, 24, P, L, LP, false, P8>(c, B, prm, teams, max_rows, mp, lc); break;
    case 5: launch_pairs_t<16, 16, P, L, LP, false, P8>(c, B, prm, teams, max_rows, mp, lc); break;
    case 6: launch_pairs_t<16, 24, P, L, LP, false, P8>(c, B, prm, teams, max_rows, mp, lc); break;
    case 7: launch_pairs_t<32, 16, P, L, LP, false, P8>(c, B, prm, teams, max_rows, mp, lc); break;
    default: fail(GPUSW_ERR_INVALID, "bad pairs kernel shape");
  }
}

void launch_pairs(gpusw_ctx* c, Bufs& B, int shape, int P, bool local, const gsw::PairsParams& prm,
                  long long max_rows, bool multipass, const LaunchCfg& lc = LaunchCfg()) {
  const int teams = pair_teams(kPairShapes[shape], prm.S.ns);
  const bool lp = prm.S.mode == gsw::kModeSemi && prm.S.free_q && prm.S.free_r;
  if (P == 2) {
    // int8 query tables when every profile value (s - go, the pad score - go, -go) fits in
    // a signed byte and the branch-free pass applies (all modes but the unpadded
    // free-query-end semiglobal one)
    const int max_sub = 32767 - prm.S.ovf_limit;  // max(0, largest substitution score)
    const bool p8 = prm.S.s_pad - prm.S.go >= -128 && max_sub - prm.S.go <= 127 &&
                    (local || lp || !(prm.S.mode == gsw::kModeSemi && prm.S.free_q));
    if (p8) {
      if (local) launch_pairs_shape<2, true, false, true>(c, B, shape, prm, teams, max_rows, multipass, lc);
      else if (lp) launch_pairs_shape<2, false, true, true>(c, B, shape, prm, teams, max_rows, multipass, lc);
      else launch_pairs_shape<2, false, false, true>(c, B, shape, prm, teams, max_rows, multipass, lc);
      return;
    }
    if (local) launch_pairs_shape<2, true, false>(c, B, shape, prm, teams, max_rows, multipass, lc);
    else if (lp) launch_pairs_shape<2, false, true>(c, B, shape, prm, teams, max_rows, multipass, lc);
    else launch_pairs_shape<2, false, false>(c, B, shape, prm, teams, max_rows, multipass, lc);
  } else {
    if (local) launch_pairs_shape<1, true, false>(c, B, shape, prm, teams, max_rows, multipass, lc);
    else if (lp) launch_pairs_shape<1, false, true>(c, B, shape, prm, teams, max_rows, multipass, lc);
    else launch_pairs_shape<1, false, false>(c, B, shape, prm, teams, max_rows, multipass, lc);
  }
}

// Inter-sequence kernel (pairs_inter_kernel): one launch over all items, boundary columns
// for every thread of the launch when a query is longer than one strip.
template <bool L, bool T>
void launch_inter_t(gpusw_ctx* c, Bufs& B, gsw::InterParams prm, int max_n, int max_m, const LaunchCfg& lc) {
  auto k = gsw::pairs_inter_kernel<L, T>;
  int bps = 1;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, gsw::kInterBlock, 0));
  long long grid = (long long)c->sms * std::max(1, bps);
  grid = std::max(1ll, std::min(grid, (prm.n_items + gsw::kInterBlock - 1) / gsw::kInterBlock));
  const bool strips = max_n > gsw::kInterW;
  const size_t need = strips ? (size_t)grid * gsw::kInterBlock * (size_t)std::max(1, max_m) : 0;
  if (lc.need) {
    *lc.need = need;
    return;
  }
  prm.stride = grid * gsw::kInterBlock;
  prm.bnd = strips ? (lc.bnd_off >= 0 ? static_cast<uint2*>(B.bnd.p) + lc.bnd_off : B.bnd.as<uint2>(need)) : nullptr;
  k<<<(int)grid, gsw::kInterBlock, 0, lc.st ? lc.st : c->stream>>>(prm);
  CK(cudaGetLastError());
  c->st.last_launches++;
}

void launch_inter(gpusw_ctx* c, Bufs& B, const gsw::InterParams& prm, int max_n, int max_m,
                  const LaunchCfg& lc = LaunchCfg()) {
  const HostScheme& h = c->sch;
  const bool local = h.mode == gsw::kModeLocal;
  // the running maximum is needed in local mode, and elsewhere only as the int16 guard
  const bool track = local || (long long)std::min(max_n, max_m) * std::max(0, h.max_sub) > prm.S.ovf_limit;
  if (local) launch_inter_t<true, true>(c, B, prm, max_n, max_m, lc);
  else if (track) launch_inter_t<false, true>(c, B, prm, max_n, max_m, lc);
  else launch_inter_t<false, false>(c, B, prm, max_n, max_m, lc);
}

// Does the inter-sequence kernel apply to an int16 call over these query and reference sets?
// Query codes 0..3 only (a 2-bit packed set) and every s - go of those columns in a byte.
bool inter_applies(const gpusw_ctx* c, const Db& q, const Db& r, int P) {
  const HostScheme& h = c->sch;
  if (!c->inter || c->plain || P != 2 || q.bits != 2 || h.ns + 1 > gsw::kInterTabMax) return false;
  auto words = [](const Db& d) {  // one past the set's last packed word
    return d.n ? d.woff[d.n - 1] + (d.len[d.n - 1] + d.per - 1) / d.per + 1 : 0ll;
  };
  if (words(q) >= (1ll << 32) || words(r) >= (1ll << 32)) return false;  // 32-bit word offsets
  for (int r = 0; r < h.ns; ++r)
    for (int col = 0; col < 4 && col < h.ns; ++col) {
      const int v = h.sub[(size_t)r * h.ns + col] - h.go;
      if (v < -128 || v > 127) return false;
    }
  return true;
}

// Items of the inter-sequence kernel over the alignments `cand`: ordered by query length, then
// reference length, longest first (two stable counting sorts), and neighbours paired into one
// thread when their query lengths are equal (any neighbours in local mode); an unpaired
// alignment takes a thread alone (b = -1). Also returns the largest item (query columns x the
// longer reference) and the sum over items, which decide whether the kernel pays.
struct InterPlan {
  std::vector<int2> items;
  int max_n = 0, max_m = 0;
  double work = 0, max_work = 0;
};

InterPlan plan_inter(const Db& q, const Db& r, const int32_t* qi, const int32_t* rj,
                     const std::vector<int>& cand, bool local) {
  InterPlan pl;
  const size_t n = cand.size();
  for (int i : cand) {
    pl.max_n = std::max(pl.max_n, q.len[qi[i]]);
    pl.max_m = std::max(pl.max_m, r.len[rj[i]]);
  }
  const int max_n = pl.max_n, max_m = pl.max_m;
  std::vector<int> by_m(n), order(n);
  {
    std::vector<int64_t> cnt((size_t)max_m + 2, 0);
    for (int i : cand) cnt[(size_t)(max_m - r.len[rj[i]]) + 1]++;
    for (int v = 0; v <= max_m; ++v) cnt[v + 1] += cnt[v];
    for (int i : cand) by_m[cnt[(size_t)(max_m - r.len[rj[i]])]++] = i;
  }
  {
    std::vector<int64_t> cnt((size_t)max_n + 2, 0);
    for (int i : cand) cnt[(size_t)(max_n - q.len[qi[i]]) + 1]++;
    for (int v = 0; v <= max_n; ++v) cnt[v + 1] += cnt[v];
    for (size_t k = 0; k < n; ++k) {
      const int i = by_m[k];
      order[cnt[(size_t)(max_n - q.len[qi[i]])]++] = i;
    }
  }
  pl.items.reserve((n + 1) / 2);
  for (size_t k = 0; k < n;) {
    const int a = order[k];
    int b = -1;
    if (k + 1 < n && (local || q.len[qi[order[k + 1]]] == q.len[qi[a]])) b = order[k + 1];
    pl.items.push_back(make_int2(a, b));
    k += b >= 0 ? 2 : 1;
    const double w = (double)std::max(q.len[qi[a]], b >= 0 ? q.len[qi[b]] : 0) *
                     std::max(r.len[rj[a]], b >= 0 ? r.len[rj[b]] : 0);
    pl.work += w;
    pl.max_work = std::max(pl.max_work, w);
  }
  return pl;
}

// Query lengths that go to the inter-sequence kernel. Against the team kernels on uniform
// pairs (kernel time, semiglobal / local): 30 x 40 2.9x / 2.8x, 100 x 120 1.35x (local),
// 150 x 200 (10^6 read/window pairs) 1.05x, 160-176 x 220 0.94x / 1.03x, 177-192 x 240
// 0.88x / 0.94x (the team kernel's 192-column pass is nearly full there), 200-224 x 270
// 1.10x / 1.05x, 250-256 x 300 0.95x / 0.89x, 384 and 512 columns 0.73-0.76x.
constexpr int kInterMaxCols = 224;
bool inter_len(int n) { return n <= 160 || (n > 192 && n <= kInterMaxCols); }

// One thread scores a whole item, so the call takes as long as its longest item unless every
// resident thread has several: the kernel is used when the items' work is at least twice the
// largest item's on every resident thread (two blocks per SM).
bool inter_pays(const gpusw_ctx* c, const InterPlan& pl) {
  return !pl.items.empty() && pl.work >= 2.0 * (double)c->sms * (2.0 * gsw::kInterBlock) * pl.max_work;
}

// Smallest pairs shape whose columns cover `ncols` and whose profile fits, else the widest
// that fits (multi-pass).
int pick_pair_shape(int ncols, int ns) {
  for (int i = 0; i < kNumPair; ++i)
    if (kPairShapes[i].cap() >= ncols && profile_bytes(kPairShapes[i], ns) <= kSmemCap) return i;
  for (int i = kNumPair - 1; i >= 0; --i)  // multi-pass: the widest shape that fits
    if (profile_bytes(kPairShapes[i], ns) <= kSmemCap) return i;
  return 0;
}

// Host staging of several arrays into one device allocation. `add` copies the bytes now;
// `add_ref` only records the pointer, and the caller keeps that memory alive and unchanged
// until `upload` has returned (the copies are issued from pageable memory, which the runtime
// stages before cudaMemcpyAsync returns).
struct Staging {
  std::vector<char> host;
  struct Ref { size_t off; const void* src; size_t bytes; };
  std::vector<Ref> refs;
  size_t end = 0;
  size_t place(size_t bytes) {
    const size_t off = (end + 255) & ~(size_t)255;
    end = off + bytes;
    return off;
  }
  size_t add(const void* src, size_t bytes) {
    const size_t off = place(bytes);
    host.resize(end);
    if (bytes) memcpy(host.data() + off, src, bytes);
    return off;
  }
  size_t add_ref(const void* src, size_t bytes) {
    const size_t off = place(bytes);
    if (bytes) refs.push_back({off, src, bytes});
    return off;
  }
  char* upload(gpusw_ctx* c, Bufs& B) {
    char* d = static_cast<char*>(B.meta.get(std::max<size_t>(end, 256)));
    // while recording a graph the plan's metadata is already in place from its eager run
    if (!B.capturing) {
      if (!host.empty())
        CK(cudaMemcpyAsync(d, host.data(), host.size(), cudaMemcpyHostToDevice, c->stream));
      for (const Ref& r : refs)
        CK(cudaMemcpyAsync(d + r.off, r.src, r.bytes, cudaMemcpyHostToDevice, c->stream));
    }
    return d;
  }
};

// Top-k of nrows score rows of ncols (row stride ncols) into (nrows, kk) outputs: the
// threshold-and-filter kernel up to 32, the multi-round kernel beyond.
void launch_topk(const int* d_scores, int nrows, int ncols, int kk, int* d_idx, int* d_sc, cudaStream_t st) {
  if (nrows <= 0 || kk <= 0) return;
  if (kk <= 32) gsw::topk_filter_kernel<<<nrows, 256, 0, st>>>(d_scores, ncols, ncols, kk, d_idx, d_sc, kk);
  else gsw::topk_kernel<<<nrows, 256, 0, st>>>(d_scores, ncols, ncols, kk, d_idx, d_sc, kk);
  CK(cudaGetLastError());
}

// Runs the n shape launches of one call, launch(i, cfg) issuing (or, with cfg.need set,
// sizing) launch i. A first pass sizes the multi-pass boundary strips of every launch and
// places them side by side in one allocation; then the launches go out round-robin on the
// context stream and its auxiliary streams, forked from the context stream's prior work and
// joined back into it. Launches of different shapes therefore overlap: a small call's
// few-item launches run side by side instead of one after another, and a large call's
// launches overlap their last waves. Recorded into a CUDA graph the fork and join become
// graph edges. The plain form keeps one stream.
template <class F>
void run_group(gpusw_ctx* c, Bufs& B, int n, F&& launch) {
  std::vector<long long> off((size_t)std::max(n, 0), -1);
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    size_t need = 0;
    LaunchCfg sz;
    sz.need = &need;
    launch(i, sz);
    if (need) {
      off[i] = (long long)total;
      total += need;
    }
  }
  if (total) B.bnd.as<uint2>(total);
  const int ns = c->plain ? 1 : std::min(n, 1 + kAuxStreams);
  if (ns > 1) {
    CK(cudaEventRecord(c->fork_ev, c->stream));
    for (int a = 0; a + 1 < ns; ++a) CK(cudaStreamWaitEvent(c->aux[a], c->fork_ev, 0));
  }
  for (int i = 0; i < n; ++i) {
    LaunchCfg lc;
    lc.st = (i % ns == 0) ? c->stream : c->aux[i % ns - 1];
    lc.bnd_off = off[i];
    launch(i, lc);
  }
  if (ns > 1) {
    for (int a = 0; a + 1 < ns; ++a) {
      CK(cudaEventRecord(c->join_ev[a], c->aux[a]));
      CK(cudaStreamWaitEvent(c->stream, c->join_ev[a], 0));
    }
  }
}

// Overflow rescoring of the int16 cells flagged by the previous launches (int32, any length).
void launch_overflow_rescore(gpusw_ctx* c, Bufs& B, const Db& q, const Db& r, int* out,
                             unsigned long long* queue_slot, const LaunchCfg& lc = LaunchCfg()) {
  gsw::PairsParams pp{};
  pp.S = make_scheme(c->sch, 1);
  pp.sub = c->sub_d;
  pp.cols = q.packed();
  pp.rows = r.packed();
  pp.item_mode = 1;
  pp.ovf_in = static_cast<const gsw::Ovf*>(B.ovf.p);
  pp.ovf_in_count = static_cast<const int*>(B.ovf_count.p);
  pp.ovf_flag = B.ovf_flag.as<int>(1);
  pp.ovf_in_cap = kOvfCap;
  pp.queue = queue_slot;
  pp.out = out;
  pp.n_items = kOvfCap;
  const int shape = pick_pair_shape(1 << 30, c->sch.ns);
  launch_pairs(c, B, shape, 1, c->sch.mode == gsw::kModeLocal, pp, std::max(q.max_len, r.max_len), true, lc);
}

void run_cross(gpusw_ctx* c, Bufs& B, const Db& q, const Db& r, const int32_t* qlist, int nq, int P,
               int* out, long long out_ld);

// Stream buffer of a reference set in sorted (batched) or input (plain) order.
// Row order of a set used as references: longest first, stable (counting sort on the length),
// and the identity order of the plain form, both on the device. Built on the set's first use
// as references, before any graph capture of that use (every cached call runs eagerly first).
void ensure_row_order(gpusw_ctx* c, Db& r) {
  if (r.order_ready) return;
  const int n = r.n;
  r.perm_desc.resize(n);
  {
    std::vector<int> cnt((size_t)r.max_len + 2, 0);
    for (int i = 0; i < n; ++i) cnt[(size_t)(r.max_len - r.len[i]) + 1]++;
    for (size_t b = 1; b < cnt.size(); ++b) cnt[b] += cnt[b - 1];
    for (int i = 0; i < n; ++i) r.perm_desc[cnt[(size_t)(r.max_len - r.len[i])]++] = i;
  }
  const size_t slots = (size_t)std::max(1, n);
  std::vector<int> img(2 * slots, 0);
  std::copy(r.perm_desc.begin(), r.perm_desc.end(), img.begin());
  std::iota(img.begin() + slots, img.begin() + slots + n, 0);
  CK(cudaMalloc(&r.order_base, img.size() * sizeof(int)));
  r.perm_d = static_cast<int*>(r.order_base);
  r.ident_d = r.perm_d + slots;
  CK(cudaMemcpy(r.order_base, img.data(), img.size() * sizeof(int), cudaMemcpyHostToDevice));
  r.bytes += (int64_t)(img.size() * sizeof(int));
  c->held += (int64_t)(img.size() * sizeof(int));
  r.order_ready = true;
}

const Db::Stream& get_stream(gpusw_ctx* c, Db& r, bool plain) {
  ensure_row_order(c, r);
  const int pad = c->sch.ns;
  const std::pair<int, int> key(plain ? 1 : 0, pad);
  for (auto& kv : r.streams)
    if (kv.first == key) return kv.second;
  Db::Stream st;
  const int R = gsw::kStreamRows, P = gsw::kStreamPadLen;
  st.n_streams = (r.n + R - 1) / R;
  std::vector<long long> off(std::max(1, st.n_streams)), row_dst(std::max(1, r.n));
  std::vector<int> total(std::max(1, st.n_streams));
  const std::vector<int>& order = r.perm_desc;
  std::vector<int> ident;
  if (plain) {
    ident.resize(r.n);
    std::iota(ident.begin(), ident.end(), 0);
  }
  const std::vector<int>& ord = plain ? ident : order;
  long long cur = 0;
  for (int sidx = 0; sidx < st.n_streams; ++sidx) {
    cur += P;
    off[sidx] = cur;
    int tot = 0;
    for (int j = sidx * R; j < std::min(r.n, sidx * R + R); ++j) {
      row_dst[j] = cur + tot;
      tot += r.len[ord[j]];
    }
    total[sidx] = tot;
    st.max_total = std::max(st.max_total, tot);
    cur += tot + P;
  }
  st.nbytes = std::max(1ll, cur) + (long long)st.n_streams * 12;
  CK(cudaMalloc(&st.bytes, std::max(1ll, cur)));
  CK(cudaMalloc(&st.off, std::max(1, st.n_streams) * sizeof(long long)));
  CK(cudaMalloc(&st.total, std::max(1, st.n_streams) * sizeof(int)));
  CK(cudaMemsetAsync(st.bytes, pad, std::max(1ll, cur), c->stream));
  CK(cudaMemcpyAsync(st.off, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(st.total, total.data(), total.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  st.total_h = total;
  if (r.n > 0) {
    long long* dst_d = nullptr;
    CK(cudaMalloc(&dst_d, r.n * sizeof(long long)));
    CK(cudaMemcpyAsync(dst_d, row_dst.data(), r.n * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    const int threads = 256;
    const long long blocks = ((long long)r.n * 32 + threads - 1) / threads;
    gsw::build_stream_kernel<<<(unsigned)blocks, threads, 0, c->stream>>>(r.packed(), plain ? r.ident_d : r.perm_d, r.n, dst_d, st.bytes);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    cudaFree(dst_d);
  }
  c->held += st.nbytes;
  r.streams.emplace_back(key, st);
  return r.streams.back().second;
}

template <int G, int W, int P>
void launch_stream_t(gpusw_ctx* c, Bufs& B, gsw::StreamParams prm, int n_streams_max_total, bool multipass,
                     const LaunchCfg& lc) {
  auto k = gsw::cross_stream_kernel<G, W, P>;
  const size_t smem = profile_bytes(Shape{G, W}, prm.S.ns);
  static int configured_dev = -1;
  static size_t configured_smem = 0;
  if (configured_dev != c->device || configured_smem < smem) {
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max(smem, configured_smem)));
    configured_smem = std::max(smem, configured_smem);
    configured_dev = c->device;
  }
  int bps = 1;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, 256, smem));
  long long grid = (long long)c->sms * std::max(1, bps);
  grid = std::max(1ll, std::min<long long>(grid, prm.n_items));
  const int nteams = 256 / G;
  const long long strip = n_streams_max_total + 2 * gsw::kStreamPadLen;
  const size_t need = multipass ? (size_t)grid * nteams * strip : 0;
  if (lc.need) {
    *lc.need = need;
    return;
  }
  if (multipass) {
    prm.bnd_strip = strip;
    prm.bnd = lc.bnd_off >= 0 ? static_cast<uint2*>(B.bnd.p) + lc.bnd_off : B.bnd.as<uint2>(need);
  } else {
    prm.bnd = nullptr;
    prm.bnd_strip = 0;
  }
  k<<<(int)grid, 256, smem, lc.st ? lc.st : c->stream>>>(prm);
  CK(cudaGetLastError());
  c->st.last_launches++;
}

template <int P>
void launch_stream_shape(gpusw_ctx* c, Bufs& B, int shape, const gsw::StreamParams& prm, int mt, bool mp,
                         const LaunchCfg& lc = LaunchCfg()) {
  switch (shape) {
    case 0: launch_stream_t<8, 4, P>(c, B, prm, mt, mp, lc); break;
    case 1: launch_stream_t<8, 8, P>(c, B, prm, mt, mp, lc); break;
    case 2: launch_stream_t<8, 12, P>(c, B, prm, mt, mp, lc); break;
    case 3: launch_stream_t<8, 16, P>(c, B, prm, mt, mp, lc); break;
    case 4: launch_stream_t<8, 24, P>(c, B, prm, mt, mp, lc); break;
    case 5: launch_stream_t<8, 32, P>(c, B, prm, mt, mp, lc); break;
    case 6: launch_stream_t<16, 16, P>(c, B, prm, mt, mp, lc); break;
    case 7: launch_stream_t<16, 20, P>(c, B, prm, mt, mp, lc); break;
    case 8: launch_stream_t<16, 24, P>(c, B, prm, mt, mp, lc); break;
    case 9: launch_stream_t<16, 32, P>(c, B, prm, mt, mp, lc); break;
    case 10: launch_stream_t<32, 16, P>(c, B, prm, mt, mp, lc); break;
    case 11: launch_stream_t<32, 20, P>(c, B, prm, mt, mp, lc); break;
    case 12: launch_stream_t<32, 24, P>(c, B, prm, mt, mp, lc); break;
    case 13: launch_stream_t<32, 32, P>(c, B, prm, mt, mp, lc); break;
    case 14: launch_stream_t<8, 20, P>(c, B, prm, mt, mp, lc); break;
    case 15: launch_stream_t<8, 28, P>(c, B, prm, mt, mp, lc); break;
    case 16: launch_stream_t<16, 28, P>(c, B, prm, mt, mp, lc); break;
    case 17: launch_stream_t<32, 28, P>(c, B, prm, mt, mp, lc); break;
    default: fail(GPUSW_ERR_INVALID, "bad stream kernel shape");
  }
}

// Every shape's items in one launch of cross_stream_multi_kernel (item.y = chunk | shape << 24).
// smem: the largest profile among the call's shapes; boundary strips for 32 teams per CTA.
template <int P>
void launch_stream_multi(gpusw_ctx* c, Bufs& B, gsw::StreamParams prm, size_t smem, int n_streams_max_total,
                         bool multipass, const LaunchCfg& lc) {
  auto k = gsw::cross_stream_multi_kernel<P>;
  static int configured_dev = -1;
  static size_t configured_smem = 0;
  if (configured_dev != c->device || configured_smem < smem) {
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max(smem, configured_smem)));
    configured_smem = std::max(smem, configured_smem);
    configured_dev = c->device;
  }
  int bps = 1;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, 256, smem));
  long long grid = (long long)c->sms * std::max(1, bps);
  grid = std::max(1ll, std::min<long long>(grid, prm.n_items));
  const long long strip = n_streams_max_total + 2 * gsw::kStreamPadLen;
  const size_t need = multipass ? (size_t)grid * 32 * strip : 0;
  if (lc.need) {
    *lc.need = need;
    return;
  }
  if (multipass) {
    prm.bnd_strip = strip;
    prm.bnd = lc.bnd_off >= 0 ? static_cast<uint2*>(B.bnd.p) + lc.bnd_off : B.bnd.as<uint2>(need);
  } else {
    prm.bnd = nullptr;
    prm.bnd_strip = 0;
  }
  k<<<(int)grid, 256, smem, lc.st ? lc.st : c->stream>>>(prm);
  CK(cudaGetLastError());
  c->st.last_launches++;
}

// Cost of scoring `ncols` columns with a shape, per reference row (lane-steps x ops).
double stream_cost(const Shape& s, int ncols) {
  const int npass = (std::max(ncols, 1) + s.cap() - 1) / s.cap();
  return (double)npass * s.G * (5.5 * s.W + 6.0);
}

// Batched form: the shape (and pass count) of least modelled cost for this column length.
// Plain form: one shape per call -- the smallest single-pass shape that covers the call's
// longest query, or the widest shape in several passes when none covers it.
int pick_stream_shape(int ncols, int ns, bool plain, const std::vector<double>* tuned = nullptr) {
  int best = -1;
  double bc = 0;
  if (plain) {
    for (int i = 0; i < kNumStream; ++i) {
      if (profile_bytes(kStreamShapes[i], ns) > kSmemCap) continue;
      const int cap = kStreamShapes[i].cap(), bcap = best < 0 ? 0 : kStreamShapes[best].cap();
      const bool covers = cap >= ncols, bcovers = bcap >= ncols;
      if (best < 0 || (covers && (!bcovers || cap < bcap)) || (!covers && !bcovers && cap > bcap))
        best = i;
    }
    return best;
  }
  for (int i = 0; i < kNumStream; ++i) {
    if (profile_bytes(kStreamShapes[i], ns) > kSmemCap) continue;
    const double cst = tuned && (*tuned)[i] > 0
                           ? (double)((std::max(ncols, 1) + kStreamShapes[i].cap() - 1) /
                                      kStreamShapes[i].cap()) * (*tuned)[i]
                           : stream_cost(kStreamShapes[i], ncols);
    if (best < 0 || cst < bc) {
      best = i;
      bc = cst;
    }
  }
  return best;
}

// Latency form, for calls too small to fill the GPU (each CTA gets at most an item or two, so
// the call lasts as long as its slowest item): an item's time is its passes x steps x the
// instructions of one step, and a step costs about 5.5 W + 6 whatever G is (G lanes work in
// parallel). So the shape of fewest passes x (5.5 W + 6), ties to the smaller team.
int pick_stream_shape_latency(int ncols, int ns) {
  int best = -1;
  double bc = 0;
  for (int i = 0; i < kNumStream; ++i) {
    const Shape& sh = kStreamShapes[i];
    if (profile_bytes(sh, ns) > kSmemCap) continue;
    const int npass = (std::max(ncols, 1) + sh.cap() - 1) / sh.cap();
    const double cst = (double)npass * (5.5 * sh.W + 6.0);
    if (best < 0 || cst < bc || (cst == bc && sh.G < kStreamShapes[best].G)) {
      best = i;
      bc = cst;
    }
  }
  return best;
}

const std::vector<double>* find_tune(gpusw_ctx* c, int P) {
  for (auto& kv : c->tune)
    if (kv.first == std::make_pair(c->sch.ns, P)) return &kv.second;
  return nullptr;
}

// Time every stream shape on synthetic full-width columns (256 queries of exactly G*W
// residues) against 4,096 synthetic references of 300 residues -- thousands of work items
// for every shape, so the GPU is full and the time measures throughput, not parallelism;
// microseconds of device time per (reference row, column pass) of one column pair. Needs
// no caller data; runs on the context's stream (about a second in all).
std::vector<double> run_autotune(gpusw_ctx* c, int P) {
  const HostScheme& h = c->sch;
  std::vector<double> us(kNumStream, 0.0);
  if (h.mode != gsw::kModeLocal || h.ns > 126) return us;
  const int nr = 4096, mr = 300, nq = 256;
  uint64_t rs = 0x9E3779B97F4A7C15ull;
  auto rnd = [&]() { rs ^= rs << 13; rs ^= rs >> 7; rs ^= rs << 17; return rs; };
  const int ncode = std::max(1, h.ns - 1);
  std::vector<uint8_t> rc((size_t)nr * mr);
  for (auto& v : rc) v = (uint8_t)(rnd() % ncode);
  std::vector<int32_t> ro(nr + 1);
  for (int i = 0; i <= nr; ++i) ro[i] = i * mr;
  int32_t rdb = 0;
  if (gpusw_db_upload(c, rc.data(), ro.data(), nr, &rdb) != GPUSW_OK) fail(GPUSW_ERR_CUDA, c->err);
  Db& r = get_db(c, rdb);
  ensure_row_order(c, r);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int saved_plain = c->plain;
  c->plain = 0;
  Bufs T;  // private buffers: never disturbs a call's shared set
  T.set_held(&c->held);
  try {
    for (int sh = 0; sh < kNumStream; ++sh) {
      const Shape S = kStreamShapes[sh];
      if (profile_bytes(S, h.ns) > kSmemCap) continue;
      std::vector<uint8_t> qc((size_t)nq * S.cap());
      for (auto& v : qc) v = (uint8_t)(rnd() % ncode);
      std::vector<int32_t> qo(nq + 1);
      for (int i = 0; i <= nq; ++i) qo[i] = i * S.cap();
      int32_t qdb = 0;
      if (gpusw_db_upload(c, qc.data(), qo.data(), nq, &qdb) != GPUSW_OK) fail(GPUSW_ERR_CUDA, c->err);
      Db& q = get_db(c, qdb);
      // force this shape: a one-shape table
      std::vector<double> only(kNumStream, 1e30);
      only[sh] = 1.0;
      std::pair<std::pair<int, int>, std::vector<double>> entry({h.ns, P}, only);
      c->tune.push_back(entry);
      std::vector<int32_t> ql(nq);
      std::iota(ql.begin(), ql.end(), 0);
      int* d_out = T.out.as<int>((size_t)nq * nr);
      double best = 1e30;
      for (int rep = 0; rep < 2; ++rep) {
        T.reset_marks();
        CK(cudaEventRecord(e0, c->stream));
        run_cross(c, T, q, r, ql.data(), nq, P, d_out, nr);
        CK(cudaEventRecord(e1, c->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0) best = std::min(best, (double)ms);
      }
      c->tune.pop_back();
      us[sh] = best * 1e3 / ((double)((nq + P - 1) / P) * nr);
      gpusw_db_free(c, qdb);
    }
  } catch (...) {
    c->plain = saved_plain;
    cudaStreamSynchronize(c->stream);
    T.release();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    gpusw_db_free(c, rdb);
    throw;
  }
  c->plain = saved_plain;
  CK(cudaStreamSynchronize(c->stream));
  T.release();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  gpusw_db_free(c, rdb);
  return us;
}

// Tune on first use (at the entry of a call, before it takes any buffer).
void ensure_tuned(gpusw_ctx* c, int P) {
  if (!c->autotune || c->plain || c->sch.mode != gsw::kModeLocal || c->sch.ns > 126) return;
  if (find_tune(c, P)) return;
  std::vector<double> us = run_autotune(c, P);
  c->tune.emplace_back(std::make_pair(c->sch.ns, P), us);
}

// Local-mode cross product through the streaming kernel (any column length).
void run_cross_stream(gpusw_ctx* c, Bufs& B, const Db& q, Db& r, const int32_t* qlist, int nq, int P,
                      int* out, long long out_ld) {
  const HostScheme& h = c->sch;
  const int nr = r.n;
  // A call whose items cannot fill the GPU even in the narrowest teams' chunks is planned for
  // latency: it lasts as long as its slowest item, so its shapes are chosen per item time
  // (pick_stream_shape_latency). When all its streams also fit one chunk, each item runs them
  // side by side and lasts as long as the longest stream: its references then stay in input
  // order, where the streams hold a mix of lengths (sorted longest first, the first stream
  // holds the eight longest). The 32 x 128 cross product went from 0.426 to 0.360 ms (plain
  // form: 0.387); with several chunks per pair input order measured mixed (-7 % to +4 %).
  const int npairs = (nq + P - 1) / P;
  const long long n_streams = ((long long)nr + gsw::kStreamRows - 1) / gsw::kStreamRows;
  const bool latency = !c->plain && (long long)npairs * ((n_streams + 31) / 32) < 2ll * c->sms;
  const bool input_order = c->plain || (latency && n_streams <= 32);
  const Db::Stream& st = get_stream(c, r, input_order);
  std::vector<int> pos(nq);
  std::iota(pos.begin(), pos.end(), 0);
  if (!c->plain)
    std::stable_sort(pos.begin(), pos.end(), [&](int a, int b) { return q.len[qlist[a]] > q.len[qlist[b]]; });
  std::vector<int2> pairs(npairs), pair_out(npairs);
  std::vector<int> pair_cols(npairs);
  for (int i = 0; i < npairs; ++i) {
    const int a = pos[i * P];
    const int b = (P == 2 && i * P + 1 < nq) ? pos[i * P + 1] : -1;
    pairs[i] = make_int2(qlist[a], b >= 0 ? qlist[b] : -1);
    pair_out[i] = make_int2(a, b);
    pair_cols[i] = std::max(q.len[qlist[a]], b >= 0 ? q.len[qlist[b]] : 0);
  }
  std::vector<std::vector<int>> bins(kNumStream);
  const int call_max = npairs ? *std::max_element(pair_cols.begin(), pair_cols.end()) : 0;
  const std::vector<double>* tuned = c->plain ? nullptr : find_tune(c, P);
  for (int i = 0; i < npairs; ++i) {
    const int sh = latency ? pick_stream_shape_latency(pair_cols[i], h.ns)
                           : pick_stream_shape(c->plain ? call_max : pair_cols[i], h.ns, c->plain != 0, tuned);
    if (sh < 0) fail(GPUSW_ERR_SCHEME, "substitution table too large for the profile");
    bins[sh].push_back(i);
  }
  Staging stg;
  const size_t off_pairs = stg.add(pairs.data(), pairs.size() * sizeof(int2));
  const size_t off_pout = stg.add(pair_out.data(), pair_out.size() * sizeof(int2));
  struct L { int shape; size_t items_off; int n_items; bool multipass; size_t smem; };
  std::vector<L> launches;
  int nshapes = 0, max_chunks = 0;
  for (int sh = 0; sh < kNumStream; ++sh) {
    if (bins[sh].empty()) continue;
    ++nshapes;
    max_chunks = std::max(max_chunks, (st.n_streams + 256 / kStreamShapes[sh].G - 1) / (256 / kStreamShapes[sh].G));
  }
  // one launch for every shape (a batched, throughput-planned call of two or more shapes):
  // items of all shapes in one queue, costliest first -- an item's time is its passes x the
  // instructions of a step x the longest stream of its chunk (streams are sorted longest first)
  const bool multi = c->stream_multi && !c->plain && !latency && nshapes >= 2 && max_chunks < (1 << 24);
  if (multi) {
    struct MI { double cost; int2 item; };
    std::vector<MI> mi;
    bool mp = false;
    size_t smem = 0;
    for (int sh = 0; sh < kNumStream; ++sh) {
      if (bins[sh].empty()) continue;
      const Shape S = kStreamShapes[sh];
      const int nteams = 256 / S.G;
      const int nchunks = (st.n_streams + nteams - 1) / nteams;
      smem = std::max(smem, profile_bytes(S, h.ns));
      for (int pi : bins[sh]) {
        const int npass = (std::max(pair_cols[pi], 1) + S.cap() - 1) / S.cap();
        mp |= npass > 1;
        const double per = (double)npass * (5.5 * S.W + 6.0);
        for (int ch = 0; ch < nchunks; ++ch)
          mi.push_back({per * st.total_h[(size_t)ch * nteams], make_int2(pi, ch | sh << 24)});
      }
    }
    std::stable_sort(mi.begin(), mi.end(), [](const MI& a, const MI& b) { return a.cost > b.cost; });
    std::vector<int2> items(mi.size());
    for (size_t i = 0; i < mi.size(); ++i) items[i] = mi[i].item;
    launches.push_back({-1, stg.add(items.data(), items.size() * sizeof(int2)), (int)items.size(), mp, smem});
  }
  for (int sh = 0; sh < kNumStream && !multi; ++sh) {
    if (bins[sh].empty()) continue;
    const int nteams = 256 / kStreamShapes[sh].G;
    const int nchunks = (st.n_streams + nteams - 1) / nteams;
    bool mp = false;
    for (int pi : bins[sh]) mp |= pair_cols[pi] > kStreamShapes[sh].cap();
    std::vector<int2> items;
    items.reserve((size_t)nchunks * bins[sh].size());
    for (int ch = 0; ch < nchunks; ++ch)
      for (int pi : bins[sh]) items.push_back(make_int2(pi, ch));
    launches.push_back({sh, stg.add(items.data(), items.size() * sizeof(int2)), (int)items.size(), mp, 0});
  }
  char* dmeta = stg.upload(c, B);
  const int nslots = (int)launches.size() + 2;
  unsigned long long* queues = B.queue.as<unsigned long long>(nslots);
  CK(cudaMemsetAsync(queues, 0, nslots * sizeof(unsigned long long), c->stream));
  if (P == 2) CK(cudaMemsetAsync(B.ovf_count.as<int>(1), 0, sizeof(int), c->stream));
  gsw::StreamParams sp{};
  sp.S = make_scheme(h, P);
  sp.sub = c->sub_d;
  sp.cols = q.packed();
  sp.row_len = r.len_d;
  sp.row_perm = input_order ? r.ident_d : r.perm_d;
  sp.n_rows = nr;
  sp.stream = st.bytes;
  sp.stream_off = st.off;
  sp.stream_total = st.total;
  sp.n_streams = st.n_streams;
  sp.pairs = reinterpret_cast<const int2*>(dmeta + off_pairs);
  sp.pair_out = reinterpret_cast<const int2*>(dmeta + off_pout);
  sp.out = out;
  sp.out_ld = out_ld;
  sp.ovf = B.ovf.as<gsw::Ovf>(kOvfCap);
  sp.ovf_count = B.ovf_count.as<int>(1);
  sp.ovf_cap = kOvfCap;
  run_group(c, B, (int)launches.size(), [&](int i, const LaunchCfg& lc) {
    const L& l = launches[i];
    gsw::StreamParams lp = sp;
    lp.items = reinterpret_cast<const int2*>(dmeta + l.items_off);
    lp.n_items = l.n_items;
    lp.queue = reinterpret_cast<int*>(queues + i);
    if (multi) {
      if (P == 2) launch_stream_multi<2>(c, B, lp, l.smem, st.max_total, l.multipass, lc);
      else launch_stream_multi<1>(c, B, lp, l.smem, st.max_total, l.multipass, lc);
    } else if (P == 2) {
      launch_stream_shape<2>(c, B, l.shape, lp, st.max_total, l.multipass, lc);
    } else {
      launch_stream_shape<1>(c, B, l.shape, lp, st.max_total, l.multipass, lc);
    }
  });
  if (P == 2) launch_overflow_rescore(c, B, q, r, out, queues + launches.size());
}

// Cross product of the queries `qlist` (a sublist of q) against every sequence of r into
// out[a * out_ld + ref] for a = position in qlist. P = 2 (int16 pairs) or 1 (int32).
// Returns the number of queue counters used (device slots at queues[...]).
void run_cross(gpusw_ctx* c, Bufs& B, const Db& q, const Db& r, const int32_t* qlist, int nq, int P,
               int* out, long long out_ld) {
  const HostScheme& h = c->sch;
  const bool local = h.mode == gsw::kModeLocal;
  const int nr = r.n;
  if (nq == 0 || nr == 0) return;
  if (local && h.ns <= 126) {
    run_cross_stream(c, B, q, const_cast<Db&>(r), qlist, nq, P, out, out_ld);
    return;
  }
  // column order: longest first (batched) or input order (plain)
  std::vector<int> pos(nq);
  std::iota(pos.begin(), pos.end(), 0);
  if (!c->plain)
    std::stable_sort(pos.begin(), pos.end(), [&](int a, int b) { return q.len[qlist[a]] > q.len[qlist[b]]; });
  // column pairs (P = 2) or singles (P = 1)
  const int npairs = (nq + P - 1) / P;
  std::vector<int2> pairs(npairs), pair_out(npairs);
  std::vector<int> pair_cols(npairs);
  for (int i = 0; i < npairs; ++i) {
    const int a = pos[i * P];
    const int b = (P == 2 && i * P + 1 < nq) ? pos[i * P + 1] : -1;
    pairs[i] = make_int2(qlist[a], b >= 0 ? qlist[b] : -1);
    pair_out[i] = make_int2(a, b);
    pair_cols[i] = std::max(q.len[qlist[a]], b >= 0 ? q.len[qlist[b]] : 0);
  }
  // Cross products the streaming kernel does not take (global and semiglobal, or codes
  // above 126) run on the pairs kernel in cross mode -- its branch-free pass, int8 tables
  // and, for semiglobal with both ends free, left padding: work item = (column pair, one
  // reference), one launch per pairs shape (the plain form: one shape for all pairs, sized
  // to the longest, references in input order).
  std::vector<std::vector<int>> pbins(kNumPair);
  const int plain_shape =
      c->plain ? pick_pair_shape(std::max(1, *std::max_element(pair_cols.begin(), pair_cols.end())), h.ns) : -1;
  for (int i = 0; i < npairs; ++i)
    pbins[c->plain ? plain_shape : pick_pair_shape(std::max(1, pair_cols[i]), h.ns)].push_back(i);
  Staging stg;
  struct PL { int shape; size_t off_p, off_o; int n; int mcol; };
  std::vector<PL> pl;
  for (int sh = 0; sh < kNumPair; ++sh) {
    if (pbins[sh].empty()) continue;
    std::vector<int2> bp, bo;
    int mcol = 0;
    for (int i : pbins[sh]) {
      bp.push_back(pairs[i]);
      bo.push_back(pair_out[i]);
      mcol = std::max(mcol, pair_cols[i]);
    }
    const size_t op = stg.add(bp.data(), bp.size() * sizeof(int2));
    const size_t oo = stg.add(bo.data(), bo.size() * sizeof(int2));
    pl.push_back({sh, op, oo, (int)bp.size(), mcol});
  }
  char* dmeta = stg.upload(c, B);
  const int nslots = (int)pl.size() + 2;
  unsigned long long* queues = B.queue.as<unsigned long long>(nslots);
  CK(cudaMemsetAsync(queues, 0, nslots * sizeof(unsigned long long), c->stream));
  if (P == 2) CK(cudaMemsetAsync(B.ovf_count.as<int>(1), 0, sizeof(int), c->stream));
  gsw::PairsParams pp{};
  pp.S = make_scheme(h, P);
  pp.sub = c->sub_d;
  pp.cols = q.packed();
  pp.rows = r.packed();
  pp.item_mode = 2;
  pp.row_perm = c->plain ? r.ident_d : r.perm_d;
  pp.n_rows = nr;
  pp.out_ld = out_ld;
  pp.out = out;
  pp.ovf = B.ovf.as<gsw::Ovf>(kOvfCap);
  pp.ovf_count = B.ovf_count.as<int>(1);
  pp.ovf_cap = kOvfCap;
  run_group(c, B, (int)pl.size(), [&](int i, const LaunchCfg& lc) {
    const PL& L = pl[i];
    gsw::PairsParams lp = pp;
    lp.pairs = reinterpret_cast<const int2*>(dmeta + L.off_p);
    lp.pair_out = reinterpret_cast<const int2*>(dmeta + L.off_o);
    lp.n_items = (long long)L.n * nr;
    lp.queue = queues + i;
    launch_pairs(c, B, L.shape, P, local, lp, r.max_len, L.mcol > kPairShapes[L.shape].cap(), lc);
  });
  if (P == 2) launch_overflow_rescore(c, B, q, r, out, queues + pl.size());
}

// Largest number of int16 cells flagged by any one launch sequence of the call (read after
// the call's device work; more than kOvfCap means some were not rescored).
int read_overflow_count(gpusw_ctx* c, Bufs& B) {
  int n = 0;
  CK(cudaMemcpyAsync(&n, B.ovf_flag.as<int>(1), sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return n;
}

// 64-bit hash of a byte range for plan keys: four interleaved multiply-xorshift lanes over
// 8-byte words (independent chains, so the multiplies overlap), chunks of 1 MiB hashed on the
// host's cores and their hashes chained in order. Not cryptographic; equal inputs give equal
// keys within a process.
uint64_t hash_chunk(const unsigned char* p, size_t bytes, uint64_t seed) {
  uint64_t h[4] = {seed, seed ^ 0x243F6A8885A308D3ull, seed ^ 0x13198A2E03707344ull,
                   seed ^ 0xA4093822299F31D0ull};
  size_t i = 0;
  for (; i + 32 <= bytes; i += 32) {
    uint64_t w[4];
    memcpy(w, p + i, 32);
    for (int l = 0; l < 4; ++l) {
      h[l] = (h[l] ^ w[l]) * 0x9E3779B97F4A7C15ull;
      h[l] ^= h[l] >> 29;
    }
  }
  uint64_t r = h[0] ^ (h[1] * 0xBF58476D1CE4E5B9ull) ^ (h[2] * 0x94D049BB133111EBull) ^ (h[3] >> 7);
  for (; i < bytes; ++i) r = (r ^ p[i]) * 1099511628211ull;
  return r ^ (uint64_t)bytes;
}

uint64_t fnv1a(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  constexpr size_t kChunk = 1 << 20;
  if (bytes < 4 * kChunk) return hash_chunk(p, bytes, h);
  const long long nch = (long long)((bytes + kChunk - 1) / kChunk);
  std::vector<uint64_t> part((size_t)nch);
  parallel_ranges_min(nch, 1, [&](long long lo, long long hi) {
    for (long long k = lo; k < hi; ++k) {
      const size_t o = (size_t)k * kChunk;
      part[(size_t)k] = hash_chunk(p + o, std::min(kChunk, bytes - o), h + (uint64_t)k);
    }
  });
  return hash_chunk(reinterpret_cast<const unsigned char*>(part.data()), part.size() * 8, h ^ bytes);
}

// Run `body` (the launches of one call) on the shared buffers, or through the plan of `key`:
// the first time eagerly on the shared buffers, the second time eagerly on the plan's own
// buffers and then recorded as a CUDA graph, afterwards by replaying the graph. Returns the
// Bufs that hold the call's results.
Plan* lookup(gpusw_ctx* c, const std::vector<long long>& key) {
  if (!c->graphs) return nullptr;
  for (auto& pl : c->plans)
    if (pl->key == key) {
      pl->last_use = ++c->use_clock;
      return pl.get();
    }
  return nullptr;
}

Bufs& replay(gpusw_ctx* c, Plan* plan) {
  CK(cudaGraphLaunch(plan->exec, c->stream));
  c->st.last_launches += plan->launches;
  return plan->B;
}

template <class F>
Bufs& execute(gpusw_ctx* c, const std::vector<long long>& key, bool cacheable, F&& body) {
  if (!cacheable || !c->graphs) {
    c->shared.reset_marks();
    CK(cudaMemsetAsync(c->shared.ovf_flag.as<int>(1), 0, sizeof(int), c->stream));
    body(c->shared);
    return c->shared;
  }
  if (Plan* hit = lookup(c, key)) return replay(c, hit);
  // A key met for the first time runs eagerly on the shared buffers; it is planned and
  // recorded as a graph when it comes back, so one-off calls pay no capture.
  auto seen = std::find(c->seen_keys.begin(), c->seen_keys.end(), key);
  if (seen == c->seen_keys.end()) {
    c->seen_keys.push_back(key);
    if (c->seen_keys.size() > 16) c->seen_keys.erase(c->seen_keys.begin());
    c->shared.reset_marks();
    CK(cudaMemsetAsync(c->shared.ovf_flag.as<int>(1), 0, sizeof(int), c->stream));
    body(c->shared);
    return c->shared;
  }
  c->seen_keys.erase(seen);
  Plan* plan = nullptr;
  if (c->plans.size() >= 4) {  // evict the least recently used plan
    auto it = std::min_element(c->plans.begin(), c->plans.end(),
                               [](const auto& a, const auto& b) { return a->last_use < b->last_use; });
    CK(cudaStreamSynchronize(c->stream));
    c->plans.erase(it);
  }
  c->plans.push_back(std::make_unique<Plan>());
  plan = c->plans.back().get();
  plan->key = key;
  plan->last_use = ++c->use_clock;
  plan->B.set_held(&c->held);
  Bufs& B = plan->B;
  // eager run: allocates every buffer and uploads the plan's metadata
  B.reset_marks();
  CK(cudaMemsetAsync(B.ovf_flag.as<int>(1), 0, sizeof(int), c->stream));
  const long long launches_before = c->st.last_launches;
  body(B);
  plan->launches = c->st.last_launches - launches_before;
  // record the same sequence (no allocation, no host copy) as a graph for later calls
  CK(cudaStreamSynchronize(c->stream));
  B.reset_marks();
  B.capturing = true;
  cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    try {
      CK(cudaMemsetAsync(B.ovf_flag.as<int>(1), 0, sizeof(int), c->stream));
      body(B);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      B.capturing = false;
      throw;
    }
    e = cudaStreamEndCapture(c->stream, &plan->graph);
  }
  B.capturing = false;
  c->st.last_launches = launches_before + plan->launches;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&plan->exec, plan->graph, 0);
  if (e != cudaSuccess) {  // a plan that cannot be recorded is simply not cached
    cudaGetLastError();
    c->plans.pop_back();
    fail(GPUSW_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e));
  }
  return B;
}

void drop_plans_of(gpusw_ctx* c, int db) {
  CK(cudaStreamSynchronize(c->stream));
  c->plans.erase(std::remove_if(c->plans.begin(), c->plans.end(),
                                [&](const auto& pl) { return pl->key[1] == db || pl->key[2] == db; }),
                 c->plans.end());
}

int choose_width(gpusw_ctx* c, int dtype, int max_n, int max_m) {
  if (!width_ok(c->sch, 1, max_n, max_m))
    fail(GPUSW_ERR_OVERFLOW, "scores of this scheme and these lengths do not fit in int32");
  if (dtype == GPUSW_DTYPE_INT32) return 1;
  return width_ok(c->sch, 2, max_n, max_m) ? 2 : 1;
}

int mark(gpusw_ctx* c, Bufs& B) {
  if (B.pool_used == (int)B.pool.size()) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    B.pool.push_back(e);
  }
  const int id = B.pool_used++;
  if (B.capturing) CK(cudaEventRecordWithFlags(B.pool[id], c->stream, cudaEventRecordExternal));
  else CK(cudaEventRecord(B.pool[id], c->stream));
  return id;
}

// Bracket the launches issued by f() with a pair of stage events.
template <class F>
void staged(gpusw_ctx* c, Bufs& B, bool topk, F&& f) {
  const int a = mark(c, B);
  f();
  const int b = mark(c, B);
  (topk ? B.topk_marks : B.score_marks).emplace_back(a, b);
}

double sum_marks(const Bufs& B, const std::vector<std::pair<int, int>>& marks) {
  double ms = 0;
  for (auto& ab : marks) {
    float x = 0;
    CK(cudaEventElapsedTime(&x, B.pool[ab.first], B.pool[ab.second]));
    ms += x;
  }
  return ms;
}

void begin_call(gpusw_ctx* c) {
  set_device(c);
  c->last_bufs = nullptr;
  c->st.last_launches = 0;
  c->st.last_inter_items = 0;
  c->st.last_overflow = 0;
  c->st.last_pairs = 0;
  c->st.last_cells = 0;
  CK(cudaEventRecord(c->ev0, c->stream));
}

void end_call(gpusw_ctx* c) {
  CK(cudaEventSynchronize(c->ev3));
  float k = 0, t = 0;
  CK(cudaEventElapsedTime(&k, c->ev1, c->ev2));
  CK(cudaEventElapsedTime(&t, c->ev0, c->ev3));
  c->st.last_kernel_ms = k;
  c->st.last_total_ms = t;
  c->st.last_score_ms = c->last_bufs ? sum_marks(*c->last_bufs, c->last_bufs->score_marks) : 0.0;
  c->st.last_topk_ms = c->last_bufs ? sum_marks(*c->last_bufs, c->last_bufs->topk_marks) : 0.0;
  c->st.total_launches += c->st.last_launches;
  c->st.total_overflow += c->st.last_overflow;
  c->st.device_bytes = c->held;
}

template <class F>
int guarded(gpusw_ctx* c, F&& f) {
  if (!c) return GPUSW_ERR_INVALID;
  try {
    f();
    return GPUSW_OK;
  } catch (const Error& e) {
    c->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    c->err = "host allocation failed";
    return GPUSW_ERR_MEMORY;
  } catch (const std::exception& e) {
    c->err = e.what();
    return GPUSW_ERR_CUDA;
  }
}

__global__ void dpx_rate_kernel(const unsigned* in, unsigned* out, int iters) {
  unsigned x[8], cst[8];
  const unsigned b = in[0];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    x[k] = in[1 + k] + threadIdx.x;
    cst[k] = in[1 + (k & 3)] ^ (threadIdx.x << 3);
  }
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = __viaddmax_s16x2(x[k], b, cst[k]);
  }
  unsigned acc = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) acc ^= x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

}  // namespace

// ================================================================================ C ABI
extern "C" {

int gpusw_version(void) { return 101; }

int gpusw_device_count(int* count) {
  if (!count) return GPUSW_ERR_INVALID;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return GPUSW_OK;
}

int gpusw_ctx_create(int device, gpusw_ctx** out) {
  if (!out) return GPUSW_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    g_create_error = "no CUDA device is available";
    return GPUSW_ERR_NO_GPU;
  }
  if (device < 0 || device >= n) {
    g_create_error = "device ordinal out of range";
    return GPUSW_ERR_INVALID;
  }
  auto* c = new gpusw_ctx();
  c->device = device;
  c->shared.set_held(&c->held);
  c->flush.held = &c->held;
  int rc = guarded(c, [&] {
    set_device(c);
    CK(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&c->ev0, &c->ev1, &c->ev2, &c->ev3}) CK(cudaEventCreate(e));
    CK(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
    for (auto& z : c->zip) {
      CK(cudaEventCreateWithFlags(&z.done, cudaEventDisableTiming));
      z.B.set_held(&c->held);
      z.image.held = &c->held;
    }
    c->zip_iota.held = &c->held;
    for (int i = 0; i < kAuxStreams; ++i) {
      CK(cudaStreamCreateWithFlags(&c->aux[i], cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&c->join_ev[i], cudaEventDisableTiming));
    }
  });
  if (rc != GPUSW_OK) {
    g_create_error = c->err;
    gpusw_ctx_destroy(c);
    return rc;
  }
  *out = c;
  return GPUSW_OK;
}

void gpusw_ctx_destroy(gpusw_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& kv : c->dbs) {
    Db& d = *kv.second;
    for (auto& st : d.streams) {
      cudaFree(st.second.bytes);
      cudaFree(st.second.off);
      cudaFree(st.second.total);
    }
    cudaFree(d.base);
    cudaFree(d.order_base);
  }
  for (int i = 0; i < kAuxStreams; ++i)
    if (c->aux[i]) cudaStreamSynchronize(c->aux[i]);
  for (auto& z : c->zip) {
    if (z.pinned) cudaFreeHost(z.pinned);
    if (z.pinned_out) cudaFreeHost(z.pinned_out);
    for (cudaEvent_t e : z.tev)
      if (e) cudaEventDestroy(e);
    z.image.release();
    z.B.release();
    if (z.done) cudaEventDestroy(z.done);
  }
  c->zip_iota.release();
  c->plans.clear();
  c->shared.release();
  c->flush.release();
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->sub_d) cudaFree(c->sub_d);
  for (cudaEvent_t e : {c->ev0, c->ev1, c->ev2, c->ev3, c->fork_ev})
    if (e) cudaEventDestroy(e);
  for (int i = 0; i < kAuxStreams; ++i) {
    if (c->join_ev[i]) cudaEventDestroy(c->join_ev[i]);
    if (c->aux[i]) cudaStreamDestroy(c->aux[i]);
  }
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* gpusw_last_error(const gpusw_ctx* c) {
  return c ? c->err.c_str() : g_create_error.c_str();
}

int gpusw_set_scheme(gpusw_ctx* c, int mode, int go, int ge, int free_q, int free_r, int ns,
                     const int32_t* sub) {
  return guarded(c, [&] {
    if (mode < 0 || mode > 2) fail(GPUSW_ERR_SCHEME, "mode must be 0 (local), 1 (global) or 2 (semiglobal)");
    if (go > 0 || ge > 0) fail(GPUSW_ERR_SCHEME, "gap_open and gap_extend must be <= 0");
    if (ns < 2 || ns > 256) fail(GPUSW_ERR_SCHEME, "substitution table side must be in [2, 256]");
    if (!sub) fail(GPUSW_ERR_INVALID, "null substitution table");
    if (go < -(1 << 24) || ge < -(1 << 24)) fail(GPUSW_ERR_SCHEME, "gap costs below -2^24 are not supported");
    HostScheme h;
    h.mode = mode;
    h.go = go;
    h.ge = ge;
    h.free_q = free_q ? 1 : 0;
    h.free_r = free_r ? 1 : 0;
    h.ns = ns;
    h.sub.assign(sub, sub + (size_t)ns * ns);
    h.max_sub = *std::max_element(h.sub.begin(), h.sub.end());
    h.min_sub = *std::min_element(h.sub.begin(), h.sub.end());
    if (h.max_sub > (1 << 24) || h.min_sub < -(1 << 24))
      fail(GPUSW_ERR_SCHEME, "substitution scores beyond +/-2^24 are not supported");
    set_device(c);
    if (c->sub_d) cudaFree(c->sub_d);
    c->sub_d = nullptr;
    CK(cudaMalloc(&c->sub_d, h.sub.size() * sizeof(int)));
    CK(cudaMemcpy(c->sub_d, h.sub.data(), h.sub.size() * sizeof(int), cudaMemcpyHostToDevice));
    c->sch = std::move(h);
    c->has_scheme = true;
    c->scheme_version++;
  });
}

int gpusw_db_upload(gpusw_ctx* c, const uint8_t* codes, const int32_t* offsets, int32_t n, int32_t* out_db) {
  return guarded(c, [&] {
    if (!offsets || !out_db || n < 0) fail(GPUSW_ERR_INVALID, "null offsets/handle or negative count");
    if (offsets[0] < 0) fail(GPUSW_ERR_INVALID, "offsets must be non-negative");
    HostTrace tr("db_upload");
    auto d = std::make_unique<Db>();
    d->n = n;
    d->len.resize(n);
    const int nt = host_threads();
    // lengths and their validation (threaded over sequences)
    {
      std::vector<int> tlen(nt + 1, 0), tbad(nt + 1, 0);
      std::atomic<int> slot{0};
      parallel_ranges(n, [&](long long lo, long long hi) {
        int mx = 0, bad = 0;
        for (long long i = lo; i < hi; ++i) {
          const int l = offsets[i + 1] - offsets[i];
          bad |= l < 0;
          d->len[i] = l;
          mx = std::max(mx, l);
        }
        const int t = slot++;
        tlen[t] = mx;
        tbad[t] = bad;
      });
      if (*std::max_element(tbad.begin(), tbad.end()))
        fail(GPUSW_ERR_INVALID, "offsets must be non-decreasing");
      d->max_len = *std::max_element(tlen.begin(), tlen.end());
    }
    const long long total = n ? (long long)offsets[n] - offsets[0] : 0;
    if (total > 0 && !codes) fail(GPUSW_ERR_INVALID, "null codes");
    // largest code (threaded) -> bits per residue
    std::vector<int> tmax(nt + 1, 0);
    {
      const uint8_t* b0 = codes ? codes + offsets[0] : nullptr;
      std::atomic<int> slot{0};
      parallel_ranges(total, [&](long long lo, long long hi) {
        uint8_t m = 0;
        for (long long k = lo; k < hi; ++k) m = std::max(m, b0[k]);
        tmax[slot++] = m;
      });
    }
    const int maxc = *std::max_element(tmax.begin(), tmax.end());
    tr.lap("lengths+max");
    d->max_code = maxc;
    d->bits = maxc < 4 ? 2 : maxc < 16 ? 4 : maxc < 32 ? 5 : 8;
    d->per = d->bits == 5 ? 6 : 32 / d->bits;
    d->woff.resize(n);
    long long w = 0;
    {
      // word offsets: every sequence starts on a 16-byte boundary (threaded two-pass scan)
      const int per = d->per;
      auto words_of = [per](int len) { return ((long long)(len + per - 1) / per + 3) & ~3ll; };
      std::vector<std::pair<long long, long long>> span((size_t)nt + 1, {0, 0});
      std::atomic<int> slot{0};
      parallel_ranges(n, [&](long long lo, long long hi) {
        long long sum = 0;
        for (long long i = lo; i < hi; ++i) sum += words_of(d->len[i]);
        span[slot++] = {lo, sum};
      });
      const int used = slot.load();
      std::sort(span.begin(), span.begin() + used);
      std::vector<std::pair<long long, long long>> start((size_t)used);
      for (int t = 0; t < used; ++t) {
        start[t] = {span[t].first, w};
        w += span[t].second;
      }
      parallel_ranges(n, [&](long long lo, long long hi) {
        // both passes split [0, n) the same way, so `lo` starts one of the first pass's ranges
        auto it = std::lower_bound(start.begin(), start.end(), std::make_pair(lo, LLONG_MIN));
        long long x = 0;
        if (it != start.end() && it->first == lo) {
          x = it->second;
        } else {  // defensive: recount from the start
          for (long long i = 0; i < lo; ++i) x += words_of(d->len[i]);
        }
        for (long long i = lo; i < hi; ++i) {
          d->woff[i] = x;
          x += words_of(d->len[i]);
        }
      });
    }
    const long long nwords = w + 64;  // tail slack for read-ahead
    // one staging image and one device allocation: words | woff (8-byte) | len (4-byte)
    const size_t words_b = (size_t)nwords * 4;
    const size_t woff_o = (words_b + 255) & ~(size_t)255;
    const size_t len_o = woff_o + (((size_t)std::max(1, n) * 8 + 255) & ~(size_t)255);
    const size_t image_b = len_o + (size_t)std::max(1, n) * 4;
    const size_t image_words = (image_b + 3) / 4;
    set_device(c);
    CK(cudaStreamSynchronize(c->stream));  // the staging buffer may still feed a copy
    if (image_words > c->pinned_words) {
      if (c->pinned) cudaFreeHost(c->pinned);
      c->pinned = nullptr;
      c->pinned_words = 0;
      CK(cudaMallocHost(&c->pinned, image_words * 4));
      c->pinned_words = image_words;
    }
    tr.lap("offsets+pinned");
    char* img = reinterpret_cast<char*>(c->pinned);
    CK(cudaMalloc(&d->base, image_b));
    d->words = reinterpret_cast<uint32_t*>(d->base);
    d->woff_d = reinterpret_cast<long long*>(static_cast<char*>(d->base) + woff_o);
    d->len_d = reinterpret_cast<int*>(static_cast<char*>(d->base) + len_o);
    d->bytes = (int64_t)image_b;
    tr.lap("malloc");
    try {
      // The tail (slack words, then word offsets and lengths) is ready first: it goes to
      // the device while the first chunk is packed.
      std::fill(c->pinned + w, c->pinned + nwords, 0u);
      if (n) {
        parallel_ranges(n, [&](long long lo, long long hi) {
          memcpy(img + woff_o + (size_t)lo * 8, d->woff.data() + lo, (size_t)(hi - lo) * 8);
          memcpy(img + len_o + (size_t)lo * 4, d->len.data() + lo, (size_t)(hi - lo) * 4);
        });
      }
      const size_t tail_o = (size_t)w * 4;
      CK(cudaMemcpyAsync(static_cast<char*>(d->base) + tail_o, img + tail_o, image_b - tail_o,
                         cudaMemcpyHostToDevice, c->stream));
      // Pack in a few chunks of sequences: the staging image is page-locked, so each
      // chunk's words go to the device (async, in order on the stream) while the pool
      // packs the next one. A chunk's words are [woff[s0], woff[s1]), contiguous because
      // word offsets increase with the sequence index.
      // offsets are relative to codes[0] in the ABI (like the reference's Encoded)
      const int chunks = n >= (1 << 18) ? 4 : 1;
      for (int k = 0; k < chunks; ++k) {
        const int s0 = (int)((long long)n * k / chunks), s1 = (int)((long long)n * (k + 1) / chunks);
        if (s0 == s1) continue;
        parallel_ranges(s1 - s0, [&](long long lo, long long hi) {
          pack_range(codes, offsets, *d, c->pinned, s0 + (int)lo, s0 + (int)hi);
        });
        const long long w0 = d->woff[s0], w1 = s1 < n ? d->woff[s1] : w;
        if (w1 > w0)
          CK(cudaMemcpyAsync(d->words + w0, c->pinned + w0, (size_t)(w1 - w0) * 4, cudaMemcpyHostToDevice,
                             c->stream));
      }
      tr.lap("pack");
      CK(cudaStreamSynchronize(c->stream));
    } catch (...) {
      cudaStreamSynchronize(c->stream);
      cudaFree(d->base);
      d->base = nullptr;
      throw;
    }
    tr.lap("copy");
    c->held += d->bytes;
    const int h = c->next_db++;
    c->dbs[h] = std::move(d);
    *out_db = h;
  });
}

// ------------------------------------------------------------ packed images (persisted sets)
// A packed set's image is the byte layout db_upload sends to the device: words (the packed
// codes, every sequence 16-byte aligned, then 64 zero slack words) | int64 word offsets |
// int32 lengths, each part starting on a 256-byte boundary.
}  // extern "C"

namespace {

struct ImageLayout {
  size_t words_b = 0, woff_o = 0, len_o = 0, image_b = 0;
};

ImageLayout image_layout(long long nwords, int n) {
  ImageLayout L;
  L.words_b = (size_t)(nwords + 64) * 4;
  L.woff_o = (L.words_b + 255) & ~(size_t)255;
  L.len_o = L.woff_o + (((size_t)std::max(1, n) * 8 + 255) & ~(size_t)255);
  L.image_b = L.len_o + (size_t)std::max(1, n) * 4;
  return L;
}

inline long long words_of(int len, int per) { return ((long long)(len + per - 1) / per + 3) & ~3ll; }

}  // namespace

extern "C" {

int gpusw_pack_image(const uint8_t* codes, const int32_t* offsets, int32_t n, void* image,
                     int64_t image_bytes, int64_t* out_need, int32_t* out_bits, int64_t* out_nwords) {
  try {
    if (!offsets || n < 0 || !out_need || !out_bits || !out_nwords)
      fail(GPUSW_ERR_INVALID, "null offsets/outputs or negative count");
    if (offsets[0] < 0) fail(GPUSW_ERR_INVALID, "offsets must be non-negative");
    Db d;
    d.n = n;
    d.len.resize(n);
    bool bad = false;
    for (int i = 0; i < n; ++i) {
      d.len[i] = offsets[i + 1] - offsets[i];
      bad |= d.len[i] < 0;
      d.max_len = std::max(d.max_len, d.len[i]);
    }
    if (bad) fail(GPUSW_ERR_INVALID, "offsets must be non-decreasing");
    const long long total = n ? (long long)offsets[n] - offsets[0] : 0;
    if (total > 0 && !codes) fail(GPUSW_ERR_INVALID, "null codes");
    std::vector<int> tmax((size_t)host_threads() + 1, 0);
    {
      const uint8_t* b0 = codes ? codes + offsets[0] : nullptr;
      std::atomic<int> slot{0};
      parallel_ranges(total, [&](long long lo, long long hi) {
        uint8_t m = 0;
        for (long long k = lo; k < hi; ++k) m = std::max(m, b0[k]);
        tmax[slot++] = m;
      });
    }
    d.max_code = *std::max_element(tmax.begin(), tmax.end());
    d.bits = d.max_code < 4 ? 2 : d.max_code < 16 ? 4 : d.max_code < 32 ? 5 : 8;
    d.per = d.bits == 5 ? 6 : 32 / d.bits;
    d.woff.resize(n);
    long long w = 0;
    for (int i = 0; i < n; ++i) {
      d.woff[i] = w;
      w += words_of(d.len[i], d.per);
    }
    const ImageLayout L = image_layout(w, n);
    *out_need = (int64_t)L.image_b;
    *out_bits = d.bits;
    *out_nwords = w;
    if (!image) return GPUSW_OK;  // sizing call
    if (image_bytes < (int64_t)L.image_b) fail(GPUSW_ERR_MEMORY, "image buffer too small");
    char* img = static_cast<char*>(image);
    uint32_t* words = reinterpret_cast<uint32_t*>(img);
    memset(img, 0, L.image_b);  // slack words and alignment gaps are zero in every image
    parallel_ranges(n, [&](long long lo, long long hi) {
      pack_range(codes, offsets, d, words, (int)lo, (int)hi);
    });
    if (n) {
      memcpy(img + L.woff_o, d.woff.data(), (size_t)n * 8);
      memcpy(img + L.len_o, d.len.data(), (size_t)n * 4);
    }
    return GPUSW_OK;
  } catch (const Error& e) {
    g_create_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_create_error = "host allocation failed";
    return GPUSW_ERR_MEMORY;
  }
}

int gpusw_db_upload_image(gpusw_ctx* c, const void* image, int64_t image_bytes, int32_t n,
                          int32_t bits, int64_t nwords, int32_t* out_db) {
  return guarded(c, [&] {
    if (!image || !out_db || n < 0 || nwords < 0) fail(GPUSW_ERR_INVALID, "null image/handle or negative count");
    if (bits != 2 && bits != 4 && bits != 5 && bits != 8) fail(GPUSW_ERR_INVALID, "bits must be 2, 4, 5 or 8");
    const ImageLayout L = image_layout(nwords, n);
    if ((size_t)image_bytes != L.image_b) fail(GPUSW_ERR_INVALID, "image size does not match its layout");
    const char* img = static_cast<const char*>(image);
    auto d = std::make_unique<Db>();
    d->n = n;
    d->bits = bits;
    d->per = bits == 5 ? 6 : 32 / bits;
    d->len.resize(n);
    d->woff.resize(n);
    if (n) {
      memcpy(d->len.data(), img + L.len_o, (size_t)n * 4);
      memcpy(d->woff.data(), img + L.woff_o, (size_t)n * 8);
    }
    // the image must describe itself consistently before any kernel reads it
    long long w = 0;
    for (int i = 0; i < n; ++i) {
      if (d->len[i] < 0 || d->woff[i] != w) fail(GPUSW_ERR_INVALID, "corrupt image: offsets or lengths");
      w += words_of(d->len[i], d->per);
      d->max_len = std::max(d->max_len, d->len[i]);
    }
    if (w != nwords) fail(GPUSW_ERR_INVALID, "corrupt image: word count");
    // largest code actually stored (threaded over sequences), checked against the scheme
    // before scoring like an uploaded set's
    const uint32_t* words = reinterpret_cast<const uint32_t*>(img);
    const uint32_t mask = (1u << bits) - 1u;
    std::vector<int> tmax((size_t)host_threads() + 1, 0);
    std::atomic<int> slot{0};
    parallel_ranges_min(n, 256, [&](long long lo, long long hi) {
      uint32_t m = 0;
      for (long long i = lo; i < hi; ++i) {
        const uint32_t* sw = words + d->woff[i];
        for (int cidx = 0; cidx < d->len[i]; ++cidx)
          m = std::max(m, (sw[cidx / d->per] >> ((cidx % d->per) * bits)) & mask);
      }
      tmax[slot++] = (int)m;
    });
    d->max_code = *std::max_element(tmax.begin(), tmax.end());
    set_device(c);
    CK(cudaStreamSynchronize(c->stream));  // the staging buffer may still feed a copy
    const size_t image_words = (L.image_b + 3) / 4;
    if (image_words > c->pinned_words) {
      if (c->pinned) cudaFreeHost(c->pinned);
      c->pinned = nullptr;
      c->pinned_words = 0;
      CK(cudaMallocHost(&c->pinned, image_words * 4));
      c->pinned_words = image_words;
    }
    char* stage = reinterpret_cast<char*>(c->pinned);
    parallel_ranges(L.image_b, [&](long long lo, long long hi) { memcpy(stage + lo, img + lo, (size_t)(hi - lo)); });
    CK(cudaMalloc(&d->base, L.image_b));
    d->words = reinterpret_cast<uint32_t*>(d->base);
    d->woff_d = reinterpret_cast<long long*>(static_cast<char*>(d->base) + L.woff_o);
    d->len_d = reinterpret_cast<int*>(static_cast<char*>(d->base) + L.len_o);
    d->bytes = (int64_t)L.image_b;
    cudaError_t e = cudaMemcpyAsync(d->base, stage, L.image_b, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      cudaFree(d->base);
      d->base = nullptr;
      fail(GPUSW_ERR_CUDA, std::string("image copy: ") + cudaGetErrorString(e));
    }
    c->held += d->bytes;
    const int h = c->next_db++;
    c->dbs[h] = std::move(d);
    *out_db = h;
  });
}

int gpusw_db_free(gpusw_ctx* c, int32_t db) {
  return guarded(c, [&] {
    Db& d = get_db(c, db);
    set_device(c);
    drop_plans_of(c, db);
    for (auto& st : d.streams) {
      cudaFree(st.second.bytes);
      cudaFree(st.second.off);
      cudaFree(st.second.total);
      c->held -= st.second.nbytes;
    }
    cudaFree(d.base);
    cudaFree(d.order_base);
    c->held -= d.bytes;
    c->dbs.erase(db);
  });
}

int gpusw_db_bits(gpusw_ctx* c, int32_t db) {
  int bits = 0;
  int rc = guarded(c, [&] { bits = get_db(c, db).bits; });
  return rc == GPUSW_OK ? bits : -rc;
}

int gpusw_score_cross(gpusw_ctx* c, int32_t qdb, int32_t rdb, const int32_t* qlist, int32_t nq,
                      int dtype, int32_t* out) {
  return guarded(c, [&] {
    Db& q = get_db(c, qdb);
    Db& r = get_db(c, rdb);
    require_scheme(c, q, r);
    ensure_row_order(c, r);
    if (nq < 0 || (nq > 0 && (!qlist || !out))) fail(GPUSW_ERR_INVALID, "null qlist/out");
    int max_n = 0;
    double qsum = 0;
    for (int a = 0; a < nq; ++a) {
      if (qlist[a] < 0 || qlist[a] >= q.n) fail(GPUSW_ERR_INVALID, "query index out of range");
      max_n = std::max(max_n, q.len[qlist[a]]);
      qsum += q.len[qlist[a]];
    }
    begin_call(c);
    const long long total = (long long)nq * r.n;
    const int P = choose_width(c, dtype, max_n, r.max_len);
    if (total > 0) ensure_tuned(c, P);
    const std::vector<long long> key = {0, qdb, rdb, c->scheme_version, P, c->plain | c->stream_multi << 1 | c->inter << 2, nq, 0,
                                        (long long)fnv1a(qlist, (size_t)nq * 4)};
    auto body = [&](Bufs& B) {
      int* d_out = B.out.as<int>(total);
      staged(c, B, false, [&] { run_cross(c, B, q, r, qlist, nq, P, d_out, r.n); });
    };
    CK(cudaEventRecord(c->ev1, c->stream));
    Bufs* B = &execute(c, key, total > 0 && !c->plain, body);
    CK(cudaEventRecord(c->ev2, c->stream));
    if (P == 2 && total > 0) {
      const int n_ovf = read_overflow_count(c, *B);
      c->st.last_overflow = n_ovf;
      if (n_ovf > kOvfCap) {  // too many to rescore one by one: redo everything in int32
        c->shared.reset_marks();
        CK(cudaEventRecord(c->ev1, c->stream));
        int* d_out = c->shared.out.as<int>(total);
        staged(c, c->shared, false, [&] { run_cross(c, c->shared, q, r, qlist, nq, 1, d_out, r.n); });
        CK(cudaEventRecord(c->ev2, c->stream));
        B = &c->shared;
      }
    }
    c->last_bufs = B;
    if (total > 0)
      CK(cudaMemcpyAsync(out, B->out.p, total * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(c->ev3, c->stream));
    double rsum = 0;
    for (int l : r.len) rsum += l;
    c->st.last_cells = qsum * rsum;
    c->st.last_pairs = total;
    end_call(c);
  });
}

int gpusw_topk(gpusw_ctx* c, int32_t qdb, int32_t rdb, const int32_t* qlist, int32_t nq, int32_t k,
               int dtype, int32_t* out_idx, int32_t* out_score) {
  return guarded(c, [&] {
    Db& q = get_db(c, qdb);
    Db& r = get_db(c, rdb);
    require_scheme(c, q, r);
    ensure_row_order(c, r);
    if (k < 0) fail(GPUSW_ERR_INVALID, "k must be >= 0");
    if (nq < 0 || (nq > 0 && !qlist)) fail(GPUSW_ERR_INVALID, "null qlist");
    const int kk = std::min(k, r.n);
    if (nq > 0 && kk > 0 && (!out_idx || !out_score)) fail(GPUSW_ERR_INVALID, "null outputs");
    int max_n = 0;
    double qsum = 0;
    for (int a = 0; a < nq; ++a) {
      if (qlist[a] < 0 || qlist[a] >= q.n) fail(GPUSW_ERR_INVALID, "query index out of range");
      max_n = std::max(max_n, q.len[qlist[a]]);
      qsum += q.len[qlist[a]];
    }
    begin_call(c);
    if (nq > 0 && kk > 0) {
      int P = choose_width(c, dtype, max_n, r.max_len);
      ensure_tuned(c, P);
      const long long row_bytes = (long long)r.n * 4;
      int qb = (int)std::max(1ll, std::min<long long>(nq, c->mem_budget / std::max(1ll, row_bytes)));
      if (c->plain) qb = std::min(qb, 16);
      auto body_w = [&](int Pw) {
        return [&, Pw](Bufs& B) {
          int* d_out = B.out.as<int>((size_t)qb * r.n);
          int* d_idx = B.idx.as<int>((size_t)nq * kk);
          int* d_sc = B.sc.as<int>((size_t)nq * kk);
          for (int b0 = 0; b0 < nq; b0 += qb) {
            const int nb = std::min(qb, nq - b0);
            staged(c, B, false, [&] { run_cross(c, B, q, r, qlist + b0, nb, Pw, d_out, r.n); });
            staged(c, B, true, [&] {
              launch_topk(d_out, nb, r.n, kk, d_idx + (size_t)b0 * kk, d_sc + (size_t)b0 * kk, c->stream);
              c->st.last_launches++;
            });
            if (c->plain && !B.capturing) {  // one batch per call: results back per batch
              CK(cudaMemcpyAsync(out_idx + (size_t)b0 * kk, d_idx + (size_t)b0 * kk, (size_t)nb * kk * 4,
                                 cudaMemcpyDeviceToHost, c->stream));
              CK(cudaMemcpyAsync(out_score + (size_t)b0 * kk, d_sc + (size_t)b0 * kk, (size_t)nb * kk * 4,
                                 cudaMemcpyDeviceToHost, c->stream));
              CK(cudaStreamSynchronize(c->stream));
            }
          }
        };
      };
      const std::vector<long long> key = {1, qdb, rdb, c->scheme_version, P, c->plain | c->stream_multi << 1 | c->inter << 2, nq, kk,
                                          (long long)fnv1a(qlist, (size_t)nq * 4), c->mem_budget};
      CK(cudaEventRecord(c->ev1, c->stream));
      Bufs* B = &execute(c, key, !c->plain, body_w(P));
      CK(cudaEventRecord(c->ev2, c->stream));
      if (P == 2) {
        const int n_ovf = read_overflow_count(c, *B);
        c->st.last_overflow = n_ovf;
        if (n_ovf > kOvfCap) {  // too many to rescore one by one: redo everything in int32
          c->shared.reset_marks();
          CK(cudaEventRecord(c->ev1, c->stream));
          body_w(1)(c->shared);
          CK(cudaEventRecord(c->ev2, c->stream));
          B = &c->shared;
        }
      }
      c->last_bufs = B;
      if (!c->plain) {
        CK(cudaMemcpyAsync(out_idx, B->idx.p, (size_t)nq * kk * 4, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(out_score, B->sc.p, (size_t)nq * kk * 4, cudaMemcpyDeviceToHost, c->stream));
      }
    } else {
      CK(cudaEventRecord(c->ev1, c->stream));
      CK(cudaEventRecord(c->ev2, c->stream));
    }
    CK(cudaEventRecord(c->ev3, c->stream));
    double rsum = 0;
    for (int l : r.len) rsum += l;
    c->st.last_cells = qsum * rsum;
    c->st.last_pairs = (long long)nq * r.n;
    end_call(c);
  });
}

int gpusw_score_pairs(gpusw_ctx* c, int32_t qdb, int32_t rdb, const int32_t* qi, const int32_t* rj,
                      int64_t n, int dtype, int32_t* out) {
  return guarded(c, [&] {
    Db& q = get_db(c, qdb);
    Db& r = get_db(c, rdb);
    require_scheme(c, q, r);
    if (n < 0 || (n > 0 && (!qi || !rj || !out))) fail(GPUSW_ERR_INVALID, "null pair arrays");
    if (n >= (1ll << 31)) fail(GPUSW_ERR_INVALID, "at most 2^31 - 1 pairs per call");
    HostTrace tr("score_pairs");
    int max_n = 0, max_m = 0;
    double cells = 0;
    {
      // validation and extents, threaded; the first bad position is reported
      struct Part { int mn = 0, mm = 0; double cells = 0; int64_t bad = -1; };
      std::vector<Part> part((size_t)host_threads() + 1);
      std::atomic<int> slot{0};
      parallel_ranges(n, [&](long long lo, long long hi) {
        Part pt;
        for (long long i = lo; i < hi; ++i) {
          if (qi[i] < 0 || qi[i] >= q.n || rj[i] < 0 || rj[i] >= r.n) {
            pt.bad = i;
            break;
          }
          const int ql = q.len[qi[i]], rl = r.len[rj[i]];
          pt.mn = std::max(pt.mn, ql);
          pt.mm = std::max(pt.mm, rl);
          pt.cells += (double)ql * rl;
        }
        part[slot++] = pt;
      });
      int64_t bad = -1;
      for (const Part& pt : part) {
        if (pt.bad >= 0 && (bad < 0 || pt.bad < bad)) bad = pt.bad;
        max_n = std::max(max_n, pt.mn);
        max_m = std::max(max_m, pt.mm);
        cells += pt.cells;
      }
      if (bad >= 0) fail(GPUSW_ERR_INVALID, "pair index out of range at position " + std::to_string(bad));
    }
    begin_call(c);
    const HostScheme& h = c->sch;
    const bool local = h.mode == gsw::kModeLocal;
    int P = n > 0 ? choose_width(c, dtype, max_n, max_m) : 1;
    const std::vector<long long> key = {2, qdb, rdb, c->scheme_version, P, c->plain | c->stream_multi << 1 | c->inter << 2, (long long)n, 0,
                                        (long long)fnv1a(rj, (size_t)n * 4, fnv1a(qi, (size_t)n * 4))};
    Bufs* B = nullptr;
    tr.lap("validate+key");
    CK(cudaEventRecord(c->ev1, c->stream));
    // Plans the call on the host and runs it (recorded as a graph when cacheable).
    auto plan_and_run = [&](int Pw, bool cacheable) -> Bufs* {
        // Short alignments (query lengths of inter_len) through the inter-sequence kernel when it
        // applies and pays; they take the excluded shape kNumPair below.
        InterPlan ipl;
        bool use_inter = false;
        if (inter_applies(c, q, r, Pw)) {
          std::vector<int> cand;
          for (int64_t i = 0; i < n; ++i)
            if (inter_len(q.len[qi[i]])) cand.push_back((int)i);
          if (!cand.empty()) {
            ipl = plan_inter(q, r, qi, rj, cand, local);
            use_inter = inter_pays(c, ipl);
          }
        }
        // Plan (host, O(n), threaded): kernel shape per alignment from its column length, then
        // a stable order by (shape, row length descending) so int16x2 partners share a shape
        // and, mostly, a row length: the input order when it already is one (checked), else a
        // counting sort on that key (a two-pass radix sort when the key range is wide).
        std::vector<int> order((size_t)n);
        std::vector<uint8_t> shp((size_t)n);
        const int plain_shape = c->plain ? pick_pair_shape(std::max(1, max_n), h.ns) : 0;
        std::vector<int> shape_of_len(4097);
        for (int L = 0; L <= 4096; ++L) shape_of_len[L] = pick_pair_shape(std::max(1, L), h.ns);
        const int big = pick_pair_shape(1 << 30, h.ns);
        struct Part {
          long long lo = 0, hi = 0;
          bool sorted = true;
          int mrow[kNumPair + 1] = {}, mcol[kNumPair + 1] = {};
          long long cnt[kNumPair + 1] = {};
        };
        std::vector<Part> part((size_t)host_threads() + 1);
        std::atomic<int> slot{0};
        auto key_of = [&](int64_t i) {
          return ((uint32_t)shp[i] << 24) | (0xFFFFFFu - (uint32_t)std::min(r.len[rj[i]], 0xFFFFFF));
        };
        parallel_ranges(n, [&](long long lo, long long hi) {
          Part pt;
          pt.lo = lo;
          pt.hi = hi;
          uint32_t prev = 0;
          for (long long i = lo; i < hi; ++i) {
            const int ql = q.len[qi[i]], rl = r.len[rj[i]];
            const int sh = c->plain ? plain_shape
                                    : (use_inter && inter_len(ql)) ? kNumPair
                                    : (ql <= 4096 ? shape_of_len[ql] : big);
            shp[i] = (uint8_t)sh;
            pt.mrow[sh] = std::max(pt.mrow[sh], rl);
            pt.mcol[sh] = std::max(pt.mcol[sh], ql);
            pt.cnt[sh]++;
            const uint32_t k = key_of(i);
            if (i > lo && k < prev) pt.sorted = false;
            prev = k;
          }
          part[slot++] = pt;
        });
        const int used = slot.load();
        std::sort(part.begin(), part.begin() + used, [](const Part& a, const Part& b) { return a.lo < b.lo; });
        bool sorted = true;
        int mrow[kNumPair + 1] = {}, mcol[kNumPair + 1] = {};
        long long cnt[kNumPair + 1] = {};
        for (int t = 0; t < used; ++t) {
          const Part& pt = part[t];
          sorted &= pt.sorted;
          if (t > 0 && pt.hi > pt.lo && part[t - 1].hi > part[t - 1].lo &&
              key_of(pt.lo) < key_of(part[t - 1].hi - 1))
            sorted = false;
          for (int sh = 0; sh <= kNumPair; ++sh) {
            mrow[sh] = std::max(mrow[sh], pt.mrow[sh]);
            mcol[sh] = std::max(mcol[sh], pt.mcol[sh]);
            cnt[sh] += pt.cnt[sh];
          }
        }
        if (c->plain || sorted) {
          std::iota(order.begin(), order.end(), 0);
        } else {
          const int mm = std::min(max_m, 0xFFFFFF);
          const size_t nb = (size_t)(kNumPair + 1) * ((size_t)mm + 1);
          if (nb <= (size_t)4 * n + 65536) {  // stable counting sort on (shape, mm - row length)
            auto bucket = [&](int64_t i) {
              return (size_t)shp[i] * ((size_t)mm + 1) + (size_t)(mm - std::min(r.len[rj[i]], 0xFFFFFF));
            };
            std::vector<int64_t> bc(nb + 1, 0);
            for (int64_t i = 0; i < n; ++i) bc[bucket(i) + 1]++;
            for (size_t bk = 0; bk < nb; ++bk) bc[bk + 1] += bc[bk];
            for (int64_t i = 0; i < n; ++i) order[bc[bucket(i)]++] = (int)i;
          } else {
            std::vector<int> tmp((size_t)n);
            std::iota(tmp.begin(), tmp.end(), 0);
            std::vector<int64_t> rc(65537);
            for (int pass = 0; pass < 2; ++pass) {
              const int sh = pass * 16;
              std::fill(rc.begin(), rc.end(), 0);
              for (int64_t i = 0; i < n; ++i) rc[((key_of(tmp[i]) >> sh) & 0xFFFF) + 1]++;
              for (int bkt = 0; bkt < 65536; ++bkt) rc[bkt + 1] += rc[bkt];
              for (int64_t i = 0; i < n; ++i) order[rc[(key_of(tmp[i]) >> sh) & 0xFFFF]++] = tmp[i];
              if (pass == 0) tmp.swap(order);
            }
          }
        }
        struct Bin { int64_t i0, i1; int shape, mrow, mcol; };
        std::vector<Bin> plan_bins;
        {
          int64_t i0 = 0;
          for (int sh = 0; sh < kNumPair; ++sh) {  // shape kNumPair (inter-sequence) sorts last
            if (!cnt[sh]) continue;
            plan_bins.push_back({i0, i0 + cnt[sh], sh, mrow[sh], mcol[sh]});
            i0 += cnt[sh];
          }
        }
        tr.lap("plan");
        Staging stg;  // qi, rj, order and the inter items stay alive until the eager run has uploaded them
        const size_t o_qi = stg.add_ref(qi, (size_t)n * 4), o_rj = stg.add_ref(rj, (size_t)n * 4);
        const size_t o_ord = stg.add_ref(order.data(), (size_t)n * 4);
        const size_t o_it = use_inter ? stg.add_ref(ipl.items.data(), ipl.items.size() * sizeof(int2)) : 0;
        const int nb_team = (int)plan_bins.size();
        auto run = [&](int Pw) {
          return [&, Pw](Bufs& Bx) {
            char* dm = stg.upload(c, Bx);
            int* d_out = Bx.out.as<int>((size_t)n);
            Bx.inter_items = use_inter ? (long long)ipl.items.size() : 0;
            const int nslots = nb_team + 3;  // team bins, the overflow rescoring, the inter launch
            unsigned long long* queues = Bx.queue.as<unsigned long long>(nslots);
            staged(c, Bx, false, [&] {
              CK(cudaMemsetAsync(queues, 0, nslots * sizeof(unsigned long long), c->stream));
              if (Pw == 2) CK(cudaMemsetAsync(Bx.ovf_count.as<int>(1), 0, sizeof(int), c->stream));
              gsw::PairsParams pp{};
              pp.S = make_scheme(h, Pw);
              pp.sub = c->sub_d;
              pp.cols = q.packed();
              pp.rows = r.packed();
              pp.qi = reinterpret_cast<const int*>(dm + o_qi);
              pp.rj = reinterpret_cast<const int*>(dm + o_rj);
              pp.item_mode = 0;
              pp.out = d_out;
              pp.ovf = Bx.ovf.as<gsw::Ovf>(kOvfCap);
              pp.ovf_count = Bx.ovf_count.as<int>(1);
              pp.ovf_cap = kOvfCap;
              gsw::InterParams ip{};
              if (use_inter) {
                ip.S = pp.S;
                ip.sub = c->sub_d;
                ip.cols = pp.cols;
                ip.rows = pp.rows;
                ip.qi = pp.qi;
                ip.rj = pp.rj;
                ip.items = reinterpret_cast<const int2*>(dm + o_it);
                ip.n_items = (long long)ipl.items.size();
                ip.queue = queues + nb_team + 1;
                ip.out = d_out;
                ip.ovf = pp.ovf;
                ip.ovf_count = pp.ovf_count;
                ip.ovf_cap = kOvfCap;
              }
              run_group(c, Bx, nb_team + (use_inter ? 1 : 0), [&](int bi, const LaunchCfg& lc) {
                if (bi == nb_team) {
                  launch_inter(c, Bx, ip, ipl.max_n, ipl.max_m, lc);
                  return;
                }
                const Bin& bn = plan_bins[bi];
                gsw::PairsParams lp = pp;
                lp.order = reinterpret_cast<const int*>(dm + o_ord) + bn.i0;
                lp.n_align = bn.i1 - bn.i0;
                lp.n_items = (lp.n_align + Pw - 1) / Pw;
                lp.queue = queues + bi;
                launch_pairs(c, Bx, bn.shape, Pw, local, lp, bn.mrow, bn.mcol > kPairShapes[bn.shape].cap(), lc);
              });
              if (Pw == 2) launch_overflow_rescore(c, Bx, q, r, d_out, queues + nb_team);
            });
          };
        };
        return &execute(c, key, cacheable, run(Pw));
    };
    if (n > 0) {
      Plan* hit = c->plain ? nullptr : lookup(c, key);
      B = hit ? &replay(c, hit) : plan_and_run(P, !c->plain);
      tr.lap(hit ? "replay" : "run");
      c->st.last_inter_items = B->inter_items;
      if (P == 2) {
        const int n_ovf = read_overflow_count(c, *B);
        c->st.last_overflow = n_ovf;
        if (n_ovf > kOvfCap) {  // too many flagged cells: all int32
          B = plan_and_run(1, false);
          c->st.last_inter_items = 0;
        }
      }
    }
    c->last_bufs = B;
    CK(cudaEventRecord(c->ev2, c->stream));
    if (n > 0) CK(cudaMemcpyAsync(out, B->out.p, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(c->ev3, c->stream));
    c->st.last_cells = cells;
    c->st.last_pairs = n;
    end_call(c);
    tr.lap("finish");
  });
}

}  // extern "C"

// ============================================================ zipped pairs, pipelined
namespace {

// One chunk of a zipped pair set: pairs [a, b) as two chunk-local packed sets, the launch
// order (by shape, then row length descending) and its bins. Kept until the chunk's results
// are read, so a chunk whose int16 overflow list filled up can be scored again in int32.
struct ZipChunk {
  long long a = 0, b = 0;
  Db q, r;
  std::vector<int> order;
  std::vector<uint8_t> shp;
  struct Bin { long long i0, i1; int shape, mrow, mcol; };
  std::vector<Bin> bins;
  size_t off_order = 0, image_bytes = 0;
  int P = 2;
  int bits_guess[2] = {2, 2};  // packing widths to try first (the previous chunk's)
};

constexpr long long kZipChunk = 1 << 17;  // pairs per pipeline chunk

// Host half of a chunk, written into the slot's page-locked image (layout: q words | r words |
// q woff | r woff | q len | r len | order, each 256-byte aligned), in two threaded passes over
// the chunk's pairs: (1) lengths, kernel shapes (shape_of[length], or plain_shape), the
// largest code of each side, word counts at every packing width, bin extents and whether the
// input is already in launch order (by shape, row length descending); (2) word offsets, the
// packed words of both sides and the metadata. Only a chunk that is out of order is sorted,
// by a stable counting sort on one thread.
void zip_prepare(gpusw_ctx* c, gpusw_ctx::ZipSlot& z, ZipChunk& ch, const uint8_t* qc,
                 const int32_t* qo, const uint8_t* rc, const int32_t* ro,
                 const std::vector<uint8_t>& shape_of, int big_shape, int plain_shape, HostTrace& tr) {
  const int nc = (int)(ch.b - ch.a);
  const HostScheme& h = c->sch;
  Db* sets[2] = {&ch.q, &ch.r};
  const uint8_t* codes[2] = {qc, rc};
  const int32_t* offs[2] = {qo + ch.a, ro + ch.a};
  for (Db* d : sets) {
    d->n = nc;
    d->len.resize(nc);
    d->woff.resize(nc);
  }
  ch.shp.resize(nc);
  constexpr int kPer[4] = {16, 8, 6, 4};  // codes per word at 2, 4, 5, 8 bits
  struct P1 {
    long long lo = 0, hi = 0;
    int maxlen[2] = {0, 0};
    long long words[2][4] = {};
    int cnt[kNumPair] = {}, mrow[kNumPair] = {}, mcol[kNumPair] = {};
    bool sorted = true;
  };
  const int nt = host_threads() + 1;
  std::vector<P1> p1((size_t)nt);
  std::atomic<int> slot{0};
  auto before = [&](int i, int j) {  // pair j may follow pair i in launch order
    const int si = ch.shp[i], sj = ch.shp[j];
    return si < sj || (si == sj && std::min(ch.r.len[j], 65535) <= std::min(ch.r.len[i], 65535));
  };
  parallel_ranges_min(nc, 4096, [&](long long lo, long long hi) {
    P1 pt;
    pt.lo = lo;
    pt.hi = hi;
    for (int k = 0; k < 2; ++k) {
      Db& d = *sets[k];
      const int32_t* o = offs[k];
      for (long long i = lo; i < hi; ++i) {
        const int l = o[i + 1] - o[i];
        d.len[i] = l;
        pt.maxlen[k] = std::max(pt.maxlen[k], l);
        for (int w = 0; w < 4; ++w) pt.words[k][w] += words_of(l, kPer[w]);
      }
    }
    for (long long i = lo; i < hi; ++i) {
      const int ql = ch.q.len[i], rl = ch.r.len[i];
      const int sh = plain_shape >= 0 ? plain_shape : (ql < (int)shape_of.size() ? shape_of[ql] : big_shape);
      ch.shp[i] = (uint8_t)sh;
      pt.cnt[sh]++;
      pt.mrow[sh] = std::max(pt.mrow[sh], rl);
      pt.mcol[sh] = std::max(pt.mcol[sh], ql);
      if (i > lo && !before((int)i - 1, (int)i)) pt.sorted = false;
    }
    p1[slot++] = pt;
  });
  const int used = slot.load();
  std::sort(p1.begin(), p1.begin() + used, [](const P1& a, const P1& b) { return a.lo < b.lo; });
  bool sorted = c->plain != 0;
  int cnt[kNumPair] = {}, mrow[kNumPair] = {}, mcol[kNumPair] = {};
  for (int t = 0; t < used; ++t) {
    const P1& pt = p1[t];
    if (!c->plain) {
      sorted = (t == 0 ? true : sorted) && pt.sorted;
      if (t > 0 && pt.hi > pt.lo && p1[t - 1].hi > p1[t - 1].lo && !before((int)p1[t - 1].hi - 1, (int)pt.lo))
        sorted = false;
    }
    for (int k = 0; k < 2; ++k) sets[k]->max_len = std::max(t ? sets[k]->max_len : 0, pt.maxlen[k]);
    for (int sh = 0; sh < kNumPair; ++sh) {
      cnt[sh] += pt.cnt[sh];
      mrow[sh] = std::max(mrow[sh], pt.mrow[sh]);
      mcol[sh] = std::max(mcol[sh], pt.mcol[sh]);
    }
  }
  if (nc == 0)
    for (Db* d : sets) d->max_len = 0;
  // packing widths: the guess (the previous chunk's widths), corrected after packing when the
  // OR of the codes shows a wider one is needed (the chunk is then packed again)
  long long wtotal[2];
  std::vector<long long> wstart[2];
  auto set_width = [&](int k, int bits) {
    Db& d = *sets[k];
    d.bits = bits;
    d.per = bits == 5 ? 6 : 32 / bits;
    const int widx = bits == 2 ? 0 : bits == 4 ? 1 : bits == 5 ? 2 : 3;
    wstart[k].resize((size_t)used);
    long long w = 0;
    for (int t = 0; t < used; ++t) {
      wstart[k][t] = w;
      w += p1[t].words[k][widx];
    }
    wtotal[k] = w;
  };
  for (int k = 0; k < 2; ++k) set_width(k, ch.bits_guess[k]);
  tr.lap("chunk: lengths, shapes");
  // launch order and bins
  ch.order.resize(nc);
  const bool identity = sorted;
  if (!identity) {  // stable counting sort on (shape, row length descending)
    const int mm = std::min(ch.r.max_len, 65535);
    auto key = [&](int i) { return (size_t)ch.shp[i] * (size_t)(mm + 1) + (size_t)(mm - std::min(ch.r.len[i], mm)); };
    std::vector<int> bc((size_t)kNumPair * (mm + 1) + 1, 0);
    for (int i = 0; i < nc; ++i) bc[key(i) + 1]++;
    for (size_t k = 0; k + 1 < bc.size(); ++k) bc[k + 1] += bc[k];
    for (int i = 0; i < nc; ++i) ch.order[bc[key(i)]++] = i;
  }
  ch.bins.clear();
  long long i0 = 0;
  for (int sh = 0; sh < kNumPair; ++sh) {
    if (!cnt[sh]) continue;
    ch.bins.push_back({i0, i0 + cnt[sh], sh, mrow[sh], mcol[sh]});
    i0 += cnt[sh];
  }
  // image layout (it depends on the widths), then pass 2: word offsets, packed words and
  // metadata, over the same ranges as pass 1, with the OR of each side's codes
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t o_w[2], o_wo[2], o_l[2];
  uint8_t side_or[2] = {0, 0};
  auto pack_pass = [&]() {
    const size_t words_b[2] = {(size_t)(wtotal[0] + 64) * 4, (size_t)(wtotal[1] + 64) * 4};
    o_w[0] = 0;
    o_w[1] = al(words_b[0]);
    o_wo[0] = al(o_w[1] + words_b[1]);
    o_wo[1] = al(o_wo[0] + (size_t)nc * 8);
    o_l[0] = al(o_wo[1] + (size_t)nc * 8);
    o_l[1] = al(o_l[0] + (size_t)nc * 4);
    ch.off_order = al(o_l[1] + (size_t)nc * 4);
    ch.image_bytes = ch.off_order + (size_t)std::max(nc, 1) * 4;
    if (ch.image_bytes > z.pinned_bytes) {
      if (z.pinned) cudaFreeHost(z.pinned);
      z.pinned = nullptr;
      z.pinned_bytes = 0;
      const size_t want = ch.image_bytes + (ch.image_bytes >> 3);  // chunks differ a little
      CK(cudaMallocHost(reinterpret_cast<void**>(&z.pinned), want));
      z.pinned_bytes = want;
    }
    char* img = z.pinned;
    for (int k = 0; k < 2; ++k) {
      uint32_t* words = reinterpret_cast<uint32_t*>(img + o_w[k]);
      std::fill(words + wtotal[k], words + wtotal[k] + 64, 0u);
    }
    std::vector<std::array<uint8_t, 2>> ors((size_t)nt, {0, 0});
    std::atomic<int> oslot{0};
    parallel_ranges_min(nc, 4096, [&](long long lo, long long hi) {
      std::array<uint8_t, 2> o = {0, 0};
      const int t = (int)(std::lower_bound(p1.begin(), p1.begin() + used, lo,
                                           [](const P1& a, long long v) { return a.lo < v; }) - p1.begin());
      for (int k = 0; k < 2; ++k) {
        Db& d = *sets[k];
        long long w = t < used && p1[t].lo == lo ? wstart[k][t] : 0;
        if (!(t < used && p1[t].lo == lo))  // defensive: the split differs, recount
          for (long long i = 0; i < lo; ++i) w += words_of(d.len[i], d.per);
        for (long long i = lo; i < hi; ++i) {
          d.woff[i] = w;
          w += words_of(d.len[i], d.per);
        }
        pack_range(codes[k], offs[k], d, reinterpret_cast<uint32_t*>(img + o_w[k]), (int)lo, (int)hi, &o[k]);
        memcpy(img + o_wo[k] + (size_t)lo * 8, d.woff.data() + lo, (size_t)(hi - lo) * 8);
        memcpy(img + o_l[k] + (size_t)lo * 4, d.len.data() + lo, (size_t)(hi - lo) * 4);
      }
      int* ord = reinterpret_cast<int*>(img + ch.off_order);
      if (identity)
        for (long long i = lo; i < hi; ++i) ord[i] = (int)i;
      else
        memcpy(ord + lo, ch.order.data() + lo, (size_t)(hi - lo) * 4);
      ors[oslot++] = o;
    });
    side_or[0] = side_or[1] = 0;
    for (int x = 0; x < oslot.load(); ++x)
      for (int k = 0; k < 2; ++k) side_or[k] |= ors[x][k];
  };
  pack_pass();
  tr.lap("chunk: pack");
  // the width each side needs (the OR has a bit at or above 2, 4 or 5 exactly when some code
  // does); a side packed too narrow is packed again, and the next chunk starts from it
  auto need_bits = [](uint8_t o) { return o < 4 ? 2 : o < 16 ? 4 : o < 32 ? 5 : 8; };
  bool again = false;
  for (int k = 0; k < 2; ++k) {
    const int nb = sets[k]->bits == 8 ? 8 : need_bits(side_or[k]);
    if (nb > sets[k]->bits) {
      set_width(k, nb);
      again = true;
    }
  }
  if (again) pack_pass();
  for (int k = 0; k < 2; ++k) {
    Db& d = *sets[k];
    ch.bits_guess[k] = d.bits;
    // the codes must index the scheme's table: the OR bounds the largest code; at 8 bits (the
    // whole words are copied, not ORed) or when the bound reaches the table, scan exactly
    int mx = side_or[k];
    if (d.bits == 8 || mx >= h.ns) {
      const int32_t* o = offs[k];
      const uint8_t* b0 = codes[k] + o[0];
      std::vector<int> tmax((size_t)nt, 0);
      std::atomic<int> sl{0};
      parallel_ranges((long long)o[nc] - o[0], [&](long long lo, long long hi) {
        uint8_t m = 0;
        for (long long x = lo; x < hi; ++x) m = std::max(m, b0[x]);
        tmax[sl++] = m;
      });
      mx = *std::max_element(tmax.begin(), tmax.end());
    }
    d.max_code = mx;
    if (d.max_code >= h.ns) fail(GPUSW_ERR_INVALID, "sequence codes exceed the scheme's substitution table");
  }
  for (int k = 0; k < 2; ++k)  // the two passes agreed on the word layout
    if (nc > 0 && sets[k]->woff[nc - 1] + words_of(sets[k]->len[nc - 1], sets[k]->per) != wtotal[k])
      fail(GPUSW_ERR_CUDA, "internal error: packed chunk layout mismatch");
  // device view of the image (filled by the slot's copy); grown with an eighth of headroom
  if (ch.image_bytes > z.image.bytes) z.image.get(ch.image_bytes + (ch.image_bytes >> 3));
  char* dimg = static_cast<char*>(z.image.p);
  for (int k = 0; k < 2; ++k) {
    Db& d = *sets[k];
    d.words = reinterpret_cast<uint32_t*>(dimg + o_w[k]);
    d.woff_d = reinterpret_cast<long long*>(dimg + o_wo[k]);
    d.len_d = reinterpret_cast<int*>(dimg + o_l[k]);
  }
}

// Device half of a chunk on stream st: the image copy (unless already resident), the
// kernels of every bin, int16 overflow rescoring, and the copy of the scores (and of the
// overflow count) into page-locked memory; then the slot's completion event.
void zip_issue(gpusw_ctx* c, gpusw_ctx::ZipSlot& z, const ZipChunk& ch, int P, cudaStream_t st,
               bool copy_image) {
  const int nc = (int)(ch.b - ch.a);
  const HostScheme& h = c->sch;
  const bool local = h.mode == gsw::kModeLocal;
  Bufs& B = z.B;
  char* dimg = static_cast<char*>(z.image.p);
  const bool tr = HostTrace::enabled();
  if (tr && !z.tev[0])
    for (cudaEvent_t& e : z.tev) CK(cudaEventCreate(&e));
  if (tr) CK(cudaEventRecord(z.tev[0], st));
  if (copy_image) CK(cudaMemcpyAsync(dimg, z.pinned, ch.image_bytes, cudaMemcpyHostToDevice, st));
  if (tr) CK(cudaEventRecord(z.tev[1], st));
  const int nslots = (int)ch.bins.size() + 2;
  unsigned long long* queues = B.queue.as<unsigned long long>(nslots);
  int* d_out = B.out.as<int>((size_t)nc);
  int* ovf_flag = B.ovf_flag.as<int>(1);
  gsw::PairsParams pp{};
  pp.S = make_scheme(h, P);
  pp.sub = c->sub_d;
  pp.cols = ch.q.packed();
  pp.rows = ch.r.packed();
  pp.qi = static_cast<const int*>(c->zip_iota.p);
  pp.rj = pp.qi;
  pp.item_mode = 0;
  pp.out = d_out;
  pp.ovf = B.ovf.as<gsw::Ovf>(kOvfCap);
  pp.ovf_count = B.ovf_count.as<int>(1);
  pp.ovf_cap = kOvfCap;
  const int* d_order = reinterpret_cast<const int*>(dimg + ch.off_order);
  // strips of every launch side by side (a sizing pass first), all on this stream
  const int nb = (int)ch.bins.size();
  std::vector<long long> off((size_t)nb + 1, -1);
  size_t total = 0;
  auto bin_launch = [&](int bi, const LaunchCfg& lc) {
    const ZipChunk::Bin& bn = ch.bins[bi];
    gsw::PairsParams lp = pp;
    lp.order = d_order + bn.i0;
    lp.n_align = bn.i1 - bn.i0;
    lp.n_items = (lp.n_align + P - 1) / P;
    lp.queue = queues + bi;
    launch_pairs(c, B, bn.shape, P, local, lp, bn.mrow, bn.mcol > kPairShapes[bn.shape].cap(), lc);
  };
  for (int bi = 0; bi <= nb; ++bi) {
    size_t need = 0;
    LaunchCfg sz;
    sz.need = &need;
    if (bi < nb) bin_launch(bi, sz);
    else if (P == 2) launch_overflow_rescore(c, B, ch.q, ch.r, d_out, queues + nb, sz);
    if (need) {
      off[bi] = (long long)total;
      total += need;
    }
  }
  if (total) B.bnd.as<uint2>(total);
  CK(cudaMemsetAsync(queues, 0, nslots * sizeof(unsigned long long), st));
  CK(cudaMemsetAsync(ovf_flag, 0, sizeof(int), st));
  if (P == 2) CK(cudaMemsetAsync(pp.ovf_count, 0, sizeof(int), st));
  for (int bi = 0; bi < nb; ++bi) {
    LaunchCfg lc;
    lc.st = st;
    lc.bnd_off = off[bi];
    bin_launch(bi, lc);
  }
  if (P == 2) {
    LaunchCfg lc;
    lc.st = st;
    lc.bnd_off = off[nb];
    launch_overflow_rescore(c, B, ch.q, ch.r, d_out, queues + nb, lc);
  }
  if (tr) CK(cudaEventRecord(z.tev[2], st));
  CK(cudaMemcpyAsync(z.pinned_out, d_out, (size_t)nc * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(z.pinned_out + nc, ovf_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (tr) CK(cudaEventRecord(z.tev[3], st));
  CK(cudaEventRecord(z.done, st));
}

}  // namespace

extern "C" {

int gpusw_score_pairs_zip(gpusw_ctx* c, const uint8_t* q_codes, const int32_t* q_offsets,
                          const uint8_t* r_codes, const int32_t* r_offsets, int64_t n, int dtype,
                          int32_t* out) {
  constexpr int kSlots = 3;  // chunks in flight: the host packs one while two are on the GPU
  cudaStream_t streams[kSlots] = {c ? c->stream : nullptr, c ? c->aux[0] : nullptr, c ? c->aux[1] : nullptr};
  return guarded(c, [&] {
    if (!c->has_scheme) fail(GPUSW_ERR_SCHEME, "no scheme set (call gpusw_set_scheme first)");
    if (n < 0 || (n > 0 && (!q_offsets || !r_offsets || !out))) fail(GPUSW_ERR_INVALID, "null arrays or negative count");
    if (n >= (1ll << 31)) fail(GPUSW_ERR_INVALID, "at most 2^31 - 1 pairs per call");
    if (n > 0 && (q_offsets[0] < 0 || r_offsets[0] < 0)) fail(GPUSW_ERR_INVALID, "offsets must be non-negative");
    HostTrace tr("score_pairs_zip");
    // lengths of every pair: validation, extents and cells (threaded)
    int max_n = 0, max_m = 0;
    double cells = 0;
    {
      struct Part { int mn = 0, mm = 0; double cells = 0; bool bad = false; };
      std::vector<Part> part((size_t)host_threads() + 1);
      std::atomic<int> slot{0};
      parallel_ranges(n, [&](long long lo, long long hi) {
        Part pt;
        for (long long i = lo; i < hi; ++i) {
          const int ql = q_offsets[i + 1] - q_offsets[i], rl = r_offsets[i + 1] - r_offsets[i];
          pt.bad |= ql < 0 || rl < 0;
          pt.mn = std::max(pt.mn, ql);
          pt.mm = std::max(pt.mm, rl);
          pt.cells += (double)ql * rl;
        }
        part[slot++] = pt;
      });
      for (const Part& pt : part) {
        if (pt.bad) fail(GPUSW_ERR_INVALID, "offsets must be non-decreasing");
        max_n = std::max(max_n, pt.mn);
        max_m = std::max(max_m, pt.mm);
        cells += pt.cells;
      }
    }
    if (n > 0 && ((q_offsets[n] > q_offsets[0] && !q_codes) || (r_offsets[n] > r_offsets[0] && !r_codes)))
      fail(GPUSW_ERR_INVALID, "null codes");
    begin_call(c);
    c->last_bufs = nullptr;
    CK(cudaEventRecord(c->ev1, c->stream));
    const int P = n > 0 ? choose_width(c, dtype, max_n, max_m) : 1;
    const long long chunk = std::min<long long>(kZipChunk, std::max<long long>(1, n));
    if (n > 0 && c->zip_iota_n < chunk) {
      std::vector<int> io((size_t)chunk);
      std::iota(io.begin(), io.end(), 0);
      CK(cudaMemcpy(c->zip_iota.get((size_t)chunk * 4), io.data(), (size_t)chunk * 4, cudaMemcpyHostToDevice));
      c->zip_iota_n = chunk;
    }
    // kernel shape of every column length up to 4,096 (longer ones: the widest shape)
    std::vector<uint8_t> shape_of(4097);
    for (int L = 0; L <= 4096; ++L) shape_of[L] = (uint8_t)pick_pair_shape(std::max(1, L), c->sch.ns);
    const int big_shape = pick_pair_shape(1 << 30, c->sch.ns);
    const int plain_shape = c->plain ? pick_pair_shape(std::max(1, max_n), c->sch.ns) : -1;
    tr.lap("validate");
    ZipChunk chs[kSlots];
    const long long K = (n + chunk - 1) / chunk;
    const int used_slots = (int)std::min<long long>(kSlots, std::max(1ll, K));
    if (used_slots > 1) {  // the other streams start after the work already on the first
      CK(cudaEventRecord(c->fork_ev, c->stream));
      for (int sl = 1; sl < used_slots; ++sl) CK(cudaStreamWaitEvent(streams[sl], c->fork_ev, 0));
    }
    // results of the chunk in slot s: copied out, or scored again in int32 if its overflow
    // list was full
    auto finish = [&](int sl) {
      gpusw_ctx::ZipSlot& z = c->zip[sl];
      ZipChunk& ch = chs[sl];
      CK(cudaEventSynchronize(z.done));
      const int nc = (int)(ch.b - ch.a);
      if (HostTrace::enabled() && z.tev[0]) {
        float a = 0, b = 0, d = 0, g = 0;
        cudaEventElapsedTime(&a, z.tev[0], z.tev[1]);
        cudaEventElapsedTime(&b, z.tev[1], z.tev[2]);
        cudaEventElapsedTime(&d, z.tev[2], z.tev[3]);
        cudaEventElapsedTime(&g, c->ev1, z.tev[0]);
        std::fprintf(stderr, "[gpusw] zip chunk %lld slot %d: starts %.3f ms after the call, copy in %.3f, kernels %.3f, copy out %.3f ms\n",
                     ch.a / kZipChunk, sl, g, a, b, d);
      }
      if (ch.P == 2 && z.pinned_out[nc] > kOvfCap) {
        ch.P = 1;
        zip_issue(c, z, ch, 1, streams[sl], false);
        CK(cudaEventSynchronize(z.done));
      }
      c->st.last_overflow = std::max<int64_t>(c->st.last_overflow, z.pinned_out[nc]);
      memcpy(out + ch.a, z.pinned_out, (size_t)nc * 4);
    };
    try {
      for (long long k = 0; k < K; ++k) {
        const int sl = (int)(k % kSlots);
        gpusw_ctx::ZipSlot& z = c->zip[sl];
        if (k >= kSlots) finish(sl);
        tr.lap("chunk: wait for the slot");
        ZipChunk& ch = chs[sl];
        ch.a = k * chunk;
        ch.b = std::min<long long>(n, ch.a + chunk);
        ch.P = P;
        const size_t nc = (size_t)(ch.b - ch.a);
        if (nc + 1 > z.pinned_out_n) {
          if (z.pinned_out) cudaFreeHost(z.pinned_out);
          z.pinned_out = nullptr;
          z.pinned_out_n = 0;
          CK(cudaMallocHost(reinterpret_cast<void**>(&z.pinned_out), (nc + 1) * 4));
          z.pinned_out_n = nc + 1;
        }
        zip_prepare(c, z, ch, q_codes, q_offsets, r_codes, r_offsets, shape_of, big_shape, plain_shape, tr);
        tr.lap("chunk: checks");
        zip_issue(c, z, ch, P, streams[sl], true);
        tr.lap("chunk: issue");
      }
      for (long long k = std::max(0ll, K - kSlots); k < K; ++k) finish((int)(k % kSlots));
    } catch (...) {
      for (cudaStream_t st : streams) cudaStreamSynchronize(st);
      throw;
    }
    tr.lap("pipeline");
    for (int sl = 1; sl < used_slots; ++sl) {
      CK(cudaEventRecord(c->join_ev[sl - 1], streams[sl]));
      CK(cudaStreamWaitEvent(c->stream, c->join_ev[sl - 1], 0));
    }
    CK(cudaEventRecord(c->ev2, c->stream));
    CK(cudaEventRecord(c->ev3, c->stream));
    c->st.last_cells = cells;
    c->st.last_pairs = n;
    end_call(c);
  });
}

int gpusw_locate_pairs(gpusw_ctx* c, int32_t qdb, int32_t rdb, const int32_t* qi, const int32_t* rj,
                       int64_t n, int anchored, int32_t* out_score, int32_t* out_rend,
                       int32_t* out_qend) {
  return guarded(c, [&] {
    Db& q = get_db(c, qdb);
    Db& r = get_db(c, rdb);
    require_scheme(c, q, r);
    if (!anchored && c->sch.mode != gsw::kModeLocal)
      fail(GPUSW_ERR_SCHEME, "locating the best local alignment needs a local-mode scheme");
    if (n < 0 || (n > 0 && (!qi || !rj || !out_score || !out_rend || !out_qend)))
      fail(GPUSW_ERR_INVALID, "null arrays");
    if (n >= (1ll << 31)) fail(GPUSW_ERR_INVALID, "at most 2^31 - 1 pairs per call");
    int max_n = 0, max_m = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (qi[i] < 0 || qi[i] >= q.n || rj[i] < 0 || rj[i] >= r.n)
        fail(GPUSW_ERR_INVALID, "pair index out of range at position " + std::to_string(i));
      max_n = std::max(max_n, q.len[qi[i]]);
      max_m = std::max(max_m, r.len[rj[i]]);
    }
    HostScheme h = c->sch;
    if (anchored) {  // same table and gaps, both sequences anchored at their start
      h.mode = gsw::kModeGlobal;
      h.free_q = h.free_r = 0;
    }
    if (!width_ok(h, 1, max_n, max_m))
      fail(GPUSW_ERR_OVERFLOW, "scores of this scheme and these lengths do not fit in int32");
    begin_call(c);
    CK(cudaEventRecord(c->ev1, c->stream));
    if (n > 0) {
      Bufs& B = c->shared;
      B.reset_marks();
      Staging stg;
      const size_t o_qi = stg.add(qi, (size_t)n * 4), o_rj = stg.add(rj, (size_t)n * 4);
      char* dm = stg.upload(c, B);
      int* d_out = B.out.as<int>((size_t)n * 3);
      unsigned long long* queue = B.queue.as<unsigned long long>(1);
      CK(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), c->stream));
      gsw::PairsParams pp{};
      pp.S = make_scheme(h, 1);
      pp.sub = c->sub_d;
      pp.cols = q.packed();
      pp.rows = r.packed();
      pp.qi = reinterpret_cast<const int*>(dm + o_qi);
      pp.rj = reinterpret_cast<const int*>(dm + o_rj);
      pp.item_mode = 0;
      pp.n_align = n;
      pp.n_items = n;
      pp.queue = queue;
      pp.out = d_out;
      pp.out_i = d_out + n;
      pp.out_j = d_out + 2 * n;
      const bool mp = max_n > kPairShapes[7].cap();
      staged(c, B, false, [&] {
        if (anchored) launch_pairs_t<32, 16, 1, false, false, true>(c, B, pp, 1, max_m, mp);
        else launch_pairs_t<32, 16, 1, true, false, true>(c, B, pp, 1, max_m, mp);
      });
      c->last_bufs = &B;
      CK(cudaEventRecord(c->ev2, c->stream));
      CK(cudaMemcpyAsync(out_score, d_out, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(out_rend, d_out + n, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(out_qend, d_out + 2 * n, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
    } else {
      CK(cudaEventRecord(c->ev2, c->stream));
    }
    CK(cudaEventRecord(c->ev3, c->stream));
    c->st.last_pairs = n;
    end_call(c);
  });
}

int gpusw_set_options(gpusw_ctx* c, int plain, int64_t mem_budget, int flags) {
  return guarded(c, [&] {
    if (mem_budget < 0) fail(GPUSW_ERR_INVALID, "negative memory budget");
    c->plain = plain ? 1 : 0;
    c->mem_budget = mem_budget ? mem_budget : (4ll << 30);
    c->autotune = (flags & GPUSW_OPT_NO_AUTOTUNE) ? 0 : 1;
    c->graphs = (flags & GPUSW_OPT_NO_GRAPHS) ? 0 : 1;
    c->stream_multi = (flags & GPUSW_OPT_ONE_LAUNCH) ? 1 : 0;
    c->inter = (flags & GPUSW_OPT_NO_INTER) ? 0 : 1;
  });
}

int gpusw_get_tune(gpusw_ctx* c, int width, double* us, int32_t n) {
  int copied = 0;
  int rc = guarded(c, [&] {
    if (!c->has_scheme) fail(GPUSW_ERR_SCHEME, "no scheme set");
    const std::vector<double>* t = find_tune(c, width);
    if (!t) return;
    for (int i = 0; i < std::min<int>(n, (int)t->size()); ++i, ++copied)
      if (us) us[i] = (*t)[i];
  });
  return rc == GPUSW_OK ? copied : -rc;
}

int gpusw_set_tune(gpusw_ctx* c, int width, const double* us, int32_t n) {
  return guarded(c, [&] {
    if (!c->has_scheme) fail(GPUSW_ERR_SCHEME, "no scheme set");
    if (width != 1 && width != 2) fail(GPUSW_ERR_INVALID, "width must be 1 or 2");
    if (!us || n != kNumStream) fail(GPUSW_ERR_INVALID, "table must have one entry per stream shape");
    std::vector<double> t(us, us + n);
    c->tune.erase(std::remove_if(c->tune.begin(), c->tune.end(),
                                 [&](const auto& kv) { return kv.first == std::make_pair(c->sch.ns, width); }),
                  c->tune.end());
    c->tune.emplace_back(std::make_pair(c->sch.ns, width), t);
    c->plans.clear();
  });
}

int gpusw_device_name(int device, char* buf, int32_t len) {
  if (!buf || len < 1) return GPUSW_ERR_INVALID;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    cudaGetLastError();
    return GPUSW_ERR_NO_GPU;
  }
  snprintf(buf, (size_t)len, "%s", prop.name);
  return GPUSW_OK;
}

int gpusw_autotune(gpusw_ctx* c, int width, double* us_per_row_pass, int32_t n) {
  return guarded(c, [&] {
    if (!c->has_scheme) fail(GPUSW_ERR_SCHEME, "no scheme set");
    if (width != 1 && width != 2) fail(GPUSW_ERR_INVALID, "width must be 1 (int32) or 2 (int16x2)");
    set_device(c);
    std::vector<double> us = run_autotune(c, width);
    c->tune.erase(std::remove_if(c->tune.begin(), c->tune.end(),
                                 [&](const auto& kv) { return kv.first == std::make_pair(c->sch.ns, width); }),
                  c->tune.end());
    c->tune.emplace_back(std::make_pair(c->sch.ns, width), us);
    c->plans.clear();  // plans were binned with the previous costs
    if (us_per_row_pass)
      for (int i = 0; i < std::min<int>(n, (int)us.size()); ++i) us_per_row_pass[i] = us[i];
  });
}

int gpusw_get_stats(gpusw_ctx* c, gpusw_stats* out) {
  return guarded(c, [&] {
    if (!out) fail(GPUSW_ERR_INVALID, "null stats");
    c->st.device_bytes = c->held;
    *out = c->st;
  });
}

int gpusw_sync(gpusw_ctx* c) {
  return guarded(c, [&] {
    set_device(c);
    CK(cudaStreamSynchronize(c->stream));
  });
}

int gpusw_measure_dpx_rate(gpusw_ctx* c, double* ops_per_s) {
  return guarded(c, [&] {
    if (!ops_per_s) fail(GPUSW_ERR_INVALID, "null output");
    set_device(c);
    const int blocks = c->sms * 8, threads = 256, iters = 4096;
    unsigned hin[16];
    for (int i = 0; i < 16; ++i) hin[i] = 0x00030005u * (i + 1);
    hin[0] = 0xFFFEFFFEu;
    unsigned* din = static_cast<unsigned*>(c->shared.meta.get(64 + (size_t)blocks * threads * 4));
    unsigned* dout = din + 16;
    CK(cudaMemcpyAsync(din, hin, 64, cudaMemcpyHostToDevice, c->stream));
    for (int w = 0; w < 3; ++w) dpx_rate_kernel<<<blocks, threads, 0, c->stream>>>(din, dout, iters);
    CK(cudaGetLastError());
    const int reps = 10;
    CK(cudaEventRecord(c->ev0, c->stream));
    for (int r = 0; r < reps; ++r) dpx_rate_kernel<<<blocks, threads, 0, c->stream>>>(din, dout, iters);
    CK(cudaEventRecord(c->ev3, c->stream));
    CK(cudaEventSynchronize(c->ev3));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev3));
    *ops_per_s = (double)blocks * threads * iters * 8 * reps / (ms * 1e-3);
  });
}

int gpusw_flush_l2(gpusw_ctx* c, int64_t bytes) {
  return guarded(c, [&] {
    if (bytes <= 0) return;
    set_device(c);
    void* p = c->flush.get((size_t)bytes);
    CK(cudaMemsetAsync(p, 0, (size_t)bytes, c->stream));
  });
}

}  // extern "C"

// ==================================================================== no-allocation entry
// gpusw_score_pairs_noalloc: explicit pairs from caller-owned device memory, with every
// byte of scratch in the file-scope array below instead of memory the library allocates.
// Layout: [0, 256) control (work counter, error word, failing pair); [256, 256 + 16 KiB)
// substitution table (ns <= 64); the rest holds multi-pass boundary strips.
namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;  // 32 MiB on every device that loads us
constexpr size_t kNoAllocSubOff = 256;
constexpr size_t kNoAllocStripOff = kNoAllocSubOff + 64 * 64 * 4;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};
// The dynamic shared-memory limit is a per-device attribute of each kernel form (local,
// left-padded semiglobal, general), so it is raised once per (form, device), under the mutex.
bool g_noalloc_smem_set[3][kNoAllocMaxDevices] = {};

void noalloc_msg(char* buf, int len, const char* msg) {
  if (buf && len > 0) snprintf(buf, (size_t)len, "%s", msg);
}

template <bool L, bool LP>
cudaError_t noalloc_launch(const gsw::NoAllocParams& prm, int dev, int grid, int teams,
                           size_t smem, cudaStream_t st) {
  auto k = gsw::pairs_noalloc_kernel<16, 16, L, LP>;
  {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    bool& set = g_noalloc_smem_set[L ? 0 : LP ? 1 : 2][dev];
    if (!set) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(kSmemCap));
      if (e != cudaSuccess) return e;
      set = true;
    }
  }
  k<<<grid, 16 * teams, smem, st>>>(prm);
  return cudaGetLastError();
}

}  // namespace

extern "C" int gpusw_score_pairs_noalloc(const uint8_t* q_codes, const int32_t* q_offsets,
                                         int32_t nq, const uint8_t* r_codes,
                                         const int32_t* r_offsets, int32_t nr, const int32_t* qi,
                                         const int32_t* rj, int32_t n, int mode, int gap_open,
                                         int gap_extend, int free_q, int free_r, int ns,
                                         const int32_t* sub, int32_t max_len, int32_t* out,
                                         void* stream, char* errbuf, int32_t errlen) {
  if (n < 0 || nq < 0 || nr < 0 || max_len < 1) {
    noalloc_msg(errbuf, errlen, "negative count or max_len < 1");
    return GPUSW_ERR_INVALID;
  }
  if (n == 0) return GPUSW_OK;
  if (!q_codes || !q_offsets || !r_codes || !r_offsets || !qi || !rj || !out || !sub) {
    noalloc_msg(errbuf, errlen, "null pointer argument");
    return GPUSW_ERR_INVALID;
  }
  if (mode < 0 || mode > 2 || gap_open > 0 || gap_extend > 0 || gap_open < -(1 << 24) ||
      gap_extend < -(1 << 24)) {
    noalloc_msg(errbuf, errlen, "bad mode or gap costs");
    return GPUSW_ERR_SCHEME;
  }
  if (ns < 2 || ns > 64) {
    noalloc_msg(errbuf, errlen, "substitution table side must be in [2, 64] for this entry point");
    return GPUSW_ERR_SCHEME;
  }
  HostScheme h;  // scalars only: no table copy, nothing allocated
  h.mode = mode;
  h.go = gap_open;
  h.ge = gap_extend;
  h.free_q = free_q ? 1 : 0;
  h.free_r = free_r ? 1 : 0;
  h.ns = ns;
  h.max_sub = h.min_sub = sub[0];
  for (int i = 0; i < ns * ns; ++i) {
    h.max_sub = std::max(h.max_sub, (int)sub[i]);
    h.min_sub = std::min(h.min_sub, (int)sub[i]);
  }
  if (h.max_sub > (1 << 24) || h.min_sub < -(1 << 24)) {
    noalloc_msg(errbuf, errlen, "substitution scores beyond +/-2^24");
    return GPUSW_ERR_SCHEME;
  }
  if (!width_ok(h, 1, max_len, max_len)) {
    noalloc_msg(errbuf, errlen, "scores of this scheme and max_len do not fit in int32");
    return GPUSW_ERR_OVERFLOW;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
    cudaGetLastError();
    noalloc_msg(errbuf, errlen, "no usable current CUDA device");
    return GPUSW_ERR_NO_GPU;
  }
  unsigned char* base = nullptr;
  {
    // once per device, with that device current: the device address of the scratch array
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) {
        cudaGetLastError();
        noalloc_msg(errbuf, errlen, "cudaGetSymbolAddress of the scratch array failed");
        return GPUSW_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = ptr;
    }
    base = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    noalloc_msg(errbuf, errlen, "cudaDeviceGetAttribute failed");
    return GPUSW_ERR_CUDA;
  }
  const Shape shape{16, 16};
  const size_t prof = profile_bytes(shape, ns);
  const int teams = (int)std::max<size_t>(1, std::min<size_t>(16, kSmemCap / prof));
  const size_t smem = prof * teams;
  // boundary strips only when a column sequence can be longer than one pass
  const bool multipass = max_len > shape.cap();
  const size_t strip_bytes = kNoAllocScratchBytes - kNoAllocStripOff;
  long long grid = (long long)sms * 2;
  if (multipass) {
    const long long fit = (long long)(strip_bytes / ((size_t)teams * (size_t)max_len * sizeof(uint2)));
    if (fit < 1) {
      char msg[160];
      snprintf(msg, sizeof msg, "max_len %d exceeds the %zu residues the no-allocation scratch holds",
               max_len, strip_bytes / ((size_t)teams * sizeof(uint2)));
      noalloc_msg(errbuf, errlen, msg);
      return GPUSW_ERR_MEMORY;
    }
    grid = std::min(grid, fit);
  }
  grid = std::max(1ll, std::min<long long>(grid, ((long long)n + teams - 1) / teams));
  gsw::NoAllocParams prm{};
  prm.S = make_scheme(h, 1);
  prm.sub = reinterpret_cast<const int*>(base + kNoAllocSubOff);
  prm.cols = gsw::ByteSeqs{q_codes, q_offsets, nq};
  prm.rows = gsw::ByteSeqs{r_codes, r_offsets, nr};
  prm.qi = qi;
  prm.rj = rj;
  prm.n = n;
  prm.out = out;
  prm.queue = reinterpret_cast<unsigned long long*>(base);
  prm.err = reinterpret_cast<int*>(base + 8);
  prm.bnd = multipass ? reinterpret_cast<uint2*>(base + kNoAllocStripOff) : nullptr;
  prm.bnd_cap = multipass ? max_len : 0;
  prm.max_len = max_len;
  // every call shares the array: clear the counter and error word, refresh the table
  cudaError_t e = cudaMemsetAsync(base, 0, 16, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + kNoAllocSubOff, sub, (size_t)ns * ns * sizeof(int32_t),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    const bool local = mode == gsw::kModeLocal, lp = mode == gsw::kModeSemi && free_q && free_r;
    e = local ? noalloc_launch<true, false>(prm, dev, (int)grid, teams, smem, st)
              : lp ? noalloc_launch<false, true>(prm, dev, (int)grid, teams, smem, st)
                   : noalloc_launch<false, false>(prm, dev, (int)grid, teams, smem, st);
  }
  int herr[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(herr, base + 8, sizeof herr, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    noalloc_msg(errbuf, errlen, cudaGetErrorString(e));
    return GPUSW_ERR_CUDA;
  }
  if (herr[0] != 0) {
    char msg[128];
    snprintf(msg, sizeof msg,
             herr[0] == 1   ? "pair index out of range at position %d"
             : herr[0] == 2 ? "row longer than max_len at pair %d"
                            : "code >= table side or decreasing offsets at pair %d",
             herr[1]);
    noalloc_msg(errbuf, errlen, msg);
    return GPUSW_ERR_INVALID;
  }
  return GPUSW_OK;
}

#include "server.cuh"
#include "fasta.cuh"
