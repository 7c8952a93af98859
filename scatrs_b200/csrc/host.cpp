// The C ABI of include/scatrs_b200.h: input checks, the cached tables, slab planning and the
// launches of K-a (mie_kernels.cu) and K-b/c/d (unit_kernel.cu).
//
// A call of the fixed-grid ensemble runs, per device and in one stream:
//   1. the node table (radii and weights w_j u(r_j) r_j per distribution) on the host;
//   2. plan_chunks: each chunk's largest number of terms N_c, copied back to the host, which
//      picks the projector bands, grows the tables if needed, and cuts the units into slabs
//      whose coefficient rows fit the arena;
//   3. per slab, K-a (one warp per chunk) then the unit kernel (one persistent CTA per SM slot).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <tuple>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/scatrs_b200.h"
#include "adaptive.h"
#include "dd.cuh"
#include "kernels.h"
#include "tables.h"

namespace sb {

static std::atomic<int64_t> g_launches{0};

// Optional per-kernel timing: CUDA events recorded around each launch on its stream, read back
// by scatrs_kernel_times (which synchronizes). Off unless scatrs_set_profiling(1).
enum KernelId {
  K_PLAN = 0,
  K_MIE = 1,
  K_UNITS = 2,
  K_NODES = 3,
  K_FINAL = 4,
  K_PROJ = 5,
  K_TM_TABLES = 6,   // tm_geom_kernel + tm_angular_kernel
  K_TM_SURFACE = 7,  // tm_surface_kernel
  K_TM_SOLVE = 8,    // tm_solve_kernel
  K_RANDOM = 9,      // the orientation average's five kernels
  K_UNITS_I8 = 10,   // unit_i8_kernel (the mixed form's int8 angle GEMMs)
  K_X_SPLIT = 11,    // x_split_kernel (the int8 chunks' digits)
  K_COUNT = 12
};
static bool g_profiling = false;
// The spheroid surface integrals' work per tm_surface_kernel launch while profiling: the sum
// over the launch's modes of K^2 (i, k) pairs times the n_theta nodes of half the surface.
static std::vector<int64_t> g_tm_pair_nodes;
struct Timed {
  int id;
  cudaEvent_t a, b;
};
static std::vector<Timed> g_timed;
static double g_kernel_ms[K_COUNT];
static int64_t g_kernel_launches[K_COUNT];

template <class F>
static void timed_launch(int id, cudaStream_t s, F f) {
  if (!g_profiling) {
    f();
    g_launches++;
    return;
  }
  Timed t{id, nullptr, nullptr};
  cudaEventCreate(&t.a);
  cudaEventCreate(&t.b);
  cudaEventRecord(t.a, s);
  f();
  cudaEventRecord(t.b, s);
  g_timed.push_back(t);
  g_launches++;
}

namespace {

constexpr int64_t kMaxGreekOrder = 1 << 21;        // MAX_GREEK_ORDER (mie/greek.rs:344)
constexpr int64_t kMaxMieValues = 1 << 27;         // scatrs-py/src/mie.rs:30
constexpr int64_t kMaxMieOrder = 1 << 20;          // MAX_MIE_ORDER (mie/mod.rs:101), check_node
constexpr int64_t kMaxLayersAbi = 16;              // layers the layered kernels carry
constexpr int64_t kMaxTmatrixOrder = 500;          // MAX_TMATRIX_ORDER (tmatrix/mod.rs:180)
constexpr int64_t kMaxGaussPoints = 1 << 17;       // special/gauss_legendre.rs:43
constexpr int64_t kMaxWignerValues = 1 << 28;      // scatrs-py/src/special.rs:24
constexpr int64_t kArenaRows = 1 << 22;            // coefficient rows per slab (1 KiB each)
constexpr int kDefaultSplit = 4;                     // work items per resident CTA and slab
// The work-division settings (scatrs_set_tuning): read once per call.
std::atomic<int> g_split{kDefaultSplit};
std::atomic<int64_t> g_arena_rows{kArenaRows};
constexpr int64_t kMaxSlabChunks = 1 << 18;        // chunks per slab
constexpr double kPi = 3.14159265358979323846264338327950288;

// A failed call: its status, its message and, for SCATRS_NOT_CONVERGED, the accuracy reached
// and the accuracy requested (scatrs::Error::NotConverged, scatrs/src/error.rs:22-28).
struct Failure {
  int status;
  std::string msg;
  double achieved = NAN;
  double requested = NAN;
};

// The last failed call's accuracies on this thread (NaN unless it was SCATRS_NOT_CONVERGED).
thread_local int g_last_status = SCATRS_OK;
thread_local double g_last_achieved = NAN;
thread_local double g_last_requested = NAN;

void set_err(char* err, size_t len, const std::string& msg) {
  if (err && len > 0) {
    size_t n = std::min(len - 1, msg.size());
    memcpy(err, msg.data(), n);
    err[n] = 0;
  }
}

// A failed runtime call becomes a SCATRS_CUDA failure; its error is also cleared from the
// runtime's last-error state, so that the next call does not report it again.
#define SB_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      cudaGetLastError();                                                                    \
      throw Failure{SCATRS_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)};        \
    }                                                                                        \
  } while (0)

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Test hooks (scatrs_testing_*): the device allocation that fails as an out-of-memory
// cudaMalloc would (0: none; k: the k-th growth from now), and a node error merged into the
// next fixed-grid call's device error word (~0: none).
std::atomic<int64_t> g_fail_allocation{0};
std::atomic<unsigned long long> g_forced_node_error{~0ull};

// A grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  void* get(size_t bytes) {
    if (bytes > cap) {
      if (p) cudaFree(p);
      p = nullptr;
      cap = 0;
      size_t want = std::max<size_t>(bytes, 256);
      if (g_fail_allocation.load() > 0 && g_fail_allocation.fetch_sub(1) == 1)
        throw Failure{SCATRS_CUDA, std::string("cudaMalloc(&p, want): ") +
                                       cudaGetErrorString(cudaErrorMemoryAllocation)};
      SB_CUDA(cudaMalloc(&p, want));
      cap = want;
    }
    return p;
  }
  template <class T>
  T* as(size_t count) {
    return static_cast<T*>(get(count * sizeof(T)));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Tables of the requested cosines: one row per cosine c (or per pair c, -c), G_E and G_O of
// orders 1..ld.
struct UserTables {
  std::vector<double> mu;
  std::vector<double> rows;  // each table row's cosine (a cosine, or a pair c, -c)
  int64_t n_orders = 0;
  int h = 0, h_pad = 0, ld = 0;
  DevBuf ge, go, map;
};

struct BandTables {
  int order = -1;
  int n_bands = 0;
  int nq_max = 0;
  std::vector<BandDesc> desc;
  std::vector<double> ge, go, d;  // host copies, appended band by band
  DevBuf ge_d, go_d, d_d, desc_d;
};

struct Context {
  int device = -1;
  int sms = 0;
  int unit_bps = 1;
  std::mutex mtx;
  UserTables user;
  std::map<int, BandTables> bands;  // by Greek order
  std::map<int64_t, std::pair<std::vector<double>, std::vector<double>>> rules;
  DevBuf radius, weight, wtheta, wthdiff, wdiff, unit_norm, wl, m, fractions, chunk_n, chunk_n_slab, chunk_row, chunk_acc, plan_units,
      unit_acc, unit_slots, slots, items, proj_items, slot_index, slot_greek, X, uz, ux,
      chunk_sums, err, acc, counter, values, phase, greek;
  // Pass 1 of the adaptive ensemble.
  DevBuf p1_radius, p1_wl, p1_wlu, p1_scratch, p1_uz, p1_ux, p1_q, p1_n, p1_status;
  DevBuf avg, mix_first, mix_part, mix_frac;
  // The Greek projection of tables at Gauss cosines: per (n_q, L) the matrices (FP64 and their
  // TF32 heads and tails), and the workspaces of the tensor-core form.
  struct Projector {
    DevBuf d, d_hi, d_lo;
  };
  std::map<std::pair<int64_t, int>, Projector> projectors;
  DevBuf tc_a_hi, tc_a_lo, tc_prod, tc_err;
  // The mixed form: digit tables (I8Tables) and the slabs' chunk digits.
  struct I8Tables {
    std::vector<double> mu;
    int64_t user_orders = 0;
    int order = -2;
    int n_bands = 0;
    std::vector<I8Table> user, band;
    DevBuf dig, scale, user_d, band_d;
  } i8;
  DevBuf xdig, xside, colmax, chunk_xoff, chunk_xidx, i8_list, i8_err;
  // Spheroid T-matrices.
  DevBuf tm_geoms, tm_jobs, tm_rules, tm_node, tm_rad, tm_ang, tm_ser, tm_J, tm_work, tm_piv, tm_T,
      tm_sums, tm_err;
  DevBuf ro_sph, ro_rank, ro_w, ro_part, ro_f, ro_greek, ro_mu, ro_proj;
  DevBuf p1_fr, p1_ml;  // layered parts of an adaptive call
  DevBuf p1_ml_aug;     // their indices with a vacuum shell (a single radius's radius)
  std::map<int64_t, std::vector<double>> dd_rules;  // n -> per node x (hi, lo), w (hi, lo)
  std::vector<int> chunk_n_host;
  int* pinned_chunk_n = nullptr;
  size_t pinned_cap = 0;
  // Two halves of pinned staging for the slabs' plans, each with the event of its last upload.
  unsigned char* staging = nullptr;
  size_t staging_cap = 0;  // bytes per half
  cudaEvent_t staged[2] = {nullptr, nullptr};
  bool staged_pending[2] = {false, false};
  // The outputs' copies to pinned host arrays, slab by slab, beside the next slabs' kernels: a
  // non-blocking stream (the kernels run on the legacy default stream) ordered by slab_done.
  cudaStream_t copies = nullptr;
  cudaEvent_t slab_done = nullptr;
  void ensure_copies() {
    if (copies) return;
    SB_CUDA(cudaStreamCreateWithFlags(&copies, cudaStreamNonBlocking));
    SB_CUDA(cudaEventCreateWithFlags(&slab_done, cudaEventDisableTiming));
  }

  void ensure_staging(size_t bytes) {
    if (!staged[0]) {
      SB_CUDA(cudaEventCreateWithFlags(&staged[0], cudaEventDisableTiming));
      SB_CUDA(cudaEventCreateWithFlags(&staged[1], cudaEventDisableTiming));
    }
    if (bytes <= staging_cap) return;
    for (int h = 0; h < 2; ++h)
      if (staged_pending[h]) SB_CUDA(cudaEventSynchronize(staged[h]));
    staged_pending[0] = staged_pending[1] = false;
    if (staging) cudaFreeHost(staging);
    staging = nullptr;
    staging_cap = 0;
    SB_CUDA(cudaMallocHost(&staging, 2 * bytes));
    staging_cap = bytes;
  }
  // Half h, once the device has read what was last uploaded from it.
  unsigned char* staging_half(int h) {
    if (staged_pending[h]) SB_CUDA(cudaEventSynchronize(staged[h]));
    staged_pending[h] = false;
    return staging + (size_t)h * staging_cap;
  }
  void staging_uploaded(int h, cudaStream_t s) {
    SB_CUDA(cudaEventRecord(staged[h], s));
    staged_pending[h] = true;
  }
};

std::mutex g_ctx_mtx;
std::vector<std::unique_ptr<Context>> g_ctx;

Context& context() {
  int dev = 0;
  SB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_ctx_mtx);
  if ((int)g_ctx.size() <= dev) g_ctx.resize(dev + 1);
  if (!g_ctx[dev]) {
    auto c = std::make_unique<Context>();
    c->device = dev;
    cudaDeviceProp prop;
    SB_CUDA(cudaGetDeviceProperties(&prop, dev));
    c->sms = prop.multiProcessorCount;
    c->unit_bps = unit_kernel_blocks_per_sm();
    g_ctx[dev] = std::move(c);
  }
  return *g_ctx[dev];
}

const std::pair<std::vector<double>, std::vector<double>>& rule(Context& c, int64_t n) {
  auto it = c.rules.find(n);
  if (it != c.rules.end()) return it->second;
  std::vector<double> x(n), w(n);
  gauss_legendre(n, x.data(), w.data());
  return c.rules.emplace(n, std::make_pair(std::move(x), std::move(w))).first->second;
}

// The tables of the requested cosines, for orders 1..n_orders at least.
void ensure_user(Context& c, const double* mu, int64_t n_mu, int64_t n_orders, cudaStream_t s) {
  UserTables& u = c.user;
  bool same = (int64_t)u.mu.size() == n_mu && u.n_orders >= n_orders &&
              (n_mu == 0 || memcmp(u.mu.data(), mu, n_mu * sizeof(double)) == 0);
  if (same) return;
  u.mu.assign(mu, mu + n_mu);
  u.n_orders = std::max<int64_t>(round_up(std::max<int64_t>(n_orders, 1), 16), u.n_orders);
  // Pair each cosine with its exact negative where the list has one.
  std::unordered_multimap<uint64_t, int> by_bits;
  for (int j = 0; j < n_mu; ++j) {
    uint64_t b;
    memcpy(&b, &mu[j], 8);
    by_bits.emplace(b, j);
  }
  std::vector<char> used(n_mu, 0);
  std::vector<double> cosines;
  std::vector<int2> map;
  for (int j = 0; j < n_mu; ++j) {
    if (used[j]) continue;
    used[j] = 1;
    int partner = -1;
    double neg = -mu[j];
    uint64_t nb;
    memcpy(&nb, &neg, 8);
    auto range = by_bits.equal_range(nb);
    for (auto it = range.first; it != range.second; ++it)
      if (!used[it->second]) {
        partner = it->second;
        break;
      }
    if (mu[j] == 0.0 && partner < 0) {
      // +0 and -0 are the same cosine.
      for (int k = j + 1; k < n_mu; ++k)
        if (!used[k] && mu[k] == 0.0) {
          partner = k;
          break;
        }
    }
    if (partner >= 0) used[partner] = 1;
    cosines.push_back(mu[j]);
    map.push_back(make_int2(j, partner));
  }
  u.h = (int)cosines.size();
  u.rows = cosines;
  u.h_pad = (int)round_up(std::max(u.h, 1), 32);
  u.ld = (int)u.n_orders;
  // Order-major (transposed) tables: element (row, order k) at k * h_pad + row, so that one
  // order of a 32-row tile is 256 contiguous bytes.
  std::vector<double> ge((size_t)u.h_pad * u.ld, 0.0), go((size_t)u.h_pad * u.ld, 0.0);
  std::vector<double> re(u.ld), ro(u.ld);
  for (int r = 0; r < u.h; ++r) {
    pi_tau_row(cosines[r], u.n_orders, re.data(), ro.data());
    for (int k = 0; k < u.ld; ++k) {
      ge[(size_t)k * u.h_pad + r] = re[k];
      go[(size_t)k * u.h_pad + r] = ro[k];
    }
  }
  SB_CUDA(cudaMemcpyAsync(u.ge.get(ge.size() * 8), ge.data(), ge.size() * 8,
                          cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(u.go.get(go.size() * 8), go.data(), go.size() * 8,
                          cudaMemcpyHostToDevice, s));
  if (!map.empty())
    SB_CUDA(cudaMemcpyAsync(u.map.get(map.size() * sizeof(int2)), map.data(),
                            map.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaStreamSynchronize(s));
}

// Bands 0..last_band for Greek order L (engine.rs:2034-2072).
BandTables& ensure_bands(Context& c, int L, int last_band, cudaStream_t s) {
  BandTables& bt = c.bands[L];
  bt.order = L;
  if (bt.n_bands > last_band) return bt;
  for (int b = bt.n_bands; b <= last_band; ++b) {
    int64_t upper = band_upper(b);
    int64_t order = std::min<int64_t>(L, 2 * upper);
    int64_t n_q = upper + (order + 2) / 2;
    const auto& r = rule(c, n_q);
    BandDesc d;
    d.upper = (int)upper;
    d.order = (int)order;
    d.n_q = (int)n_q;
    int64_t lo = n_q / 2;
    d.h = (int)(n_q - lo);
    d.h_pad = (int)round_up(d.h, 32);
    d.ld = (int)round_up(upper, 16);
    d.g_off = (int64_t)bt.ge.size();
    d.d_off = (int64_t)bt.d.size();
    bt.ge.resize(bt.ge.size() + (size_t)d.h_pad * d.ld, 0.0);
    bt.go.resize(bt.go.size() + (size_t)d.h_pad * d.ld, 0.0);
    {
      // Order-major, as the requested cosines' tables.
      std::vector<double> re(upper), ro(upper);
      for (int i = 0; i < d.h; ++i) {
        pi_tau_row(r.first[lo + i], upper, re.data(), ro.data());
        for (int64_t k = 0; k < upper; ++k) {
          bt.ge[d.g_off + (size_t)k * d.h_pad + i] = re[k];
          bt.go[d.g_off + (size_t)k * d.h_pad + i] = ro[k];
        }
      }
    }
    int64_t len = order + 1;
    bt.d.resize(bt.d.size() + 4 * (size_t)n_q * len);
    std::vector<double> buf(len);
    const int mn[4][2] = {{0, 0}, {2, 2}, {2, -2}, {0, 2}};
    for (int f = 0; f < 4; ++f)
      for (int64_t k = 0; k < n_q; ++k) {
        wigner_d(mn[f][0], mn[f][1], r.first[k], buf.data(), len);
        double* dst = &bt.d[d.d_off + ((size_t)f * n_q + k) * len];
        for (int64_t l = 0; l < len; ++l) dst[l] = (double)(2 * l + 1) * 0.5 * r.second[k] * buf[l];
      }
    bt.desc.push_back(d);
    bt.nq_max = std::max(bt.nq_max, d.n_q);
  }
  bt.n_bands = last_band + 1;
  SB_CUDA(cudaMemcpyAsync(bt.ge_d.get(bt.ge.size() * 8), bt.ge.data(), bt.ge.size() * 8,
                          cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(bt.go_d.get(bt.go.size() * 8), bt.go.data(), bt.go.size() * 8,
                          cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(bt.d_d.get(bt.d.size() * 8), bt.d.data(), bt.d.size() * 8,
                          cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(bt.desc_d.get(bt.desc.size() * sizeof(BandDesc)), bt.desc.data(),
                          bt.desc.size() * sizeof(BandDesc), cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaStreamSynchronize(s));
  return bt;
}

// The digits of one table of the mixed form (kernels.h): pairs [0, h) whose E and O rows over
// orders 0 .. n_orders - 1 row(pair, e, o) writes (zero beyond), in M tiles of kI8Pairs pairs
// (MMA rows 2p and 2p + 1: the E and O rows of the tile's pair p) and n_kb K blocks; each MMA row's power of two 2^e puts
// its largest |value| below 127 2^-e (in [63.5, 127) 2^-e), and F = rint(value 2^(e + 32))
// goes out as its five balanced digits (each in [-128, 127]: the low ones the sign-extended low
// byte of what is left) into the 64-byte swizzle (16-byte chunk q of row r at chunk
// q ^ ((r >> 1) & 3)). The scale written per row is 2^-e (0 for a zero row).
template <class Row>
I8Table i8_table(int h, int64_t n_orders, int n_kb, Row row, std::vector<unsigned char>& dig,
                 std::vector<double>& scale) {
  I8Table t;
  t.off = (int64_t)dig.size();
  t.scale_off = (int64_t)scale.size();
  t.n_kb = n_kb;
  t.n_tiles = (h + kI8Pairs - 1) / kI8Pairs;
  const int64_t K = (int64_t)n_kb * kI8KB;
  dig.resize(dig.size() + (size_t)t.n_tiles * n_kb * kI8TileBytes, 0);
  scale.resize(scale.size() + (size_t)t.n_tiles * 128, 0.0);
  std::vector<double> e_row(K), o_row(K);
  for (int tile = 0; tile < t.n_tiles; ++tile) {
    for (int pp = 0; pp < kI8Pairs; ++pp) {
      const int pair = tile * kI8Pairs + pp;
      if (pair >= h) break;
      std::fill(e_row.begin(), e_row.end(), 0.0);
      std::fill(o_row.begin(), o_row.end(), 0.0);
      row(pair, std::min<int64_t>(n_orders, K), e_row.data(), o_row.data());
      for (int side = 0; side < 2; ++side) {
        const std::vector<double>& v = side ? o_row : e_row;
        const int r = 2 * pp + side;  // a pair's E and O rows side by side
        double m = 0.0;
        for (int64_t k = 0; k < K; ++k) m = std::max(m, std::fabs(v[k]));
        if (!(m > 0.0)) continue;
        int ex = 0;
        std::frexp(m, &ex);
        int e = 7 - ex;
        if (std::ldexp(m, e) >= 127.0) --e;
        scale[t.scale_off + (size_t)tile * 128 + r] = std::ldexp(1.0, -e);
        for (int64_t k = 0; k < K; ++k) {
          long long f = std::llrint(std::ldexp(v[k], e + 32));
          const int kb = (int)(k / kI8KB), kk = (int)(k % kI8KB);
          const int q = kk / 16, b = kk % 16, qs = q ^ ((r >> 1) & 3);
          const size_t at = (size_t)t.off + ((size_t)(tile * n_kb + kb) * kI8Levels) * 8192 +
                            (size_t)r * kI8KB + qs * 16 + b;
          int d[kI8Levels];
          for (int s2 = kI8Levels - 1; s2 > 0; --s2) {
            d[s2] = (int)(signed char)(f & 0xff);
            f = (f - d[s2]) >> 8;
          }
          d[0] = (int)f;
          for (int s2 = 0; s2 < kI8Levels; ++s2)
            dig[at + (size_t)s2 * 8192] = (unsigned char)(d[s2] & 0xff);
        }
      }
    }
  }
  return t;
}

// The mixed form's digit tables for the requested cosines (versions v = 0, 1, ... covering
// orders < 64 2^v up to n_max, each row scaled over its version's orders, so that a chunk's
// rows keep their bits relative to the orders it uses) and for bands 0 .. n_bands - 1 of Greek
// order L (L < 0: none); cached per context until the cosines, the order or the reach change.
void ensure_i8(Context& c, int64_t n_max, const BandTables* bt, cudaStream_t s) {
  Context::I8Tables& T = c.i8;
  const int L = bt ? bt->order : -1;
  const int nb = bt ? bt->n_bands : 0;
  int n_ver = 1;
  while (((int64_t)kI8KB << (n_ver - 1)) < std::min<int64_t>(n_max, kI8MaxTerms)) ++n_ver;
  if (T.mu == c.user.mu && T.user_orders >= ((int64_t)kI8KB << (n_ver - 1)) && T.order == L &&
      T.n_bands >= nb)
    return;
  std::vector<unsigned char> dig;
  std::vector<double> scale;
  T.user.clear();
  T.band.clear();
  const int h_u = c.user.h;
  const std::vector<double>& cosines = c.user.rows;
  for (int v = 0; v < n_ver; ++v) {
    const int n_kb = 1 << v;
    const int64_t K = (int64_t)n_kb * kI8KB;
    T.user.push_back(i8_table(
        h_u, K, n_kb,
        [&](int pair, int64_t n, double* e, double* o) { pi_tau_row(cosines[pair], n, e, o); },
        dig, scale));
  }
  for (int b = 0; b < nb; ++b) {
    const BandDesc& d = bt->desc[b];
    const int n_kb = (d.upper + kI8KB - 1) / kI8KB;
    T.band.push_back(i8_table(
        d.h, d.upper, n_kb,
        [&](int pair, int64_t n, double* e, double* o) {
          for (int64_t k = 0; k < n; ++k) {
            e[k] = bt->ge[d.g_off + (size_t)k * d.h_pad + pair];
            o[k] = bt->go[d.g_off + (size_t)k * d.h_pad + pair];
          }
        },
        dig, scale));
  }
  if (T.band.empty()) T.band.push_back(I8Table{});
  SB_CUDA(cudaMemcpyAsync(T.dig.get(std::max<size_t>(dig.size(), 16)), dig.data(), dig.size(),
                          cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(T.scale.get(std::max<size_t>(scale.size(), 1) * 8), scale.data(),
                          scale.size() * 8, cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(T.user_d.get(T.user.size() * sizeof(I8Table)), T.user.data(),
                          T.user.size() * sizeof(I8Table), cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(T.band_d.get(T.band.size() * sizeof(I8Table)), T.band.data(),
                          T.band.size() * sizeof(I8Table), cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaStreamSynchronize(s));
  T.mu = c.user.mu;
  T.user_orders = (int64_t)kI8KB << (n_ver - 1);
  T.order = L;
  T.n_bands = nb;
}

// A distribution's density at r: its closed form, or a tabulated one's interpolation.
double node_density(const scatrs_distribution& d, double r) {
  return d.kind == kTabulated ? table_density(d.table, d.table_len, r)
                              : density(d.kind, d.param, r);
}

void check_options(const scatrs_fixed_options* o, int64_t n_units, int64_t n_mu,
                   const double* mu, int n_derivs = 0) {
  if (!o) throw Failure{SCATRS_INVALID_INPUT, "options must not be NULL"};
  if (o->n_nodes < 1) throw Failure{SCATRS_INVALID_INPUT, "n_nodes must be >= 1"};
  if (o->greek_order < -1 || o->greek_order > kMaxGreekOrder)
    throw Failure{SCATRS_INVALID_INPUT, "the Greek order must be at most 2097152"};
  if (n_mu < 0) throw Failure{SCATRS_INVALID_INPUT, "n_mu must be >= 0"};
  for (int64_t j = 0; j < n_mu; ++j)
    if (!(std::isfinite(mu[j]) && mu[j] >= -1.0 && mu[j] <= 1.0))
      throw Failure{SCATRS_INVALID_INPUT,
                    "a cosine of the scattering angle must be finite and in [-1, 1]"};
  // The output bound of scatrs-py/src/ensemble.rs:388-399.
  int64_t per = 11 + 4 * n_mu + (o->greek_order >= 0 ? 6 * ((int64_t)o->greek_order + 1) : 0);
  per *= 1 + n_derivs;
  if ((double)n_units * (double)per * 2.0 > 2.0 * (double)kMaxMieValues)
    throw Failure{SCATRS_INVALID_INPUT,
                  "the ensemble outputs would exceed 2 * MAX_MIE_VALUES = 268435456 real values"};
}

std::string node_message(int status, double lambda, double r) {
  char buf[256];
  snprintf(buf, sizeof buf, "at wavelength %e, radius %e: %s", lambda, r,
           status == 3 ? "the size parameter and refractive index are outside the validated "
                         "domain x in [1e-06, 2e4], 0 < Re m <= 10, 0 <= Im m <= 10, |m| >= 0.1"
                       : "the size parameter x must be in [1e-30, 1e6] and the refractive "
                         "index finite with Re m >= 0, Im m >= 0 and |m| in [1e-6, 1e3]");
  return buf;
}

struct FixedCall {
  // Host copies needed for error messages.
  std::vector<double> radius;  // [n_dist][n_nodes], or [n_units][n_nodes] with per_unit
  std::vector<double> wl_host;
  int64_t n_dist = 0, n_wl = 0, n_nodes = 0;
  bool per_unit = false;
  // Pinned host outputs (values, and phase and greek when they have a length): each slab's units
  // are copied there on the copy stream once its final kernel is done (Context::copies).
  double* h_values = nullptr;
  double* h_phase = nullptr;
  double* h_greek = nullptr;
  // The mixed form (values of homogeneous spheres): chunks with i8_above < N_c <=
  // kI8MaxTerms run their angle GEMMs on int8 digits (unit_i8_kernel); 0 for plain FP64.
  int i8_above = 0;
  int i8_levels = 5;           // product levels kept (5 or 6)
  unsigned* i8_err = nullptr;  // the int8 kernel's timeout flag, checked with the errors
};

// The device pipeline; wl_dev and m_dev are device arrays, outputs device arrays.
// Layered spheres: L layers, per distribution the L - 1 radius fractions (host) and the
// layers' indices per wavelength (device, [n_dist][L][n_wl] complex).
struct LayerInput {
  int n_layers = 1;
  const double* fractions = nullptr;
  const double* m_dev = nullptr;
};

// Derivative outputs (homogeneous spheres, every distribution of one kind): along the
// distribution's n_theta parameters, then Re m and Im m; device arrays d_values [P][11][n],
// d_phase [P][6][n][n_mu], d_greek [P][6][n][L + 1].
struct DerivOutput {
  bool on = false;
  int n_theta = 0;
  int dir = 0;  // layered spheres: the direction of the pass (MieFixedArgs::deriv_dir)
  double* d_values = nullptr;
  double* d_phase = nullptr;
  double* d_greek = nullptr;
};

// Adaptive panels (pass 2 of the adaptive ensemble): each unit's own nodes, two GK15 panels per
// chunk of 32 (host arrays [n_units][n_nodes], radius 0 for padding), the error weights, the
// per-unit normalization (8 doubles, see FinalArgs) and the device error outputs.
struct AdaptiveInput {
  bool on = false;
  const double* radius = nullptr;
  const double* weight = nullptr;
  const double* wdiff = nullptr;
  const double* unit_norm = nullptr;
  double* avg = nullptr;  // the units' averages, mixed and assembled by mix_assemble_kernel
  // With derivatives (and DerivOutput::on with n_theta parameters): per unit and node the
  // parameters' Kronrod weights w_K (du/dtheta) r and error weights (w_K - w_G) (du/dtheta) r
  // ([n_units][n_nodes][3]); unit_norm then holds kNormStrideD doubles per unit and avg the
  // per-block averages of final_adaptive_d_kernel.
  const double* wtheta = nullptr;
  const double* wthdiff = nullptr;
};

void run_fixed(Context& c, const scatrs_distribution* dists, int64_t n_dist, const double* wl_dev,
               int64_t n_wl, const double* m_dev, const double* mu, int64_t n_mu,
               const scatrs_fixed_options* opt, double* values, double* phase, double* greek,
               cudaStream_t s, FixedCall* call, const LayerInput& layers = LayerInput(),
               const DerivOutput& dv = DerivOutput(),
               const AdaptiveInput& ad = AdaptiveInput()) {
  const int64_t n_units = n_dist * n_wl;
  check_options(opt, n_units, n_mu, mu, dv.on ? dv.n_theta + 2 : 0);
  if (n_units == 0) return;
  const int64_t n_nodes = opt->n_nodes;
  const int cpu = (int)((n_nodes + 31) / 32);
  const int64_t n_chunks = n_units * cpu;
  if (n_chunks > (int64_t)INT32_MAX / 32)
    throw Failure{SCATRS_INVALID_INPUT, "too many (distribution, wavelength, node) triples"};
  // 1. Node table.
  const auto& gl = rule(c, n_nodes);
  std::vector<double> radius(n_dist * n_nodes), weight(n_dist * n_nodes);
  std::vector<double> wtheta(dv.on ? n_dist * n_nodes * 3 : 0);
  if (dv.on && !ad.on) {
    for (int64_t d = 0; d < n_dist; ++d)
      if (parameter_count(dists[d].kind) != dv.n_theta)
        throw Failure{SCATRS_INVALID_INPUT,
                      "derivatives need every distribution of one kind (distribution " +
                          std::to_string(d) + " differs)"};
  }
  for (int64_t d = 0; d < n_dist && !ad.on; ++d) {
    std::string msg;
    if (!(dists[d].kind == kTabulated
              ? validate_table(dists[d].table, dists[d].table_len, &msg)
              : validate_distribution(dists[d].kind, dists[d].param, &msg)))
      throw Failure{SCATRS_INVALID_INPUT, "distribution " + std::to_string(d) + ": " + msg};
    if (!(dists[d].r_lo > 0.0 && dists[d].r_hi > dists[d].r_lo && std::isfinite(dists[d].r_hi)))
      throw Failure{SCATRS_INVALID_INPUT, "distribution " + std::to_string(d) +
                                              ": the grid needs 0 < r_lo < r_hi < inf"};
    double a = std::log(dists[d].r_lo), b = std::log(dists[d].r_hi);
    double ctr = 0.5 * (a + b), h = 0.5 * (b - a);
    for (int64_t j = 0; j < n_nodes; ++j) {
      double t = ctr + h * gl.first[j];
      double r = std::exp(t);
      const double w = h * gl.second[j];
      double u;
      if (dv.on) {
        double g[3];
        if (dists[d].kind == kTabulated) {
          u = node_density(dists[d], r);
          g[0] = g[1] = g[2] = 0.0;
        } else {
          u = density_gradient(dists[d].kind, dists[d].param, r, g);
        }
        for (int p = 0; p < 3; ++p) wtheta[(d * n_nodes + j) * 3 + p] = w * (g[p] * r);
      } else {
        u = node_density(dists[d], r);
      }
      radius[d * n_nodes + j] = r;
      weight[d * n_nodes + j] = w * (u * r);
    }
  }
  const int L_layers = layers.n_layers;
  if (L_layers < 1 || L_layers > kMaxLayersAbi)
    throw Failure{SCATRS_INVALID_INPUT, "the GPU path takes 1 to 16 layers"};
  if (L_layers > 1) {
    for (int64_t d = 0; d < n_dist; ++d)
      for (int l = 0; l < L_layers - 1; ++l) {
        const double f = layers.fractions[d * (L_layers - 1) + l];
        const double prev = l > 0 ? layers.fractions[d * (L_layers - 1) + l - 1] : 0.0;
        if (!(f > 0.0 && f <= 1.0 && f >= prev))
          throw Failure{SCATRS_INVALID_INPUT,
                        "distribution " + std::to_string(d) +
                            ": radius fractions must be nondecreasing in (0, 1]"};
      }
    SB_CUDA(cudaMemcpyAsync(c.fractions.get(n_dist * (L_layers - 1) * 8), layers.fractions,
                            n_dist * (L_layers - 1) * 8, cudaMemcpyHostToDevice, s));
  }
  if (ad.on) {
    // Nodes per unit.
    const size_t cnt = (size_t)n_units * n_nodes;
    SB_CUDA(cudaMemcpyAsync(c.radius.get(cnt * 8), ad.radius, cnt * 8, cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(c.weight.get(cnt * 8), ad.weight, cnt * 8, cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(c.wdiff.get(cnt * 8), ad.wdiff, cnt * 8, cudaMemcpyHostToDevice, s));
    const size_t norm_bytes = (size_t)n_units * (dv.on ? kNormStrideD : 8) * 8;
    SB_CUDA(cudaMemcpyAsync(c.unit_norm.get(norm_bytes), ad.unit_norm, norm_bytes,
                            cudaMemcpyHostToDevice, s));
    if (dv.on) {
      SB_CUDA(cudaMemcpyAsync(c.wtheta.get(cnt * 24), ad.wtheta, cnt * 24,
                              cudaMemcpyHostToDevice, s));
      SB_CUDA(cudaMemcpyAsync(c.wthdiff.get(cnt * 24), ad.wthdiff, cnt * 24,
                              cudaMemcpyHostToDevice, s));
    }
  } else {
    SB_CUDA(cudaMemcpyAsync(c.radius.get(radius.size() * 8), radius.data(), radius.size() * 8,
                            cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(c.weight.get(weight.size() * 8), weight.data(), weight.size() * 8,
                            cudaMemcpyHostToDevice, s));
  }
  if (dv.on && !ad.on)
    SB_CUDA(cudaMemcpyAsync(c.wtheta.get(wtheta.size() * 8), wtheta.data(), wtheta.size() * 8,
                            cudaMemcpyHostToDevice, s));
  // Blocks of sums per quantity (values, then each derivative) and coefficient rows per term
  // of a chunk (two 16-node halves with derivatives).
  // Adaptive calls add the error sums of every block (a second set of n_blk / 2).
  const int n_blk = (dv.on ? 3 + dv.n_theta : 1) * (ad.on ? 2 : 1);
  const int rows_per_term = dv.on ? 2 : 1;  unsigned long long* err = c.err.as<unsigned long long>(2);
  SB_CUDA(cudaMemsetAsync(err, 0xff, 2 * sizeof(unsigned long long), s));
  // 2. Plan: every chunk's largest number of terms.
  PlanArgs pa{};
  pa.radius = c.radius.as<double>(0);
  pa.wl = wl_dev;
  pa.n_dist = (int)n_dist;
  pa.n_wl = (int)n_wl;
  pa.n_nodes = (int)n_nodes;
  pa.cpu = cpu;
  pa.n_chunks = n_chunks;
  int* chunk_n_all = c.chunk_n.as<int>(n_chunks);
  pa.chunk_n = chunk_n_all;
  pa.per_unit = ad.on ? 1 : 0;
  timed_launch(K_PLAN, s, [&] { launch_plan_chunks(pa, s); });
  SB_CUDA(cudaGetLastError());
  if (c.pinned_cap < (size_t)n_chunks) {
    if (c.pinned_chunk_n) cudaFreeHost(c.pinned_chunk_n);
    c.pinned_chunk_n = nullptr;
    c.pinned_cap = 0;
    SB_CUDA(cudaMallocHost(&c.pinned_chunk_n, n_chunks * sizeof(int)));
    c.pinned_cap = n_chunks;
  }
  const int* cn = c.pinned_chunk_n;
  SB_CUDA(cudaMemcpyAsync(c.pinned_chunk_n, chunk_n_all, n_chunks * sizeof(int),
                          cudaMemcpyDeviceToHost, s));
  SB_CUDA(cudaStreamSynchronize(s));
  int n_max = 1;
  for (int64_t k = 0; k < n_chunks; ++k) n_max = std::max(n_max, cn[k]);
  // Tables.
  const int L = opt->greek_order;
  ensure_user(c, mu, n_mu, n_max, s);
  BandTables* bt = nullptr;
  if (L >= 0) bt = &ensure_bands(c, L, band_index(n_max), s);
  // The mixed form: values of the fixed grid only.
  const int i8_above = (call && !ad.on && !dv.on) ? call->i8_above : 0;
  auto on_i8 = [&](int nc) { return i8_above > 0 && nc > i8_above && nc <= kI8MaxTerms; };
  unsigned* i8_err = nullptr;
  if (i8_above > 0) {
    ensure_i8(c, n_max, bt, s);
    i8_err = c.i8_err.as<unsigned>(1);
    SB_CUDA(cudaMemsetAsync(i8_err, 0, sizeof(unsigned), s));
    call->i8_err = i8_err;
  }
  // 3. Slabs. Each unit's work: its chunks' rows times the table rows they meet.
  const int nb = bt ? bt->n_bands : 0;
  std::vector<int> band_of_n(n_max + 1, -1), band_tiles(nb), band_nq(nb);
  if (bt) {
    int b = 0;
    for (int n = 1; n <= n_max; ++n) {
      while (bt->desc[b].upper < n) ++b;
      band_of_n[n] = b;
    }
    for (int k = 0; k < nb; ++k) {
      band_tiles[k] = (bt->desc[k].h + 31) / 32;
      band_nq[k] = bt->desc[k].n_q;
    }
  }
  const int t_user = (c.user.h + 31) / 32;
  const int64_t acc_head = 4 * n_mu * n_blk;
  std::vector<int64_t> urows(n_units), uacc(n_units), ui8(n_units, 0), ui8n(n_units, 0);
  std::vector<int> uslots(n_units), utiles(n_units);
  std::vector<double> ucost(n_units);
  int64_t total_rows = 0;
  double total_cost = 0.0;
  for (int64_t u = 0; u < n_units; ++u) {
    const int* cu = cn + u * cpu;
    int64_t rows = 0, acc = acc_head;
    double cost = 0.0;
    int prev = -1, slots = 0, max_tiles = 1;
    for (int k = 0; k < cpu; ++k) {
      const int nc = cu[k];
      rows += (int64_t)rows_per_term * nc;
      if (on_i8(nc)) {
        ui8[u] += 2 * (int64_t)((nc + kI8KB - 1) / kI8KB) * kI8HalfBytes;
        ui8n[u] += 1;
      }
      int tiles = t_user;
      if (bt && nc > 0) {
        const int b = band_of_n[nc];
        tiles += band_tiles[b];
        if (b != prev) {
          acc += 4 * (int64_t)band_nq[b] * n_blk;
          slots += n_blk;
          prev = b;
        }
      }
      cost += (double)tiles * ((double)nc + 24.0) * rows_per_term * (dv.on ? 1.5 : 1.0);
      max_tiles = std::max(max_tiles, tiles);
    }
    urows[u] = rows;
    uacc[u] = acc;
    uslots[u] = slots;
    utiles[u] = max_tiles;
    ucost[u] = cost;
    total_rows += rows;
    total_cost += cost;
  }
  const int64_t max_urows = *std::max_element(urows.begin(), urows.end());
  const int64_t arena = std::max<int64_t>(g_arena_rows.load(), 2 * max_urows);
  std::vector<int> by_cost(n_units);
  for (int64_t u = 0; u < n_units; ++u) by_cost[u] = (int)u;
  std::sort(by_cost.begin(), by_cost.end(), [&](int x, int y) {
    return ucost[x] != ucost[y] ? ucost[x] > ucost[y] : x < y;
  });
  // Cut the units, in order, into slabs of consecutive units (so that a slab's outputs are a few
  // contiguous ranges, copied out while the next slabs run) of about equal work, each within the
  // arena and the chunk limit.
  int64_t n_slabs = std::max<int64_t>(1, (total_rows + arena - 1) / arena);
  n_slabs = std::max<int64_t>(n_slabs, (n_chunks + kMaxSlabChunks - 1) / kMaxSlabChunks);
  std::vector<int> slab_of(n_units);
  std::vector<int64_t> slab_lo;  // the first unit of each slab
  {
    const double target = total_cost / (double)n_slabs;
    int64_t rows = 0, chunks = 0;
    double cost = 0.0;
    for (int64_t u = 0; u < n_units; ++u) {
      if (u == 0 || rows + urows[u] > arena || chunks + cpu > kMaxSlabChunks ||
          cost >= target) {
        slab_lo.push_back(u);
        rows = chunks = 0;
        cost = 0.0;
      }
      slab_of[u] = (int)slab_lo.size() - 1;
      rows += urows[u];
      chunks += cpu;
      cost += ucost[u];
    }
    n_slabs = (int64_t)slab_lo.size();
  }
  // A large unit's row tiles split into work items of about item_target work each.
  const int grid_max = c.sms * c.unit_bps;
  const double item_target =
      std::max(1.0, total_cost / (double)n_slabs / ((double)g_split.load() * grid_max));
  std::vector<int> ugroups(n_units);
  for (int64_t u = 0; u < n_units; ++u)
    ugroups[u] = (int)std::min<double>(std::max(1.0, std::ceil(ucost[u] / item_target)),
                                       (double)utiles[u]);
  struct Slab {
    int64_t u0 = 0, nu = 0;      // units (flat list, slab-major)
    int64_t sl0 = 0, n_slots = 0;
    int64_t pi0 = 0, pi_cap = 0;  // projection items: nb + n_slots / 32 at most
    int64_t it0 = 0, n_items = 0;
    int64_t acc_len = 0;
    int64_t n_proj = 0;
    int64_t i8_bytes = 0, i8_chunks = 0;  // the mixed form's chunk digits
  };
  std::vector<Slab> slabs(n_slabs);
  std::vector<int> members(n_units);
  {
    std::vector<int64_t> count(n_slabs, 0);
    for (int64_t u = 0; u < n_units; ++u) {
      Slab& S = slabs[slab_of[u]];
      count[slab_of[u]]++;
      S.n_slots += uslots[u];
      S.n_items += ugroups[u];
      S.acc_len += uacc[u];
      S.i8_bytes += ui8[u];
      S.i8_chunks += ui8n[u];
    }
    int64_t u0 = 0, sl0 = 0, pi0 = 0, it0 = 0;
    for (int64_t sl = 0; sl < n_slabs; ++sl) {
      Slab& S = slabs[sl];
      S.u0 = u0;
      S.nu = count[sl];
      S.sl0 = sl0;
      S.pi0 = pi0;
      S.pi_cap = 2 * nb + S.n_slots / 32 + 1;
      S.it0 = it0;
      u0 += S.nu;
      sl0 += S.n_slots;
      pi0 += S.pi_cap;
      it0 += S.n_items;
    }
    // by_cost order within each slab: the largest units first.
    std::vector<int64_t> fill(n_slabs, 0);
    for (int64_t k = 0; k < n_units; ++k) {
      const int u = by_cost[k];
      const int sl = slab_of[u];
      members[slabs[sl].u0 + fill[sl]++] = u;
    }
  }
  int64_t acc_max = 1, slots_max = 1, stage_max = 0, n_slots_all = 0, n_proj_all = 0,
          n_items_all = 0, i8_bytes_max = 16, i8_chunks_max = 1;
  auto stage_bytes = [&](const Slab& S) {
    return S.nu * (int64_t)(sizeof(int) + 8 + sizeof(int2)) +
           S.nu * cpu * (int64_t)(sizeof(int) + 16) +
           S.n_slots * (int64_t)(sizeof(BandSlot) + sizeof(int)) +
           S.pi_cap * (int64_t)sizeof(ProjItem) + S.n_items * (int64_t)sizeof(WorkItem) +
           (i8_above > 0 ? S.nu * cpu * (int64_t)(8 + 2 * sizeof(int)) + 64 : 0) + 256;
  };
  for (const Slab& S : slabs) {
    acc_max = std::max(acc_max, S.acc_len);
    slots_max = std::max(slots_max, S.n_slots);
    stage_max = std::max(stage_max, stage_bytes(S));
    n_slots_all += S.n_slots;
    n_proj_all += S.pi_cap;
    n_items_all += S.n_items;
    i8_bytes_max = std::max(i8_bytes_max, S.i8_bytes);
    i8_chunks_max = std::max(i8_chunks_max, S.i8_chunks);
  }
  // Device buffers: the plan's flat arrays (every slab its own segment), arena, scratch, sums.
  int* units_d = c.plan_units.as<int>(n_units);
  int* chunk_n_d = c.chunk_n_slab.as<int>(n_chunks);
  int64_t* chunk_row_d = c.chunk_row.as<int64_t>(n_chunks);
  int64_t* chunk_acc_d = c.chunk_acc.as<int64_t>(n_chunks);
  int64_t* unit_acc_d = c.unit_acc.as<int64_t>(n_units);
  int2* unit_slots_d = c.unit_slots.as<int2>(n_units);
  BandSlot* slots_d = c.slots.as<BandSlot>(std::max<int64_t>(n_slots_all, 1));
  int* slot_index_d = c.slot_index.as<int>(std::max<int64_t>(n_slots_all, 1));
  ProjItem* proj_d = c.proj_items.as<ProjItem>(std::max<int64_t>(n_proj_all, 1));
  WorkItem* items_d = c.items.as<WorkItem>(std::max<int64_t>(n_items_all, 1));
  double* X = c.X.as<double>((size_t)arena * 128);
  const int n_arr = L_layers > 1 ? 2 * L_layers - 1 : 1;
  // Layered derivatives keep each ratio array's derivative beside it.
  const int arr_factor = dv.on && L_layers > 1 ? 2 : 1;
  double2* uz =
      c.uz.as<double2>((size_t)(arena + 2 * kMaxSlabChunks) * 32 * n_arr * arr_factor);
  double* ux = c.ux.as<double>((size_t)(arena + 2 * kMaxSlabChunks) * 32);
  double* chunk_sums = c.chunk_sums.as<double>((size_t)kMaxSlabChunks * 8 * n_blk);
  double* acc = c.acc.as<double>((size_t)acc_max);
  double* slot_greek =
      L >= 0 ? c.slot_greek.as<double>((size_t)slots_max * 6 * (L + 1)) : nullptr;
  int* counter = c.counter.as<int>(64);
  int64_t* chunk_xoff_d = nullptr;
  int* chunk_xidx_d = nullptr;
  int* i8_list_d = nullptr;
  unsigned char* xdig = nullptr;
  double* xside = nullptr;
  double* colmax = nullptr;
  if (i8_above > 0) {
    chunk_xoff_d = c.chunk_xoff.as<int64_t>(n_chunks);
    chunk_xidx_d = c.chunk_xidx.as<int>(n_chunks);
    i8_list_d = c.i8_list.as<int>(n_chunks);
    xdig = c.xdig.as<unsigned char>((size_t)i8_bytes_max);
    xside = c.xside.as<double>((size_t)i8_chunks_max * kI8Side);
    colmax = c.colmax.as<double>((size_t)kMaxSlabChunks * 128);
  }
  c.ensure_staging((size_t)stage_max);
  // 4. Per slab: build its plan into pinned staging, upload it, launch its kernels. The host
  // builds the next slab while the device runs this one.
  MieFixedArgs ka{};
  ka.radius = c.radius.as<double>(0);
  ka.weight = c.weight.as<double>(0);
  ka.wl = wl_dev;
  ka.m = reinterpret_cast<const double2*>(m_dev);
  ka.n_dist = (int)n_dist;
  ka.n_wl = (int)n_wl;
  ka.n_nodes = (int)n_nodes;
  ka.cpu = cpu;
  ka.n_layers = L_layers;
  if (L_layers > 1) {
    ka.fractions = c.fractions.as<double>(0);
    ka.m_layers = reinterpret_cast<const double2*>(layers.m_dev);
  }
  ka.X = X;
  ka.colmax = colmax;  // the mixed form's digit scales; null otherwise
  ka.uz = uz;
  ka.ux = ux;
  ka.chunk_sums = chunk_sums;
  ka.err = err;
  ka.allow_unvalidated = opt->allow_unvalidated;
  if (dv.on) {
    ka.deriv = 1;
    ka.deriv_dir = dv.dir;
    ka.n_theta = dv.n_theta;
    ka.wtheta = c.wtheta.as<double>(0);
  }
  if (ad.on) {
    ka.per_unit = 1;
    ka.wdiff = c.wdiff.as<double>(0);
    if (dv.on) ka.wthdiff = c.wthdiff.as<double>(0);
  }
  UnitArgs ua{};
  ua.radius = ka.radius;
  ua.weight = ka.weight;
  ua.wl = wl_dev;
  ua.n_dist = (int)n_dist;
  ua.n_wl = (int)n_wl;
  ua.n_nodes = (int)n_nodes;
  ua.cpu = cpu;
  ua.X = X;
  ua.n_mu = (int)n_mu;
  ua.h_u = c.user.h;
  ua.h_u_pad = c.user.h_pad;
  ua.ge_u = c.user.ge.as<double>(0);
  ua.go_u = c.user.go.as<double>(0);
  ua.user_map = c.user.map.as<int2>(0);
  ua.greek_order = L;
  if (bt) {
    ua.bands = bt->desc_d.as<BandDesc>(0);
    ua.band_ge = bt->ge_d.as<double>(0);
    ua.band_go = bt->go_d.as<double>(0);
  }
  ua.acc = acc;
  ua.work_counter = counter;
  ua.deriv = ka.deriv;
  ua.n_theta = ka.n_theta;
  ua.wtheta = ka.wtheta;
  ua.per_unit = ka.per_unit;
  ua.wdiff = ka.wdiff;
  ua.wthdiff = ka.wthdiff;
  ua.i8_above = i8_above;
  ProjArgs pj{};
  pj.cpu = cpu;
  pj.greek_order = L;
  pj.acc = acc;
  pj.chunk_sums = chunk_sums;
  pj.slot_greek = slot_greek;
  pj.raw = dv.on && !ad.on ? 1 : 0;
  if (ad.on) pj.unit_norm = c.unit_norm.as<double>(0);
  if (ad.on && dv.on) {
    pj.ad_blocks = 3 + dv.n_theta;
    pj.n_theta = dv.n_theta;
  }
  if (bt) {
    pj.bands = bt->desc_d.as<BandDesc>(0);
    pj.band_d = bt->d_d.as<double>(0);
  }
  FinalArgs fa{};
  fa.cpu = cpu;
  fa.n_dist = (int)n_dist;
  fa.n_wl = (int)n_wl;
  fa.chunk_sums = chunk_sums;
  fa.n_mu = (int)n_mu;
  fa.greek_order = L;
  if (bt) fa.bands = ua.bands;
  fa.slot_greek = slot_greek;
  fa.acc = acc;
  fa.n_units_total = n_units;
  fa.values = values;
  fa.phase = n_mu > 0 ? phase : nullptr;
  fa.greek = L >= 0 ? greek : nullptr;
  fa.normalized = opt->normalized;
  fa.err = err;
  if (dv.on) {
    fa.n_theta = dv.n_theta;
    fa.d_values = dv.d_values;
    fa.d_phase = n_mu > 0 ? dv.d_phase : nullptr;
    fa.d_greek = L >= 0 ? dv.d_greek : nullptr;
  }
  if (ad.on) {
    fa.unit_norm = c.unit_norm.as<double>(0);
    fa.avg = ad.avg;
    if (dv.on) {
      fa.ad_blocks = 3 + dv.n_theta;
      fa.n_theta = dv.n_theta;
      fa.d_values = nullptr;
      fa.d_phase = nullptr;
      fa.d_greek = nullptr;
    }
  }
  std::vector<std::pair<double, int64_t>> order;  // work items by cost
  std::vector<int> per_band;
  for (int64_t sl = 0; sl < n_slabs; ++sl) {
    Slab& S = slabs[sl];
    if (S.nu == 0) continue;
    const int64_t nch = S.nu * cpu;
    // Staging layout of this slab.
    unsigned char* base = c.staging_half(sl & 1);
    auto take = [&](size_t bytes) {
      unsigned char* p = base;
      base += (bytes + 15) / 16 * 16;
      return p;
    };
    int* P_units = (int*)take(S.nu * sizeof(int));
    int64_t* P_uacc = (int64_t*)take(S.nu * 8);
    int2* P_uslots = (int2*)take(S.nu * sizeof(int2));
    int* P_cn = (int*)take(nch * sizeof(int));
    int64_t* P_row = (int64_t*)take(nch * 8);
    int64_t* P_cacc = (int64_t*)take(nch * 8);
    BandSlot* P_slots = (BandSlot*)take(S.n_slots * sizeof(BandSlot));
    int* P_sidx = (int*)take(S.n_slots * sizeof(int));
    ProjItem* P_proj = (ProjItem*)take(S.pi_cap * sizeof(ProjItem));
    WorkItem* P_items = (WorkItem*)take(S.n_items * sizeof(WorkItem));
    int64_t* P_xoff = i8_above > 0 ? (int64_t*)take(nch * 8) : nullptr;
    int* P_xidx = i8_above > 0 ? (int*)take(nch * sizeof(int)) : nullptr;
    int* P_list = i8_above > 0 ? (int*)take(nch * sizeof(int)) : nullptr;
    int64_t xoff = 0;
    int n_i8 = 0;
    const size_t used = (size_t)(base - c.staging_half(sl & 1));
    int64_t row = 0, accpos = 0, nslot = 0;
    order.clear();
    for (int64_t lu = 0; lu < S.nu; ++lu) {
      const int u = members[S.u0 + lu];
      P_units[lu] = u;
      P_uacc[lu] = accpos;
      int64_t band_acc = accpos + acc_head;
      int2 us = make_int2((int)nslot, 0);
      int prev = -1;
      for (int k = 0; k < cpu; ++k) {
        const int64_t ci = lu * cpu + k;
        const int nc = cn[(int64_t)u * cpu + k];
        P_cn[ci] = nc;
        P_row[ci] = row;
        if (P_xoff) {
          P_xoff[ci] = -1;
          P_xidx[ci] = 0;
          if (on_i8(nc)) {
            P_xoff[ci] = xoff;
            P_xidx[ci] = n_i8;
            P_list[n_i8++] = (int)ci;
            xoff += 2 * (int64_t)((nc + kI8KB - 1) / kI8KB) * kI8HalfBytes;
          }
        }
        row += (int64_t)rows_per_term * nc;
        P_cacc[ci] = -1;
        if (bt && nc > 0) {
          const int b = band_of_n[nc];
          if (b != prev) {
            // One slot per block of sums, their tables 4 n_q doubles apart.
            for (int blk = 0; blk < n_blk; ++blk) {
              P_slots[nslot].band = b;
              P_slots[nslot].unit = (int)lu;
              P_slots[nslot].off = band_acc;
              // Adaptive: the value slots, then the error slots; pad is the block.
              P_slots[nslot].kind = ad.on ? (2 * blk >= n_blk ? 1 : 0) : 0;
              P_slots[nslot].pad = ad.on ? blk % (n_blk / 2) : 0;
              band_acc += 4 * (int64_t)band_nq[b];
              ++nslot;
            }
            us.y += n_blk;
            prev = b;
          }
          P_cacc[ci] = P_slots[nslot - n_blk].off;
        }
      }
      P_uslots[lu] = us;
      accpos += uacc[u];
      const int G = ugroups[u];
      for (int g = 0; g < G; ++g) order.emplace_back(-ucost[u] / G, lu * 65536 + g);
    }
    std::stable_sort(order.begin(), order.end(),
                     [](const std::pair<double, int64_t>& x, const std::pair<double, int64_t>& y) {
                       return x.first < y.first;
                     });
    for (size_t k = 0; k < order.size(); ++k) {
      const int64_t lu = order[k].second / 65536;
      P_items[k].unit = (int)lu;
      P_items[k].group = (int)(order[k].second % 65536);
      P_items[k].n_groups = ugroups[P_units[lu]];
      P_items[k].pad = 0;
    }
    // Projection tiles: the slab's slots grouped by band (largest bands first), 32 at a time.
    S.n_proj = 0;
    if (bt && S.n_slots > 0) {
      // Slots grouped by (band, kind): a tile's slots share the band's matrices and the kind
      // (values or bounds) of its projection.
      const int nk = ad.on ? 2 : 1, ng = nb * nk;
      per_band.assign(ng + 1, 0);
      auto key = [&](const BandSlot& x) { return x.band * nk + (nk > 1 ? x.kind : 0); };
      for (int64_t k = 0; k < S.n_slots; ++k) per_band[key(P_slots[k]) + 1]++;
      std::vector<int64_t> start(ng + 1, 0), cursor(ng, 0);
      // Bands in descending order occupy the slot-index list from the front.
      int64_t pos = 0;
      for (int g = ng - 1; g >= 0; --g) {
        start[g] = pos;
        pos += per_band[g + 1];
      }
      for (int g = 0; g < ng; ++g) cursor[g] = start[g];
      for (int64_t k = 0; k < S.n_slots; ++k) P_sidx[cursor[key(P_slots[k])]++] = (int)k;
      for (int g = ng - 1; g >= 0; --g)
        for (int64_t k0 = 0; k0 < per_band[g + 1]; k0 += 32) {
          ProjItem& pi = P_proj[S.n_proj++];
          pi.band = g / nk;
          pi.kind = g % nk;
          pi.pad = 0;
          pi.count = (int)std::min<int64_t>(32, per_band[g + 1] - k0);
          pi.first = start[g] + k0;
        }
    }
    // Upload (pinned source: asynchronous) once the staging half's previous upload is done.
    (void)used;
    SB_CUDA(cudaMemcpyAsync(units_d + S.u0, P_units, S.nu * sizeof(int), cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(unit_acc_d + S.u0, P_uacc, S.nu * 8, cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(unit_slots_d + S.u0, P_uslots, S.nu * sizeof(int2),
                            cudaMemcpyHostToDevice, s));
    const int64_t ch0 = S.u0 * cpu;
    SB_CUDA(cudaMemcpyAsync(chunk_n_d + ch0, P_cn, nch * sizeof(int), cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(chunk_row_d + ch0, P_row, nch * 8, cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(chunk_acc_d + ch0, P_cacc, nch * 8, cudaMemcpyHostToDevice, s));
    if (S.n_slots > 0) {
      SB_CUDA(cudaMemcpyAsync(slots_d + S.sl0, P_slots, S.n_slots * sizeof(BandSlot),
                              cudaMemcpyHostToDevice, s));
      SB_CUDA(cudaMemcpyAsync(slot_index_d + S.sl0, P_sidx, S.n_slots * sizeof(int),
                              cudaMemcpyHostToDevice, s));
    }
    if (S.n_proj > 0)
      SB_CUDA(cudaMemcpyAsync(proj_d + S.pi0, P_proj, S.n_proj * sizeof(ProjItem),
                              cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(items_d + S.it0, P_items, S.n_items * sizeof(WorkItem),
                            cudaMemcpyHostToDevice, s));
    if (i8_above > 0) {
      SB_CUDA(cudaMemcpyAsync(chunk_xoff_d + ch0, P_xoff, nch * 8, cudaMemcpyHostToDevice, s));
      SB_CUDA(cudaMemcpyAsync(chunk_xidx_d + ch0, P_xidx, nch * sizeof(int),
                              cudaMemcpyHostToDevice, s));
      if (n_i8 > 0)
        SB_CUDA(cudaMemcpyAsync(i8_list_d + ch0, P_list, n_i8 * sizeof(int),
                                cudaMemcpyHostToDevice, s));
    }
    c.staging_uploaded(sl & 1, s);
    // Launches.
    ka.units = units_d + S.u0;
    ka.n_chunks = (int)nch;
    ka.chunk_n = chunk_n_d + ch0;
    ka.chunk_row = chunk_row_d + ch0;
    timed_launch(K_MIE, s, [&] { launch_mie_fixed(ka, s); });
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaMemsetAsync(acc, 0, (size_t)S.acc_len * 8, s));
    SB_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), s));
    ua.units = ka.units;
    ua.n_items = (int)S.n_items;
    ua.items = items_d + S.it0;
    ua.chunk_n = ka.chunk_n;
    ua.chunk_row = ka.chunk_row;
    ua.chunk_acc = chunk_acc_d + ch0;
    ua.unit_acc = unit_acc_d + S.u0;
    const int grid = (int)std::min<int64_t>(grid_max, S.n_items);
    timed_launch(K_UNITS, s, [&] { launch_units(ua, grid, s); });
    SB_CUDA(cudaGetLastError());
    if (i8_above > 0 && n_i8 > 0) {
      // The mixed form: the int8 chunks' digits, then their angle GEMMs on the tensor cores.
      XSplitArgs xa{};
      xa.X = X;
      xa.colmax = colmax;
      xa.chunk_row = ua.chunk_row;
      xa.chunk_n = ua.chunk_n;
      xa.list = i8_list_d + ch0;
      xa.n = n_i8;
      xa.chunk_xoff = chunk_xoff_d + ch0;
      xa.chunk_xidx = chunk_xidx_d + ch0;
      xa.xdig = xdig;
      xa.xside = xside;
      xa.radius = ua.radius;
      xa.weight = ua.weight;
      xa.wl = wl_dev;
      xa.units = ua.units;
      xa.n_wl = (int)n_wl;
      xa.n_nodes = (int)n_nodes;
      xa.cpu = cpu;
      timed_launch(K_X_SPLIT, s, [&] { launch_x_split(xa, s); });
      SB_CUDA(cudaGetLastError());
      UnitI8Args ia{};
      ia.radius = ua.radius;
      ia.weight = ua.weight;
      ia.wl = wl_dev;
      ia.n_dist = (int)n_dist;
      ia.n_wl = (int)n_wl;
      ia.n_nodes = (int)n_nodes;
      ia.cpu = cpu;
      ia.units = ua.units;
      ia.n_items = ua.n_items;
      ia.items = ua.items;
      ia.chunk_n = ua.chunk_n;
      ia.chunk_acc = ua.chunk_acc;
      ia.unit_acc = ua.unit_acc;
      ia.n_mu = (int)n_mu;
      ia.h_u = c.user.h;
      ia.user_map = ua.user_map;
      ia.greek_order = L;
      ia.bands = ua.bands;
      ia.acc = acc;
      ia.chunk_xoff = xa.chunk_xoff;
      ia.chunk_xidx = xa.chunk_xidx;
      ia.xdig = xdig;
      ia.xside = xside;
      ia.tdig = c.i8.dig.as<unsigned char>(0);
      ia.tscale = c.i8.scale.as<double>(0);
      ia.user_tabs = c.i8.user_d.as<I8Table>(0);
      ia.n_user_tabs = (int)c.i8.user.size();
      ia.band_tabs = c.i8.band_d.as<I8Table>(0);
      ia.levels = call->i8_levels;
      ia.err = i8_err;
      const int grid8 = (int)std::min<int64_t>(c.sms, S.n_items);
      cudaError_t le = cudaSuccess;
      timed_launch(K_UNITS_I8, s, [&] { le = launch_units_i8(ia, grid8, s); });
      SB_CUDA(le);
    }
    if (bt && S.n_proj > 0) {
      pj.items = proj_d + S.pi0;
      pj.n_items = (int)S.n_proj;
      pj.slot_index = slot_index_d + S.sl0;
      pj.slots = slots_d + S.sl0;
      pj.units = ka.units;
      timed_launch(K_PROJ, s, [&] { launch_proj(pj, s); });
      SB_CUDA(cudaGetLastError());
    }
    fa.units = ka.units;
    fa.n_units = (int)S.nu;
    fa.unit_acc = ua.unit_acc;
    fa.unit_slots = unit_slots_d + S.u0;
    fa.slots = slots_d + S.sl0;
    timed_launch(K_FINAL, s, [&] { launch_final(fa, s); });
    SB_CUDA(cudaGetLastError());
    if (call && call->h_values && !ad.on && !dv.on) {
      // This slab's units are [lo, hi): copy their outputs out beside the next slabs.
      const int64_t lo = slab_lo[sl], hi = sl + 1 < n_slabs ? slab_lo[sl + 1] : n_units;
      const int64_t nu = hi - lo, glen = opt->greek_order + 1;
      SB_CUDA(cudaEventRecord(c.slab_done, s));
      SB_CUDA(cudaStreamWaitEvent(c.copies, c.slab_done, 0));
      for (int k = 0; k < 11; ++k)
        SB_CUDA(cudaMemcpyAsync(call->h_values + k * n_units + lo, values + k * n_units + lo,
                                nu * 8, cudaMemcpyDeviceToHost, c.copies));
      for (int e = 0; e < 6 && call->h_phase && n_mu > 0; ++e)
        SB_CUDA(cudaMemcpyAsync(call->h_phase + (e * n_units + lo) * n_mu,
                                phase + (e * n_units + lo) * n_mu, nu * n_mu * 8,
                                cudaMemcpyDeviceToHost, c.copies));
      for (int e = 0; e < 6 && call->h_greek && glen > 0; ++e)
        SB_CUDA(cudaMemcpyAsync(call->h_greek + (e * n_units + lo) * glen,
                                greek + (e * n_units + lo) * glen, nu * glen * 8,
                                cudaMemcpyDeviceToHost, c.copies));
    }
  }
  if (call && !ad.on) {
    call->radius = std::move(radius);
    call->n_dist = n_dist;
    call->n_wl = n_wl;
    call->n_nodes = n_nodes;
  }
}

// Reads the error words of the last call (synchronizes the stream).
void check_device_errors(Context& c, cudaStream_t s, const FixedCall* call) {
  unsigned long long h[2];
  SB_CUDA(cudaMemcpyAsync(h, c.err.as<unsigned long long>(2), sizeof h, cudaMemcpyDeviceToHost, s));
  SB_CUDA(cudaStreamSynchronize(s));
  // A forced node error (test hook) merges as a kernel's atomicMin would: the first in order.
  h[0] = std::min(h[0], g_forced_node_error.exchange(~0ull));
  if (call && call->i8_err) {
    unsigned f = 0;
    SB_CUDA(cudaMemcpy(&f, call->i8_err, sizeof f, cudaMemcpyDeviceToHost));
    if (f)
      throw Failure{SCATRS_CUDA,
                    "the int8 angle GEMMs gave up waiting on the tensor cores or the copies "
                    "(bounded wait)"};
  }
  if (h[0] != ~0ull) {
    int status = (int)(h[0] & 3);
    unsigned long long key = h[0] >> 2;
    std::string msg = "a size node's inputs are invalid";
    if (call && call->n_nodes > 0) {
      int64_t j = key % call->n_nodes;
      int64_t d = (key / call->n_nodes) % call->n_dist;
      int64_t i = key / call->n_nodes / call->n_dist;
      double lam = i < (int64_t)call->wl_host.size() ? call->wl_host[i] : NAN;
      const int64_t row = call->per_unit ? d * call->n_wl + i : d;
      const size_t at = (size_t)(row * call->n_nodes + j);
      msg = node_message(status, lam, at < call->radius.size() ? call->radius[at] : NAN);
    }
    throw Failure{status, msg};
  }
  if (h[1] != ~0ull) {
    int which = (int)(h[1] & 3);
    const char* what = which == 1 ? "<C_ext>" : which == 2 ? "<C_sca>" : "<C_back>";
    throw Failure{SCATRS_INVALID_INPUT,
                  std::string("the ensemble's ") + what +
                      " is 0 or not finite, so its ratios (albedo, asymmetry parameter, lidar "
                      "ratio) are undefined (does m = 1?)"};
  }
}

// One part of an adaptive call (engine.rs:78-112): a distribution (or a mode of one), its
// sphere's m per wavelength (host), its number fraction in its output unit, that unit, and the
// prefix of its validation errors.
struct AdPart {
  int kind;
  double p[3];
  const double* m;
  double f;
  int out;
  std::string who;
  const double* table = nullptr;  // a tabulated distribution's table
  int64_t table_len = 0;
  // Derivatives (engine.rs:95-115, 153-176): the requested distribution parameters (indices
  // into the density's gradient) and their result columns, the columns along the particle's
  // directions (-1: not requested; a sphere's Re m and Im m, a layered sphere's Re m_l and
  // Im m_l per layer and then each radius fraction), and the part's component, mode (-1:
  // none) and weights w (the component's), v (the mode's) and v_total (the component's mode
  // weights' sum).
  std::vector<int> grads, theta_cols;
  std::vector<int> dir_cols = std::vector<int>(2, -1);
  int component = 0, mode = -1;
  double w = 1.0, v = 1.0, v_total = 1.0;
};

// The derivative outputs of an adaptive call: the requested parameters and the arrays
// d_values, d_errors [P][11][n], d_phase, d_phase_err [P][6][n][n_mu], d_greek, d_greek_err
// [P][6][n][L + 1].
struct AdDerivs {
  const scatrs_param* params = nullptr;
  int64_t n = 0;
  double *d_values = nullptr, *d_errors = nullptr, *d_phase = nullptr, *d_phase_err = nullptr,
         *d_greek = nullptr, *d_greek_err = nullptr;
};

// Lin (ensemble/lin.rs:7-68): a value with its error estimate, its derivatives along the
// requested parameters and theirs, through the ratios with the quotient rule and first-order
// bounds.
struct LinD {
  double v = 0.0, e = 0.0;
  std::vector<double> d, de;
  static LinD constant(double v, size_t n) {
    LinD x;
    x.v = v;
    x.d.assign(n, 0.0);
    x.de.assign(n, 0.0);
    return x;
  }
  LinD div(const LinD& b) const {
    LinD o;
    o.v = v / b.v;
    o.e = (e + std::fabs(o.v) * b.e) / std::fabs(b.v);
    const size_t n = d.size();
    o.d.resize(n);
    o.de.resize(n);
    for (size_t k = 0; k < n; ++k) o.d[k] = (d[k] - o.v * b.d[k]) / b.v;
    for (size_t k = 0; k < n; ++k)
      o.de[k] = (de[k] + std::fabs(o.v) * b.de[k] + std::fabs(o.d[k]) * b.e +
                 o.e * std::fabs(b.d[k])) /
                std::fabs(b.v);
    return o;
  }
  LinD scale(double c) const {
    LinD o = *this;
    o.v = c * v;
    o.e = std::fabs(c) * e;
    for (size_t k = 0; k < d.size(); ++k) {
      o.d[k] = c * d[k];
      o.de[k] = std::fabs(c) * de[k];
    }
    return o;
  }
};

struct AdOutputs {
  double *values, *errors, *phase, *phase_err, *greek, *greek_err;
  int8_t* converged;
  int64_t* panels;
};

// The adaptive ensemble of `parts` mixed into n_out output units (engine.rs:236-296 run and
// run_batch, 1964-2250 wavelength): the parts' cut-offs and moments; pass 1 with each part on its
// own panels, or (batch) every part with a range on one shared group per wavelength; pass 2 on
// the final panels; each part's averages; the mixing and the outputs per (output unit,
// wavelength), unit-major.
// With layers (n_layers > 1), every part p is a layered sphere with the fractions
// layers->fractions[p][L - 1] and indices layers->m[p][L][n_wl] (the parts' m unused).
// converged: every part of the output unit; panels: the sum over its distinct groups
// (engine.rs:2228-2236).
void adaptive_flags(const std::vector<AdPart>& in, const std::vector<adaptive::Job>& jobs,
                    const std::vector<int>& job_of, const std::vector<char>& unit_converged,
                    const std::vector<int64_t>& unit_panels, int n_out, int64_t n_wl,
                    const AdOutputs& res) {
  (void)jobs;
  for (int ou = 0; ou < n_out; ++ou)
    for (int64_t i = 0; i < n_wl; ++i) {
      bool conv = true;
      int64_t pan = 0;
      std::vector<int> seen;
      for (size_t p = 0; p < in.size(); ++p) {
        if (in[p].out != ou) continue;
        const int64_t u = (int64_t)p * n_wl + i;
        conv = conv && unit_converged[u];
        const int g = job_of[u];
        if (g >= 0 && std::find(seen.begin(), seen.end(), g) == seen.end()) {
          seen.push_back(g);
          pan += unit_panels[u];
        }
      }
      if (res.converged) res.converged[ou * n_wl + i] = conv ? 1 : 0;
      if (res.panels) res.panels[ou * n_wl + i] = pan;
    }
}

// The mixing and outputs of an adaptive call with derivatives, on the host from the parts'
// per-block averages (final_adaptive_d_kernel's rows): per output unit and wavelength, the
// number fractions f (engine.rs:2121-2140) on the values, errors and each block's column, the
// weight derivatives df (2141-2176: of w/w_total for a component's weight, of v/v_total for a
// mode's), then the ratios, normalizations and bounds with the derivatives (lin.rs,
// engine.rs:2396-2497) and the Greek coefficients normalized by the mixture's alpha1_0.
// hav_x: with single radii whose radius is asked for, the rows of the pass along x, whose Re m
// block is d/dx of every slot at fixed m; d/dr = (2 pi / lambda) d/dx there (pi r^2 (2/x^2) is
// constant: the 2 pi r Q term of engine.rs:1158-1170 cancels the -2/x Q of dQ/dx), with 2 r and
// 3 r^2 for <r^2> and <r^3>.
void mix_derivatives(const std::vector<AdPart>& in, const std::vector<adaptive::Part>& parts,
                     int n_out, int64_t n_wl, int64_t n_mu, int greek_order, bool normalized,
                     int n_theta, const std::vector<double>& hav, const AdDerivs& dd,
                     const AdOutputs& res, const double* wavelengths,
                     const std::vector<double>& hav_x) {
  // Blocks per part: the values, n_theta parameters, then every direction of the particle.
  const int n_dirs = in.empty() ? 2 : (int)in[0].dir_cols.size();
  const int B = 1 + n_theta + n_dirs;
  const int64_t glen = greek_order >= 0 ? greek_order + 1 : 0;
  const int64_t row = 8 + 4 * n_mu + 6 * glen, stride = 2 * B * row;
  const size_t P = (size_t)dd.n;
  const int64_t n_outs = (int64_t)n_out * n_wl;
  // The result column of block b of part p (-1: none).
  auto column = [&](const AdPart& a, int b) {
    if (b >= 1 && b <= n_theta) return b - 1 < (int)a.theta_cols.size() ? a.theta_cols[b - 1] : -1;
    const int k = b - n_theta - 1;
    if (k >= 0 && k < (int)a.dir_cols.size()) return a.dir_cols[k];
    return -1;
  };
  std::vector<double> v(row), e(row), d(P * row), de(P * row);
  for (int ou = 0; ou < n_out; ++ou) {
    double w_total = 0.0;
    {
      std::vector<int> comps;
      for (const AdPart& a : in)
        if (a.out == ou && std::find(comps.begin(), comps.end(), a.component) == comps.end()) {
          comps.push_back(a.component);
          w_total += a.w;
        }
    }
    for (int64_t i = 0; i < n_wl; ++i) {
      std::fill(v.begin(), v.end(), 0.0);
      std::fill(e.begin(), e.end(), 0.0);
      std::fill(d.begin(), d.end(), 0.0);
      std::fill(de.begin(), de.end(), 0.0);
      for (size_t p = 0; p < in.size(); ++p) {
        const AdPart& a = in[p];
        if (a.out != ou) continue;
        const double* av = hav.data() + ((int64_t)p * n_wl + i) * stride;
        for (int64_t k = 0; k < row; ++k) {
          v[k] += a.f * av[k];
          e[k] += a.f * av[row + k];
        }
        for (int b = 1; b < B; ++b) {
          const int col = column(a, b);
          if (col < 0) continue;
          for (int64_t k = 0; k < row; ++k) {
            d[col * row + k] += a.f * av[2 * b * row + k];
            de[col * row + k] += a.f * av[(2 * b + 1) * row + k];
          }
        }
        if (parts[p].support == adaptive::POINT && !a.grads.empty() && !hav_x.empty()) {
          // monodisperse (engine.rs:1857-1883): exact, no error estimate.
          const int col = a.theta_cols[0];
          const double r = parts[p].lo, kw = 2.0 * kPi / wavelengths[i];
          const double* ax = hav_x.data() + ((int64_t)p * n_wl + i) * stride +
                             2 * (n_theta + 1) * row;
          for (int64_t k = 1; k < row; ++k)
            d[col * row + k] += a.f * (k == 6 ? 2.0 * r : k == 7 ? 3.0 * r * r : kw * ax[k]);
        }
      }
      for (size_t col = 0; col < P; ++col) {
        const scatrs_param& pr = dd.params[col];
        if (pr.kind != SCATRS_PARAM_WEIGHT) continue;
        for (size_t p = 0; p < in.size(); ++p) {
          const AdPart& a = in[p];
          if (a.out != ou) continue;
          const double f = a.w / w_total * a.v / a.v_total;
          double df;
          if (pr.mode < 0) {
            const double own = a.component == pr.component ? a.v / a.v_total : 0.0;
            df = (own - f) / w_total;
          } else if (a.component != pr.component) {
            df = 0.0;
          } else {
            const double own = a.mode == pr.mode ? 1.0 : 0.0;
            df = a.w / w_total * (own - a.v / a.v_total) / a.v_total;
          }
          const double* av = hav.data() + ((int64_t)p * n_wl + i) * stride;
          for (int64_t k = 0; k < row; ++k) {
            d[col * row + k] += df * av[k];
            de[col * row + k] += std::fabs(df) * av[row + k];
          }
        }
      }
      auto lin = [&](int64_t k) {
        LinD x;
        x.v = v[k];
        x.e = e[k];
        x.d.resize(P);
        x.de.resize(P);
        for (size_t c = 0; c < P; ++c) {
          x.d[c] = d[c * row + k];
          x.de[c] = de[c * row + k];
        }
        return x;
      };
      const LinD ext = lin(1), sca = lin(2), scag = lin(3), ab = lin(4), back = lin(5),
                 r2 = lin(6), r3 = lin(7);
      const LinD* dens[3] = {&ext, &sca, &back};
      const char* names[3] = {"<C_ext>", "<C_sca>", "<C_back>"};
      for (int k = 0; k < 3; ++k)
        if (!(std::isfinite(dens[k]->v) && dens[k]->v != 0.0))
          throw Failure{SCATRS_INVALID_INPUT,
                        std::string("the ensemble's ") + names[k] +
                            " is 0 or not finite, so its ratios (albedo, asymmetry parameter, "
                            "lidar ratio) are undefined (does m = 1?)"};
      const LinD sc[11] = {ext,
                           sca,
                           ab,
                           back,
                           sca.div(ext),
                           scag.div(sca),
                           ext.div(back).scale(4.0 * kPi),
                           LinD::constant(0.0, P),
                           r3.div(r2),
                           r2.scale(kPi),
                           r3.scale(4.0 * kPi / 3.0)};
      const int64_t ox = ou * n_wl + i;
      for (int k = 0; k < 11; ++k) {
        res.values[k * n_outs + ox] = sc[k].v;
        if (res.errors) res.errors[k * n_outs + ox] = sc[k].e;
        for (size_t c = 0; c < P; ++c) {
          if (dd.d_values) dd.d_values[(c * 11 + k) * n_outs + ox] = sc[k].d[c];
          if (dd.d_errors) dd.d_errors[(c * 11 + k) * n_outs + ox] = sc[k].de[c];
        }
      }
      if (n_mu > 0) {
        const int src[6] = {0, 1, 0, 2, 3, 2};
        for (int el = 0; el < 6; ++el)
          for (int64_t j = 0; j < n_mu; ++j) {
            LinD f = lin(8 + src[el] * n_mu + j);
            if (normalized) f = f.div(sca);
            const int64_t at = (el * n_outs + ox) * n_mu + j;
            if (res.phase) res.phase[at] = f.v;
            if (res.phase_err) res.phase_err[at] = f.e;
            for (size_t c = 0; c < P; ++c) {
              const int64_t atd = (((int64_t)c * 6 + el) * n_outs + ox) * n_mu + j;
              if (dd.d_phase) dd.d_phase[atd] = f.d[c];
              if (dd.d_phase_err) dd.d_phase_err[atd] = f.de[c];
            }
          }
      }
      if (glen > 0) {
        const int64_t g0 = 8 + 4 * n_mu;
        const LinD a0 = lin(g0);
        for (int el = 0; el < 6; ++el)
          for (int64_t l = 0; l < glen; ++l) {
            LinD x = lin(g0 + el * glen + l);
            if (normalized) x = (el == 0 && l == 0) ? LinD::constant(1.0, P) : x.div(a0);
            const int64_t at = (el * n_outs + ox) * glen + l;
            if (res.greek) res.greek[at] = x.v;
            if (res.greek_err) res.greek_err[at] = x.e;
            for (size_t c = 0; c < P; ++c) {
              const int64_t atd = (((int64_t)c * 6 + el) * n_outs + ox) * glen + l;
              if (dd.d_greek) dd.d_greek[atd] = x.d[c];
              if (dd.d_greek_err) dd.d_greek_err[atd] = x.de[c];
            }
          }
      }
    }
  }
}

// With dd (derivatives), pass 1 refines the requested parameters' blocks too, pass 2 runs the
// derivative blocks of every part, and the mixing (with the weight derivatives) and the
// outputs are assembled on the host from the parts' per-block averages.
// The parts' averages of an adaptive call (final_adaptive_kernel's rows, per (part, wavelength)
// unit: 8 scalars, 4 n_mu cosine values, 6 (L + 1) Greek coefficients, then their errors), with
// each unit's converged flag and panel count, for a mixture's host assembly.
struct PartRows {
  std::vector<double> rows;
  int64_t stride = 0;
  std::vector<char> converged;
  std::vector<int64_t> panels;
};

// A single radius's radius derivative (engine.rs:1158-1170, 1857-1883) into its first parameter
// block of an adaptive call's per-block rows (zero there: a point has no weight derivatives), as
// mix_derivatives adds it: d/dr = (2 pi / lambda) d/dx of every slot from the x rows hav_x,
// 2 r and 3 r^2 for <r^2> and <r^3>, no error estimate.
void place_radius_rows(const std::vector<AdPart>& in, const std::vector<adaptive::Part>& parts,
                       int64_t n_wl, const double* wavelengths, int n_theta, int64_t row,
                       int64_t stride, const std::vector<double>& hav_x, std::vector<double>& hav) {
  for (size_t p = 0; p < parts.size(); ++p) {
    if (parts[p].support != adaptive::POINT || in[p].grads.empty()) continue;
    const double r = parts[p].lo;
    for (int64_t i = 0; i < n_wl; ++i) {
      const int64_t u = (int64_t)p * n_wl + i;
      double* blk = hav.data() + u * stride + 2 * row;
      const double* ax = hav_x.data() + u * stride + 2 * (n_theta + 1) * row;
      const double kw = 2.0 * kPi / wavelengths[i];
      for (int64_t k = 0; k < row; ++k) {
        blk[k] = k == 0 ? 0.0 : k == 6 ? 2.0 * r : k == 7 ? 3.0 * r * r : kw * ax[k];
        blk[row + k] = 0.0;
      }
    }
  }
}

// With n_max_out, only pass 1 runs (and its errors are reported): n_max_out receives each
// (part, wavelength) unit's largest number of terms, its group's (engine.rs:1987-2030). With
// rows_out, the parts' averages go there instead of the outputs: without derivatives as
// PartRows describes, with them final_adaptive_d_kernel's rows (per block, values then
// errors, 8 + 4 n_mu + 6 (L + 1) each; blocks the values, n_theta parameters and every
// direction of the particle).
void adaptive_call_order(const std::vector<AdPart>& in, int n_out, bool batch,
                         const double* wavelengths, int64_t n_wl, const double* mu, int64_t n_mu,
                         const scatrs_adaptive_options* options, const AdOutputs& res,
                         const scatrs_layers* layers = nullptr, const AdDerivs* dd = nullptr,
                         std::vector<int64_t>* n_max_out = nullptr,
                         PartRows* rows_out = nullptr) {
  if (!options) throw Failure{SCATRS_INVALID_INPUT, "options must not be NULL"};
  if (n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
  const adaptive::Options o{options->rtol, options->max_panels, options->allow_unvalidated != 0,
                            options->refine_backscatter != 0};
  // ensemble/mod.rs:688-720.
  if (!(o.rtol >= 1e-13 && o.rtol <= 0.1)) {
    char buf[80];
    snprintf(buf, sizeof buf, "rtol must be in [1e-13, 0.1], got %g", o.rtol);
    throw Failure{SCATRS_INVALID_INPUT, buf};
  }
  if (o.max_panels < 1) throw Failure{SCATRS_INVALID_INPUT, "max_panels must be at least 1"};
  for (int64_t i = 0; i < n_wl; ++i)
    if (!(std::isfinite(wavelengths[i]) && wavelengths[i] > 0.0))
      throw Failure{SCATRS_INVALID_INPUT,
                    "wavelength " + std::to_string(i) + " must be finite and > 0"};
  scatrs_fixed_options fo{32, options->greek_order, options->normalized,
                          options->allow_unvalidated};
  const int64_t n_parts = (int64_t)in.size();
  const int64_t n_units = n_parts * n_wl;  // pipeline units: (part, wavelength)
  check_options(&fo, (int64_t)n_out * n_wl, n_mu, mu);
  if (n_units == 0 || n_out == 0) return;
  const bool deriv = dd && dd->n > 0;
  std::vector<adaptive::Part> parts;
  bool radius_x = false;  // a single radius's radius: a pass along x
  int n_theta = 0;  // the most requested distribution parameters of a part
  bool any_dirs = false;
  for (const AdPart& p : in) {
    try {
      parts.push_back(adaptive::make_part(p.kind, p.p, o.rtol, p.table, p.table_len, p.grads));
    } catch (const adaptive::Error& e) {
      throw Failure{e.status, p.who + e.msg};
    }
    if ((int)p.dir_cols.size() > adaptive::kMaxAllDirs)
      throw Failure{SCATRS_INVALID_INPUT, "the GPU path takes 1 to 16 layers"};
    parts.back().dirs.assign(p.dir_cols.size(), 0);
    for (size_t k = 0; k < p.dir_cols.size(); ++k) parts.back().dirs[k] = p.dir_cols[k] >= 0;
    n_theta = std::max(n_theta, (int)p.grads.size());
    any_dirs = any_dirs || parts.back().dir_derivatives();
    if (!p.grads.empty() && parts.back().support == adaptive::POINT) radius_x = true;
  }
  Context& c = context();
  std::lock_guard<std::mutex> lk(c.mtx);
  cudaStream_t s = 0;
  double* wl_d = c.wl.as<double>(n_wl);
  SB_CUDA(cudaMemcpyAsync(wl_d, wavelengths, n_wl * 8, cudaMemcpyHostToDevice, s));
  // Each pipeline unit's m, and a distinct index per (part, wavelength) for pass 1.
  const int L = layers && layers->n_layers > 1 ? layers->n_layers : 1;
  if (L > kMaxLayersAbi) throw Failure{SCATRS_INVALID_INPUT, "the GPU path takes 1 to 16 layers"};
  if (L > 1 && (!layers->fractions || !layers->m))
    throw Failure{SCATRS_INVALID_INPUT, "layers must give fractions and m"};
  if (L > 1 && radius_x && L + 1 > kMaxLayersAbi)
    throw Failure{SCATRS_INVALID_INPUT,
                  "the radius derivative of a single layered sphere takes at most 15 layers"};
  // A layered sphere's direction groups with a requested direction (any part's): group l < L is
  // layer l's index (directions 2 l, 2 l + 1), group L + f the radius fraction f (direction
  // 2 L + f).
  std::vector<int> groups;
  const int n_dirs_all = L > 1 ? 3 * L - 1 : 2;
  if (L > 1 && any_dirs)
    for (int g = 0; g < 2 * L - 1; ++g) {
      bool want = false;
      for (const AdPart& p : in) {
        if ((int)p.dir_cols.size() != n_dirs_all)
          throw Failure{SCATRS_INVALID_INPUT, "a layered part's directions must number 3 L - 1"};
        if (g < L)
          want = want || p.dir_cols[2 * g] >= 0 || p.dir_cols[2 * g + 1] >= 0;
        else
          want = want || p.dir_cols[2 * L + (g - L)] >= 0;
      }
      if (want) groups.push_back(g);
    }
  std::vector<double> m_unit(2 * n_units, 0.0);
  if (L == 1)
    for (int64_t u = 0; u < n_units; ++u) {
      const int64_t p = u / n_wl, i = u % n_wl;
      m_unit[2 * u] = in[p].m[2 * i];
      m_unit[2 * u + 1] = in[p].m[2 * i + 1];
    }
  double* m_d = c.m.as<double>(2 * n_units);
  SB_CUDA(cudaMemcpyAsync(m_d, m_unit.data(), 2 * n_units * 8, cudaMemcpyHostToDevice, s));
  // Layered parts: the fractions and layer indices on the device for pass 1 and pass 2.
  double* fr_d = nullptr;
  double* ml_d = nullptr;
  if (L > 1) {
    for (int64_t p = 0; p < n_parts; ++p)
      for (int l = 0; l < L - 1; ++l) {
        const double f = layers->fractions[p * (L - 1) + l];
        const double prev = l > 0 ? layers->fractions[p * (L - 1) + l - 1] : 0.0;
        if (!(f > 0.0 && f <= 1.0 && f >= prev))
          throw Failure{SCATRS_INVALID_INPUT,
                        in[p].who + "radius fractions must be nondecreasing in (0, 1]"};
      }
    fr_d = c.p1_fr.as<double>((size_t)n_parts * (L - 1));
    ml_d = c.p1_ml.as<double>((size_t)2 * n_parts * L * n_wl);
    SB_CUDA(cudaMemcpyAsync(fr_d, layers->fractions, (size_t)n_parts * (L - 1) * 8,
                            cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(ml_d, layers->m, (size_t)2 * n_parts * L * n_wl * 8,
                            cudaMemcpyHostToDevice, s));
  }
  // Node evaluations on the device (queries carry the pipeline unit in `wl`), in batches of at
  // most kRows scratch rows.
  constexpr int64_t kRows = int64_t(1) << 26;
  double* wl_unit_d = c.p1_wlu.as<double>(n_units);
  {
    std::vector<double> wlu(n_units);
    for (int64_t u = 0; u < n_units; ++u) wlu[u] = wavelengths[u % n_wl];
    SB_CUDA(cudaMemcpyAsync(wl_unit_d, wlu.data(), n_units * 8, cudaMemcpyHostToDevice, s));
  }
  // A layered sphere's derivatives: each node's kGroup quantities per direction (all
  // 3 L - 1), filled by one pass per requested group, read by pass 1 through NodeResult::dq.
  const bool layered_dirs = L > 1 && any_dirs;
  std::vector<double> dq_store;
  const int64_t row_cap =
      layered_dirs ? std::max<int64_t>(int64_t(1) << 20, kRows / (2 * (2 * L - 1))) : kRows;
  auto eval = [&](const std::vector<adaptive::Query>& qs, std::vector<adaptive::NodeResult>& out) {
    size_t k0 = 0;
    std::vector<double> r;
    std::vector<int> wi;
    std::vector<int64_t> off;
    const int64_t dstride = (int64_t)n_dirs_all * adaptive::kGroup;
    if (layered_dirs) dq_store.assign(qs.size() * (size_t)dstride, 0.0);
    while (k0 < qs.size()) {
      r.clear();
      wi.clear();
      off.assign(1, 0);
      size_t k1 = k0;
      while (k1 < qs.size()) {
        const double x =
            2.0 * 3.14159265358979323846 * qs[k1].r / wavelengths[qs[k1].wl % n_wl];
        const int64_t cap = (std::isfinite(x) && x > 0.0 && x <= 1e6)
                                ? (int64_t)std::ceil(x + 6.0 * std::cbrt(x) + 3.0) + 4
                                : 0;
        if (k1 > k0 && off.back() + cap > row_cap) break;
        r.push_back(qs[k1].r);
        wi.push_back(qs[k1].wl);
        off.push_back(off.back() + cap);
        ++k1;
      }
      const int64_t n = (int64_t)r.size(), rows = std::max<int64_t>(off.back(), 1);
      Pass1Args a{};
      a.radius = c.p1_radius.as<double>(n);
      a.wl_index = c.p1_wl.as<int>(n);
      a.scratch = c.p1_scratch.as<int64_t>(n + 1);
      a.uz = c.p1_uz.as<double2>((size_t)rows * (2 * L - 1));
      a.ux = c.p1_ux.as<double>(rows);
      // A sphere's directions come with its values; a layered sphere's in the group passes.
      const bool sphere_dirs = any_dirs && L == 1;
      const int nq = sphere_dirs ? adaptive::kSphereQ : adaptive::kPass1;
      a.deriv = sphere_dirs ? 1 : 0;
      a.q = c.p1_q.as<double>(nq * n);
      a.n_terms = c.p1_n.as<int64_t>(n);
      a.status = c.p1_status.as<int>(n);
      a.wl = wl_unit_d;
      a.m = reinterpret_cast<const double2*>(m_d);
      a.n = n;
      a.allow_unvalidated = o.allow_unvalidated ? 1 : 0;
      a.n_layers = L;
      a.n_wl = (int)n_wl;
      a.fractions = fr_d;
      a.m_layers = reinterpret_cast<const double2*>(ml_d);
      SB_CUDA(cudaMemcpyAsync((void*)a.radius, r.data(), n * 8, cudaMemcpyHostToDevice, s));
      SB_CUDA(cudaMemcpyAsync((void*)a.wl_index, wi.data(), n * 4, cudaMemcpyHostToDevice, s));
      SB_CUDA(cudaMemcpyAsync((void*)a.scratch, off.data(), (n + 1) * 8, cudaMemcpyHostToDevice,
                              s));
      timed_launch(K_NODES, s, [&] { launch_pass1(a, s); });
      SB_CUDA(cudaGetLastError());
      std::vector<double> q(nq * n);
      std::vector<int64_t> nt(n);
      std::vector<int> st(n);
      SB_CUDA(cudaMemcpyAsync(q.data(), a.q, nq * n * 8, cudaMemcpyDeviceToHost, s));
      SB_CUDA(cudaMemcpyAsync(nt.data(), a.n_terms, n * 8, cudaMemcpyDeviceToHost, s));
      SB_CUDA(cudaMemcpyAsync(st.data(), a.status, n * 4, cudaMemcpyDeviceToHost, s));
      SB_CUDA(cudaStreamSynchronize(s));
      for (int64_t k = 0; k < n; ++k) {
        adaptive::NodeResult& x = out[k0 + k];
        for (int j = 0; j < adaptive::kNodeQ; ++j) x.q[j] = j < nq ? q[nq * k + j] : 0.0;
        x.n = nt[k];
        x.status = st[k];
        x.dq = layered_dirs ? dq_store.data() + (k0 + k) * dstride : nullptr;
        x.msg = nullptr;
      }
      // A layered sphere's requested direction groups, one pass each (nodes that failed above
      // fail the same way there and keep zeros).
      for (int g : groups) {
        Pass1Args b = a;
        b.deriv = 1;
        b.deriv_dir = g;
        b.uz = c.p1_uz.as<double2>((size_t)rows * 2 * (2 * L - 1));
        b.q = c.p1_q.as<double>(16 * n);
        timed_launch(K_NODES, s, [&] { launch_pass1_layered_deriv(b, s); });
        SB_CUDA(cudaGetLastError());
        std::vector<double> qd(16 * n);
        std::vector<int> sd(n);
        SB_CUDA(cudaMemcpyAsync(qd.data(), b.q, 16 * n * 8, cudaMemcpyDeviceToHost, s));
        SB_CUDA(cudaMemcpyAsync(sd.data(), b.status, n * 4, cudaMemcpyDeviceToHost, s));
        SB_CUDA(cudaStreamSynchronize(s));
        for (int64_t k = 0; k < n; ++k) {
          adaptive::NodeResult& x = out[k0 + k];
          if (x.status == 0 && sd[k] != 0) {
            x.status = sd[k];
            if (sd[k] == 3)
              x.msg = "the layered sphere's derivatives are outside their validated domain "
                      "x_L <= 1000";
          }
          double* o = dq_store.data() + (k0 + k) * dstride;
          if (g < L) {
            for (int j = 0; j < 2 * adaptive::kGroup; ++j)
              o[2 * g * adaptive::kGroup + j] = qd[16 * k + 6 + j];
          } else {
            for (int j = 0; j < adaptive::kGroup; ++j)
              o[(2 * L + (g - L)) * adaptive::kGroup + j] = qd[16 * k + 6 + j];
          }
        }
      }
      k0 = k1;
    }
  };
  // Jobs: pass-1 groups per wavelength. The pass-1 callback's `wl` is the pipeline unit of the
  // group's first part (its m and wavelength serve every part of a batch: one particle).
  std::vector<adaptive::Job> jobs;
  std::vector<int> job_of(n_units, -1), place(n_units, 0);
  std::vector<double> wl_of_job;
  for (int64_t i = 0; i < n_wl; ++i) {
    if (batch) {
      adaptive::Job jb;
      for (int64_t p = 0; p < n_parts; ++p)
        if (parts[p].support != adaptive::POINT) {
          if (jb.parts.empty()) jb.wl = (int)(p * n_wl + i);
          place[p * n_wl + i] = (int)jb.parts.size();
          job_of[p * n_wl + i] = (int)jobs.size();
          jb.parts.push_back((int)p);
        }
      if (!jb.parts.empty()) jobs.push_back(jb);
    } else {
      for (int64_t p = 0; p < n_parts; ++p)
        if (parts[p].support != adaptive::POINT) {
          job_of[p * n_wl + i] = (int)jobs.size();
          adaptive::Job jb;
          jb.wl = (int)(p * n_wl + i);
          jb.parts = {(int)p};
          jobs.push_back(jb);
        }
    }
  }
  // Pass 1 sees the wavelength of each job's unit.
  std::vector<double> wl_units(n_units);
  for (int64_t u = 0; u < n_units; ++u) wl_units[u] = wavelengths[u % n_wl];
  // Single radii: their node checked once.
  std::vector<adaptive::Query> points;
  std::vector<int64_t> point_unit;
  for (int64_t p = 0; p < n_parts; ++p)
    if (parts[p].support == adaptive::POINT)
      for (int64_t i = 0; i < n_wl; ++i) {
        points.push_back({parts[p].lo, (int)(p * n_wl + i)});
        point_unit.push_back(p * n_wl + i);
      }
  std::vector<adaptive::NodeResult> point_res(points.size());
  if (!points.empty()) eval(points, point_res);
  adaptive::pass1(jobs, parts, wl_units.data(), o, eval);
  // The first error in (wavelength, part) order.
  {
    int64_t first = n_units;
    int status = 0;
    std::string msg;
    for (int64_t u = 0; u < n_units; ++u) {
      const int64_t key = (u % n_wl) * n_parts + u / n_wl;
      if (job_of[u] >= 0 && jobs[job_of[u]].status != 0 && key < first) {
        first = key;
        status = jobs[job_of[u]].status;
        msg = jobs[job_of[u]].msg;
      }
    }
    for (size_t k = 0; k < points.size(); ++k) {
      const int64_t u = point_unit[k], key = (u % n_wl) * n_parts + u / n_wl;
      if (point_res[k].status != 0 && key < first) {
        first = key;
        status = point_res[k].status;
        msg = node_message(point_res[k].status, wavelengths[u % n_wl], points[k].r);
      }
    }
    if (status != 0) throw Failure{status, msg};
  }
  if (n_max_out) {
    // Per (part, wavelength) unit: its group's largest number of terms (a point's own).
    n_max_out->assign(n_units, 0);
    for (int64_t u = 0; u < n_units; ++u)
      if (job_of[u] >= 0) (*n_max_out)[u] = jobs[job_of[u]].n_terms;
    for (size_t k = 0; k < points.size(); ++k) (*n_max_out)[point_unit[k]] = point_res[k].n;
    return;
  }
  // Pass 2: every unit's nodes, up to two panels per chunk of 32 (nodes 0-14 and 16-30), two
  // only when their projector bands agree, so that each panel's tables go to its own band
  // (engine.rs:1530-1543).
  std::vector<std::vector<int64_t>> slot_of(jobs.size());
  int64_t n_nodes = 32;
  for (size_t k = 0; k < jobs.size(); ++k) {
    const auto& jb = jobs[k];
    int64_t next = 0;  // the next free half-chunk (16 nodes)
    for (size_t pi = 0; pi < jb.panels.size(); ++pi) {
      if (next % 2 == 1 && bucket(jb.panel_terms[pi]) != bucket(jb.panel_terms[pi - 1])) ++next;
      slot_of[k].push_back(16 * next);
      ++next;
    }
    n_nodes = std::max<int64_t>(n_nodes, 32 * ((next + 1) / 2));
  }
  if ((double)n_units * (double)n_nodes > 4e9)
    throw Failure{SCATRS_INVALID_INPUT, "too many (unit, node) pairs for one call"};
  const int ns = deriv ? kNormStrideD : 8;  // unit_norm doubles per unit
  std::vector<double> radius((size_t)n_units * n_nodes, 0.0), weight(radius.size(), 0.0),
      wdiff(radius.size(), 0.0), norm((size_t)n_units * ns, 0.0);
  std::vector<double> wth(deriv ? 3 * radius.size() : 0, 0.0), wthd(wth.size(), 0.0);
  std::vector<char> unit_converged(n_units, 1);
  std::vector<int64_t> unit_panels(n_units, 0);
  // Every unit's nodes and weights on its own (the host's threads; each unit writes its rows).
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t u = 0; u < n_units; ++u) {
    const int64_t p = u / n_wl;
    const adaptive::Part& part = parts[p];
    double* nr = &radius[(size_t)u * n_nodes];
    double* nw = &weight[(size_t)u * n_nodes];
    double* nd = &wdiff[(size_t)u * n_nodes];
    double* un = &norm[(size_t)u * ns];
    if (part.support == adaptive::POINT) {
      nr[0] = part.lo;
      nw[0] = 1.0;
      un[0] = 1.0;
      un[3] = 1.0;
      continue;
    }
    const adaptive::Job& jb = jobs[job_of[u]];
    for (size_t pi = 0; pi < jb.panels.size(); ++pi) {
      adaptive::Node g[15];
      adaptive::gk15(jb.panels[pi].first, jb.panels[pi].second, g);
      const size_t base = (size_t)slot_of[job_of[u]][pi];
      for (int k = 0; k < 15; ++k) {
        const double r = std::exp(g[k].t);
        double grad[3];
        const double ur = (part.grads.empty() ? part.u(r) : part.u(r, grad)) * r;
        nr[base + k] = r;
        nw[base + k] = g[k].wk * ur;
        nd[base + k] = g[k].wk * ur - g[k].wg * ur;
        // Each requested parameter's weights w (du/dtheta) r (engine.rs:1637-1644).
        for (size_t b = 0; b < part.grads.size(); ++b) {
          const double dw = grad[part.grads[b]] * r;
          const size_t at = ((size_t)u * n_nodes + base + k) * 3 + b;
          wth[at] = g[k].wk * dw;
          wthd[at] = g[k].wk * dw - g[k].wg * dw;
        }
      }
    }
    un[0] = part.mom.z;
    un[1] = part.mom.ez;
    un[2] = part.support == adaptive::UNBOUNDED ? 0.2 * o.rtol : 0.0;
    un[4] = part.mom.v[0];
    un[5] = part.mom.e[0];
    un[6] = part.mom.v[1];
    un[7] = part.mom.e[1];
    for (size_t b = 0; deriv && b < part.grads.size(); ++b) {
      un[8 + b] = part.mom.dz[b];
      un[11 + b] = part.mom.dez[b];
      un[14 + 4 * b] = part.mom.d[b][0];
      un[15 + 4 * b] = part.mom.de[b][0];
      un[16 + 4 * b] = part.mom.d[b][1];
      un[17 + 4 * b] = part.mom.de[b][1];
    }
    unit_converged[u] = jb.converged[place[u]] ? 1 : 0;
    unit_panels[u] = (int64_t)jb.panels.size();
  }
  fo.n_nodes = (int32_t)n_nodes;
  const int glen = options->greek_order >= 0 ? options->greek_order + 1 : 0;
  // The parts' averages: values and errors, or per block of a call with derivatives (values,
  // n_theta parameters, Re m, Im m).
  const int n_blocks = 3 + n_theta;
  const int64_t row = 8 + 4 * n_mu + 6 * (int64_t)glen;
  const int64_t stride = deriv ? 2 * n_blocks * row : 16 + 8 * n_mu + 12 * (int64_t)glen;
  double* avg = c.avg.as<double>((size_t)n_units * stride);
  AdaptiveInput ad;
  ad.on = true;
  ad.radius = radius.data();
  ad.weight = weight.data();
  ad.wdiff = wdiff.data();
  ad.unit_norm = norm.data();
  ad.avg = avg;
  DerivOutput dvo;
  if (deriv) {
    ad.wtheta = wth.data();
    ad.wthdiff = wthd.data();
    dvo.on = true;
    dvo.n_theta = n_theta;
  }
  FixedCall call;
  call.wl_host.assign(wavelengths, wavelengths + n_wl);
  call.per_unit = true;
  call.n_dist = n_parts;
  call.n_wl = n_wl;
  call.n_nodes = n_nodes;
  std::vector<scatrs_distribution> dummy(n_parts);
  LayerInput li;
  if (L > 1) {
    li.n_layers = L;
    li.fractions = layers->fractions;
    li.m_dev = ml_d;
  }
  if (L > 1 && deriv) {
    // A layered sphere: the derivative pipeline once per requested direction group (K-a along
    // the group's direction, engine.rs:1047-1109 with Solved::direction), each pass's values and
    // parameter blocks alike; the direction blocks gathered into one row per unit of the values,
    // the n_theta parameters and all 3 L - 1 directions for the mixing.
    const std::vector<int> passes = groups.empty() ? std::vector<int>{0} : groups;
    const int n_all = 1 + n_theta + n_dirs_all;
    const int64_t cstride = 2 * (int64_t)n_all * row;
    std::vector<double> hav((size_t)n_units * cstride, 0.0), one((size_t)n_units * stride);
    call.radius = radius;
    for (size_t pi = 0; pi < passes.size(); ++pi) {
      const int g = passes[pi];
      DerivOutput dvg = dvo;
      dvg.dir = g;
      run_fixed(c, dummy.data(), n_parts, wl_d, n_wl, m_d, mu, n_mu, &fo, nullptr, nullptr,
                nullptr, s, &call, li, dvg, ad);
      check_device_errors(c, s, &call);
      SB_CUDA(cudaMemcpyAsync(one.data(), avg, one.size() * 8, cudaMemcpyDeviceToHost, s));
      SB_CUDA(cudaStreamSynchronize(s));
      auto copy_block = [&](const double* src, double* dst, int from, int to) {
        std::copy(src + 2 * from * row, src + (2 * from + 2) * row, dst + 2 * to * row);
      };
      for (int64_t u = 0; u < n_units; ++u) {
        const double* src = one.data() + u * stride;
        double* dst = hav.data() + u * cstride;
        if (pi == 0)
          for (int b = 0; b <= n_theta; ++b) copy_block(src, dst, b, b);
        if (groups.empty()) continue;
        if (g < L) {
          copy_block(src, dst, n_theta + 1, 1 + n_theta + 2 * g);
          copy_block(src, dst, n_theta + 2, 2 + n_theta + 2 * g);
        } else {
          copy_block(src, dst, n_theta + 1, 1 + n_theta + 2 * L + (g - L));
        }
      }
    }
    // A single layered radius's radius (particle.rs:221-237 size_derivative: the sum over
    // the interfaces of f_l d/dx_l and the outer surface's d/dx_L): the particle with a vacuum
    // shell of zero thickness around it (fractions f_0..f_{L-2}, 1; index 1 outside) has the
    // same coefficients, and its interface l's direction is x d/dx_l with the outer surface
    // moving beneath the fixed vacuum radius; so d/dx = (1/x) sum_l f_l (its direction l's
    // block), f_{L-1} = 1, one pass per interface. The sum goes where mix_derivatives and
    // place_radius_rows read the x rows of a sphere.
    std::vector<double> hav_x;
    if (radius_x) {
      const int la = L + 1;
      std::vector<double> fr_aug((size_t)n_parts * L), ml_aug((size_t)2 * n_parts * la * n_wl);
      for (int64_t p = 0; p < n_parts; ++p) {
        for (int l = 0; l < L - 1; ++l) fr_aug[p * L + l] = layers->fractions[p * (L - 1) + l];
        fr_aug[p * L + L - 1] = 1.0;
        for (int l = 0; l < L; ++l)
          for (int64_t i = 0; i < n_wl; ++i)
            for (int k = 0; k < 2; ++k)
              ml_aug[2 * ((p * la + l) * n_wl + i) + k] =
                  layers->m[2 * ((p * L + l) * n_wl + i) + k];
        for (int64_t i = 0; i < n_wl; ++i) {
          ml_aug[2 * ((p * la + L) * n_wl + i)] = 1.0;
          ml_aug[2 * ((p * la + L) * n_wl + i) + 1] = 0.0;
        }
      }
      double* mla_d = c.p1_ml_aug.as<double>(ml_aug.size());
      SB_CUDA(cudaMemcpyAsync(mla_d, ml_aug.data(), ml_aug.size() * 8, cudaMemcpyHostToDevice, s));
      LayerInput lia;
      lia.n_layers = la;
      lia.fractions = fr_aug.data();
      lia.m_dev = mla_d;
      hav_x.assign((size_t)n_units * cstride, 0.0);
      for (int l = 0; l < L; ++l) {
        DerivOutput dvg = dvo;
        dvg.dir = la + l;
        run_fixed(c, dummy.data(), n_parts, wl_d, n_wl, m_d, mu, n_mu, &fo, nullptr, nullptr,
                  nullptr, s, &call, lia, dvg, ad);
        check_device_errors(c, s, &call);
        SB_CUDA(cudaMemcpyAsync(one.data(), avg, one.size() * 8, cudaMemcpyDeviceToHost, s));
        SB_CUDA(cudaStreamSynchronize(s));
        for (int64_t p = 0; p < n_parts; ++p) {
          if (parts[p].support != adaptive::POINT || in[p].grads.empty()) continue;
          const double f = fr_aug[p * L + l];
          for (int64_t i = 0; i < n_wl; ++i) {
            const int64_t u = p * n_wl + i;
            const double x = 2.0 * kPi * parts[p].lo / wavelengths[i];
            const double* src = one.data() + u * stride + 2 * (n_theta + 1) * row;
            double* dst = hav_x.data() + u * cstride + 2 * (n_theta + 1) * row;
            for (int64_t k = 0; k < row; ++k) dst[k] += f / x * src[k];
          }
        }
      }
    }
    if (rows_out) {  // a mixture's host assembly: the per-block rows by unit
      if (radius_x)
        place_radius_rows(in, parts, n_wl, wavelengths, n_theta, row, cstride, hav_x, hav);
      rows_out->stride = cstride;
      rows_out->rows = std::move(hav);
      rows_out->converged = unit_converged;
      rows_out->panels = unit_panels;
      return;
    }
    mix_derivatives(in, parts, n_out, n_wl, n_mu, options->greek_order, options->normalized != 0,
                    n_theta, hav, *dd, res, wavelengths, hav_x);
    adaptive_flags(in, jobs, job_of, unit_converged, unit_panels, n_out, n_wl, res);
    return;
  }
  run_fixed(c, dummy.data(), n_parts, wl_d, n_wl, m_d, mu, n_mu, &fo, nullptr, nullptr, nullptr,
            s, &call, li, dvo, ad);
  if (deriv) {
    call.radius = std::move(radius);
    check_device_errors(c, s, &call);
    std::vector<double> hav((size_t)n_units * stride), hav_x;
    SB_CUDA(cudaMemcpyAsync(hav.data(), avg, hav.size() * 8, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    if (radius_x) {
      // The single radii's derivatives along x (engine.rs:1158-1170, 1857-1883): the pipeline
      // again with K-a's x direction in place of Re m.
      DerivOutput dvx = dvo;
      dvx.dir = 1;
      run_fixed(c, dummy.data(), n_parts, wl_d, n_wl, m_d, mu, n_mu, &fo, nullptr, nullptr,
                nullptr, s, &call, li, dvx, ad);
      check_device_errors(c, s, &call);
      hav_x.resize(hav.size());
      SB_CUDA(cudaMemcpyAsync(hav_x.data(), avg, hav_x.size() * 8, cudaMemcpyDeviceToHost, s));
      SB_CUDA(cudaStreamSynchronize(s));
    }
    if (rows_out) {  // a mixture's host assembly: the per-block rows by unit
      if (radius_x)
        place_radius_rows(in, parts, n_wl, wavelengths, n_theta, row, stride, hav_x, hav);
      rows_out->stride = stride;
      rows_out->rows = std::move(hav);
      rows_out->converged = unit_converged;
      rows_out->panels = unit_panels;
      return;
    }
    mix_derivatives(in, parts, n_out, n_wl, n_mu, options->greek_order, options->normalized != 0,
                    n_theta, hav, *dd, res, wavelengths, hav_x);
    adaptive_flags(in, jobs, job_of, unit_converged, unit_panels, n_out, n_wl, res);
    return;
  }
  if (rows_out) {
    call.radius = std::move(radius);
    check_device_errors(c, s, &call);
    rows_out->stride = stride;
    rows_out->rows.resize((size_t)n_units * stride);
    SB_CUDA(cudaMemcpyAsync(rows_out->rows.data(), avg, rows_out->rows.size() * 8,
                            cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    rows_out->converged = unit_converged;
    rows_out->panels = unit_panels;
    return;
  }
  // Mixing and outputs.
  const int64_t n_outs = (int64_t)n_out * n_wl;
  int64_t vl, pl, gl;
  scatrs_ensemble_fixed_sizes(n_outs, n_mu, options->greek_order, &vl, &pl, &gl);
  double* v_d = c.values.as<double>(2 * vl);
  double* p_d = pl > 0 ? c.phase.as<double>(2 * pl) : nullptr;
  double* g_d = gl > 0 ? c.greek.as<double>(2 * gl) : nullptr;
  std::vector<int> first(n_out + 1, 0), member;
  std::vector<double> frac;
  for (int ou = 0; ou < n_out; ++ou) {
    for (int64_t p = 0; p < n_parts; ++p)
      if (in[p].out == ou) {
        member.push_back((int)p);
        frac.push_back(in[p].f);
      }
    first[ou + 1] = (int)member.size();
  }
  int* first_d = c.mix_first.as<int>(first.size());
  int* member_d = c.mix_part.as<int>(std::max<size_t>(member.size(), 1));
  double* frac_d = c.mix_frac.as<double>(std::max<size_t>(frac.size(), 1));
  SB_CUDA(cudaMemcpyAsync(first_d, first.data(), first.size() * 4, cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(member_d, member.data(), member.size() * 4, cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(frac_d, frac.data(), frac.size() * 8, cudaMemcpyHostToDevice, s));
  MixArgs mx{};
  mx.n_out = n_out;
  mx.n_wl = (int)n_wl;
  mx.n_mu = (int)n_mu;
  mx.greek_order = options->greek_order;
  mx.normalized = options->normalized;
  mx.first = first_d;
  mx.part = member_d;
  mx.fraction = frac_d;
  mx.avg = avg;
  mx.values = v_d;
  mx.errors = v_d + vl;
  mx.phase = p_d;
  mx.phase_err = p_d ? p_d + pl : nullptr;
  mx.greek = g_d;
  mx.greek_err = g_d ? g_d + gl : nullptr;
  mx.err = c.err.as<unsigned long long>(2);
  timed_launch(K_FINAL, s, [&] { launch_mix(mx, s); });
  SB_CUDA(cudaGetLastError());
  call.radius = std::move(radius);
  check_device_errors(c, s, &call);
  SB_CUDA(cudaMemcpyAsync(res.values, v_d, vl * 8, cudaMemcpyDeviceToHost, s));
  if (res.errors) SB_CUDA(cudaMemcpyAsync(res.errors, v_d + vl, vl * 8, cudaMemcpyDeviceToHost, s));
  if (pl > 0 && res.phase)
    SB_CUDA(cudaMemcpyAsync(res.phase, p_d, pl * 8, cudaMemcpyDeviceToHost, s));
  if (pl > 0 && res.phase_err)
    SB_CUDA(cudaMemcpyAsync(res.phase_err, p_d + pl, pl * 8, cudaMemcpyDeviceToHost, s));
  if (gl > 0 && res.greek)
    SB_CUDA(cudaMemcpyAsync(res.greek, g_d, gl * 8, cudaMemcpyDeviceToHost, s));
  if (gl > 0 && res.greek_err)
    SB_CUDA(cudaMemcpyAsync(res.greek_err, g_d + gl, gl * 8, cudaMemcpyDeviceToHost, s));
  SB_CUDA(cudaStreamSynchronize(s));
  adaptive_flags(in, jobs, job_of, unit_converged, unit_panels, n_out, n_wl, res);
}

// The Greek coefficients of the thread's last greek="all" call, (6, n, width) and with
// derivatives (P, 6, n, width), zero above each wavelength's order.
struct GreekAll {
  int64_t width = 0, n = 0, p = 0;
  std::vector<double> g, ge, dg, dge;
};
thread_local GreekAll t_greek_all;

// adaptive_call_order, and greek="all" (GreekOrder::All, engine.rs:2016-2020: every order up to
// 2 N_max, N_max the largest number of terms of the call at that wavelength: every part of a
// batch, else the output unit's own parts; ensemble.rs:419-429 pads the arrays to the longest):
// pass 1 finds the N_max, then the wavelengths of one order run together at that order (all
// output units of a batch, else each unit alone), so that each band projects to
// min(2 N_max, 2 N_band) as the reference's. The coefficients go to t_greek_all.
void adaptive_call(const std::vector<AdPart>& in, int n_out, bool batch, const double* wavelengths,
                   int64_t n_wl, const double* mu, int64_t n_mu,
                   const scatrs_adaptive_options* options, const AdOutputs& res,
                   const scatrs_layers* layers = nullptr, const AdDerivs* dd = nullptr) {
  if (!options || options->greek_order != SCATRS_GREEK_ALL) {
    adaptive_call_order(in, n_out, batch, wavelengths, n_wl, mu, n_mu, options, res, layers, dd);
    return;
  }
  scatrs_adaptive_options o1 = *options;
  o1.greek_order = -1;
  std::vector<int64_t> n_max;
  adaptive_call_order(in, n_out, batch, wavelengths, n_wl, mu, n_mu, &o1, AdOutputs{}, layers,
                      dd, &n_max);
  const int64_t n_parts = (int64_t)in.size();
  // Each output unit's order at each wavelength: 2 N_max over the parts of its call (a batch is
  // one call over every part; otherwise each output unit is a call of its own).
  std::vector<int64_t> order((size_t)n_out * n_wl, 0);
  for (int64_t p = 0; p < n_parts && !n_max.empty(); ++p)
    for (int64_t i = 0; i < n_wl; ++i)
      for (int o = 0; o < n_out; ++o)
        if (batch || in[p].out == o)
          order[o * n_wl + i] = std::max(order[o * n_wl + i], 2 * n_max[p * n_wl + i]);
  int64_t width = 1;
  for (int64_t x : order) width = std::max(width, x + 1);
  const int64_t n_outs = (int64_t)n_out * n_wl, P = dd ? dd->n : 0;
  GreekAll& ga = t_greek_all;
  ga.width = width;
  ga.n = n_outs;
  ga.p = P;
  ga.g.assign(6 * n_outs * width, 0.0);
  ga.ge.assign(ga.g.size(), 0.0);
  ga.dg.assign(P * ga.g.size(), 0.0);
  ga.dge.assign(ga.dg.size(), 0.0);
  const int nl = layers && layers->n_layers > 1 ? layers->n_layers : 1;
  // One call per set of output units run together (all of a batch, else each alone) and order.
  std::vector<std::vector<int>> sets;
  if (batch) {
    sets.push_back({});
    for (int o = 0; o < n_out; ++o) sets[0].push_back(o);
  } else {
    for (int o = 0; o < n_out; ++o) sets.push_back({o});
  }
  for (const std::vector<int>& outs : sets) {
    std::map<int64_t, std::vector<int64_t>> by_order;
    for (int64_t i = 0; i < n_wl; ++i) by_order[order[outs[0] * n_wl + i]].push_back(i);
    // The set's parts, their output units renumbered.
    std::vector<int64_t> ps;
    for (int64_t p = 0; p < n_parts; ++p)
      if (std::find(outs.begin(), outs.end(), in[p].out) != outs.end()) ps.push_back(p);
    const int no = (int)outs.size(), np = (int)ps.size();
    for (const auto& kv : by_order) {
      const int64_t L = kv.first;
      const std::vector<int64_t>& ws = kv.second;
      const int64_t nw = (int64_t)ws.size(), ns = (int64_t)no * nw, glen = L + 1;
      std::vector<double> wl_s(nw);
      for (int64_t k = 0; k < nw; ++k) wl_s[k] = wavelengths[ws[k]];
      std::vector<AdPart> in_s;
      std::vector<std::vector<double>> m_s(np);
      for (int q = 0; q < np; ++q) {
        AdPart a = in[ps[q]];
        a.out = (int)(std::find(outs.begin(), outs.end(), a.out) - outs.begin());
        if (a.m) {
          m_s[q].resize(2 * nw);
          for (int64_t k = 0; k < nw; ++k) {
            m_s[q][2 * k] = a.m[2 * ws[k]];
            m_s[q][2 * k + 1] = a.m[2 * ws[k] + 1];
          }
          a.m = m_s[q].data();
        }
        in_s.push_back(a);
      }
      scatrs_layers lay_s{};
      std::vector<double> ml_s, fr_s;
      if (nl > 1) {
        lay_s = *layers;
        ml_s.resize(2 * (size_t)np * nl * nw);
        fr_s.resize((size_t)np * (nl - 1));
        for (int q = 0; q < np; ++q) {
          for (int l = 0; l + 1 < nl; ++l) fr_s[q * (nl - 1) + l] = layers->fractions[ps[q] * (nl - 1) + l];
          for (int l = 0; l < nl; ++l)
            for (int64_t k = 0; k < nw; ++k)
              for (int c = 0; c < 2; ++c)
                ml_s[2 * ((q * nl + l) * nw + k) + c] =
                    layers->m[2 * ((ps[q] * nl + l) * n_wl + ws[k]) + c];
        }
        lay_s.m = ml_s.data();
        lay_s.fractions = fr_s.data();
      }
      std::vector<double> v(11 * ns), e(11 * ns), ph(6 * ns * n_mu), phe(ph.size()),
          g(6 * ns * glen), ge(g.size()), dv(P * v.size()), de(dv.size()), dph(P * ph.size()),
          dphe(dph.size()), dg(P * g.size()), dge(dg.size());
      std::vector<int8_t> conv(ns);
      std::vector<int64_t> pan(ns);
      AdOutputs out_s{v.data(), e.data(), ph.data(), phe.data(), g.data(), ge.data(),
                      conv.data(), pan.data()};
      AdDerivs dd_s;
      if (dd) {
        dd_s = *dd;
        dd_s.d_values = dv.data();
        dd_s.d_errors = de.data();
        dd_s.d_phase = dph.data();
        dd_s.d_phase_err = dphe.data();
        dd_s.d_greek = dg.data();
        dd_s.d_greek_err = dge.data();
      }
      scatrs_adaptive_options o2 = *options;
      o2.greek_order = (int32_t)L;
      adaptive_call_order(in_s, no, batch, wl_s.data(), nw, mu, n_mu, &o2, out_s,
                          nl > 1 ? &lay_s : nullptr, dd ? &dd_s : nullptr);
      // Back to the call's output units and wavelengths.
      for (int q = 0; q < no; ++q)
        for (int64_t k = 0; k < nw; ++k) {
          const int64_t x = q * nw + k, y = outs[q] * n_wl + ws[k];
          for (int c2 = 0; c2 < 11; ++c2) {
            res.values[c2 * n_outs + y] = v[c2 * ns + x];
            if (res.errors) res.errors[c2 * n_outs + y] = e[c2 * ns + x];
            for (int64_t c = 0; c < P; ++c) {
              if (dd->d_values) dd->d_values[(c * 11 + c2) * n_outs + y] = dv[(c * 11 + c2) * ns + x];
              if (dd->d_errors) dd->d_errors[(c * 11 + c2) * n_outs + y] = de[(c * 11 + c2) * ns + x];
            }
          }
          for (int el = 0; el < 6; ++el) {
            for (int64_t j = 0; j < n_mu; ++j) {
              const int64_t a = (el * n_outs + y) * n_mu + j, b = (el * ns + x) * n_mu + j;
              if (res.phase) res.phase[a] = ph[b];
              if (res.phase_err) res.phase_err[a] = phe[b];
              for (int64_t c = 0; c < P; ++c) {
                const int64_t ad = ((c * 6 + el) * n_outs + y) * n_mu + j;
                const int64_t bd = ((c * 6 + el) * ns + x) * n_mu + j;
                if (dd->d_phase) dd->d_phase[ad] = dph[bd];
                if (dd->d_phase_err) dd->d_phase_err[ad] = dphe[bd];
              }
            }
            for (int64_t l = 0; l < glen; ++l) {
              ga.g[(el * n_outs + y) * width + l] = g[(el * ns + x) * glen + l];
              ga.ge[(el * n_outs + y) * width + l] = ge[(el * ns + x) * glen + l];
              for (int64_t c = 0; c < P; ++c) {
                ga.dg[((c * 6 + el) * n_outs + y) * width + l] =
                    dg[((c * 6 + el) * ns + x) * glen + l];
                ga.dge[((c * 6 + el) * n_outs + y) * width + l] =
                    dge[((c * 6 + el) * ns + x) * glen + l];
              }
            }
          }
          if (res.converged) res.converged[y] = conv[x];
          if (res.panels) res.panels[y] = pan[x];
        }
    }
  }
}

// The driver's tensor-map encoder, found once through the runtime.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) throw Failure{SCATRS_CUDA, "cuTensorMapEncodeTiled is not available"};
  return fn;
}

// A 2-D FP32 tensor map over rows of n_q_pad values, boxes of 32 x box_rows, 128-byte swizzle,
// zero fill outside.
CUtensorMap tensor_map_2d(float* base, int64_t n_q_pad, int64_t rows, int box_rows) {
  CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)n_q_pad, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)n_q_pad * 4};
  const cuuint32_t box[2] = {32, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides,
                                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw Failure{SCATRS_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")"};
  return m;
}

// The projection matrices (2l+1)/2 w_k d_l(mu_k) of d00, d22, d2-2, d02 ([4][n_q][L + 1]) on the
// n_q-point Gauss rule (greek.rs:131-335), and their TF32 heads and tails transposed.
Context::Projector& projector(Context& c, int64_t n_q, int L, cudaStream_t s) {
  auto key = std::make_pair(n_q, L);
  auto it = c.projectors.find(key);
  if (it != c.projectors.end()) return it->second;
  Context::Projector& p = c.projectors[key];
  const auto& r = rule(c, n_q);
  const int64_t len = L + 1;
  std::vector<double> d(4 * (size_t)n_q * len), buf(len);
  const int mn[4][2] = {{0, 0}, {2, 2}, {2, -2}, {0, 2}};
  for (int f = 0; f < 4; ++f)
    for (int64_t k = 0; k < n_q; ++k) {
      wigner_d(mn[f][0], mn[f][1], r.first[k], buf.data(), len);
      for (int64_t l = 0; l < len; ++l)
        d[((size_t)f * n_q + k) * len + l] = (double)(2 * l + 1) * 0.5 * r.second[k] * buf[l];
    }
  double* dd = p.d.as<double>(d.size());
  SB_CUDA(cudaMemcpyAsync(dd, d.data(), d.size() * 8, cudaMemcpyHostToDevice, s));
  const int64_t n_q_pad = round_up(n_q, 4);
  float* hi = p.d_hi.as<float>(4 * (size_t)len * n_q_pad);
  float* lo = p.d_lo.as<float>(4 * (size_t)len * n_q_pad);
  launch_greek_split_d(dd, (int)n_q, (int)n_q_pad, (int)len, hi, lo, s);
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaStreamSynchronize(s));
  return p;
}

// ---------------------------------------------------------------------------------------
// Spheroid T-matrices (tmatrix.cu) and the convergence in N and n_theta (driver.rs).
// ---------------------------------------------------------------------------------------
struct TmSpec {
  double x, eps, s_re, s_im;
  int m, N, n_theta;
};

void check_tm_spec(const TmSpec& t) {
  if (!(std::isfinite(t.x) && t.x > 0.0 && t.x <= 1e4))
    throw Failure{SCATRS_INVALID_INPUT, "the size parameter must be finite and in (0, 1e4]"};
  if (!(std::isfinite(t.eps) && t.eps > 0.0))
    throw Failure{SCATRS_INVALID_INPUT, "the aspect ratio must be finite and > 0"};
  if (!(std::isfinite(t.s_re) && std::isfinite(t.s_im) && t.s_re > 0.0 && t.s_im >= 0.0))
    throw Failure{SCATRS_INVALID_INPUT, "the refractive index needs Re m > 0 and Im m >= 0"};
  if (t.N < 1 || t.N > 500 || t.m < 0 || t.m > t.N || t.n_theta < 2 || t.n_theta > 4000)
    throw Failure{SCATRS_INVALID_INPUT,
                  "a T-matrix needs 1 <= N <= 500, 0 <= m <= N and 2 <= n_theta <= 4000"};
}

// The n-point Gauss-Legendre rule on [-1, 1] in double-double: the double rule's nodes refined
// by Newton's method on P_n (three-term recurrence) in the host's 113-bit __float128
// arithmetic, the weights 2 / ((1 - x^2) P_n'(x)^2), each rounded to a double-double pair.
const std::vector<double>& dd_rule(Context& c, int64_t n) {
  auto it = c.dd_rules.find(n);
  if (it != c.dd_rules.end()) return it->second;
  typedef __float128 q128;
  const auto& r = rule(c, n);
  std::vector<double> out(4 * (size_t)n);
  auto legendre = [&](q128 t, q128* p, q128* dp) {
    q128 p0 = 1, p1 = t;
    for (int64_t k = 2; k <= n; ++k) {
      const q128 p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    *p = p1;
    *dp = n * (p0 - t * p1) / ((1 - t) * (1 + t));
  };
  auto split = [](q128 v, double* o) {
    o[0] = (double)v;
    o[1] = (double)(v - (q128)o[0]);
  };
  for (int64_t i = 0; i < n; ++i) {
    q128 t = r.first[i], p, dp;
    for (int it2 = 0; it2 < 3; ++it2) {
      legendre(t, &p, &dp);
      t -= p / dp;
    }
    legendre(t, &p, &dp);
    split(t, &out[4 * i]);
    split(2 / ((1 - t) * (1 + t) * dp * dp), &out[4 * i + 2]);
  }
  return c.dd_rules.emplace(n, std::move(out)).first->second;
}

// The form each element of Q is assembled in: -1 (the cleanest of the three exact ones, the
// default) or, for diagnostics, the environment's SCATRS_TMATRIX_FORM: 0 plain, 1 without the
// y-part's terms of power < 0, 2 without those of power <= 0 (each where it applies).
int tm_form_override() {
  const char* v = std::getenv("SCATRS_TMATRIX_FORM");
  if (!v || !*v) return -1;
  const int f = std::atoi(v);
  return f >= 0 && f <= 2 ? f : -1;
}

// Runs the T-matrices of specs in batches of bounded memory. Consecutive specs of the same
// spheroid at the same N and n_theta share one geometry (nodes and radial functions). Per
// spec j: sums[3 j] = -Re tr T, sums[3 j + 1] = sum |T|^2, sums[3 j + 2] = the refinement's
// last relative correction; each T (row-major (2K)^2 complex) into t_out if given.
//
// With greek_out, every spheroid's specs must be its modes 0..N in order: its orientation
// average (random.cu) then runs on the device-resident T, and greek_out gets, per spheroid in
// order, the unnormalized Greek coefficients [6][2N + 1] (alpha1_0 = C_sca / (4 pi), 1/k^2).
void run_tmatrices(Context& c, const std::vector<TmSpec>& specs, std::vector<double>& sums,
                   std::vector<std::vector<double>>* t_out, cudaStream_t s,
                   std::vector<std::vector<double>>* greek_out = nullptr) {
  sums.assign(3 * specs.size(), 0.0);
  if (t_out) t_out->assign(specs.size(), {});
  if (greek_out) greek_out->clear();
  constexpr double kBudget = 8.0e9;  // bytes of device workspace per batch
  const bool ro = greek_out != nullptr;
  auto same_geom = [](const TmSpec& p, const TmSpec& q) {
    return p.x == q.x && p.eps == q.eps && p.s_re == q.s_re && p.s_im == q.s_im && p.N == q.N &&
           p.n_theta == q.n_theta;
  };
  size_t j0 = 0;
  while (j0 < specs.size()) {
    std::vector<TmGeom> geoms;
    std::vector<TmJob> jobs;
    std::map<int64_t, int64_t> rule_at;
    std::vector<double> rules;
    int64_t nodes = 0, rad = 0, ang_nodes = 0, ang = 0, pairs = 0, J = 0, W = 0, P = 0, T = 0;
    int64_t ser = 0, ser_threads = 0, forms_threads = 0;
    double bytes = 0.0;
    size_t j1 = j0;
    for (; j1 < specs.size(); ++j1) {
      const TmSpec& t = specs[j1];
      check_tm_spec(t);
      const bool new_geom = j1 == j0 || t.m == 0 || !same_geom(specs[j1 - 1], t);
      const int K = t.N - std::max(t.m, 1) + 1, n2 = 2 * K, nq = 2 * t.n_theta;
      double b = 8.0 * ((double)nq * (t.N + 1) * 6 + 32.0 * K * K + 14.0 * n2 * n2 +
                        (t_out || ro ? 2.0 * n2 * n2 : 0.0)) + 4.0 * n2;
      if (new_geom)
        b += 8.0 * ((double)nq * 16 + (double)nq * (t.N + 1) * 20 +
                    (double)t.n_theta * (t.N + 1) * tm_series_slot(t.N));
      if (ro && new_geom) {
        if (t.m != 0 || t.N > kRoMaxN)
          throw Failure{SCATRS_INVALID_INPUT,
                        "the orientation average needs the modes 0..N in order and N <= " +
                            std::to_string(kRoMaxN)};
        const double n1 = t.N + 1, S = 2 * t.N + 1, Q = 2 * t.N + 3, q = 2 * t.N + 1;
        b += 16.0 * (4 * n1 * n1 * S + Q * 4 * S * n1 + Q * 16 * q) + 8.0 * 12 * q;
      }
      if (ro && !new_geom && t.m != specs[j1 - 1].m + 1)
        throw Failure{SCATRS_INVALID_INPUT, "the orientation average needs the modes 0..N in order"};
      // Batches break between spheroids when their modes must stay together.
      if (j1 > j0 && bytes + b > kBudget && (!ro || new_geom)) break;
      bytes += b;
      if (new_geom) {
        if (!rule_at.count(nq)) {
          rule_at[nq] = (int64_t)rules.size() / 4;
          const auto& r = dd_rule(c, nq);
          rules.insert(rules.end(), r.begin(), r.end());
        }
        TmGeom g{};
        g.a = t.x * std::cbrt(t.eps);
        g.c = g.a / t.eps;
        g.s_re = t.s_re;
        g.s_im = t.s_im;
        g.N = t.N;
        g.n_theta = t.n_theta;
        g.node0 = nodes;
        g.rule = rule_at[nq];
        g.rad0 = rad;
        g.ser0 = ser;
        g.sth0 = ser_threads;
        g.fth0 = forms_threads;
        nodes += nq;
        rad += (int64_t)nq * (t.N + 1) * 20;
        ser += (int64_t)t.n_theta * (t.N + 1) * tm_series_slot(t.N);
        ser_threads += (int64_t)t.n_theta * t.N;
        forms_threads += (int64_t)t.n_theta * t.N * t.N;
        geoms.push_back(g);
      }
      TmJob jb{};
      jb.geom = (int)geoms.size() - 1;
      jb.m = t.m;
      jb.K = K;
      jb.ang_node0 = ang_nodes;
      jb.ang0 = ang;
      jb.pair0 = pairs;
      jb.J0 = J;
      jb.W0 = W;
      jb.piv0 = P;
      jb.T0 = T;
      ang_nodes += nq;
      ang += (int64_t)nq * (t.N + 1) * 6;
      pairs += (int64_t)K * K;
      J += 8 * (int64_t)K * K;
      W += 14 * (int64_t)n2 * n2;
      P += n2;
      T += (int64_t)n2 * n2;
      jobs.push_back(jb);
    }
    TmArgs a{};
    a.n_geoms = (int)geoms.size();
    a.n_jobs = (int)jobs.size();
    a.n_node_total = nodes;
    a.n_ang_total = ang_nodes;
    a.n_pair_total = pairs;
    a.geoms = c.tm_geoms.as<TmGeom>(geoms.size());
    a.jobs = c.tm_jobs.as<TmJob>(jobs.size());
    double* rl = c.tm_rules.as<double>(rules.size());
    a.rule = rl;
    a.node = c.tm_node.as<double>(16 * (size_t)nodes);
    a.rad = c.tm_rad.as<double>((size_t)rad);
    a.ang = c.tm_ang.as<double>((size_t)ang);
    a.ser = c.tm_ser.as<double>((size_t)ser);
    a.n_ser_total = ser_threads;
    a.n_forms_total = forms_threads;
    a.form = tm_form_override();
    a.J = c.tm_J.as<double>(4 * (size_t)J);
    a.work = c.tm_work.as<double>((size_t)W);
    a.piv = c.tm_piv.as<int>((size_t)P);
    a.T = t_out || ro ? c.tm_T.as<double>(2 * (size_t)T) : nullptr;
    a.sums = c.tm_sums.as<double>(3 * jobs.size());
    a.err = c.tm_err.as<unsigned>(1);
    a.max_sweeps = 4;
    SB_CUDA(cudaMemcpyAsync((void*)a.geoms, geoms.data(), geoms.size() * sizeof(TmGeom),
                            cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync((void*)a.jobs, jobs.data(), jobs.size() * sizeof(TmJob),
                            cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(rl, rules.data(), rules.size() * 8, cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemsetAsync(a.err, 0, sizeof(unsigned), s));
    if (g_profiling) {
      int64_t pn = 0;
      for (const TmJob& jb : jobs) pn += (int64_t)jb.K * jb.K * geoms[jb.geom].n_theta;
      g_tm_pair_nodes.push_back(pn);
    }
    timed_launch(K_TM_TABLES, s, [&] { launch_tm_tables(a, s); });
    timed_launch(K_TM_SURFACE, s, [&] { launch_tm_surface(a, s); });
    timed_launch(K_TM_SOLVE, s, [&] { launch_tm_solve(a, s); });
    SB_CUDA(cudaGetLastError());
    std::vector<double> greek_all;
    std::vector<RoSph> sph;
    if (ro) {
      RoArgs r{};
      std::vector<double> mus;
      std::vector<const double*> projs;
      int64_t rank = 0, w = 0, part = 0, f = 0, g = 0;
      for (size_t k = 0; k < jobs.size(); ++k) {
        if (jobs[k].m != 0) continue;
        const TmGeom& gm = geoms[jobs[k].geom];
        RoSph e{};
        e.N = gm.N;
        e.L = 2 * gm.N;
        e.nq = gm.N + (e.L + 2) / 2;
        e.job0 = (int)k;
        const int64_t n1 = e.N + 1, S = 2 * e.N + 1, Q = 2 * e.N + 3;
        e.rank0 = rank;
        e.w0 = w;
        e.part0 = part;
        e.f0 = f;
        e.g0 = g;
        e.mu0 = (int64_t)mus.size();
        e.t_rank = r.n_rank;
        e.t_w = r.n_w;
        e.t_phi = r.n_phi;
        e.t_f = r.n_f;
        e.t_g = r.n_g;
        rank += 2 * 4 * n1 * n1 * S;
        w += 2 * Q * 4 * S * n1;
        part += 2 * Q * 16 * e.nq;
        f += 6 * e.nq;
        g += 6 * (e.L + 1);
        r.n_rank += (int64_t)e.N * e.N;
        r.n_w += Q * 2 * e.N;
        r.n_phi += Q * ((e.nq + 31) / 32);  // blocks: a tile of 32 cosines per q
        r.max_n = std::max(r.max_n, e.N);
        r.n_f += e.nq;
        r.n_g += e.L + 1;
        const auto& rl = rule(c, e.nq);
        mus.insert(mus.end(), rl.first.begin(), rl.first.end());
        projs.push_back(projector(c, e.nq, e.L, s).d.as<double>(0));
        sph.push_back(e);
      }
      r.sph = c.ro_sph.as<RoSph>(sph.size());
      r.n_sph = (int)sph.size();
      r.jobs = a.jobs;
      r.T = a.T;
      r.rank = c.ro_rank.as<double>((size_t)rank);
      r.w = c.ro_w.as<double>((size_t)w);
      r.part = c.ro_part.as<double>((size_t)part);
      r.f = c.ro_f.as<double>((size_t)f);
      r.greek = c.ro_greek.as<double>((size_t)g);
      double* mu_d = c.ro_mu.as<double>(mus.size());
      const double** proj_d = c.ro_proj.as<const double*>(projs.size());
      r.mu = mu_d;
      r.proj = proj_d;
      SB_CUDA(cudaMemcpyAsync((void*)r.sph, sph.data(), sph.size() * sizeof(RoSph),
                              cudaMemcpyHostToDevice, s));
      SB_CUDA(cudaMemcpyAsync(mu_d, mus.data(), mus.size() * 8, cudaMemcpyHostToDevice, s));
      SB_CUDA(cudaMemcpyAsync((void*)proj_d, projs.data(), projs.size() * sizeof(double*),
                              cudaMemcpyHostToDevice, s));
      timed_launch(K_RANDOM, s, [&] { launch_random(r, s); });
      SB_CUDA(cudaGetLastError());
      greek_all.resize((size_t)g);
      SB_CUDA(cudaMemcpyAsync(greek_all.data(), r.greek, (size_t)g * 8, cudaMemcpyDeviceToHost, s));
    }
    unsigned flag = 0;
    SB_CUDA(cudaMemcpyAsync(sums.data() + 3 * j0, a.sums, 3 * jobs.size() * 8,
                            cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaMemcpyAsync(&flag, a.err, sizeof flag, cudaMemcpyDeviceToHost, s));
    std::vector<double> all;
    if (t_out) {
      all.resize(2 * (size_t)T);
      SB_CUDA(cudaMemcpyAsync(all.data(), a.T, all.size() * 8, cudaMemcpyDeviceToHost, s));
    }
    SB_CUDA(cudaStreamSynchronize(s));
    if (flag & 2u)
      throw Failure{SCATRS_INVALID_INPUT,
                    "a spheroid's radial series needs more than 4000 terms (size too large)"};
    if (flag) throw Failure{SCATRS_INVALID_INPUT, "a spheroid's Q matrix is singular"};
    for (const RoSph& e : sph)
      greek_out->emplace_back(greek_all.begin() + e.g0, greek_all.begin() + e.g0 + 6 * (e.L + 1));
    if (t_out)
      for (size_t k = 0; k < jobs.size(); ++k) {
        const int n2 = 2 * jobs[k].K;
        (*t_out)[j0 + k].assign(all.begin() + 2 * jobs[k].T0,
                                all.begin() + 2 * jobs[k].T0 + 2 * (int64_t)n2 * n2);
      }
    j0 = j1;
  }
}

// driver.rs:166-214.
double tm_x_max(double x, double eps) {
  const double a = x * std::cbrt(eps);
  return std::max(a, a / eps);
}
// The validated domain of spheroids (tmatrix/domain.rs:45-79): aspect ratios 0.2 to 5,
// equal-volume x >= 1e-6, |m| x_max <= 60 (x_max of the longest semi-axis), 1.3 <= Re m <= 3,
// 0 <= Im m <= 0.5, rtol >= 1e-12.
constexpr double kTmDomainRtolMin = 1e-12;
bool tm_in_domain(double x, double eps, double mr, double mi) {
  return eps >= 0.2 && eps <= 5.0 && x >= 1e-6 && std::hypot(mr, mi) * tm_x_max(x, eps) <= 60.0 &&
         mr >= 1.3 && mr <= 3.0 && mi >= 0.0 && mi <= 0.5;
}
int tm_wiscombe(double xm) { return std::max((int)std::ceil(xm + 4.0 * std::cbrt(xm)) + 2, 4); }
int tm_theta_of(int n, double eps, double rtol) {
  const double h = std::max(eps, 1.0 / eps);
  const int shape =
      h <= 1.0 ? 0 : (int)std::ceil(std::log(1e4 / rtol) / (2.0 * std::log((h + 1.0) / (h - 1.0))));
  return std::max(2 * n, shape);
}

// One spheroid's converged solution: N, n_theta, the efficiencies (tmatrix/mod.rs:437-462:
// Q_back = 4 pi F11(180 deg) / (pi x^2) and g = alpha1_1 / (3 alpha1_0) from the Greek
// expansion, NaN without it), the raw Greek coefficients [6][2N + 1] and the largest last
// relative correction of the modes' refinement.
struct SpheroidResult {
  int n = 0, nth = 0;
  double q_ext = 0, q_sca = 0, q_abs = 0, q_back = NAN, g = NAN, err_est = 0;
  std::vector<double> greek;
};

// The T-matrices of n spheroids converged as driver.rs:343-420 converges them: N grown by
// max(N/8, 2) on mode 0 until its cross sections settle to rtol, then n_theta by a tenth (each
// loop skipped when n_fixed / theta_fixed > 0 fixes it), both within their caps; then every mode
// at the final N and n_theta, with the orientation average if `greek`. All spheroids of a step
// run as one batch of device work.
void spheroid_solve(Context& c, int64_t n, const double* x, const double* aspect_ratio,
                    const double* m, double rtol, int n_fixed, int theta_fixed, bool greek,
                    std::vector<SpheroidResult>& out, cudaStream_t s, bool allow_unvalidated) {
  if (!x || !aspect_ratio || !m)
    throw Failure{SCATRS_INVALID_INPUT, "x, aspect_ratio and m are required"};
  if (!(rtol >= 1e-13 && rtol <= 0.1))
    throw Failure{SCATRS_INVALID_INPUT, "rtol must be in [1e-13, 0.1]"};
  for (int64_t i = 0; i < n; ++i)
    check_tm_spec({x[i], aspect_ratio[i], m[2 * i], m[2 * i + 1], 0,
                   n_fixed > 0 ? n_fixed : 1, theta_fixed > 0 ? theta_fixed : 2});
  if (!allow_unvalidated) {
    // mod.rs:280-292: outside the validated domain only when asked for.
    if (rtol < kTmDomainRtolMin) {
      char buf[120];
      snprintf(buf, sizeof buf, "outside the validated domain: rtol %e is below %e", rtol,
               kTmDomainRtolMin);
      throw Failure{SCATRS_OUTSIDE_VALIDATED_DOMAIN, buf};
    }
    for (int64_t i = 0; i < n; ++i)
      if (!tm_in_domain(x[i], aspect_ratio[i], m[2 * i], m[2 * i + 1])) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "outside the validated domain: aspect ratio %g, x = %g, m = %g%+gi (spheroid %lld)",
                 aspect_ratio[i], x[i], m[2 * i], m[2 * i + 1], (long long)i);
        throw Failure{SCATRS_OUTSIDE_VALIDATED_DOMAIN, buf};
      }
  }
  struct St {
    int n, nth, cap, th_cap, stage;  // stage 0: N, 1: n_theta, 2: done
    double e, sc;
    double change = INFINITY;  // the last step's relative change of the cross sections
  };
  std::vector<St> st(n);
  std::vector<TmSpec> specs;
  auto theta = [&](int64_t i, int nn) {
    return theta_fixed > 0 ? theta_fixed
                           : std::min(tm_theta_of(nn, aspect_ratio[i], rtol), st[i].th_cap);
  };
  for (int64_t i = 0; i < n; ++i) {
    const double mag = std::hypot(m[2 * i], m[2 * i + 1]);
    const int start = tm_wiscombe(tm_x_max(x[i], aspect_ratio[i]));
    st[i].cap = std::min(2 * tm_wiscombe(tm_x_max(x[i], aspect_ratio[i]) * std::max(mag, 1.0)) + 20,
                         500);
    st[i].n = n_fixed > 0 ? n_fixed : std::min(start, st[i].cap);
    // mod.rs:293-300: n_theta's cap is 4 theta(start) + 40.
    st[i].th_cap = 4 * tm_theta_of(std::min(start, st[i].cap), aspect_ratio[i], rtol) + 40;
    st[i].nth = theta(i, st[i].n);
    st[i].stage = n_fixed > 0 ? (theta_fixed > 0 ? 2 : 1) : 0;
    if (st[i].stage < 2)
      specs.push_back({x[i], aspect_ratio[i], m[2 * i], m[2 * i + 1], 0, st[i].n, st[i].nth});
  }
  std::vector<double> sums;
  if (!specs.empty()) {
    run_tmatrices(c, specs, sums, nullptr, s);
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i)
      if (st[i].stage < 2) {
        st[i].e = sums[3 * k];
        st[i].sc = sums[3 * k + 1];
        ++k;
      }
  }
  for (;;) {
    std::vector<int64_t> who;
    specs.clear();
    for (int64_t i = 0; i < n; ++i) {
      St& z = st[i];
      if (z.stage == 2) continue;
      if ((z.stage == 0 && z.n >= z.cap) || (z.stage == 1 && z.nth >= z.th_cap)) {
        // driver.rs:356-359: achieved is the last relative change, requested the rtol.
        char buf[240];
        snprintf(buf, sizeof buf,
                 "not converged: achieved %e, requested %e (spheroid %lld: the cross sections "
                 "did not settle within N = %d, n_theta = %d)",
                 z.change, rtol, (long long)i, z.cap, z.th_cap);
        throw Failure{SCATRS_NOT_CONVERGED, buf, z.change, rtol};
      }
      int nn = z.n, nt = z.nth;
      if (z.stage == 0) {
        nn = std::min(z.n + std::max(z.n / 8, 2), z.cap);
        nt = theta(i, nn);
      } else {
        nt = std::min(z.nth + std::max(z.nth / 10, 2), z.th_cap);
      }
      specs.push_back({x[i], aspect_ratio[i], m[2 * i], m[2 * i + 1], 0, nn, nt});
      who.push_back(i);
    }
    if (who.empty()) break;
    run_tmatrices(c, specs, sums, nullptr, s);
    for (size_t k = 0; k < who.size(); ++k) {
      St& z = st[who[k]];
      const double e1 = sums[3 * k], s1 = sums[3 * k + 1];
      const double ch =
          std::max(std::fabs(e1 - z.e) / std::fabs(e1), std::fabs(s1 - z.sc) / std::fabs(s1));
      z.n = specs[k].N;
      z.nth = specs[k].n_theta;
      z.e = e1;
      z.sc = s1;
      z.change = ch;
      if (ch < rtol) z.stage += 1;
    }
  }
  // Every mode at the final N and n_theta.
  specs.clear();
  std::vector<int64_t> owner;
  for (int64_t i = 0; i < n; ++i)
    for (int mm = 0; mm <= st[i].n; ++mm) {
      specs.push_back({x[i], aspect_ratio[i], m[2 * i], m[2 * i + 1], mm, st[i].n, st[i].nth});
      owner.push_back(i);
    }
  std::vector<std::vector<double>> greeks;
  run_tmatrices(c, specs, sums, nullptr, s, greek ? &greeks : nullptr);
  out.assign(n, SpheroidResult{});
  std::vector<double> ext(n, 0.0), sca(n, 0.0);
  for (size_t k = 0; k < specs.size(); ++k) {
    const double w = specs[k].m == 0 ? 1.0 : 2.0;
    ext[owner[k]] += w * sums[3 * k];
    sca[owner[k]] += w * sums[3 * k + 1];
    out[owner[k]].err_est = std::max(out[owner[k]].err_est, sums[3 * k + 2]);
  }
  const double pi = 3.14159265358979323846;
  for (int64_t i = 0; i < n; ++i) {
    SpheroidResult& r = out[i];
    const double area = pi * x[i] * x[i];
    r.n = st[i].n;
    r.nth = st[i].nth;
    r.q_ext = 2.0 * pi * ext[i] / area;
    r.q_sca = 2.0 * pi * sca[i] / area;
    r.q_abs = r.q_ext - r.q_sca;
    if (greek) {
      r.greek = std::move(greeks[i]);
      const int64_t len = 2 * (int64_t)r.n + 1;
      const double a0 = r.greek[0];
      r.g = a0 > 0.0 ? (len > 1 ? r.greek[1] : 0.0) / (3.0 * a0) : 0.0;
      double f11 = 0.0;
      for (int64_t l = 0; l < len; ++l) f11 += (l % 2 ? -1.0 : 1.0) * r.greek[l];
      r.q_back = 4.0 * pi * f11 / area;
    }
  }
}

// The outputs of spheroids at a given truncation N and node count n_theta each (no convergence
// loop): every mode at that discretization, the orientation average, and per spheroid the
// efficiencies (Q_ext, Q_sca, Q_abs, Q_back, g) followed by the Greek coefficients [6][L + 1]
// (normalized by alpha1_0, or unnormalized: times 4 / x^2; zero above 2N), as
// scatrs_spheroid_compute reports them.
struct SphEval {
  double x, eps, m_re, m_im;
  int N, nth;
};
void spheroid_fixed_outputs(Context& c, const std::vector<SphEval>& ev, int order,
                            bool normalized, std::vector<std::vector<double>>& out,
                            cudaStream_t s) {
  std::vector<TmSpec> specs;
  std::vector<int64_t> owner;
  for (size_t i = 0; i < ev.size(); ++i)
    for (int mm = 0; mm <= ev[i].N; ++mm) {
      specs.push_back({ev[i].x, ev[i].eps, ev[i].m_re, ev[i].m_im, mm, ev[i].N, ev[i].nth});
      owner.push_back((int64_t)i);
    }
  std::vector<double> sums;
  std::vector<std::vector<double>> greeks;
  run_tmatrices(c, specs, sums, nullptr, s, &greeks);
  std::vector<double> ext(ev.size(), 0.0), sca(ev.size(), 0.0);
  for (size_t k = 0; k < specs.size(); ++k) {
    const double w = specs[k].m == 0 ? 1.0 : 2.0;
    ext[owner[k]] += w * sums[3 * k];
    sca[owner[k]] += w * sums[3 * k + 1];
  }
  const double pi = 3.14159265358979323846;
  const int64_t len = (int64_t)order + 1;
  out.assign(ev.size(), {});
  for (size_t i = 0; i < ev.size(); ++i) {
    const double x = ev[i].x, area = pi * x * x;
    const std::vector<double>& gr = greeks[i];
    const int64_t have = 2 * (int64_t)ev[i].N + 1;
    const double a0 = gr[0];
    double f11 = 0.0;
    for (int64_t l = 0; l < have; ++l) f11 += (l % 2 ? -1.0 : 1.0) * gr[l];
    std::vector<double>& o = out[i];
    o.assign(5 + (order >= 0 ? 6 * len : 0), 0.0);
    o[0] = 2.0 * pi * ext[i] / area;
    o[1] = 2.0 * pi * sca[i] / area;
    o[2] = o[0] - o[1];
    o[3] = 4.0 * pi * f11 / area;
    o[4] = a0 > 0.0 ? (have > 1 ? gr[1] : 0.0) / (3.0 * a0) : 0.0;
    if (order < 0) continue;
    const double scale = normalized ? 1.0 / a0 : 4.0 / (x * x);
    for (int f = 0; f < 6; ++f)
      for (int64_t l = 0; l < len; ++l)
        o[5 + f * len + l] = l < have ? scale * gr[f * have + l] : 0.0;
    if (normalized) o[5] = 1.0;
  }
}

// The derivatives of those outputs along x, the aspect ratio, Re m and Im m at each spheroid's
// converged (N, n_theta) -- the derivatives of the discretized solution, as the reference's
// compute_with_derivatives takes them (tmatrix/mod.rs:231-245). They are formed from the
// outputs at perturbed parameters, solved at the same (N, n_theta) in one batch: per direction
// the central differences at steps h and h/2 (h = 1e-4 of x, of the aspect ratio, of |m|),
// Richardson-extrapolated (truncation O(h^4)); along Im m, whose values cannot go below zero,
// the one-sided fourth-order stencil on the steps h, 2h, 3h, 4h when Im m < 4h. d[dir][i] holds
// spheroid i's output vector's derivative.
void spheroid_fixed_derivs(Context& c, const std::vector<SphEval>& base, int order,
                           bool normalized, std::vector<std::vector<double>> d[4],
                           cudaStream_t s, unsigned dir_mask = 0xF) {
  std::vector<SphEval> ev;
  struct Plan {
    double h;
    bool forward;
  };
  std::vector<Plan> plan(4 * base.size());
  for (size_t i = 0; i < base.size(); ++i) {
    const SphEval& b = base[i];
    const double mag = std::hypot(b.m_re, b.m_im);
    const double hs[4] = {1e-4 * b.x, 1e-4 * b.eps, 1e-4 * mag, 1e-4 * mag};
    for (int dir = 0; dir < 4; ++dir) {
      Plan& p = plan[4 * i + dir];
      p.h = hs[dir];
      if (!(dir_mask >> dir & 1u)) continue;
      p.forward = dir == 3 && b.m_im < 4.0 * p.h;
      const double steps_c[4] = {p.h, -p.h, 0.5 * p.h, -0.5 * p.h};
      const double steps_f[4] = {p.h, 2.0 * p.h, 3.0 * p.h, 4.0 * p.h};
      for (int k = 0; k < 4; ++k) {
        const double st = p.forward ? steps_f[k] : steps_c[k];
        SphEval e = b;
        if (dir == 0) e.x += st;
        if (dir == 1) e.eps += st;
        if (dir == 2) e.m_re += st;
        if (dir == 3) e.m_im += st;
        ev.push_back(e);
      }
    }
  }
  std::vector<std::vector<double>> val, at;
  spheroid_fixed_outputs(c, base, order, normalized, val, s);
  spheroid_fixed_outputs(c, ev, order, normalized, at, s);
  const int n_dirs = __builtin_popcount(dir_mask & 0xFu);
  for (int dir = 0; dir < 4; ++dir) d[dir].assign(base.size(), {});
  for (size_t i = 0; i < base.size(); ++i)
    for (int dir = 0, slot = 0; dir < 4; ++dir) {
      if (!(dir_mask >> dir & 1u)) continue;
      const Plan& p = plan[4 * i + dir];
      const size_t k0 = 4 * (n_dirs * i + slot++);
      const std::vector<double>& f0 = val[i];
      std::vector<double>& o = d[dir][i];
      o.assign(f0.size(), 0.0);
      for (size_t q = 0; q < f0.size(); ++q) {
        const double a = at[k0][q], b = at[k0 + 1][q], a2 = at[k0 + 2][q], b2 = at[k0 + 3][q];
        if (p.forward) {
          // f'(0) = (-25 f0 + 48 f1 - 36 f2 + 16 f3 - 3 f4) / (12 h)
          o[q] = (-25.0 * f0[q] + 48.0 * a - 36.0 * b + 16.0 * a2 - 3.0 * b2) / (12.0 * p.h);
        } else {
          const double dh = (a - b) / (2.0 * p.h), dh2 = (a2 - b2) / p.h;
          o[q] = (4.0 * dh2 - dh) / 3.0;
        }
      }
    }
}

// A value and its error bound, propagated to first order through the ratios (lin.rs:7-68,
// without derivatives).
struct LinE {
  double v = 0.0, e = 0.0;
};
LinE lin_div(const LinE& a, const LinE& b) {
  const double v = a.v / b.v;
  return {v, (a.e + std::fabs(v) * b.e) / std::fabs(b.v)};
}
LinE lin_scale(const LinE& a, double c) { return {c * a.v, std::fabs(c) * a.e}; }

// The adaptive ensemble of randomly oriented spheroids (Particle::Spheroid on the engine's
// direct path, engine.rs:369-449 for pass 1, 1207-1339 and 1558-1740 for pass 2, 1782-1836
// for the averages, 2396-2497 for the outputs). Pass 1's node evaluations are spheroid batches
// on the GPU (T-matrix converged to the ensemble's rtol / 100 clamped to [1e-12, 1e-8],
// engine.rs:87, with the orientation average when Greek coefficients or phase are asked for),
// kept for pass 2, which integrates them without solving again. Every distribution of every
// particle is an output unit of its own (batch, one particle: panels shared per wavelength);
// the direct order at a wavelength follows the largest N of all the call's spheroids there
// (engine.rs:2073-2086). With rows, the parts' averages go there instead of the outputs (a
// mixture's host assembly).
struct SphParticle {
  const scatrs_distribution* dists;
  int64_t n_dist;
  double eps;
  const double* m;  // complex per wavelength
};
struct SphRows {
  std::vector<std::vector<double>> av, ae;  // per (part, wavelength): 9 + 6 (ld + 1) doubles
  std::vector<int64_t> ld;                  // per wavelength: the direct order, or -1
  std::vector<char> converged;
  std::vector<int64_t> panels;
};

void spheroid_call(const std::vector<SphParticle>& ps, bool batch, const double* wavelengths,
                   int64_t n_wl, const double* mu, int64_t n_mu,
                   const scatrs_adaptive_options* options, const AdOutputs& res,
                   SphRows* rows = nullptr) {
  if (!options) throw Failure{SCATRS_INVALID_INPUT, "options must not be NULL"};
  int64_t n_dist = 0;
  for (const SphParticle& q : ps) n_dist += q.n_dist;
  if (n_dist < 0 || n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
  if (batch && ps.size() > 1) throw Failure{SCATRS_INVALID_INPUT, "a batch has one particle"};
  const bool all_orders = options->greek_order == SCATRS_GREEK_ALL;
  const adaptive::Options o{options->rtol, options->max_panels, options->allow_unvalidated != 0,
                            options->refine_backscatter != 0};
  if (!(o.rtol >= 1e-13 && o.rtol <= 0.1)) {
    char buf[80];
    snprintf(buf, sizeof buf, "rtol must be in [1e-13, 0.1], got %g", o.rtol);
    throw Failure{SCATRS_INVALID_INPUT, buf};
  }
  if (o.max_panels < 1) throw Failure{SCATRS_INVALID_INPUT, "max_panels must be at least 1"};
  for (int64_t i = 0; i < n_wl; ++i)
    if (!(std::isfinite(wavelengths[i]) && wavelengths[i] > 0.0))
      throw Failure{SCATRS_INVALID_INPUT,
                    "wavelength " + std::to_string(i) + " must be finite and > 0"};
  for (const SphParticle& q : ps)
    if (!(std::isfinite(q.eps) && q.eps > 0.0))
      throw Failure{SCATRS_INVALID_INPUT, "the aspect ratio must be finite and > 0"};
  scatrs_fixed_options fo{32, all_orders ? -1 : options->greek_order, options->normalized,
                          options->allow_unvalidated};
  const int64_t n_units = n_dist * n_wl;
  check_options(&fo, n_units, n_mu, mu);
  if (n_units == 0) return;
  std::vector<adaptive::Part> parts;
  std::vector<int> particle_of;  // per part
  for (size_t q = 0; q < ps.size(); ++q)
    for (int64_t d = 0; d < ps[q].n_dist; ++d) {
      const scatrs_distribution& dd = ps[q].dists[d];
      try {
        parts.push_back(
            adaptive::make_part(dd.kind, dd.param, o.rtol, dd.table, dd.table_len));
      } catch (const adaptive::Error& e) {
        throw Failure{e.status, "distribution " + std::to_string(d) + ": " + e.msg};
      }
      particle_of.push_back((int)q);
    }
  const double rtol_t = std::min(std::max(o.rtol / 100.0, 1e-12), 1e-8);
  const bool keep_greek = options->greek_order >= 0 || all_orders || n_mu > 0;
  const double pi = 3.14159265358979323846;
  Context& c = context();
  std::lock_guard<std::mutex> lk(c.mtx);
  cudaStream_t s = 0;
  // Solved nodes by (particle, wavelength, radius bits).
  std::map<std::tuple<int, int64_t, uint64_t>, SpheroidResult> cache;
  auto key_of = [](int q, int64_t i, double r) {
    uint64_t b;
    memcpy(&b, &r, 8);
    return std::make_tuple(q, i, b);
  };
  auto eval = [&](const std::vector<adaptive::Query>& qs, std::vector<adaptive::NodeResult>& out) {
    std::vector<double> xs, es, ms;
    std::vector<size_t> which;
    for (size_t k = 0; k < qs.size(); ++k) {
      const int64_t i = qs[k].wl % n_wl;
      const int q = particle_of[qs[k].wl / n_wl];
      if (cache.count(key_of(q, i, qs[k].r))) continue;
      xs.push_back(2.0 * pi * qs[k].r / wavelengths[i]);
      es.push_back(ps[q].eps);
      ms.push_back(ps[q].m[2 * i]);
      ms.push_back(ps[q].m[2 * i + 1]);
      which.push_back(k);
    }
    if (!which.empty()) {
      std::vector<SpheroidResult> r;
      // The orientation average always: Q_back, g and the depolarization numerator come
      // from it (particle.rs:334-343).
      spheroid_solve(c, (int64_t)which.size(), xs.data(), es.data(), ms.data(), rtol_t, 0, 0,
                     true, r, s, o.allow_unvalidated);
      for (size_t k = 0; k < which.size(); ++k) {
        const adaptive::Query& q = qs[which[k]];
        cache[key_of(particle_of[q.wl / n_wl], q.wl % n_wl, q.r)] = std::move(r[k]);
      }
    }
    for (size_t k = 0; k < qs.size(); ++k) {
      const SpheroidResult& v =
          cache.at(key_of(particle_of[qs[k].wl / n_wl], qs[k].wl % n_wl, qs[k].r));
      const double area = pi * qs[k].r * qs[k].r;
      adaptive::NodeResult& x = out[k];
      const double q[6] = {1.0, area * v.q_ext, area * v.q_sca, area * v.q_sca * v.g,
                           area * v.q_back, area * v.q_abs};
      for (int j = 0; j < 6; ++j) x.q[j] = q[j];
      x.n = v.n;
      x.status = 0;
    }
  };
  // Pass 1 per (group, wavelength): every distribution on its own, or one batch.
  std::vector<adaptive::Job> jobs;
  std::vector<int> job_of(n_units, -1), place(n_units, 0);
  for (int64_t i = 0; i < n_wl; ++i) {
    adaptive::Job shared;
    for (int64_t p = 0; p < n_dist; ++p) {
      if (parts[p].support == adaptive::POINT) continue;
      const int64_t u = p * n_wl + i;
      if (batch) {
        if (shared.parts.empty()) shared.wl = (int)u;
        place[u] = (int)shared.parts.size();
        job_of[u] = -2;  // fixed below
        shared.parts.push_back((int)p);
      } else {
        job_of[u] = (int)jobs.size();
        adaptive::Job jb;
        jb.wl = (int)u;
        jb.parts = {(int)p};
        jobs.push_back(jb);
      }
    }
    if (batch && !shared.parts.empty()) {
      for (int p : shared.parts) job_of[p * n_wl + i] = (int)jobs.size();
      jobs.push_back(shared);
    }
  }
  std::vector<double> wl_units(n_units);
  for (int64_t u = 0; u < n_units; ++u) wl_units[u] = wavelengths[u % n_wl];
  std::vector<adaptive::Query> points;
  for (int64_t p = 0; p < n_dist; ++p)
    if (parts[p].support == adaptive::POINT)
      for (int64_t i = 0; i < n_wl; ++i) points.push_back({parts[p].lo, (int)(p * n_wl + i)});
  std::vector<adaptive::NodeResult> point_res(points.size());
  if (!points.empty()) eval(points, point_res);
  adaptive::pass1(jobs, parts, wl_units.data(), o, eval);
  for (const adaptive::Job& jb : jobs)
    if (jb.status != 0) throw Failure{jb.status, jb.msg};
  // The direct order per wavelength: every order to 2N for the phase matrix, else to the
  // requested one (engine.rs:2073-2086).
  // N_max of each unit's call at its wavelength (engine.rs:1987-2030, p1.n_terms over the
  // final panels): the unit's own part, or every part of a batch or a mixture.
  std::vector<int64_t> n_own(n_units, 0), n_direct(n_units, 0), n_at(n_wl, 0);
  for (int64_t u = 0; u < n_units; ++u) {
    const int64_t p = u / n_wl, i = u % n_wl;
    n_own[u] = parts[p].support == adaptive::POINT
                   ? cache.at(key_of(particle_of[p], i, parts[p].lo)).n
                   : jobs[job_of[u]].n_terms;
    n_at[i] = std::max(n_at[i], n_own[u]);
  }
  for (int64_t u = 0; u < n_units; ++u) n_direct[u] = batch || rows ? n_at[u % n_wl] : n_own[u];
  // greek='all': every order to 2 N_max (GreekOrder::All), padded to the longest.
  int64_t width = 0;
  if (all_orders && !rows) {  // a mixture's rows: the mixture sets its own coefficients
    for (int64_t u = 0; u < n_units; ++u) width = std::max(width, 2 * n_direct[u] + 1);
    GreekAll& ga = t_greek_all;
    ga.width = width;
    ga.n = n_units;
    ga.p = 0;
    ga.g.assign(6 * n_units * width, 0.0);
    ga.ge.assign(ga.g.size(), 0.0);
    ga.dg.clear();
    ga.dge.clear();
  }
  if (rows) {
    rows->av.assign(n_units, {});
    rows->ae.assign(n_units, {});
    rows->ld.assign(n_wl, -1);
    rows->converged.assign(n_units, 1);
    rows->panels.assign(n_units, 0);
  }
  constexpr int kS = 9;  // ONE, EXT, SCA, SCAG, ABS, BACK, R2, R3, DEPOL
  for (int64_t u = 0; u < n_units; ++u) {
    const int64_t p = u / n_wl, i = u % n_wl;
    const double lambda = wavelengths[i];
    const adaptive::Part& part = parts[p];
    const int L = all_orders ? (int)(2 * n_direct[u]) : options->greek_order;
    const int64_t ld = !keep_greek ? -1 : n_mu == 0 ? std::min<int64_t>(L, 2 * n_direct[u])
                                                      : 2 * n_direct[u];
    const int64_t glen = ld + 1;  // 0 without a direct segment
    const int64_t len = kS + 6 * glen;
    // One node's direct quantities and declared errors (direct_scalars, direct_node).
    std::vector<double> g(len), ge(len);
    auto direct_node = [&](double r) {
      const SpheroidResult& v = cache.at(key_of(particle_of[p], i, r));
      const double area = pi * r * r;
      const double tau = std::max(rtol_t, v.err_est);
      const double c4 = 4.0 * tau, c16 = 16.0 * tau;
      const int64_t have = 2 * (int64_t)v.n + 1;
      const double x = 2.0 * pi * r / lambda, un = 4.0 / (x * x);
      double depol = 0.0;
      for (int64_t l = 0; l < have; ++l) {
        const double t = un * (v.greek[l] - 0.5 * (v.greek[have + l] - v.greek[2 * have + l]));
        depol += l % 2 ? -t : t;
      }
      const double sv[kS] = {1.0,         area * v.q_ext, area * v.q_sca, area * v.q_sca * v.g,
                             area * v.q_abs, area * v.q_back, r * r, r * r * r, area * depol};
      const double back = area * std::max(std::fabs(v.q_back), std::fabs(v.q_sca));
      const double se[kS] = {0.0,
                             c4 * std::fabs(sv[1]),
                             c4 * std::fabs(sv[2]),
                             c4 * std::fabs(sv[2]) * (1.0 + std::fabs(v.g)),
                             c16 * std::fabs(sv[1]),
                             c16 * back,
                             0.0,
                             0.0,
                             2.0 * c16 * back};
      for (int k = 0; k < kS; ++k) {
        g[k] = sv[k];
        ge[k] = se[k];
      }
      if (glen > 0) {
        double big = 0.0;
        for (int64_t l = 0; l < have; ++l) big = std::max(big, std::fabs(un * v.greek[l]));
        const double ce = c16 * area * big;
        for (int f = 0; f < 6; ++f)
          for (int64_t l = 0; l < glen; ++l) {
            g[kS + f * glen + l] = l < have ? area * un * v.greek[f * have + l] : 0.0;
            ge[kS + f * glen + l] = ce;
          }
      }
    };
    std::vector<double> av(len, 0.0), ae(len, 0.0);
    bool conv = true;
    int64_t panels = 0;
    if (part.support == adaptive::POINT) {
      // monodisperse_direct (engine.rs:1896-1961): the particle itself.
      direct_node(part.lo);
      av = g;
      ae = ge;
    } else {
      const adaptive::Job& jb = jobs[job_of[u]];
      conv = jb.converged[place[u]];
      panels = (int64_t)jb.panels.size();
      std::vector<double> S(len, 0.0), E(len, 0.0);
      for (const auto& ab : jb.panels) {
        adaptive::Node nd[15];
        adaptive::gk15(ab.first, ab.second, nd);
        std::vector<double> ks(len, 0.0), gs(len, 0.0), ne(len, 0.0);
        for (int k = 0; k < 15; ++k) {
          const double r = std::exp(nd[k].t), ur = part.u(r) * r;
          direct_node(r);
          for (int64_t j = 0; j < len; ++j) {
            ks[j] += nd[k].wk * ur * g[j];
            gs[j] += nd[k].wg * ur * g[j];
            ne[j] += std::fabs(nd[k].wk * ur) * ge[j];
          }
        }
        for (int64_t j = 0; j < len; ++j) {
          S[j] += ks[j];
          E[j] += std::fabs(ks[j] - gs[j]) + ne[j];
        }
      }
      // averages (engine.rs:1782-1836).
      const double z = part.mom.z, ez = part.mom.ez;
      const double trunc = part.support == adaptive::UNBOUNDED ? 0.2 * o.rtol : 0.0;
      for (int64_t j = 0; j < len; ++j) {
        av[j] = S[j] / z;
        ae[j] = (E[j] + std::fabs(av[j]) * ez) / z + trunc * std::fabs(av[j]);
      }
      av[6] = part.mom.v[0];
      ae[6] = part.mom.e[0];
      av[7] = part.mom.v[1];
      ae[7] = part.mom.e[1];
    }
    if (rows) {
      rows->av[u] = std::move(av);
      rows->ae[u] = std::move(ae);
      rows->ld[i] = ld;
      rows->converged[u] = conv ? 1 : 0;
      rows->panels[u] = panels;
      continue;
    }
    // assemble (engine.rs:2396-2497).
    auto lin = [&](int64_t j) { return LinE{av[j], ae[j]}; };
    const LinE ext = lin(1), sca = lin(2), scag = lin(3), abs_ = lin(4), back = lin(5),
               r2 = lin(6), r3 = lin(7), num = lin(8);
    for (const auto& w : {std::make_pair("<C_ext>", ext), std::make_pair("<C_sca>", sca),
                          std::make_pair("<C_back>", back)})
      if (!(std::isfinite(w.second.v) && w.second.v != 0.0))
        throw Failure{SCATRS_INVALID_INPUT,
                      std::string("the ensemble's ") + w.first +
                          " is zero or not finite, so its ratios are undefined (does m = 1?)"};
    const LinE den{2.0 * back.v - num.v, 2.0 * back.e + num.e};
    const LinE outs[11] = {ext,
                           sca,
                           abs_,
                           back,
                           lin_div(sca, ext),
                           lin_div(scag, sca),
                           lin_scale(lin_div(ext, back), 4.0 * pi),
                           lin_div(num, den),
                           lin_div(r3, r2),
                           lin_scale(r2, pi),
                           lin_scale(r3, 4.0 * pi / 3.0)};
    for (int k = 0; k < 11; ++k) {
      res.values[k * n_units + u] = outs[k].v;
      if (res.errors) res.errors[k * n_units + u] = outs[k].e;
    }
    const bool norm = options->normalized != 0;
    auto G = [&](int f, int64_t l) { return LinE{av[kS + f * glen + l], ae[kS + f * glen + l]}; };
    if (L >= 0 && (res.greek || all_orders)) {
      const LinE a0 = G(0, 0);
      double* gv = all_orders ? t_greek_all.g.data() : res.greek;
      double* ge_out = all_orders ? t_greek_all.ge.data() : res.greek_err;
      const int64_t w = all_orders ? width : L + 1;
      for (int f = 0; f < 6; ++f)
        for (int64_t l = 0; l <= L; ++l) {
          LinE x = l < glen ? G(f, l) : LinE{};
          if (norm) x = (f == 0 && l == 0) ? LinE{1.0, 0.0} : lin_div(x, a0);
          gv[((int64_t)f * n_units + u) * w + l] = x.v;
          if (ge_out) ge_out[((int64_t)f * n_units + u) * w + l] = x.e;
        }
    }
    if (n_mu > 0 && res.phase) {
      // greek_phase (engine.rs:2359-2390): combinations with exact weights, errors as bounds.
      std::vector<double> d00(glen), d22(glen), d2m2(glen), d02(glen);
      for (int64_t j = 0; j < n_mu; ++j) {
        wigner_d(0, 0, mu[j], d00.data(), glen);
        wigner_d(2, 2, mu[j], d22.data(), glen);
        wigner_d(2, -2, mu[j], d2m2.data(), glen);
        wigner_d(0, 2, mu[j], d02.data(), glen);
        LinE f[6];
        for (int64_t l = 0; l < glen; ++l) {
          const double plus = 0.5 * (d22[l] + d2m2[l]), minus = 0.5 * (d22[l] - d2m2[l]);
          const double w[6][2] = {{d00[l], 0}, {d02[l], 0}, {plus, minus},
                                  {minus, plus}, {d02[l], 0}, {d00[l], 0}};
          const int src[6][2] = {{0, -1}, {4, -1}, {1, 2}, {1, 2}, {5, -1}, {3, -1}};
          for (int k = 0; k < 6; ++k)
            for (int t = 0; t < 2; ++t) {
              if (src[k][t] < 0) continue;
              const LinE x = G(src[k][t], l);
              f[k].v += w[k][t] * x.v;
              f[k].e += std::fabs(w[k][t]) * x.e;
            }
        }
        for (int k = 0; k < 6; ++k) {
          const LinE x = norm ? lin_div(f[k], sca) : f[k];
          res.phase[((int64_t)k * n_units + u) * n_mu + j] = x.v;
          if (res.phase_err) res.phase_err[((int64_t)k * n_units + u) * n_mu + j] = x.e;
        }
      }
    }
    if (res.converged) res.converged[u] = conv ? 1 : 0;
    if (res.panels) res.panels[u] = panels;
  }
}

// The adaptive ensemble of spheroid distributions with derivatives (EnsembleOptions::
// derivatives on the engine's direct path): pass 1 refines the requested distribution
// parameters' blocks and the derivatives of C_ext, C_sca, C_sca g, C_back and C_abs along each
// requested direction of the particle (Re m, Im m, the aspect ratio; engine.rs:379-471,
// 620-720); pass 2 integrates the stored node values and their derivatives with their declared
// errors (direct_node, engine.rs:1281-1340; the node errors summed with the absolute weights,
// 1682-1740); the averages follow the quotient rule against the moments' dZ (averages,
// engine.rs:1782-1836; a single radius: monodisperse_direct, 1896-1961, with the radius
// derivative 2/r g + (2 pi / lambda) dg/dx); the outputs carry the derivatives through the
// ratios (assemble, engine.rs:2396-2497; lin.rs). A node's derivatives are those of its
// discretized solution at its converged N and n_theta (spheroid_fixed_derivs), where the
// reference carries dual numbers through its T-matrix (tmatrix/mod.rs:231-245). Every
// distribution of every particle is a part on its own panels; reqs holds each part's request
// (particle-major). Alone (one part) the call writes the outputs; with rows (a mixture's host
// assembly) each (part, wavelength) unit's averages go there, the direct order at a wavelength
// following the largest N of all its spheroids (engine.rs:2073-2086).
struct SphDerivReq {
  std::vector<int> grads, theta_cols;  // distribution parameters and their result columns
  int dir_cols[3] = {-1, -1, -1};      // result columns along Re m, Im m, the aspect ratio
};
// Per (part, wavelength) unit: the 9 scalars and the direct segment (9 + 6 (ld + 1)) with their
// errors, and per result column (P of them, column-major) their derivatives and errors.
struct SphRowsD {
  std::vector<std::vector<double>> av, ae, dv, de;
  std::vector<int64_t> ld;  // per wavelength, or -1
  std::vector<char> converged;
  std::vector<int64_t> panels;
};

void spheroid_call_d(const std::vector<SphParticle>& ps, const std::vector<SphDerivReq>& reqs,
                     const double* wavelengths, int64_t n_wl, const double* mu, int64_t n_mu,
                     const scatrs_adaptive_options* options, const AdOutputs& res,
                     const AdDerivs& dd, SphRowsD* rows = nullptr) {
  if (!options) throw Failure{SCATRS_INVALID_INPUT, "options must not be NULL"};
  int64_t n_parts = 0;
  for (const SphParticle& q : ps) n_parts += q.n_dist;
  if ((int64_t)reqs.size() != n_parts)
    throw Failure{SCATRS_INVALID_INPUT, "one derivative request per distribution"};
  if (!rows && n_parts != 1) throw Failure{SCATRS_INVALID_INPUT, "one distribution"};
  if (n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
  const bool all_orders = options->greek_order == SCATRS_GREEK_ALL;
  const adaptive::Options o{options->rtol, options->max_panels, options->allow_unvalidated != 0,
                            options->refine_backscatter != 0};
  if (!(o.rtol >= 1e-13 && o.rtol <= 0.1)) {
    char buf[80];
    snprintf(buf, sizeof buf, "rtol must be in [1e-13, 0.1], got %g", o.rtol);
    throw Failure{SCATRS_INVALID_INPUT, buf};
  }
  if (o.max_panels < 1) throw Failure{SCATRS_INVALID_INPUT, "max_panels must be at least 1"};
  for (int64_t i = 0; i < n_wl; ++i)
    if (!(std::isfinite(wavelengths[i]) && wavelengths[i] > 0.0))
      throw Failure{SCATRS_INVALID_INPUT,
                    "wavelength " + std::to_string(i) + " must be finite and > 0"};
  for (const SphParticle& q : ps)
    if (!(std::isfinite(q.eps) && q.eps > 0.0))
      throw Failure{SCATRS_INVALID_INPUT, "the aspect ratio must be finite and > 0"};
  scatrs_fixed_options fo{32, all_orders ? -1 : options->greek_order, options->normalized,
                          options->allow_unvalidated};
  const int64_t n_units = n_parts * n_wl;
  check_options(&fo, n_units, n_mu, mu);
  if (n_units == 0) return;
  std::vector<adaptive::Part> parts;
  std::vector<int> particle_of;
  bool any_dir = false, along_x = false;
  for (size_t q = 0; q < ps.size(); ++q)
    for (int64_t d = 0; d < ps[q].n_dist; ++d) {
      const scatrs_distribution& dist = ps[q].dists[d];
      const SphDerivReq& rq = reqs[parts.size()];
      try {
        parts.push_back(adaptive::make_part(dist.kind, dist.param, o.rtol, dist.table,
                                            dist.table_len, rq.grads));
      } catch (const adaptive::Error& e) {
        throw Failure{e.status, "distribution " + std::to_string(d) + ": " + e.msg};
      }
      for (int k = 0; k < 3; ++k) parts.back().dirs[k] = rq.dir_cols[k] >= 0;
      any_dir = any_dir || parts.back().dir_derivatives();
      along_x = along_x || (parts.back().support == adaptive::POINT && !rq.grads.empty());
      particle_of.push_back((int)q);
    }
  // The directions solved at each node: every one of the particle's when any is asked for
  // (engine.rs:1438-1440), and x for a single radius's radius. spheroid_fixed_derivs orders
  // them x, aspect ratio, Re m, Im m; here the directions are Re m, Im m, aspect ratio, x.
  const unsigned mask = (any_dir ? 0xEu : 0u) | (along_x ? 0x1u : 0u);
  const int sfd_of[4] = {2, 3, 1, 0};
  const double rtol_t = std::min(std::max(o.rtol / 100.0, 1e-12), 1e-8);
  const double pi = 3.14159265358979323846;
  Context& c = context();
  std::lock_guard<std::mutex> lk(c.mtx);
  cudaStream_t s = 0;
  // Solved nodes by (particle, wavelength, radius bits): the values, and per direction the
  // derivatives of (Q_ext, Q_sca, Q_abs, Q_back, g, then the six unnormalized Greek arrays to
  // 2N). A query's `wl` is its unit, part * n_wl + wavelength.
  struct Node {
    SpheroidResult v;
    std::vector<double> d[4];
  };
  std::map<std::tuple<int, int64_t, uint64_t>, Node> cache;
  auto key_of = [](int q, int64_t i, double r) {
    uint64_t b;
    memcpy(&b, &r, 8);
    return std::make_tuple(q, i, b);
  };
  auto key_u = [&](int64_t u, double r) { return key_of(particle_of[u / n_wl], u % n_wl, r); };
  auto solve = [&](const std::vector<adaptive::Query>& qs) {
    std::vector<double> xs, es, ms;
    std::vector<std::pair<int64_t, double>> which;
    std::set<std::tuple<int, int64_t, uint64_t>> batch;  // parts of one particle may share nodes
    for (const adaptive::Query& q : qs) {
      const int64_t i = q.wl % n_wl;
      const SphParticle& sp = ps[particle_of[q.wl / n_wl]];
      if (cache.count(key_u(q.wl, q.r)) || !batch.insert(key_u(q.wl, q.r)).second) continue;
      xs.push_back(2.0 * pi * q.r / wavelengths[i]);
      es.push_back(sp.eps);
      ms.push_back(sp.m[2 * i]);
      ms.push_back(sp.m[2 * i + 1]);
      which.push_back({q.wl, q.r});
    }
    if (which.empty()) return;
    std::vector<SpheroidResult> r;
    spheroid_solve(c, (int64_t)which.size(), xs.data(), es.data(), ms.data(), rtol_t, 0, 0, true,
                   r, s, o.allow_unvalidated);
    std::vector<SphEval> ev(which.size());
    int order = 0;
    for (size_t k = 0; k < which.size(); ++k) {
      ev[k] = {xs[k], es[k], ms[2 * k], ms[2 * k + 1], r[k].n, r[k].nth};
      order = std::max(order, 2 * r[k].n);
    }
    std::vector<std::vector<double>> d[4];
    if (mask) spheroid_fixed_derivs(c, ev, order, false, d, s, mask);
    const int64_t len = (int64_t)order + 1;
    for (size_t k = 0; k < which.size(); ++k) {
      Node nd;
      const int64_t have = 2 * (int64_t)r[k].n + 1;
      for (int dir = 0; dir < 4; ++dir) {
        if (!(mask >> sfd_of[dir] & 1u)) continue;
        const std::vector<double>& src = d[sfd_of[dir]][k];
        std::vector<double>& dst = nd.d[dir];
        dst.assign(5 + 6 * have, 0.0);
        for (int j = 0; j < 5; ++j) dst[j] = src[j];
        for (int f = 0; f < 6; ++f)
          for (int64_t l = 0; l < have; ++l) dst[5 + f * have + l] = src[5 + f * len + l];
      }
      nd.v = std::move(r[k]);
      cache[key_u(which[k].first, which[k].second)] = std::move(nd);
    }
  };
  // The pass-1 quantities (quantities1, engine.rs:379-417): the values, then per direction
  // d C_ext, d C_sca, d(C_sca g), d C_back, d C_abs.
  auto eval = [&](const std::vector<adaptive::Query>& qs, std::vector<adaptive::NodeResult>& out) {
    solve(qs);
    for (size_t k = 0; k < qs.size(); ++k) {
      const Node& nd = cache.at(key_u(qs[k].wl, qs[k].r));
      const SpheroidResult& v = nd.v;
      const double area = pi * qs[k].r * qs[k].r;
      adaptive::NodeResult& x = out[k];
      const double q[6] = {1.0, area * v.q_ext, area * v.q_sca, area * v.q_sca * v.g,
                           area * v.q_back, area * v.q_abs};
      for (int j = 0; j < adaptive::kNodeQ; ++j) x.q[j] = 0.0;
      for (int j = 0; j < 6; ++j) x.q[j] = q[j];
      for (int dir = 0; dir < 3 && any_dir; ++dir) {
        const std::vector<double>& dq = nd.d[dir];
        double* o5 = x.q + adaptive::kPass1 + adaptive::kGroup * dir;
        o5[0] = area * dq[0];
        o5[1] = area * dq[1];
        o5[2] = area * (dq[1] * v.g + v.q_sca * dq[4]);
        o5[3] = area * dq[3];
        o5[4] = area * dq[2];
      }
      x.n = v.n;
      x.status = 0;
    }
  };
  // Pass 1 per (part, wavelength) unit, each part on its own panels; single radii themselves.
  std::vector<adaptive::Job> jobs;
  std::vector<int> job_of(n_units, -1);
  std::vector<adaptive::Query> points;
  for (int64_t u = 0; u < n_units; ++u) {
    const adaptive::Part& pt = parts[u / n_wl];
    if (pt.support == adaptive::POINT) {
      points.push_back({pt.lo, (int)u});
      continue;
    }
    job_of[u] = (int)jobs.size();
    adaptive::Job jb;
    jb.wl = (int)u;
    jb.parts = {(int)(u / n_wl)};
    jobs.push_back(jb);
  }
  std::vector<double> wl_units(n_units);
  for (int64_t u = 0; u < n_units; ++u) wl_units[u] = wavelengths[u % n_wl];
  std::vector<adaptive::NodeResult> point_res(points.size());
  if (!points.empty()) eval(points, point_res);
  adaptive::pass1(jobs, parts, wl_units.data(), o, eval);
  for (const adaptive::Job& jb : jobs)
    if (jb.status != 0) throw Failure{jb.status, jb.msg};
  // The direct order: each unit's own N_max, or in a mixture the largest at its wavelength.
  std::vector<int64_t> n_direct(n_units), n_at(n_wl, 0);
  int64_t width = 0;
  for (int64_t u = 0; u < n_units; ++u) {
    const adaptive::Part& pt = parts[u / n_wl];
    n_direct[u] = pt.support == adaptive::POINT ? cache.at(key_u(u, pt.lo)).v.n
                                                : jobs[job_of[u]].n_terms;
    n_at[u % n_wl] = std::max(n_at[u % n_wl], n_direct[u]);
  }
  for (int64_t u = 0; u < n_units; ++u) {
    if (rows) n_direct[u] = n_at[u % n_wl];
    width = std::max(width, 2 * n_direct[u] + 1);
  }
  if (rows) {
    rows->av.assign(n_units, {});
    rows->ae.assign(n_units, {});
    rows->dv.assign(n_units, {});
    rows->de.assign(n_units, {});
    rows->ld.assign(n_wl, -1);
    rows->converged.assign(n_units, 1);
    rows->panels.assign(n_units, 0);
  }
  const int64_t P = dd.n;
  if (all_orders && !rows) {  // a mixture's rows: the mixture sets its own coefficients
    GreekAll& ga = t_greek_all;
    ga.width = width;
    ga.n = n_units;
    ga.p = P;
    ga.g.assign(6 * n_units * width, 0.0);
    ga.ge.assign(ga.g.size(), 0.0);
    ga.dg.assign(P * ga.g.size(), 0.0);
    ga.dge.assign(ga.dg.size(), 0.0);
  }
  const bool keep_greek = options->greek_order >= 0 || all_orders || n_mu > 0;
  constexpr int kS = 9;  // ONE, EXT, SCA, SCAG, ABS, BACK, R2, R3, DEPOL
  for (int64_t u = 0; u < n_units; ++u) {
    const int64_t i = u % n_wl;
    const adaptive::Part& part = parts[u / n_wl];
    const SphDerivReq& req = reqs[u / n_wl];
    const bool point = part.support == adaptive::POINT;
    const int nt = (int)req.grads.size();
    const double lambda = wavelengths[i];
    const int L = all_orders ? (int)(2 * n_direct[u]) : options->greek_order;
    const int64_t ld = !keep_greek ? -1 : n_mu == 0 ? std::min<int64_t>(L, 2 * n_direct[u])
                                                      : 2 * n_direct[u];
    const int64_t glen = ld + 1;  // 0 without a direct segment
    const int64_t len = kS + 6 * glen;
    // A node's rows (direct_node, direct_scalars): the values and their declared errors, and
    // per direction (Re m, Im m, aspect ratio, x) the derivatives and theirs, relative to the
    // derivatives themselves.
    std::vector<double> g(len), ge(len), dg(4 * len), dge(4 * len);
    auto rows_at = [&](double r) {
      const Node& nd = cache.at(key_u(u, r));
      const SpheroidResult& v = nd.v;
      const double area = pi * r * r;
      const double tau = std::max(rtol_t, v.err_est);
      const double c4 = 4.0 * tau, c16 = 16.0 * tau;
      const int64_t have = 2 * (int64_t)v.n + 1;
      const double x = 2.0 * pi * r / lambda, un = 4.0 / (x * x);
      double depol = 0.0;
      for (int64_t l = 0; l < have; ++l) {
        const double t = un * (v.greek[l] - 0.5 * (v.greek[have + l] - v.greek[2 * have + l]));
        depol += l % 2 ? -t : t;
      }
      const double sv[kS] = {1.0,         area * v.q_ext, area * v.q_sca, area * v.q_sca * v.g,
                             area * v.q_abs, area * v.q_back, r * r, r * r * r, area * depol};
      const double back = area * std::max(std::fabs(v.q_back), std::fabs(v.q_sca));
      const double se[kS] = {0.0,
                             c4 * std::fabs(sv[1]),
                             c4 * std::fabs(sv[2]),
                             c4 * std::fabs(sv[2]) * (1.0 + std::fabs(v.g)),
                             c16 * std::fabs(sv[1]),
                             c16 * back,
                             0.0,
                             0.0,
                             2.0 * c16 * back};
      for (int k = 0; k < kS; ++k) {
        g[k] = sv[k];
        ge[k] = se[k];
      }
      if (glen > 0) {
        double big = 0.0;
        for (int64_t l = 0; l < have; ++l) big = std::max(big, std::fabs(un * v.greek[l]));
        const double ce = c16 * area * big;
        for (int f = 0; f < 6; ++f)
          for (int64_t l = 0; l < glen; ++l) {
            g[kS + f * glen + l] = l < have ? area * un * v.greek[f * have + l] : 0.0;
            ge[kS + f * glen + l] = ce;
          }
      }
      for (int dir = 0; dir < 4; ++dir) {
        double* d = dg.data() + dir * len;
        double* de = dge.data() + dir * len;
        if (nd.d[dir].empty()) {
          std::fill(d, d + len, 0.0);
          std::fill(de, de + len, 0.0);
          continue;
        }
        // The unnormalized Greek arrays' derivatives (4/x^2 times the coefficients').
        const double* dq = nd.d[dir].data();
        const double* gr = dq + 5;
        double ddepol = 0.0;
        for (int64_t l = 0; l < have; ++l) {
          const double t = gr[l] - 0.5 * (gr[have + l] - gr[2 * have + l]);
          ddepol += l % 2 ? -t : t;
        }
        const double sd[kS] = {0.0,
                               area * dq[0],
                               area * dq[1],
                               area * (dq[1] * v.g + v.q_sca * dq[4]),
                               area * dq[2],
                               area * dq[3],
                               0.0,
                               0.0,
                               area * ddepol};
        const double cd[kS] = {0.0, c4, c4, c4, c16, c16, 0.0, 0.0, c16};
        for (int k = 0; k < kS; ++k) {
          d[k] = sd[k];
          de[k] = cd[k] * std::fabs(sd[k]);
        }
        for (int f = 0; f < 6; ++f)
          for (int64_t l = 0; l < glen; ++l) {
            const double y = l < have ? area * gr[f * have + l] : 0.0;
            d[kS + f * glen + l] = y;
            de[kS + f * glen + l] = c16 * std::fabs(y);
          }
      }
    };
    std::vector<double> av(len, 0.0), ae(len, 0.0), dv(P * len, 0.0), de(P * len, 0.0);
    bool conv = true;
    int64_t panels = 0;
    if (point) {
      // monodisperse_direct (engine.rs:1896-1961): the particle itself; its radius
      // d/dr = 2/r g + (2 pi / lambda) dg/dx, errors likewise, exact r^2 and r^3.
      const double r = part.lo;
      rows_at(r);
      av = g;
      ae = ge;
      if (nt > 0) {
        const int col = req.theta_cols[0];
        const double k = 2.0 * pi / lambda;
        const double* gx = dg.data() + 3 * len;
        const double* ex = dge.data() + 3 * len;
        for (int64_t j = 0; j < len; ++j) {
          dv[col * len + j] = 2.0 / r * g[j] + k * gx[j];
          de[col * len + j] = 2.0 / r * ge[j] + k * ex[j];
        }
        dv[col * len + 0] = 0.0;
        dv[col * len + 6] = 2.0 * r;
        dv[col * len + 7] = 3.0 * r * r;
        de[col * len + 0] = de[col * len + 6] = de[col * len + 7] = 0.0;
      }
      for (int dir = 0; dir < 3; ++dir) {
        const int col = req.dir_cols[dir];
        if (col < 0) continue;
        for (int64_t j = 0; j < len; ++j) {
          dv[col * len + j] = dg[dir * len + j];
          de[col * len + j] = dge[dir * len + j];
        }
      }
    } else {
      const adaptive::Job& jb = jobs[job_of[u]];
      conv = jb.converged[0];
      panels = (int64_t)jb.panels.size();
      // Blocks: the values (weights u r), each parameter's (weights du/dtheta r on the values),
      // each requested direction's (weights u r on its derivative rows).
      std::vector<int> dirs;
      for (int dir = 0; dir < 3; ++dir)
        if (req.dir_cols[dir] >= 0) dirs.push_back(dir);
      const int nb = 1 + nt + (int)dirs.size();
      std::vector<double> S(nb * len, 0.0), E(nb * len, 0.0);
      std::vector<double> ks(nb * len), gs(nb * len), ne(nb * len);
      double grad[3] = {0.0, 0.0, 0.0};
      for (const auto& ab : jb.panels) {
        adaptive::Node nd[15];
        adaptive::gk15(ab.first, ab.second, nd);
        std::fill(ks.begin(), ks.end(), 0.0);
        std::fill(gs.begin(), gs.end(), 0.0);
        std::fill(ne.begin(), ne.end(), 0.0);
        for (int k = 0; k < 15; ++k) {
          const double r = std::exp(nd[k].t);
          const double ur = (nt > 0 ? part.u(r, grad) : part.u(r)) * r;
          rows_at(r);
          for (int b = 0; b < nb; ++b) {
            double w;
            const double *row, *err;
            if (b == 0) {
              w = ur;
              row = g.data();
              err = ge.data();
            } else if (b <= nt) {
              w = grad[req.grads[b - 1]] * r;
              row = g.data();
              err = ge.data();
            } else {
              w = ur;
              row = dg.data() + dirs[b - 1 - nt] * len;
              err = dge.data() + dirs[b - 1 - nt] * len;
            }
            double* kb = ks.data() + b * len;
            double* gb = gs.data() + b * len;
            double* nb_ = ne.data() + b * len;
            const double wk = nd[k].wk * w, wg = nd[k].wg * w, wa = std::fabs(wk);
            for (int64_t j = 0; j < len; ++j) {
              kb[j] += wk * row[j];
              gb[j] += wg * row[j];
              nb_[j] += wa * err[j];
            }
          }
        }
        for (int64_t j = 0; j < nb * len; ++j) {
          S[j] += ks[j];
          E[j] += std::fabs(ks[j] - gs[j]) + ne[j];
        }
      }
      // averages (engine.rs:1782-1836).
      const adaptive::Moments& mom = part.mom;
      const double z = mom.z, ez = mom.ez;
      const double trunc = part.support == adaptive::UNBOUNDED ? 0.2 * o.rtol : 0.0;
      for (int64_t j = 0; j < len; ++j) {
        av[j] = S[j] / z;
        ae[j] = (E[j] + std::fabs(av[j]) * ez) / z + trunc * std::fabs(av[j]);
      }
      for (int b = 0; b < nt; ++b) {
        const int col = req.theta_cols[b];
        const double dz = mom.dz[b], edz = mom.dez[b];
        const double* sb = S.data() + (1 + b) * len;
        const double* eb = E.data() + (1 + b) * len;
        for (int64_t j = 0; j < len; ++j) {
          const double x = (sb[j] - av[j] * dz) / z;
          dv[col * len + j] = x;
          de[col * len + j] = (eb[j] + std::fabs(av[j]) * edz + std::fabs(x) * ez +
                               ae[j] * std::fabs(dz)) /
                                  z +
                              trunc * std::fabs(x);
        }
      }
      for (size_t c2 = 0; c2 < dirs.size(); ++c2) {
        const int col = req.dir_cols[dirs[c2]];
        const double* sb = S.data() + (1 + nt + c2) * len;
        const double* eb = E.data() + (1 + nt + c2) * len;
        for (int64_t j = 0; j < len; ++j) {
          const double x = sb[j] / z;
          dv[col * len + j] = x;
          de[col * len + j] = (eb[j] + std::fabs(x) * ez) / z + trunc * std::fabs(x);
        }
      }
      // <r^2>, <r^3> from the moments, with their parameter derivatives.
      for (int k = 0; k < 2; ++k) {
        av[6 + k] = mom.v[k];
        ae[6 + k] = mom.e[k];
        for (int64_t col = 0; col < P; ++col) {
          dv[col * len + 6 + k] = 0.0;
          de[col * len + 6 + k] = 0.0;
        }
        for (int b = 0; b < nt; ++b) {
          dv[req.theta_cols[b] * len + 6 + k] = mom.d[b][k];
          de[req.theta_cols[b] * len + 6 + k] = mom.de[b][k];
        }
      }
    }
    if (rows) {
      rows->av[u] = std::move(av);
      rows->ae[u] = std::move(ae);
      rows->dv[u] = std::move(dv);
      rows->de[u] = std::move(de);
      rows->ld[i] = ld;
      rows->converged[u] = conv ? 1 : 0;
      rows->panels[u] = panels;
      continue;
    }
    // assemble (engine.rs:2396-2497) with the derivatives (lin.rs).
    auto lin = [&](int64_t j) {
      LinD x;
      x.v = av[j];
      x.e = ae[j];
      x.d.resize(P);
      x.de.resize(P);
      for (int64_t col = 0; col < P; ++col) {
        x.d[col] = dv[col * len + j];
        x.de[col] = de[col * len + j];
      }
      return x;
    };
    // sum of c_k terms_k for exact constants (Lin::combine).
    auto combine = [&](std::initializer_list<std::pair<double, const LinD*>> terms) {
      LinD out = LinD::constant(0.0, (size_t)P);
      for (const auto& t : terms) {
        const double cw = t.first;
        const LinD& x = *t.second;
        out.v += cw * x.v;
        out.e += std::fabs(cw) * x.e;
        for (int64_t k = 0; k < P; ++k) {
          out.d[k] += cw * x.d[k];
          out.de[k] += std::fabs(cw) * x.de[k];
        }
      }
      return out;
    };
    const LinD ext = lin(1), sca = lin(2), scag = lin(3), abs_ = lin(4), back = lin(5),
               r2 = lin(6), r3 = lin(7), num = lin(8);
    for (const auto& w : {std::make_pair("<C_ext>", &ext), std::make_pair("<C_sca>", &sca),
                          std::make_pair("<C_back>", &back)})
      if (!(std::isfinite(w.second->v) && w.second->v != 0.0))
        throw Failure{SCATRS_INVALID_INPUT,
                      std::string("the ensemble's ") + w.first +
                          " is zero or not finite, so its ratios are undefined (does m = 1?)"};
    const LinD outs[11] = {ext,
                           sca,
                           abs_,
                           back,
                           sca.div(ext),
                           scag.div(sca),
                           ext.div(back).scale(4.0 * pi),
                           num.div(combine({{2.0, &back}, {-1.0, &num}})),
                           r3.div(r2),
                           r2.scale(pi),
                           r3.scale(4.0 * pi / 3.0)};
    for (int k = 0; k < 11; ++k) {
      res.values[k * n_units + u] = outs[k].v;
      if (res.errors) res.errors[k * n_units + u] = outs[k].e;
      for (int64_t col = 0; col < P; ++col) {
        if (dd.d_values) dd.d_values[(col * 11 + k) * n_units + u] = outs[k].d[col];
        if (dd.d_errors) dd.d_errors[(col * 11 + k) * n_units + u] = outs[k].de[col];
      }
    }
    const bool norm = options->normalized != 0;
    auto G = [&](int f, int64_t l) { return lin(kS + f * glen + l); };
    if (L >= 0 && (res.greek || all_orders)) {
      const LinD a0 = glen > 0 ? G(0, 0) : LinD::constant(0.0, (size_t)P);
      const int64_t w = all_orders ? width : L + 1;
      GreekAll& ga = t_greek_all;
      for (int f = 0; f < 6; ++f)
        for (int64_t l = 0; l <= L; ++l) {
          LinD x = l < glen ? G(f, l) : LinD::constant(0.0, (size_t)P);
          if (norm) x = (f == 0 && l == 0) ? LinD::constant(1.0, (size_t)P) : x.div(a0);
          const int64_t at = ((int64_t)f * n_units + u) * w + l;
          if (all_orders) {
            ga.g[at] = x.v;
            ga.ge[at] = x.e;
          } else {
            res.greek[at] = x.v;
            if (res.greek_err) res.greek_err[at] = x.e;
          }
          for (int64_t col = 0; col < P; ++col) {
            const int64_t atd = ((col * 6 + f) * n_units + u) * w + l;
            if (all_orders) {
              ga.dg[atd] = x.d[col];
              ga.dge[atd] = x.de[col];
            } else {
              if (dd.d_greek) dd.d_greek[atd] = x.d[col];
              if (dd.d_greek_err) dd.d_greek_err[atd] = x.de[col];
            }
          }
        }
    }
    if (n_mu > 0 && res.phase) {
      // greek_phase (engine.rs:2359-2390): combinations with exact weights, errors as bounds.
      std::vector<double> d00(glen), d22(glen), d2m2(glen), d02(glen);
      for (int64_t j = 0; j < n_mu; ++j) {
        wigner_d(0, 0, mu[j], d00.data(), glen);
        wigner_d(2, 2, mu[j], d22.data(), glen);
        wigner_d(2, -2, mu[j], d2m2.data(), glen);
        wigner_d(0, 2, mu[j], d02.data(), glen);
        LinD f[6];
        for (int k = 0; k < 6; ++k) f[k] = LinD::constant(0.0, (size_t)P);
        for (int64_t l = 0; l < glen; ++l) {
          const double plus = 0.5 * (d22[l] + d2m2[l]), minus = 0.5 * (d22[l] - d2m2[l]);
          const double wt[6][2] = {{d00[l], 0}, {d02[l], 0}, {plus, minus},
                                   {minus, plus}, {d02[l], 0}, {d00[l], 0}};
          const int src[6][2] = {{0, -1}, {4, -1}, {1, 2}, {1, 2}, {5, -1}, {3, -1}};
          for (int k = 0; k < 6; ++k)
            for (int t = 0; t < 2; ++t) {
              if (src[k][t] < 0) continue;
              const LinD x = G(src[k][t], l);
              f[k] = combine({{1.0, &f[k]}, {wt[k][t], &x}});
            }
        }
        for (int k = 0; k < 6; ++k) {
          const LinD x = norm ? f[k].div(sca) : f[k];
          const int64_t at = ((int64_t)k * n_units + u) * n_mu + j;
          res.phase[at] = x.v;
          if (res.phase_err) res.phase_err[at] = x.e;
          for (int64_t col = 0; col < P; ++col) {
            const int64_t atd = ((col * 6 + k) * n_units + u) * n_mu + j;
            if (dd.d_phase) dd.d_phase[atd] = x.d[col];
            if (dd.d_phase_err) dd.d_phase_err[atd] = x.de[col];
          }
        }
      }
    }
    if (res.converged) res.converged[u] = conv ? 1 : 0;
    if (res.panels) res.panels[u] = panels;
  }
}

FixedCall g_last_call;  // for scatrs_check_errors

template <class F>
int guarded(char* err, size_t err_len, F f) {
  g_last_status = SCATRS_OK;
  g_last_achieved = g_last_requested = NAN;
  try {
    f();
    return SCATRS_OK;
  } catch (const Failure& e) {
    set_err(err, err_len, e.msg);
    g_last_status = e.status;
    g_last_achieved = e.achieved;
    g_last_requested = e.requested;
    return e.status;
  } catch (const std::bad_alloc&) {
    set_err(err, err_len, "host allocation failed");
    g_last_status = SCATRS_INVALID_INPUT;
    return SCATRS_INVALID_INPUT;
  }
}

// Whether a mixture has components other than homogeneous spheres.
bool heterogeneous(const scatrs_component* components, int64_t n_comp) {
  for (int64_t c = 0; c < n_comp && components; ++c)
    if (components[c].n_layers > 1 || components[c].aspect_ratio != 0.0) return true;
  return false;
}

// The parts of a mixture (ensemble/mod.rs:609-625, 688-780 validation; engine.rs:141-223): each
// mode of each component with its number fraction w / w_total * v / v_total (engine.rs:2131).
std::vector<AdPart> mixture_parts(const scatrs_component* components, int64_t n_comp) {
  if (n_comp < 1) throw Failure{SCATRS_INVALID_INPUT, "a mixture needs a component"};
  double total = 0.0;
  for (int64_t c = 0; c < n_comp; ++c) {
    const scatrs_component& k = components[c];
    const std::string who = "component " + std::to_string(c);
    if (!(std::isfinite(k.weight) && k.weight >= 0.0))
      throw Failure{SCATRS_INVALID_INPUT, "the weight of " + who + " must be finite and >= 0"};
    if (k.n_modes < 1 || !k.modes || !k.m)
      throw Failure{SCATRS_INVALID_INPUT, who + ": needs a distribution and m"};
    if (k.n_modes > 1) {
      if (!k.mode_weights) throw Failure{SCATRS_INVALID_INPUT, who + ": needs mode weights"};
      double sum = 0.0;
      for (int j = 0; j < k.n_modes; ++j) sum += k.mode_weights[j];
      if (!std::isfinite(sum))
        throw Failure{SCATRS_INVALID_INPUT, who + ": the mode weights must have a finite sum"};
    }
    total += k.weight;
  }
  if (!(std::isfinite(total) && total > 0.0))
    throw Failure{SCATRS_INVALID_INPUT,
                  "the mixture weights must have a finite, positive sum"};
  std::vector<AdPart> parts;
  for (int64_t c = 0; c < n_comp; ++c) {
    const scatrs_component& k = components[c];
    double v_total = 0.0;
    for (int j = 0; j < k.n_modes; ++j) v_total += k.n_modes > 1 ? k.mode_weights[j] : 1.0;
    for (int j = 0; j < k.n_modes; ++j) {
      const double v = k.n_modes > 1 ? k.mode_weights[j] : 1.0;
      const scatrs_distribution& d = k.modes[j];
      parts.push_back(AdPart{d.kind, {d.param[0], d.param[1], d.param[2]}, k.m,
                             k.weight / total * v / v_total, 0,
                             "component " + std::to_string(c) + ": ", d.table, d.table_len});
      AdPart& a = parts.back();
      a.component = (int)c;
      a.mode = k.mode_weights ? j : -1;
      a.w = k.weight;
      a.v = v;
      a.v_total = v_total;
    }
  }
  return parts;
}

// A mixture whose components are not all homogeneous spheres (engine.rs:1964-2250 over
// components of different particles): the spheres in one adaptive call, the layered spheres in
// one per number of layers, the spheroids in one spheroid call (one direct order per
// wavelength over all of them), each returning its parts' averages; then per wavelength the
// number-fraction mixing on one layout (scalars with the depolarization numerator, the spheres'
// cosine tables and projected Greek coefficients, the spheroids' direct segment) and the
// assembly: ratios and bounds (lin.rs), the depolarization ratio, the Greek coefficients of the
// spheres plus the spheroids', the phase matrix of the spheres' tables plus the spheroids'
// averaged expansion (greek_phase, engine.rs:2363-2390), normalized by alpha1_0 and <C_sca>.
void mixture_hetero(const scatrs_component* components, int64_t n_comp,
                    const double* wavelengths, int64_t n_wl, const double* mu, int64_t n_mu,
                    const scatrs_adaptive_options* options, const AdOutputs& res) {
  if (!options) throw Failure{SCATRS_INVALID_INPUT, "options must not be NULL"};
  const bool all_orders = options->greek_order == SCATRS_GREEK_ALL;
  const std::vector<AdPart> parts = mixture_parts(components, n_comp);
  const int64_t np = (int64_t)parts.size();
  for (int64_t c = 0; c < n_comp; ++c) {
    const scatrs_component& k = components[c];
    const std::string who = "component " + std::to_string(c) + ": ";
    if (!(std::isfinite(k.aspect_ratio) && k.aspect_ratio >= 0.0))
      throw Failure{SCATRS_INVALID_INPUT, who + "the aspect ratio must be finite and > 0"};
    if (k.aspect_ratio > 0.0 && k.n_layers > 1)
      throw Failure{SCATRS_INVALID_INPUT, who + "a particle is layered or a spheroid, not both"};
    if (k.n_layers > kMaxLayersAbi) throw Failure{SCATRS_INVALID_INPUT, who + "at most 16 layers"};
    if (k.n_layers > 1 && !k.fractions)
      throw Failure{SCATRS_INVALID_INPUT, who + "a layered sphere needs its fractions"};
  }
  // Spheroids: one particle per component, its modes its distributions. They run first: with
  // greek='all' their N at each wavelength (ld = 2 N) enters the mixture's order.
  std::vector<SphParticle> sph;
  std::vector<int64_t> sph_parts;  // the parts in the order of the spheroid call's
  for (int64_t c = 0; c < n_comp; ++c) {
    const scatrs_component& k = components[c];
    if (k.aspect_ratio == 0.0) continue;
    sph.push_back(SphParticle{k.modes, k.n_modes, k.aspect_ratio, k.m});
    for (int64_t p = 0; p < np; ++p)
      if (parts[p].component == c) sph_parts.push_back(p);
  }
  std::vector<int64_t> ld(n_wl, -1);
  SphRows srows;
  if (!sph.empty()) {
    spheroid_call(sph, false, wavelengths, n_wl, mu, n_mu, options, AdOutputs{}, &srows);
    ld = srows.ld;
  }
  // Spheres, and layered spheres by their number of layers.
  std::map<int, std::vector<int64_t>> by_layers;
  for (int64_t p = 0; p < np; ++p) {
    const scatrs_component& k = components[parts[p].component];
    if (k.aspect_ratio == 0.0) by_layers[k.n_layers > 1 ? k.n_layers : 1].push_back(p);
  }
  // A class's parts (output unit 0) with their layers' fractions and indices.
  struct Cls {
    std::vector<AdPart> sub;
    std::vector<double> fr, ml;
    int nl;
  };
  auto make_cls = [&](int nl, const std::vector<int64_t>& ps) {
    Cls k{{}, {}, {}, nl};
    for (int64_t p : ps) {
      AdPart a = parts[p];
      a.out = 0;
      k.sub.push_back(a);
      if (nl > 1) {
        const scatrs_component& c = components[parts[p].component];
        k.fr.insert(k.fr.end(), c.fractions, c.fractions + nl - 1);
        k.ml.insert(k.ml.end(), c.m, c.m + 2 * (size_t)nl * n_wl);
      }
    }
    return k;
  };
  // The Greek order at each wavelength: the requested one, or with greek='all' 2 N_max over
  // every part of the mixture (GreekOrder::All, engine.rs:2016-2036: spheres, layered spheres
  // and spheroids alike), the sphere classes' N_max from their pass 1.
  std::vector<int64_t> order(n_wl, options->greek_order);
  if (all_orders) {
    std::fill(order.begin(), order.end(), 0);
    for (int64_t i = 0; i < n_wl; ++i)
      if (ld[i] >= 0) order[i] = ld[i];
    scatrs_adaptive_options o1 = *options;
    o1.greek_order = -1;
    for (const auto& kv : by_layers) {
      Cls k = make_cls(kv.first, kv.second);
      scatrs_layers lay{k.nl, 0, k.fr.data(), k.ml.data()};
      std::vector<int64_t> n_max;
      adaptive_call_order(k.sub, 1, false, wavelengths, n_wl, mu, n_mu, &o1, AdOutputs{},
                          k.nl > 1 ? &lay : nullptr, nullptr, &n_max);
      for (size_t q = 0; q < k.sub.size() && !n_max.empty(); ++q)
        for (int64_t i = 0; i < n_wl; ++i)
          order[i] = std::max(order[i], 2 * n_max[q * n_wl + i]);
    }
  }
  // The Greek coefficients' width in the rows: the order plus one (the longest with 'all').
  int64_t gw = 0;
  for (int64_t i = 0; i < n_wl; ++i) gw = std::max(gw, order[i] + 1);
  // Each part's averages at each wavelength: 9 scalars (the last the depolarization
  // numerator), 4 n_mu cosine values, 6 gw Greek coefficients (zero above the wavelength's
  // order), each with its error, and the spheroids' direct segment.
  struct Avg {
    std::vector<double> v, e, dv, de;  // v, e: 9 + 4 n_mu + 6 gw; dv, de: 6 (ld + 1)
    bool converged = true;
    int64_t panels = 0;
  };
  const int64_t row = 9 + 4 * n_mu + 6 * gw;
  std::vector<Avg> avg((size_t)np * n_wl);
  for (const auto& kv : by_layers) {
    const std::vector<int64_t>& ps = kv.second;
    const Cls k = make_cls(kv.first, ps);
    // The wavelengths of one order run together (all of them without 'all').
    std::map<int64_t, std::vector<int64_t>> by_order;
    for (int64_t i = 0; i < n_wl; ++i) by_order[order[i]].push_back(i);
    for (const auto& ko : by_order) {
      const int64_t L = ko.first, glen = L >= 0 ? L + 1 : 0;
      const std::vector<int64_t>& ws = ko.second;
      const int64_t nw = (int64_t)ws.size();
      std::vector<double> wl_s(nw);
      for (int64_t j = 0; j < nw; ++j) wl_s[j] = wavelengths[ws[j]];
      std::vector<AdPart> sub = k.sub;
      std::vector<std::vector<double>> m_s(sub.size());
      std::vector<double> ml_s(k.ml.size() / std::max<int64_t>(n_wl, 1) * nw);
      for (size_t q = 0; q < sub.size(); ++q) {
        if (sub[q].m) {
          m_s[q].resize(2 * nw);
          for (int64_t j = 0; j < nw; ++j) {
            m_s[q][2 * j] = sub[q].m[2 * ws[j]];
            m_s[q][2 * j + 1] = sub[q].m[2 * ws[j] + 1];
          }
          sub[q].m = m_s[q].data();
        }
        for (int l = 0; k.nl > 1 && l < k.nl; ++l)
          for (int64_t j = 0; j < nw; ++j)
            for (int c = 0; c < 2; ++c)
              ml_s[2 * ((q * k.nl + l) * nw + j) + c] =
                  k.ml[2 * ((q * k.nl + l) * n_wl + ws[j]) + c];
      }
      scatrs_layers lay{k.nl, 0, k.fr.data(), ml_s.data()};
      scatrs_adaptive_options oL = *options;
      oL.greek_order = (int)L;
      PartRows rows;
      adaptive_call_order(sub, 1, false, wl_s.data(), nw, mu, n_mu, &oL, AdOutputs{},
                          k.nl > 1 ? &lay : nullptr, nullptr, nullptr, &rows);
      const int64_t n2 = 4 * n_mu, base_t = 16, base_g = 16 + 8 * n_mu;
      for (size_t q = 0; q < ps.size(); ++q)
        for (int64_t j = 0; j < nw; ++j) {
          const int64_t i = ws[j];
          const double* r = rows.rows.data() + ((int64_t)q * nw + j) * rows.stride;
          Avg& a = avg[ps[q] * n_wl + i];
          a.v.assign(row, 0.0);
          a.e.assign(row, 0.0);
          for (int c = 0; c < 8; ++c) {
            a.v[c] = r[c];
            a.e[c] = r[8 + c];
          }
          for (int64_t t = 0; t < n2; ++t) {
            a.v[9 + t] = r[base_t + t];
            a.e[9 + t] = r[base_t + n2 + t];
          }
          for (int f = 0; f < 6; ++f)
            for (int64_t l = 0; l < glen; ++l) {
              a.v[9 + n2 + f * gw + l] = r[base_g + f * glen + l];
              a.e[9 + n2 + f * gw + l] = r[base_g + 6 * glen + f * glen + l];
            }
          a.converged = rows.converged[q * nw + j] != 0;
          a.panels = rows.panels[q * nw + j];
        }
    }
  }
  for (size_t q = 0; q < sph_parts.size(); ++q)
    for (int64_t i = 0; i < n_wl; ++i) {
      const std::vector<double>& sv = srows.av[q * n_wl + i];
      const std::vector<double>& se = srows.ae[q * n_wl + i];
      Avg& a = avg[sph_parts[q] * n_wl + i];
      a.v.assign(row, 0.0);
      a.e.assign(row, 0.0);
      for (int k = 0; k < 9; ++k) {
        a.v[k] = sv[k];
        a.e[k] = se[k];
      }
      a.dv.assign(sv.begin() + 9, sv.end());
      a.de.assign(se.begin() + 9, se.end());
      a.converged = srows.converged[q * n_wl + i] != 0;
      a.panels = srows.panels[q * n_wl + i];
    }
  if (all_orders) {
    GreekAll& ga = t_greek_all;
    ga.width = gw;
    ga.n = n_wl;
    ga.p = 0;
    ga.g.assign(6 * n_wl * gw, 0.0);
    ga.ge.assign(ga.g.size(), 0.0);
    ga.dg.clear();
    ga.dge.clear();
  }
  // Mixing and assembly per wavelength.
  const bool norm = options->normalized != 0;
  for (int64_t i = 0; i < n_wl; ++i) {
    const int64_t ldi = ld[i], dlen = ldi >= 0 ? 6 * (ldi + 1) : 0;
    std::vector<double> v(row, 0.0), e(row, 0.0), dv(dlen, 0.0), de(dlen, 0.0);
    bool has_direct = false, conv = true;
    int64_t panels = 0;
    for (int64_t p = 0; p < np; ++p) {
      const Avg& a = avg[p * n_wl + i];
      const double f = parts[p].f;
      for (int64_t k = 0; k < row; ++k) {
        v[k] += f * a.v[k];
        e[k] += f * a.e[k];
      }
      if (components[parts[p].component].aspect_ratio > 0.0) {
        has_direct = true;
        for (int64_t k = 0; k < dlen; ++k) {
          dv[k] += f * a.dv[k];
          de[k] += f * a.de[k];
        }
      }
      conv = conv && a.converged;
      panels += a.panels;
    }
    auto lin = [&](int64_t k) { return LinE{v[k], e[k]}; };
    const LinE ext = lin(1), sca = lin(2), scag = lin(3), abs_ = lin(4), back = lin(5),
               r2 = lin(6), r3 = lin(7), num = lin(8);
    for (const auto& w : {std::make_pair("<C_ext>", ext), std::make_pair("<C_sca>", sca),
                          std::make_pair("<C_back>", back)})
      if (!(std::isfinite(w.second.v) && w.second.v != 0.0))
        throw Failure{SCATRS_INVALID_INPUT,
                      std::string("the ensemble's ") + w.first +
                          " is 0 or not finite, so its ratios (albedo, asymmetry parameter, "
                          "lidar ratio) are undefined (does m = 1?)"};
    const LinE depol = has_direct ? lin_div(num, LinE{2.0 * back.v - num.v, 2.0 * back.e + num.e})
                                  : LinE{0.0, 0.0};
    const LinE outs[11] = {ext,
                           sca,
                           abs_,
                           back,
                           lin_div(sca, ext),
                           lin_div(scag, sca),
                           lin_scale(lin_div(ext, back), 4.0 * kPi),
                           depol,
                           lin_div(r3, r2),
                           lin_scale(r2, kPi),
                           lin_scale(r3, 4.0 * kPi / 3.0)};
    for (int k = 0; k < 11; ++k) {
      res.values[k * n_wl + i] = outs[k].v;
      if (res.errors) res.errors[k * n_wl + i] = outs[k].e;
    }
    auto D = [&](int f, int64_t l) {
      return LinE{dv[f * (ldi + 1) + l], de[f * (ldi + 1) + l]};
    };
    const int64_t g0 = 9 + 4 * n_mu, glen = order[i] + 1;
    double* g_out = all_orders ? t_greek_all.g.data() : res.greek;
    double* ge_out = all_orders ? t_greek_all.ge.data() : res.greek_err;
    if (glen > 0 && g_out) {
      // The spheres' coefficients plus the spheroids' (engine.rs:2196-2216).
      auto G = [&](int f, int64_t l) {
        LinE x = lin(g0 + f * gw + l);
        if (has_direct && l <= ldi) {
          const LinE y = D(f, l);
          x.v += y.v;
          x.e += y.e;
        }
        return x;
      };
      const LinE a0 = G(0, 0);
      for (int f = 0; f < 6; ++f)
        for (int64_t l = 0; l < glen; ++l) {
          LinE x = G(f, l);
          if (norm) x = (f == 0 && l == 0) ? LinE{1.0, 0.0} : lin_div(x, a0);
          g_out[(f * n_wl + i) * gw + l] = x.v;
          if (ge_out) ge_out[(f * n_wl + i) * gw + l] = x.e;
        }
    }
    if (n_mu > 0 && res.phase) {
      const int src[6] = {0, 1, 0, 2, 3, 2};
      std::vector<double> d00, d22, d2m2, d02;
      if (has_direct && ldi >= 0) {
        d00.resize(ldi + 1);
        d22.resize(ldi + 1);
        d2m2.resize(ldi + 1);
        d02.resize(ldi + 1);
      }
      for (int64_t j = 0; j < n_mu; ++j) {
        LinE fd[6];
        if (has_direct && ldi >= 0) {
          wigner_d(0, 0, mu[j], d00.data(), ldi + 1);
          wigner_d(2, 2, mu[j], d22.data(), ldi + 1);
          wigner_d(2, -2, mu[j], d2m2.data(), ldi + 1);
          wigner_d(0, 2, mu[j], d02.data(), ldi + 1);
          auto acc = [](LinE& t, double w, const LinE& x) {
            t.v += w * x.v;
            t.e += std::fabs(w) * x.e;
          };
          for (int64_t l = 0; l <= ldi; ++l) {
            const double pl = 0.5 * (d22[l] + d2m2[l]), mn = 0.5 * (d22[l] - d2m2[l]);
            acc(fd[0], d00[l], D(0, l));
            acc(fd[1], d02[l], D(4, l));
            acc(fd[2], pl, D(1, l));
            acc(fd[2], mn, D(2, l));
            acc(fd[3], mn, D(1, l));
            acc(fd[3], pl, D(2, l));
            acc(fd[4], d02[l], D(5, l));
            acc(fd[5], d00[l], D(3, l));
          }
        }
        for (int el = 0; el < 6; ++el) {
          LinE x = lin(9 + src[el] * n_mu + j);
          x.v += fd[el].v;
          x.e += fd[el].e;
          if (norm) x = lin_div(x, sca);
          res.phase[(el * n_wl + i) * n_mu + j] = x.v;
          if (res.phase_err) res.phase_err[(el * n_wl + i) * n_mu + j] = x.e;
        }
      }
    }
    if (res.converged) res.converged[i] = conv ? 1 : 0;
    if (res.panels) res.panels[i] = panels;
  }
}

// mixture_hetero with the derivatives along `dd`'s parameters (engine.rs:1964-2250 with
// EnsembleOptions::derivatives): each part's averages with its derivative blocks from its own
// engine (spheres and layered spheres: adaptive_call_order's per-block rows, one call per number
// of layers; spheroids: spheroid_call_d's rows on the mixture's direct order), placed by result
// column; then per wavelength the number-fraction mixing with the weight derivatives
// (engine.rs:2121-2176) and the assembly of mixture_hetero with Lin (lin.rs): ratios, the
// depolarization ratio, the spheres' Greek coefficients plus the spheroids' direct segment, and
// the phase matrix of the spheres' tables plus the spheroids' expansion.
void mixture_hetero_d(const scatrs_component* components, int64_t n_comp,
                      const double* wavelengths, int64_t n_wl, const double* mu, int64_t n_mu,
                      const scatrs_adaptive_options* options, const AdOutputs& res,
                      const AdDerivs& dd) {
  if (!options) throw Failure{SCATRS_INVALID_INPUT, "options must not be NULL"};
  const bool all_orders = options->greek_order == SCATRS_GREEK_ALL;
  std::vector<AdPart> parts = mixture_parts(components, n_comp);
  const int64_t np = (int64_t)parts.size(), P = dd.n;
  for (int64_t c = 0; c < n_comp; ++c) {
    const scatrs_component& k = components[c];
    const std::string who = "component " + std::to_string(c) + ": ";
    if (!(std::isfinite(k.aspect_ratio) && k.aspect_ratio >= 0.0))
      throw Failure{SCATRS_INVALID_INPUT, who + "the aspect ratio must be finite and > 0"};
    if (k.aspect_ratio > 0.0 && k.n_layers > 1)
      throw Failure{SCATRS_INVALID_INPUT, who + "a particle is layered or a spheroid, not both"};
    if (k.n_layers > kMaxLayersAbi) throw Failure{SCATRS_INVALID_INPUT, who + "at most 16 layers"};
    if (k.n_layers > 1 && !k.fractions)
      throw Failure{SCATRS_INVALID_INPUT, who + "a layered sphere needs its fractions"};
  }
  // Each part's parameters and the columns of its particle's directions.
  for (AdPart& a : parts) {
    const scatrs_component& k = components[a.component];
    const int L = k.n_layers > 1 ? k.n_layers : 1;
    a.dir_cols.assign(k.aspect_ratio > 0.0 ? 3 : L > 1 ? 3 * L - 1 : 2, -1);
    for (int64_t c = 0; c < P; ++c) {
      const scatrs_param& q = dd.params[c];
      if (q.component != a.component) continue;
      switch (q.kind) {
        case SCATRS_PARAM_DISTRIBUTION:
          if (q.mode == a.mode) {
            a.grads.push_back(q.index);
            a.theta_cols.push_back((int)c);
          }
          break;
        case SCATRS_PARAM_REFR_REAL: a.dir_cols[0] = (int)c; break;
        case SCATRS_PARAM_REFR_IMAG: a.dir_cols[1] = (int)c; break;
        case SCATRS_PARAM_ASPECT_RATIO: a.dir_cols[2] = (int)c; break;
        case SCATRS_PARAM_LAYER_REFR_REAL: a.dir_cols[2 * q.index] = (int)c; break;
        case SCATRS_PARAM_LAYER_REFR_IMAG: a.dir_cols[2 * q.index + 1] = (int)c; break;
        case SCATRS_PARAM_RADIUS_FRACTION: a.dir_cols[2 * L + q.index] = (int)c; break;
        default: break;  // a weight: the mixing's
      }
    }
  }
  // Each (part, wavelength)'s averages on the common layout (9 scalars, the last the
  // depolarization numerator; 4 n_mu cosine values; 6 gw Greek coefficients) with their errors,
  // and per column their derivatives (P x row); a spheroid's direct segment likewise. The
  // layout's width gw follows the spheroids' and the sphere classes' orders.
  struct PD {
    std::vector<double> v, e, d, de, sv, se, sd, sde;
    bool converged = true;
    int64_t panels = 0;
  };
  std::vector<PD> avg((size_t)np * n_wl);
  int64_t gw = 0, row = 0;
  std::vector<int64_t> order(n_wl, options->greek_order);
  // Spheroids first: their direct order.
  std::vector<SphParticle> sph;
  std::vector<SphDerivReq> sreq;
  std::vector<int64_t> sph_parts;
  for (int64_t c = 0; c < n_comp; ++c) {
    const scatrs_component& k = components[c];
    if (k.aspect_ratio == 0.0) continue;
    sph.push_back(SphParticle{k.modes, k.n_modes, k.aspect_ratio, k.m});
    for (int64_t p = 0; p < np; ++p)
      if (parts[p].component == c) {
        sph_parts.push_back(p);
        SphDerivReq r;
        r.grads = parts[p].grads;
        r.theta_cols = parts[p].theta_cols;
        for (int j = 0; j < 3; ++j) r.dir_cols[j] = parts[p].dir_cols[j];
        sreq.push_back(r);
      }
  }
  std::vector<int64_t> ld(n_wl, -1);
  SphRowsD srows;
  if (!sph.empty()) {
    spheroid_call_d(sph, sreq, wavelengths, n_wl, mu, n_mu, options, AdOutputs{}, dd, &srows);
    ld = srows.ld;
  }
  // Spheres, and layered spheres by their number of layers.
  std::map<int, std::vector<int64_t>> by_layers;
  for (int64_t p = 0; p < np; ++p) {
    const scatrs_component& k = components[parts[p].component];
    if (k.aspect_ratio == 0.0) by_layers[k.n_layers > 1 ? k.n_layers : 1].push_back(p);
  }
  // A class's parts (output unit 0) with their layers' fractions and indices.
  struct Cls {
    std::vector<AdPart> sub;
    std::vector<double> fr, ml;
    int nl = 1, n_theta = 0;
  };
  auto make_cls = [&](int nl, const std::vector<int64_t>& ps) {
    Cls k;
    k.nl = nl;
    for (int64_t p : ps) {
      AdPart a = parts[p];
      a.out = 0;
      k.n_theta = std::max(k.n_theta, (int)a.grads.size());
      k.sub.push_back(a);
      if (nl > 1) {
        const scatrs_component& c = components[parts[p].component];
        k.fr.insert(k.fr.end(), c.fractions, c.fractions + nl - 1);
        k.ml.insert(k.ml.end(), c.m, c.m + 2 * (size_t)nl * n_wl);
      }
    }
    return k;
  };
  // greek='all': every wavelength's order 2 N_max over every part (engine.rs:2016-2036), the
  // sphere classes' N_max from their pass 1.
  if (all_orders) {
    std::fill(order.begin(), order.end(), 0);
    for (int64_t i = 0; i < n_wl; ++i)
      if (ld[i] >= 0) order[i] = ld[i];
    scatrs_adaptive_options o1 = *options;
    o1.greek_order = -1;
    for (const auto& kv : by_layers) {
      Cls k = make_cls(kv.first, kv.second);
      scatrs_layers lay{k.nl, 0, k.fr.data(), k.ml.data()};
      std::vector<int64_t> n_max;
      adaptive_call_order(k.sub, 1, false, wavelengths, n_wl, mu, n_mu, &o1, AdOutputs{},
                          k.nl > 1 ? &lay : nullptr, nullptr, &n_max);
      for (size_t q = 0; q < k.sub.size() && !n_max.empty(); ++q)
        for (int64_t i = 0; i < n_wl; ++i)
          order[i] = std::max(order[i], 2 * n_max[q * n_wl + i]);
    }
  }
  for (int64_t i = 0; i < n_wl; ++i) gw = std::max(gw, order[i] + 1);
  row = 9 + 4 * n_mu + 6 * gw;
  for (PD& a : avg) {
    a.v.assign(row, 0.0);
    a.e.assign(row, 0.0);
    a.d.assign((size_t)P * row, 0.0);
    a.de.assign((size_t)P * row, 0.0);
  }
  if (!sph.empty()) {
    for (size_t q = 0; q < sph_parts.size(); ++q)
      for (int64_t i = 0; i < n_wl; ++i) {
        const int64_t u = (int64_t)q * n_wl + i;
        const std::vector<double>& sv = srows.av[u];
        const int64_t len = (int64_t)sv.size(), dlen = len - 9;
        PD& a = avg[sph_parts[q] * n_wl + i];
        for (int k = 0; k < 9; ++k) {
          a.v[k] = sv[k];
          a.e[k] = srows.ae[u][k];
        }
        a.sv.assign(sv.begin() + 9, sv.end());
        a.se.assign(srows.ae[u].begin() + 9, srows.ae[u].end());
        a.sd.assign((size_t)P * dlen, 0.0);
        a.sde.assign((size_t)P * dlen, 0.0);
        for (int64_t col = 0; col < P; ++col) {
          for (int k = 0; k < 9; ++k) {
            a.d[col * row + k] = srows.dv[u][col * len + k];
            a.de[col * row + k] = srows.de[u][col * len + k];
          }
          for (int64_t t = 0; t < dlen; ++t) {
            a.sd[col * dlen + t] = srows.dv[u][col * len + 9 + t];
            a.sde[col * dlen + t] = srows.de[u][col * len + 9 + t];
          }
        }
        a.converged = srows.converged[u] != 0;
        a.panels = srows.panels[u];
      }
  }
  // The sphere classes: one adaptive call per class and group of wavelengths of one order (all
  // of them without 'all'), its per-block rows placed by column.
  for (const auto& kv : by_layers) {
    const Cls k = make_cls(kv.first, kv.second);
    const std::vector<int64_t>& ps = kv.second;
    std::map<int64_t, std::vector<int64_t>> by_order;
    for (int64_t i = 0; i < n_wl; ++i) by_order[order[i]].push_back(i);
    for (const auto& ko : by_order) {
      const int64_t glen = ko.first >= 0 ? ko.first + 1 : 0;
      const std::vector<int64_t>& ws = ko.second;
      const int64_t nw = (int64_t)ws.size();
      std::vector<double> wl_s(nw);
      for (int64_t j = 0; j < nw; ++j) wl_s[j] = wavelengths[ws[j]];
      std::vector<AdPart> sub = k.sub;
      std::vector<std::vector<double>> m_s(sub.size());
      std::vector<double> ml_s(k.ml.size() / std::max<int64_t>(n_wl, 1) * nw);
      for (size_t q = 0; q < sub.size(); ++q) {
        if (sub[q].m) {
          m_s[q].resize(2 * nw);
          for (int64_t j = 0; j < nw; ++j) {
            m_s[q][2 * j] = sub[q].m[2 * ws[j]];
            m_s[q][2 * j + 1] = sub[q].m[2 * ws[j] + 1];
          }
          sub[q].m = m_s[q].data();
        }
        for (int l = 0; k.nl > 1 && l < k.nl; ++l)
          for (int64_t j = 0; j < nw; ++j)
            for (int c = 0; c < 2; ++c)
              ml_s[2 * ((q * k.nl + l) * nw + j) + c] =
                  k.ml[2 * ((q * k.nl + l) * n_wl + ws[j]) + c];
      }
      scatrs_layers lay{k.nl, 0, k.fr.data(), ml_s.data()};
      scatrs_adaptive_options oL = *options;
      oL.greek_order = (int32_t)ko.first;
      PartRows rows;
      adaptive_call_order(sub, 1, false, wl_s.data(), nw, mu, n_mu, &oL, AdOutputs{},
                          k.nl > 1 ? &lay : nullptr, &dd, nullptr, &rows);
      const int n_theta = k.n_theta;
      const int64_t hrow = 8 + 4 * n_mu + 6 * glen;
      const int B = 1 + n_theta + (int)sub[0].dir_cols.size();
      if (rows.stride != 2 * (int64_t)B * hrow)
        throw Failure{SCATRS_CUDA, "internal: the rows of a mixture's sphere class"};
      // One row of the per-block layout onto the common one (depolarization numerator 0).
      auto put = [&](const double* src, double* dst) {
        for (int c = 0; c < 8; ++c) dst[c] = src[c];
        dst[8] = 0.0;
        for (int64_t t = 0; t < 4 * n_mu; ++t) dst[9 + t] = src[8 + t];
        for (int f = 0; f < 6; ++f)
          for (int64_t l = 0; l < glen; ++l)
            dst[9 + 4 * n_mu + f * gw + l] = src[8 + 4 * n_mu + f * glen + l];
      };
      for (size_t q = 0; q < ps.size(); ++q) {
        const AdPart& a = sub[q];
        for (int64_t j = 0; j < nw; ++j) {
          const int64_t i = ws[j];
          const double* r = rows.rows.data() + ((int64_t)q * nw + j) * rows.stride;
          PD& x = avg[ps[q] * n_wl + i];
          put(r, x.v.data());
          put(r + hrow, x.e.data());
          for (int b = 1; b < B; ++b) {
            int col = -1;
            if (b <= n_theta) {
              if (b - 1 < (int)a.theta_cols.size()) col = a.theta_cols[b - 1];
            } else {
              col = a.dir_cols[b - n_theta - 1];
            }
            if (col < 0) continue;
            put(r + 2 * b * hrow, x.d.data() + col * row);
            put(r + (2 * b + 1) * hrow, x.de.data() + col * row);
          }
          x.converged = rows.converged[q * nw + j] != 0;
          x.panels = rows.panels[q * nw + j];
        }
      }
    }
  }
  if (all_orders) {
    GreekAll& ga = t_greek_all;
    ga.width = gw;
    ga.n = n_wl;
    ga.p = P;
    ga.g.assign(6 * n_wl * gw, 0.0);
    ga.ge.assign(ga.g.size(), 0.0);
    ga.dg.assign(P * ga.g.size(), 0.0);
    ga.dge.assign(ga.dg.size(), 0.0);
  }
  // Mixing (with the weight derivatives) and assembly per wavelength.
  double w_total = 0.0;
  {
    std::vector<int> comps;
    for (const AdPart& a : parts)
      if (std::find(comps.begin(), comps.end(), a.component) == comps.end()) {
        comps.push_back(a.component);
        w_total += a.w;
      }
  }
  const bool norm = options->normalized != 0;
  for (int64_t i = 0; i < n_wl; ++i) {
    const int64_t ldi = ld[i], dlen = ldi >= 0 ? 6 * (ldi + 1) : 0;
    std::vector<double> v(row, 0.0), e(row, 0.0), d((size_t)P * row, 0.0),
        de((size_t)P * row, 0.0), sv(dlen, 0.0), se(dlen, 0.0), sd((size_t)P * dlen, 0.0),
        sde((size_t)P * dlen, 0.0);
    bool has_direct = false, conv = true;
    int64_t panels = 0;
    for (int64_t p = 0; p < np; ++p) {
      const PD& a = avg[p * n_wl + i];
      const double f = parts[p].f;
      const bool direct = components[parts[p].component].aspect_ratio > 0.0;
      for (int64_t k = 0; k < row; ++k) {
        v[k] += f * a.v[k];
        e[k] += f * a.e[k];
      }
      for (int64_t k = 0; k < P * row; ++k) {
        d[k] += f * a.d[k];
        de[k] += f * a.de[k];
      }
      if (direct) {
        has_direct = true;
        for (int64_t k = 0; k < dlen; ++k) {
          sv[k] += f * a.sv[k];
          se[k] += f * a.se[k];
        }
        for (int64_t k = 0; k < P * dlen; ++k) {
          sd[k] += f * a.sd[k];
          sde[k] += f * a.sde[k];
        }
      }
      conv = conv && a.converged;
      panels += a.panels;
    }
    for (int64_t col = 0; col < P; ++col) {
      const scatrs_param& pr = dd.params[col];
      if (pr.kind != SCATRS_PARAM_WEIGHT) continue;
      for (int64_t p = 0; p < np; ++p) {
        const AdPart& a = parts[p];
        const double f = a.w / w_total * a.v / a.v_total;
        double df;
        if (pr.mode < 0) {
          const double own = a.component == pr.component ? a.v / a.v_total : 0.0;
          df = (own - f) / w_total;
        } else if (a.component != pr.component) {
          df = 0.0;
        } else {
          const double own = a.mode == pr.mode ? 1.0 : 0.0;
          df = a.w / w_total * (own - a.v / a.v_total) / a.v_total;
        }
        const PD& x = avg[p * n_wl + i];
        for (int64_t k = 0; k < row; ++k) {
          d[col * row + k] += df * x.v[k];
          de[col * row + k] += std::fabs(df) * x.e[k];
        }
        if (components[a.component].aspect_ratio > 0.0)
          for (int64_t k = 0; k < dlen; ++k) {
            sd[col * dlen + k] += df * x.sv[k];
            sde[col * dlen + k] += std::fabs(df) * x.se[k];
          }
      }
    }
    auto lin = [&](int64_t k) {
      LinD x;
      x.v = v[k];
      x.e = e[k];
      x.d.resize(P);
      x.de.resize(P);
      for (int64_t c = 0; c < P; ++c) {
        x.d[c] = d[c * row + k];
        x.de[c] = de[c * row + k];
      }
      return x;
    };
    auto D = [&](int f, int64_t l) {
      const int64_t k = f * (ldi + 1) + l;
      LinD x;
      x.v = sv[k];
      x.e = se[k];
      x.d.resize(P);
      x.de.resize(P);
      for (int64_t c = 0; c < P; ++c) {
        x.d[c] = sd[c * dlen + k];
        x.de[c] = sde[c * dlen + k];
      }
      return x;
    };
    // x + c y for an exact c (Lin::combine).
    auto add = [&](LinD x, double c, const LinD& y) {
      x.v += c * y.v;
      x.e += std::fabs(c) * y.e;
      for (int64_t k = 0; k < P; ++k) {
        x.d[k] += c * y.d[k];
        x.de[k] += std::fabs(c) * y.de[k];
      }
      return x;
    };
    const LinD ext = lin(1), sca = lin(2), scag = lin(3), abs_ = lin(4), back = lin(5),
               r2 = lin(6), r3 = lin(7), num = lin(8);
    for (const auto& w : {std::make_pair("<C_ext>", &ext), std::make_pair("<C_sca>", &sca),
                          std::make_pair("<C_back>", &back)})
      if (!(std::isfinite(w.second->v) && w.second->v != 0.0))
        throw Failure{SCATRS_INVALID_INPUT,
                      std::string("the ensemble's ") + w.first +
                          " is 0 or not finite, so its ratios (albedo, asymmetry parameter, "
                          "lidar ratio) are undefined (does m = 1?)"};
    const LinD depol = has_direct ? num.div(add(back.scale(2.0), -1.0, num))
                                  : LinD::constant(0.0, (size_t)P);
    const LinD outs[11] = {ext,
                           sca,
                           abs_,
                           back,
                           sca.div(ext),
                           scag.div(sca),
                           ext.div(back).scale(4.0 * kPi),
                           depol,
                           r3.div(r2),
                           r2.scale(kPi),
                           r3.scale(4.0 * kPi / 3.0)};
    for (int k = 0; k < 11; ++k) {
      res.values[k * n_wl + i] = outs[k].v;
      if (res.errors) res.errors[k * n_wl + i] = outs[k].e;
      for (int64_t c = 0; c < P; ++c) {
        if (dd.d_values) dd.d_values[(c * 11 + k) * n_wl + i] = outs[k].d[c];
        if (dd.d_errors) dd.d_errors[(c * 11 + k) * n_wl + i] = outs[k].de[c];
      }
    }
    const int64_t g0 = 9 + 4 * n_mu, glen = order[i] + 1;
    double* g_out = all_orders ? t_greek_all.g.data() : res.greek;
    double* ge_out = all_orders ? t_greek_all.ge.data() : res.greek_err;
    double* dg_out = all_orders ? t_greek_all.dg.data() : dd.d_greek;
    double* dge_out = all_orders ? t_greek_all.dge.data() : dd.d_greek_err;
    if (glen > 0 && g_out) {
      // The spheres' coefficients plus the spheroids' (engine.rs:2196-2216).
      auto G = [&](int f, int64_t l) {
        LinD x = lin(g0 + f * gw + l);
        if (has_direct && l <= ldi) x = add(x, 1.0, D(f, l));
        return x;
      };
      const LinD a0 = G(0, 0);
      for (int f = 0; f < 6; ++f)
        for (int64_t l = 0; l < glen; ++l) {
          LinD x = G(f, l);
          if (norm) x = (f == 0 && l == 0) ? LinD::constant(1.0, (size_t)P) : x.div(a0);
          const int64_t at = (f * n_wl + i) * gw + l;
          g_out[at] = x.v;
          if (ge_out) ge_out[at] = x.e;
          for (int64_t c = 0; c < P; ++c) {
            const int64_t atd = ((c * 6 + f) * n_wl + i) * gw + l;
            if (dg_out) dg_out[atd] = x.d[c];
            if (dge_out) dge_out[atd] = x.de[c];
          }
        }
    }
    if (n_mu > 0 && res.phase) {
      const int src[6] = {0, 1, 0, 2, 3, 2};
      std::vector<double> d00, d22, d2m2, d02;
      if (has_direct && ldi >= 0) {
        d00.resize(ldi + 1);
        d22.resize(ldi + 1);
        d2m2.resize(ldi + 1);
        d02.resize(ldi + 1);
      }
      for (int64_t j = 0; j < n_mu; ++j) {
        LinD fd[6];
        for (int k = 0; k < 6; ++k) fd[k] = LinD::constant(0.0, (size_t)P);
        if (has_direct && ldi >= 0) {
          wigner_d(0, 0, mu[j], d00.data(), ldi + 1);
          wigner_d(2, 2, mu[j], d22.data(), ldi + 1);
          wigner_d(2, -2, mu[j], d2m2.data(), ldi + 1);
          wigner_d(0, 2, mu[j], d02.data(), ldi + 1);
          for (int64_t l = 0; l <= ldi; ++l) {
            const double pl = 0.5 * (d22[l] + d2m2[l]), mn = 0.5 * (d22[l] - d2m2[l]);
            fd[0] = add(fd[0], d00[l], D(0, l));
            fd[1] = add(fd[1], d02[l], D(4, l));
            fd[2] = add(add(fd[2], pl, D(1, l)), mn, D(2, l));
            fd[3] = add(add(fd[3], mn, D(1, l)), pl, D(2, l));
            fd[4] = add(fd[4], d02[l], D(5, l));
            fd[5] = add(fd[5], d00[l], D(3, l));
          }
        }
        for (int el = 0; el < 6; ++el) {
          LinD x = add(lin(9 + src[el] * n_mu + j), 1.0, fd[el]);
          if (norm) x = x.div(sca);
          const int64_t at = (el * n_wl + i) * n_mu + j;
          res.phase[at] = x.v;
          if (res.phase_err) res.phase_err[at] = x.e;
          for (int64_t c = 0; c < P; ++c) {
            const int64_t atd = ((c * 6 + el) * n_wl + i) * n_mu + j;
            if (dd.d_phase) dd.d_phase[atd] = x.d[c];
            if (dd.d_phase_err) dd.d_phase_err[atd] = x.de[c];
          }
        }
      }
    }
    if (res.converged) res.converged[i] = conv ? 1 : 0;
    if (res.panels) res.panels[i] = panels;
  }
}


}  // namespace
}  // namespace sb

using namespace sb;

extern "C" {

void scatrs_ensemble_fixed_sizes(int64_t n_units, int64_t n_mu, int32_t greek_order,
                                 int64_t* values_len, int64_t* phase_len, int64_t* greek_len) {
  if (values_len) *values_len = 11 * n_units;
  if (phase_len) *phase_len = 6 * n_units * n_mu;
  if (greek_len) *greek_len = greek_order >= 0 ? 6 * n_units * ((int64_t)greek_order + 1) : 0;
}

}  // extern "C"

namespace sb {
namespace {
// The mixed form's options into a call (NULL or i8_above <= 0: the plain form).
void set_mixed(FixedCall& call, const scatrs_mixed_options* mixed) {
  if (!mixed || mixed->i8_above <= 0) return;
  if (mixed->levels != 0 && mixed->levels != 5 && mixed->levels != 6)
    throw Failure{SCATRS_INVALID_INPUT, "the mixed form keeps 5 or 6 product levels (0: 5)"};
  call.i8_above = mixed->i8_above;
  call.i8_levels = mixed->levels == 0 ? 5 : mixed->levels;
}
// scatrs_ensemble_fixed and its mixed form.
int fixed_host(const scatrs_distribution* dists, int64_t n_dist, const double* wavelengths,
               int64_t n_wl, const double* m, const double* mu, int64_t n_mu,
               const scatrs_fixed_options* options, double* values, double* phase,
               double* greek, const scatrs_mixed_options* mixed, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_dist < 0 || n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    for (int64_t i = 0; i < n_wl; ++i)
      if (!(std::isfinite(wavelengths[i]) && wavelengths[i] > 0.0))
        throw Failure{SCATRS_INVALID_INPUT, "wavelengths must be finite and > 0"};
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    cudaStream_t s = 0;
    const int64_t n_units = n_dist * n_wl;
    check_options(options, n_units, n_mu, mu);
    if (n_units == 0) return;
    double* wl_d = c.wl.as<double>(n_wl);
    double* m_d = c.m.as<double>(2 * n_units);
    SB_CUDA(cudaMemcpyAsync(wl_d, wavelengths, n_wl * 8, cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(m_d, m, 2 * n_units * 8, cudaMemcpyHostToDevice, s));
    int64_t vl, pl, gl;
    scatrs_ensemble_fixed_sizes(n_units, n_mu, options->greek_order, &vl, &pl, &gl);
    double* v_d = c.values.as<double>(vl);
    double* p_d = pl > 0 ? c.phase.as<double>(pl) : nullptr;
    double* g_d = gl > 0 ? c.greek.as<double>(gl) : nullptr;
    FixedCall call;
    call.wl_host.assign(wavelengths, wavelengths + n_wl);
    set_mixed(call, mixed);
    // Pinned outputs are copied slab by slab beside the computation; others at the end.
    auto pinned = [](const void* p) {
      cudaPointerAttributes at{};
      if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      return at.type == cudaMemoryTypeHost;
    };
    const bool overlap = pinned(values) && (pl == 0 || !phase || pinned(phase)) &&
                         (gl == 0 || !greek || pinned(greek));
    // Waits for the slab copies into the caller's pinned arrays on every exit, the error
    // exits included, so that no copy outlives the call.
    struct CopyWait {
      cudaStream_t st = nullptr;
      ~CopyWait() {
        if (st && cudaStreamSynchronize(st) != cudaSuccess) cudaGetLastError();
      }
    } copy_wait;
    if (overlap) {
      c.ensure_copies();
      copy_wait.st = c.copies;
      call.h_values = values;
      call.h_phase = pl > 0 ? phase : nullptr;
      call.h_greek = gl > 0 ? greek : nullptr;
    }
    run_fixed(c, dists, n_dist, wl_d, n_wl, m_d, mu, n_mu, options, v_d, p_d, g_d, s, &call);
    if (overlap) {
      copy_wait.st = nullptr;
      const cudaError_t e = cudaStreamSynchronize(c.copies);
      check_device_errors(c, s, &call);
      SB_CUDA(e);
      return;
    }
    check_device_errors(c, s, &call);
    SB_CUDA(cudaMemcpyAsync(values, v_d, vl * 8, cudaMemcpyDeviceToHost, s));
    if (pl > 0 && phase) SB_CUDA(cudaMemcpyAsync(phase, p_d, pl * 8, cudaMemcpyDeviceToHost, s));
    if (gl > 0 && greek) SB_CUDA(cudaMemcpyAsync(greek, g_d, gl * 8, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
  });
}

// scatrs_ensemble_fixed_device and its mixed form.
int fixed_device(const scatrs_distribution* dists_host, int64_t n_dist,
                 const double* wavelengths_dev, int64_t n_wl, const double* m_dev,
                 const double* mu_host, int64_t n_mu, const scatrs_fixed_options* options,
                 double* values_dev, double* phase_dev, double* greek_dev, void* stream,
                 const scatrs_mixed_options* mixed, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_dist < 0 || n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    FixedCall call;
    set_mixed(call, mixed);
    call.wl_host.resize(n_wl);
    if (n_wl > 0)
      SB_CUDA(cudaMemcpyAsync(call.wl_host.data(), wavelengths_dev, n_wl * 8,
                              cudaMemcpyDeviceToHost, s));
    run_fixed(c, dists_host, n_dist, wavelengths_dev, n_wl, m_dev, mu_host, n_mu, options,
              values_dev, phase_dev, greek_dev, s, &call);
    g_last_call = std::move(call);
  });
}
}  // namespace
}  // namespace sb

extern "C" {

int scatrs_ensemble_fixed(const scatrs_distribution* dists, int64_t n_dist,
                          const double* wavelengths, int64_t n_wl, const double* m,
                          const double* mu, int64_t n_mu, const scatrs_fixed_options* options,
                          double* values, double* phase, double* greek, char* err,
                          size_t err_len) {
  return fixed_host(dists, n_dist, wavelengths, n_wl, m, mu, n_mu, options, values, phase,
                    greek, nullptr, err, err_len);
}

int scatrs_ensemble_fixed_mixed(const scatrs_distribution* dists, int64_t n_dist,
                                const double* wavelengths, int64_t n_wl, const double* m,
                                const double* mu, int64_t n_mu,
                                const scatrs_fixed_options* options,
                                const scatrs_mixed_options* mixed, double* values,
                                double* phase, double* greek, char* err, size_t err_len) {
  return fixed_host(dists, n_dist, wavelengths, n_wl, m, mu, n_mu, options, values, phase,
                    greek, mixed, err, err_len);
}

int scatrs_ensemble_fixed_mixed_device(const scatrs_distribution* dists_host, int64_t n_dist,
                                       const double* wavelengths_dev, int64_t n_wl,
                                       const double* m_dev, const double* mu_host, int64_t n_mu,
                                       const scatrs_fixed_options* options,
                                       const scatrs_mixed_options* mixed, double* values_dev,
                                       double* phase_dev, double* greek_dev, void* stream,
                                       char* err, size_t err_len) {
  return fixed_device(dists_host, n_dist, wavelengths_dev, n_wl, m_dev, mu_host, n_mu, options,
                      values_dev, phase_dev, greek_dev, stream, mixed, err, err_len);
}

}  // extern "C"

namespace sb {
namespace {
// The wavelengths on the host for checks and messages: a copy of device ones.
std::vector<double> host_wavelengths(const double* wl, int64_t n_wl, bool device, cudaStream_t s) {
  std::vector<double> h(std::max<int64_t>(n_wl, 0));
  if (n_wl <= 0) return h;
  if (device) {
    SB_CUDA(cudaMemcpyAsync(h.data(), wl, n_wl * 8, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
  } else {
    h.assign(wl, wl + n_wl);
  }
  for (int64_t i = 0; i < n_wl; ++i)
    if (!(std::isfinite(h[i]) && h[i] > 0.0))
      throw Failure{SCATRS_INVALID_INPUT, "wavelengths must be finite and > 0"};
  return h;
}

// scatrs_ensemble_fixed_d with host (device = false) or device arrays.
void fixed_d_impl(const scatrs_distribution* dists, int64_t n_dist, const double* wavelengths,
                  int64_t n_wl, const double* m, const double* mu, int64_t n_mu,
                  const scatrs_fixed_options* options, double* values, double* phase,
                  double* greek, double* d_values, double* d_phase, double* d_greek, bool device,
                  cudaStream_t s) {
  if (n_dist < 0 || n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
  DerivOutput dv;
  dv.on = true;
  dv.n_theta = n_dist > 0 ? parameter_count(dists[0].kind) : 2;
  const int P = dv.n_theta + 2;
  Context& c = context();
  std::lock_guard<std::mutex> lk(c.mtx);
  const std::vector<double> wl_host = host_wavelengths(wavelengths, n_wl, device, s);
  const int64_t n_units = n_dist * n_wl;
  check_options(options, n_units, n_mu, mu, P);
  if (n_units == 0) return;
  const cudaMemcpyKind in = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind out = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  double* wl_d = c.wl.as<double>(n_wl);
  double* m_d = c.m.as<double>(2 * n_units);
  SB_CUDA(cudaMemcpyAsync(wl_d, wavelengths, n_wl * 8, in, s));
  SB_CUDA(cudaMemcpyAsync(m_d, m, 2 * n_units * 8, in, s));
  int64_t vl, pl, gl;
  scatrs_ensemble_fixed_sizes(n_units, n_mu, options->greek_order, &vl, &pl, &gl);
  if (device && ((pl > 0 && (!phase || !d_phase)) || (gl > 0 && (!greek || !d_greek)) ||
                 !values || !d_values))
    throw Failure{SCATRS_INVALID_INPUT,
                  "the device entry needs every output array the options call for"};
  // One allocation per output kind: the values, then the P derivative blocks.
  double* v_d = c.values.as<double>(vl * (1 + P));
  double* p_d = pl > 0 ? c.phase.as<double>(pl * (1 + P)) : nullptr;
  double* g_d = gl > 0 ? c.greek.as<double>(gl * (1 + P)) : nullptr;
  dv.d_values = v_d + vl;
  dv.d_phase = p_d ? p_d + pl : nullptr;
  dv.d_greek = g_d ? g_d + gl : nullptr;
  FixedCall call;
  call.wl_host = wl_host;
  run_fixed(c, dists, n_dist, wl_d, n_wl, m_d, mu, n_mu, options, v_d, p_d, g_d, s, &call,
            LayerInput(), dv);
  check_device_errors(c, s, &call);
  SB_CUDA(cudaMemcpyAsync(values, v_d, vl * 8, out, s));
  if (d_values) SB_CUDA(cudaMemcpyAsync(d_values, dv.d_values, P * vl * 8, out, s));
  if (pl > 0 && phase) SB_CUDA(cudaMemcpyAsync(phase, p_d, pl * 8, out, s));
  if (pl > 0 && d_phase) SB_CUDA(cudaMemcpyAsync(d_phase, dv.d_phase, P * pl * 8, out, s));
  if (gl > 0 && greek) SB_CUDA(cudaMemcpyAsync(greek, g_d, gl * 8, out, s));
  if (gl > 0 && d_greek) SB_CUDA(cudaMemcpyAsync(d_greek, dv.d_greek, P * gl * 8, out, s));
  SB_CUDA(cudaStreamSynchronize(s));
}
}  // namespace
}  // namespace sb

extern "C" {

int scatrs_ensemble_fixed_d(const scatrs_distribution* dists, int64_t n_dist,
                            const double* wavelengths, int64_t n_wl, const double* m,
                            const double* mu, int64_t n_mu, const scatrs_fixed_options* options,
                            double* values, double* phase, double* greek, double* d_values,
                            double* d_phase, double* d_greek, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    fixed_d_impl(dists, n_dist, wavelengths, n_wl, m, mu, n_mu, options, values, phase, greek,
                 d_values, d_phase, d_greek, false, 0);
  });
}

int scatrs_ensemble_fixed_d_device(const scatrs_distribution* dists_host, int64_t n_dist,
                                   const double* wavelengths_dev, int64_t n_wl,
                                   const double* m_dev, const double* mu_host, int64_t n_mu,
                                   const scatrs_fixed_options* options, double* values_dev,
                                   double* phase_dev, double* greek_dev, double* d_values_dev,
                                   double* d_phase_dev, double* d_greek_dev, void* stream,
                                   char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    fixed_d_impl(dists_host, n_dist, wavelengths_dev, n_wl, m_dev, mu_host, n_mu, options,
                 values_dev, phase_dev, greek_dev, d_values_dev, d_phase_dev, d_greek_dev, true,
                 static_cast<cudaStream_t>(stream));
  });
}

int scatrs_ensemble_adaptive(const scatrs_distribution* dists, int64_t n_dist, int32_t batch,
                             const double* wavelengths, int64_t n_wl, const double* m,
                             const double* mu, int64_t n_mu,
                             const scatrs_adaptive_options* options, double* values,
                             double* errors, double* phase, double* phase_err, double* greek,
                             double* greek_err, int8_t* converged, int64_t* panels, char* err,
                             size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_dist < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    std::vector<AdPart> parts;
    for (int64_t d = 0; d < n_dist; ++d)
      parts.push_back(AdPart{dists[d].kind, {dists[d].param[0], dists[d].param[1],
                                             dists[d].param[2]},
                             m, 1.0, (int)d, "distribution " + std::to_string(d) + ": ",
                             dists[d].table, dists[d].table_len});
    AdOutputs out{values, errors, phase, phase_err, greek, greek_err, converged, panels};
    adaptive_call(parts, (int)n_dist, batch != 0, wavelengths, n_wl, mu, n_mu, options, out);
  });
}

int scatrs_ensemble_adaptive_layered(const scatrs_distribution* dists, int64_t n_dist,
                                     int32_t batch, const double* wavelengths, int64_t n_wl,
                                     const scatrs_layers* layers, const double* mu, int64_t n_mu,
                                     const scatrs_adaptive_options* options, double* values,
                                     double* errors, double* phase, double* phase_err,
                                     double* greek, double* greek_err, int8_t* converged,
                                     int64_t* panels, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_dist < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    if (!layers || layers->n_layers < 1 || !layers->m ||
        (layers->n_layers > 1 && !layers->fractions))
      throw Failure{SCATRS_INVALID_INPUT, "layers must give n_layers >= 1, fractions and m"};
    // One layer: a homogeneous sphere with m = layers->m[d][0][n_wl].
    std::vector<AdPart> parts;
    for (int64_t d = 0; d < n_dist; ++d)
      parts.push_back(AdPart{dists[d].kind, {dists[d].param[0], dists[d].param[1],
                                             dists[d].param[2]},
                             layers->m + 2 * d * layers->n_layers * n_wl, 1.0, (int)d,
                             "distribution " + std::to_string(d) + ": ", dists[d].table,
                             dists[d].table_len});
    AdOutputs out{values, errors, phase, phase_err, greek, greek_err, converged, panels};
    adaptive_call(parts, (int)n_dist, batch != 0, wavelengths, n_wl, mu, n_mu, options, out,
                  layers);
  });
}

int scatrs_ensemble_adaptive_spheroid(const scatrs_distribution* dists, int64_t n_dist,
                                      int32_t batch, const double* wavelengths, int64_t n_wl,
                                      double aspect_ratio, const double* m, const double* mu,
                                      int64_t n_mu, const scatrs_adaptive_options* options,
                                      double* values, double* errors, double* phase,
                                      double* phase_err, double* greek, double* greek_err,
                                      int8_t* converged, int64_t* panels, char* err,
                                      size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!values || !m) throw Failure{SCATRS_INVALID_INPUT, "values and m are required"};
    AdOutputs out{values, errors, phase, phase_err, greek, greek_err, converged, panels};
    spheroid_call({SphParticle{dists, n_dist, aspect_ratio, m}}, batch != 0, wavelengths, n_wl,
                  mu, n_mu, options, out);
  });
}

int scatrs_ensemble_mixture_d(const scatrs_component* components, int64_t n_comp,
                              const double* wavelengths, int64_t n_wl, const double* mu,
                              int64_t n_mu, const scatrs_adaptive_options* options,
                              const scatrs_param* params, int64_t n_params, double* values,
                              double* errors, double* d_values, double* d_errors, double* phase,
                              double* phase_err, double* d_phase, double* d_phase_err,
                              double* greek, double* greek_err, double* d_greek,
                              double* d_greek_err, int8_t* converged, int64_t* panels, char* err,
                              size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_params < 0 || (n_params > 0 && !params))
      throw Failure{SCATRS_INVALID_INPUT, "params must hold n_params parameters"};
    // One spheroid distribution takes its derivatives on the direct path (spheroid_call_d).
    const bool spheroid_alone = n_comp == 1 && components && components[0].aspect_ratio > 0.0 &&
                                components[0].n_layers <= 1 && components[0].n_modes == 1 &&
                                !components[0].mode_weights;
    // One layered component (plain or multimodal) takes them on the adaptive pipeline with
    // its layers.
    const bool layered_alone = n_comp == 1 && components && components[0].n_layers > 1 &&
                               components[0].aspect_ratio == 0.0;
    if (heterogeneous(components, n_comp) && n_params == 0) {
      AdOutputs out{values, errors, phase, phase_err, greek, greek_err, converged, panels};
      mixture_hetero(components, n_comp, wavelengths, n_wl, mu, n_mu, options, out);
      return;
    }
    std::vector<AdPart> parts = mixture_parts(components, n_comp);
    // ensemble/mod.rs:781-799: every parameter once and among the mixture's (mod.rs:254-337).
    bool mixture = n_comp > 1;
    for (int64_t k = 0; k < n_params; ++k)
      mixture = mixture || (params[k].kind == SCATRS_PARAM_WEIGHT && params[k].mode < 0);
    auto name = [&](const scatrs_param& q) {
      static const char* dist_names[7][3] = {{"", "", ""},
                                             {"median_radius", "width", ""},
                                             {"effective_radius", "effective_variance", ""},
                                             {"alpha", "b", "gamma"},
                                             {"exponent", "", ""},
                                             {"radius", "", ""},
                                             {"", "", ""}};
      std::string out = mixture ? "c" + std::to_string(q.component) + "." : "";
      if (q.mode >= 0) out += "mode" + std::to_string(q.mode) + ".";
      switch (q.kind) {
        case SCATRS_PARAM_DISTRIBUTION: {
          const bool ok = q.component >= 0 && q.component < n_comp && q.mode >= -1 &&
                          q.mode < components[q.component].n_modes;
          const int kind = ok ? components[q.component].modes[q.mode < 0 ? 0 : q.mode].kind : 0;
          out += kind >= 0 && kind < 7 && q.index >= 0 && q.index < 3 && dist_names[kind][q.index][0]
                     ? dist_names[kind][q.index]
                     : "parameter" + std::to_string(q.index);
          break;
        }
        case SCATRS_PARAM_REFR_REAL: out += "m_real"; break;
        case SCATRS_PARAM_REFR_IMAG: out += "m_imag"; break;
        case SCATRS_PARAM_WEIGHT: out += "weight"; break;
        case SCATRS_PARAM_ASPECT_RATIO: out += "aspect_ratio"; break;
        case SCATRS_PARAM_LAYER_REFR_REAL: out += "layer" + std::to_string(q.index) + ".m_real"; break;
        case SCATRS_PARAM_LAYER_REFR_IMAG: out += "layer" + std::to_string(q.index) + ".m_imag"; break;
        case SCATRS_PARAM_RADIUS_FRACTION:
          out += "layer" + std::to_string(q.index) + ".radius_fraction";
          break;
        default: out += "kind" + std::to_string(q.kind);
      }
      return out;
    };
    for (int64_t k = 0; k < n_params; ++k) {
      const scatrs_param& q = params[k];
      for (int64_t j = 0; j < k; ++j)
        if (params[j].component == q.component && params[j].mode == q.mode &&
            params[j].kind == q.kind && params[j].index == q.index)
          throw Failure{SCATRS_INVALID_INPUT, "parameter " + name(q) + " requested twice"};
      bool allowed = q.component >= 0 && q.component < n_comp;
      if (allowed) {
        const scatrs_component& cp = components[q.component];
        const bool multi = cp.mode_weights != nullptr;
        switch (q.kind) {
          case SCATRS_PARAM_DISTRIBUTION: {
            const bool mode_ok = multi ? (q.mode >= 0 && q.mode < cp.n_modes) : q.mode == -1;
            const int kind = mode_ok ? cp.modes[q.mode < 0 ? 0 : q.mode].kind : 0;
            const int np = kind == adaptive::kMonodisperse ? 1 : parameter_count(kind);
            allowed = mode_ok && q.index >= 0 && q.index < np;
            break;
          }
          case SCATRS_PARAM_REFR_REAL:
          case SCATRS_PARAM_REFR_IMAG: allowed = q.mode == -1 && cp.n_layers <= 1; break;
          case SCATRS_PARAM_ASPECT_RATIO: allowed = q.mode == -1 && cp.aspect_ratio > 0.0; break;
          case SCATRS_PARAM_LAYER_REFR_REAL:
          case SCATRS_PARAM_LAYER_REFR_IMAG:
            allowed = q.mode == -1 && cp.n_layers > 1 && q.index >= 0 && q.index < cp.n_layers;
            break;
          case SCATRS_PARAM_RADIUS_FRACTION:
            allowed = q.mode == -1 && cp.n_layers > 1 && q.index >= 0 &&
                      q.index < cp.n_layers - 1;
            break;
          case SCATRS_PARAM_WEIGHT:
            allowed = q.mode == -1 || (multi && q.mode >= 0 && q.mode < cp.n_modes);
            break;
          default: allowed = false;
        }
      }
      if (!allowed) throw Failure{SCATRS_INVALID_INPUT, "no parameter " + name(q) + " here"};
    }
    if (heterogeneous(components, n_comp) && !spheroid_alone && !layered_alone) {
      // Components of different particles (or a multimodal spheroid): every part on its own
      // engine, mixed and assembled on the host with the derivatives.
      if (!d_values) throw Failure{SCATRS_INVALID_INPUT, "d_values is required with parameters"};
      AdOutputs out{values, errors, phase, phase_err, greek, greek_err, converged, panels};
      AdDerivs dd;
      dd.params = params;
      dd.n = n_params;
      dd.d_values = d_values;
      dd.d_errors = d_errors;
      dd.d_phase = d_phase;
      dd.d_phase_err = d_phase_err;
      dd.d_greek = d_greek;
      dd.d_greek_err = d_greek_err;
      mixture_hetero_d(components, n_comp, wavelengths, n_wl, mu, n_mu, options, out, dd);
      return;
    }
    if (spheroid_alone) {
      if (n_params > 0 && !d_values)
        throw Failure{SCATRS_INVALID_INPUT, "d_values is required with parameters"};
      SphDerivReq req;
      for (int64_t k = 0; k < n_params; ++k) {
        const scatrs_param& q = params[k];
        if (q.kind == SCATRS_PARAM_DISTRIBUTION) {
          req.grads.push_back(q.index);
          req.theta_cols.push_back((int)k);
        } else if (q.kind == SCATRS_PARAM_REFR_REAL) {
          req.dir_cols[0] = (int)k;
        } else if (q.kind == SCATRS_PARAM_REFR_IMAG) {
          req.dir_cols[1] = (int)k;
        } else if (q.kind == SCATRS_PARAM_ASPECT_RATIO) {
          req.dir_cols[2] = (int)k;
        }  // a single component's weight: its number fraction is 1 whatever it is
      }
      AdOutputs out{values, errors, phase, phase_err, greek, greek_err, converged, panels};
      AdDerivs dd;
      dd.params = params;
      dd.n = n_params;
      dd.d_values = d_values;
      dd.d_errors = d_errors;
      dd.d_phase = d_phase;
      dd.d_phase_err = d_phase_err;
      dd.d_greek = d_greek;
      dd.d_greek_err = d_greek_err;
      for (int64_t k = 0; k < n_params * 11 * n_wl && d_values; ++k) d_values[k] = 0.0;
      for (int64_t k = 0; k < n_params * 11 * n_wl && d_errors; ++k) d_errors[k] = 0.0;
      const scatrs_component& cp = components[0];
      spheroid_call_d({SphParticle{cp.modes, 1, cp.aspect_ratio, cp.m}}, {req}, wavelengths, n_wl,
                      mu, n_mu, options, out, dd);
      return;
    }
    if (layered_alone) {
      // Each mode a part with the component's layers; the directions each layer's Re m and
      // Im m, then each radius fraction (particle.rs:119-145).
      const scatrs_component& cp = components[0];
      const int L = cp.n_layers;
      if (!cp.fractions || !cp.m)
        throw Failure{SCATRS_INVALID_INPUT, "component 0: a layered sphere needs fractions and m"};
      const int64_t np = (int64_t)parts.size();
      std::vector<double> fr((size_t)np * (L - 1)), ml((size_t)np * 2 * L * n_wl);
      for (int64_t p = 0; p < np; ++p) {
        std::copy(cp.fractions, cp.fractions + (L - 1), fr.begin() + p * (L - 1));
        std::copy(cp.m, cp.m + 2 * L * n_wl, ml.begin() + p * 2 * L * n_wl);
      }
      for (AdPart& a : parts) {
        a.dir_cols.assign(3 * L - 1, -1);
        for (int64_t k = 0; k < n_params; ++k) {
          const scatrs_param& q = params[k];
          if (q.kind == SCATRS_PARAM_DISTRIBUTION && q.mode == a.mode) {
            a.grads.push_back(q.index);
            a.theta_cols.push_back((int)k);
          } else if (q.kind == SCATRS_PARAM_LAYER_REFR_REAL) {
            a.dir_cols[2 * q.index] = (int)k;
          } else if (q.kind == SCATRS_PARAM_LAYER_REFR_IMAG) {
            a.dir_cols[2 * q.index + 1] = (int)k;
          } else if (q.kind == SCATRS_PARAM_RADIUS_FRACTION) {
            a.dir_cols[2 * L + q.index] = (int)k;
          }
        }
      }
      scatrs_layers lay{L, 0, fr.data(), ml.data()};
      AdOutputs out{values, errors, phase, phase_err, greek, greek_err, converged, panels};
      AdDerivs dd;
      dd.params = params;
      dd.n = n_params;
      dd.d_values = d_values;
      dd.d_errors = d_errors;
      dd.d_phase = d_phase;
      dd.d_phase_err = d_phase_err;
      dd.d_greek = d_greek;
      dd.d_greek_err = d_greek_err;
      if (!d_values) throw Failure{SCATRS_INVALID_INPUT, "d_values is required with parameters"};
      adaptive_call(parts, 1, false, wavelengths, n_wl, mu, n_mu, options, out, &lay, &dd);
      return;
    }
    // engine.rs:153-176: each part's parameters and their columns.
    for (AdPart& a : parts)
      for (int64_t k = 0; k < n_params; ++k) {
        const scatrs_param& q = params[k];
        if (q.component != a.component) continue;
        if (q.kind == SCATRS_PARAM_DISTRIBUTION && q.mode == a.mode) {
          a.grads.push_back(q.index);
          a.theta_cols.push_back((int)k);
        } else if (q.kind == SCATRS_PARAM_REFR_REAL) {
          a.dir_cols[0] = (int)k;
        } else if (q.kind == SCATRS_PARAM_REFR_IMAG) {
          a.dir_cols[1] = (int)k;
        }
      }
    AdOutputs out{values, errors, phase, phase_err, greek, greek_err, converged, panels};
    AdDerivs dd;
    dd.params = params;
    dd.n = n_params;
    dd.d_values = d_values;
    dd.d_errors = d_errors;
    dd.d_phase = d_phase;
    dd.d_phase_err = d_phase_err;
    dd.d_greek = d_greek;
    dd.d_greek_err = d_greek_err;
    if (n_params > 0 && !d_values)
      throw Failure{SCATRS_INVALID_INPUT, "d_values is required with parameters"};
    adaptive_call(parts, 1, false, wavelengths, n_wl, mu, n_mu, options, out, nullptr,
                  n_params > 0 ? &dd : nullptr);
  });
}

int scatrs_ensemble_mixture(const scatrs_component* components, int64_t n_comp,
                            const double* wavelengths, int64_t n_wl, const double* mu,
                            int64_t n_mu, const scatrs_adaptive_options* options, double* values,
                            double* errors, double* phase, double* phase_err, double* greek,
                            double* greek_err, int8_t* converged, int64_t* panels, char* err,
                            size_t err_len) {
  return guarded(err, err_len, [&] {
    AdOutputs out{values, errors, phase, phase_err, greek, greek_err, converged, panels};
    if (heterogeneous(components, n_comp)) {
      mixture_hetero(components, n_comp, wavelengths, n_wl, mu, n_mu, options, out);
      return;
    }
    std::vector<AdPart> parts = mixture_parts(components, n_comp);
    adaptive_call(parts, 1, false, wavelengths, n_wl, mu, n_mu, options, out);
  });
}


int scatrs_project_greek_device(const double* phase_dev, int64_t n_units, int64_t n_q,
                                int32_t order, int32_t precision, double* greek_dev,
                                void* stream, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_units < 0 || n_q < 1 || order < 0 || order > kMaxGreekOrder)
      throw Failure{SCATRS_INVALID_INPUT, "needs n_units >= 0, n_q >= 1 and 0 <= order"};
    if (n_q > kMaxGaussPoints || (double)n_q * ((double)order + 1.0) > (double)kMaxWignerValues)
      throw Failure{SCATRS_INVALID_INPUT,
                    "the projection tables would exceed MAX_GAUSS_LEGENDRE_POINTS cosines or "
                    "MAX_WIGNER_D_VALUES Wigner values"};
    if (precision != 0 && precision != 1)
      throw Failure{SCATRS_INVALID_INPUT, "precision must be 0 (FP64) or 1 (3xTF32)"};
    if (n_units == 0) return;
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Context::Projector& p = projector(c, n_q, order, s);
    const int len = order + 1;
    if (precision == 0) {
      timed_launch(K_PROJ, s, [&] {
        launch_greek_fp64(phase_dev, n_units, (int)n_q, len, p.d.as<double>(0), greek_dev, s);
      });
      SB_CUDA(cudaGetLastError());
      return;
    }
    if (n_units > (int64_t)INT32_MAX / 6)
      throw Failure{SCATRS_INVALID_INPUT, "too many tables for one tensor-core projection"};
    const int64_t n_q_pad = round_up(n_q, 4);
    float* a_hi = c.tc_a_hi.as<float>(6 * (size_t)n_units * n_q_pad);
    float* a_lo = c.tc_a_lo.as<float>(6 * (size_t)n_units * n_q_pad);
    float* prod = c.tc_prod.as<float>(6 * (size_t)n_units * len);
    unsigned* flag = c.tc_err.as<unsigned>(1);
    SB_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned), s));
    launch_greek_split(phase_dev, n_units, (int)n_q, (int)n_q_pad, a_hi, a_lo, s);
    SB_CUDA(cudaGetLastError());
    const CUtensorMap maps[4] = {
        tensor_map_2d(a_hi, n_q_pad, 6 * n_units, 128), tensor_map_2d(a_lo, n_q_pad, 6 * n_units, 128),
        tensor_map_2d(p.d_hi.as<float>(0), n_q_pad, 4 * (int64_t)len, 256),
        tensor_map_2d(p.d_lo.as<float>(0), n_q_pad, 4 * (int64_t)len, 256)};
    TcArgs ta{(int)n_units, (int)n_q_pad, len, prod, flag};
    cudaError_t e = cudaSuccess;
    timed_launch(K_PROJ, s, [&] { e = launch_greek_tc(maps, ta, s); });
    if (e != cudaSuccess)
      throw Failure{SCATRS_CUDA, std::string("greek_tc_kernel: ") + cudaGetErrorString(e)};
    launch_greek_assemble(prod, n_units, len, greek_dev, s);
    SB_CUDA(cudaGetLastError());
    unsigned h = 0;
    SB_CUDA(cudaMemcpyAsync(&h, flag, sizeof h, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    if (h) throw Failure{SCATRS_CUDA, "the tensor-core projection's pipeline timed out"};
  });
}

int scatrs_spheroid_tmatrix(double x, double aspect_ratio, const double* m, int32_t mode,
                            int32_t n_terms, int32_t n_theta, double* t, char* err,
                            size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!m || !t) throw Failure{SCATRS_INVALID_INPUT, "m and t are required"};
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    std::vector<double> sums;
    std::vector<std::vector<double>> ts;
    run_tmatrices(c, {TmSpec{x, aspect_ratio, m[0], m[1], mode, n_terms, n_theta}}, sums, &ts, 0);
    std::copy(ts[0].begin(), ts[0].end(), t);
  });
}

int scatrs_spheroid_efficiencies(int64_t n, const double* x, const double* aspect_ratio,
                                 const double* m, double rtol, double* q, int32_t* n_terms,
                                 int32_t* n_theta, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    if (n == 0) return;
    if (!q) throw Failure{SCATRS_INVALID_INPUT, "q is required"};
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    std::vector<SpheroidResult> res;
    spheroid_solve(c, n, x, aspect_ratio, m, rtol, 0, 0, false, res, 0, true);
    for (int64_t i = 0; i < n; ++i) {
      q[3 * i] = res[i].q_ext;
      q[3 * i + 1] = res[i].q_sca;
      q[3 * i + 2] = res[i].q_abs;
      if (n_terms) n_terms[i] = res[i].n;
      if (n_theta) n_theta[i] = res[i].nth;
    }
  });
}

int scatrs_spheroid_compute(int64_t n, const double* x, const double* aspect_ratio,
                            const double* m, const scatrs_spheroid_options* options, double* eff,
                            double* greek, int32_t* n_terms, int32_t* n_theta,
                            double* error_estimate, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    if (!options) throw Failure{SCATRS_INVALID_INPUT, "options are required"};
    const scatrs_spheroid_options& o = *options;
    if (o.n_terms < 0 || o.n_theta < 0 || o.greek_order < -1 || o.greek_order > (1 << 20))
      throw Failure{SCATRS_INVALID_INPUT, "n_terms, n_theta >= 0 and greek_order >= -1 needed"};
    if (n == 0) return;
    if (!eff) throw Failure{SCATRS_INVALID_INPUT, "eff is required"};
    if (o.greek_order >= 0 && !greek)
      throw Failure{SCATRS_INVALID_INPUT, "greek is required with greek_order >= 0"};
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    std::vector<SpheroidResult> res;
    spheroid_solve(c, n, x, aspect_ratio, m, o.rtol, o.n_terms, o.n_theta, true, res, 0,
                   o.allow_unvalidated != 0);
    const int64_t len = (int64_t)o.greek_order + 1;
    for (int64_t i = 0; i < n; ++i) {
      const SpheroidResult& r = res[i];
      eff[5 * i] = r.q_ext;
      eff[5 * i + 1] = r.q_sca;
      eff[5 * i + 2] = r.q_abs;
      eff[5 * i + 3] = r.q_back;
      eff[5 * i + 4] = r.g;
      if (n_terms) n_terms[i] = r.n;
      if (n_theta) n_theta[i] = r.nth;
      if (error_estimate) error_estimate[i] = r.err_est;
      if (o.greek_order < 0) continue;
      // tmatrix/mod.rs:464-491: truncated or zero-padded to the order; normalized by alpha1_0,
      // or unnormalized (alpha1_0 = C_sca / (4 pi) in 1/k^2, so times 4 / x^2).
      const int64_t have = 2 * (int64_t)r.n + 1;
      const double a0 = r.greek[0];
      const double scale = o.normalized ? 1.0 / a0 : 4.0 / (x[i] * x[i]);
      double* out = greek + 6 * len * i;
      for (int f = 0; f < 6; ++f)
        for (int64_t l = 0; l < len; ++l)
          out[f * len + l] = l < have ? scale * r.greek[f * have + l] : 0.0;
      if (o.normalized) out[0] = 1.0;
    }
  });
}

int scatrs_spheroid_compute_d(int64_t n, const double* x, const double* aspect_ratio,
                              const double* m, const scatrs_spheroid_options* options,
                              double* eff, double* greek, double* d_eff, double* d_greek,
                              int32_t* n_terms, int32_t* n_theta, double* error_estimate,
                              char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    if (!options) throw Failure{SCATRS_INVALID_INPUT, "options are required"};
    const scatrs_spheroid_options& o = *options;
    if (o.n_terms < 0 || o.n_theta < 0 || o.greek_order < -1 || o.greek_order > (1 << 20))
      throw Failure{SCATRS_INVALID_INPUT, "n_terms, n_theta >= 0 and greek_order >= -1 needed"};
    if (n == 0) return;
    if (!eff || !d_eff) throw Failure{SCATRS_INVALID_INPUT, "eff and d_eff are required"};
    if (o.greek_order >= 0 && (!greek || !d_greek))
      throw Failure{SCATRS_INVALID_INPUT, "greek and d_greek are required with greek_order >= 0"};
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    std::vector<SpheroidResult> res;
    spheroid_solve(c, n, x, aspect_ratio, m, o.rtol, o.n_terms, o.n_theta, false, res, 0,
                   o.allow_unvalidated != 0);
    std::vector<SphEval> base(n);
    for (int64_t i = 0; i < n; ++i) {
      base[i] = {x[i], aspect_ratio[i], m[2 * i], m[2 * i + 1], res[i].n, res[i].nth};
      if (n_terms) n_terms[i] = res[i].n;
      if (n_theta) n_theta[i] = res[i].nth;
      if (error_estimate) error_estimate[i] = res[i].err_est;
    }
    std::vector<std::vector<double>> val, d[4];
    spheroid_fixed_outputs(c, base, o.greek_order, o.normalized != 0, val, 0);
    spheroid_fixed_derivs(c, base, o.greek_order, o.normalized != 0, d, 0);
    const int64_t len = (int64_t)o.greek_order + 1;
    for (int64_t i = 0; i < n; ++i) {
      for (int q = 0; q < 5; ++q) eff[5 * i + q] = val[i][q];
      for (int dir = 0; dir < 4; ++dir)
        for (int q = 0; q < 5; ++q) d_eff[(dir * n + i) * 5 + q] = d[dir][i][q];
      if (o.greek_order < 0) continue;
      for (int64_t q = 0; q < 6 * len; ++q) {
        greek[6 * len * i + q] = val[i][5 + q];
        for (int dir = 0; dir < 4; ++dir)
          d_greek[(dir * n + i) * 6 * len + q] = d[dir][i][5 + q];
      }
    }
  });
}

int scatrs_ensemble_fixed_spheroid(const scatrs_distribution* dists, int64_t n_dist,
                                   const double* wavelengths, int64_t n_wl,
                                   const double* aspect_ratio, const double* m, const double* mu,
                                   int64_t n_mu, const scatrs_fixed_options* options,
                                   double tmatrix_rtol, double* values, double* phase,
                                   double* greek, int32_t* node_terms, char* err,
                                   size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_dist < 0 || n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    for (int64_t i = 0; i < n_wl; ++i)
      if (!(std::isfinite(wavelengths[i]) && wavelengths[i] > 0.0))
        throw Failure{SCATRS_INVALID_INPUT, "wavelengths must be finite and > 0"};
    const int64_t n_units = n_dist * n_wl;
    check_options(options, n_units, n_mu, mu);
    if (n_units == 0) return;
    if (!aspect_ratio || !m || !values)
      throw Failure{SCATRS_INVALID_INPUT, "aspect_ratio, m and values are required"};
    const int64_t n_nodes = options->n_nodes;
    const int L = options->greek_order;
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    // The nodes of each distribution, as the sphere grid's: Gauss-Legendre in ln r over
    // [r_lo, r_hi], weights w u(r) r (engine.rs:1636-1651).
    const auto& gl = rule(c, n_nodes);
    std::vector<double> radius(n_dist * n_nodes), weight(n_dist * n_nodes);
    for (int64_t d = 0; d < n_dist; ++d) {
      std::string msg;
      if (!(dists[d].kind == kTabulated
                ? validate_table(dists[d].table, dists[d].table_len, &msg)
                : validate_distribution(dists[d].kind, dists[d].param, &msg)))
        throw Failure{SCATRS_INVALID_INPUT, "distribution " + std::to_string(d) + ": " + msg};
      if (!(dists[d].r_lo > 0.0 && dists[d].r_hi > dists[d].r_lo && std::isfinite(dists[d].r_hi)))
        throw Failure{SCATRS_INVALID_INPUT, "distribution " + std::to_string(d) +
                                                ": the grid needs 0 < r_lo < r_hi < inf"};
      const double a = std::log(dists[d].r_lo), b = std::log(dists[d].r_hi);
      const double ctr = 0.5 * (a + b), h = 0.5 * (b - a);
      for (int64_t j = 0; j < n_nodes; ++j) {
        const double r = std::exp(ctr + h * gl.first[j]);
        radius[d * n_nodes + j] = r;
        weight[d * n_nodes + j] = h * gl.second[j] * (node_density(dists[d], r) * r);
      }
    }
    // Every node of every unit is one spheroid of the batch (particle.rs:317-366).
    const int64_t n_sph = n_units * n_nodes;
    std::vector<double> xs(n_sph), es(n_sph), ms(2 * n_sph);
    const double pi = 3.14159265358979323846;
    for (int64_t d = 0; d < n_dist; ++d)
      for (int64_t w = 0; w < n_wl; ++w)
        for (int64_t j = 0; j < n_nodes; ++j) {
          const int64_t u = d * n_wl + w, k = u * n_nodes + j;
          xs[k] = 2.0 * pi * radius[d * n_nodes + j] / wavelengths[w];
          es[k] = aspect_ratio[d];
          ms[2 * k] = m[2 * u];
          ms[2 * k + 1] = m[2 * u + 1];
        }
    std::vector<SpheroidResult> res;
    spheroid_solve(c, n_sph, xs.data(), es.data(), ms.data(), tmatrix_rtol, 0, 0, true, res, 0,
                   options->allow_unvalidated != 0);
    // The direct path's per-particle quantities and segment (engine.rs:1207-1339) summed over
    // each unit's nodes in order, then the averages and the outputs of engine.rs:2396-2497.
    std::vector<double> d00, d22, d2m2, d02;
    for (int64_t u = 0; u < n_units; ++u) {
      const int64_t d = u / n_wl;
      double Z = 0, ext = 0, sca = 0, scag = 0, ab = 0, back = 0, r2 = 0, r3 = 0, dep = 0;
      int64_t top = 0;
      for (int64_t j = 0; j < n_nodes; ++j) top = std::max<int64_t>(top, 2 * res[u * n_nodes + j].n);
      const int64_t glen = std::max<int64_t>(top, L) + 1;
      std::vector<double> G(6 * glen, 0.0);
      for (int64_t j = 0; j < n_nodes; ++j) {
        const SpheroidResult& v = res[u * n_nodes + j];
        const double r = radius[d * n_nodes + j], W = weight[d * n_nodes + j];
        const double x = xs[u * n_nodes + j], area = pi * r * r;
        const int64_t have = 2 * (int64_t)v.n + 1;
        // Unnormalized Greek coefficients (alpha1_0 = Q_sca): the raw ones times 4 / x^2.
        const double un = 4.0 / (x * x);
        double depol = 0.0;  // Q_back - Q_sca F22(180 deg) (particle.rs:276-285)
        for (int64_t l = 0; l < have; ++l) {
          const double t = un * (v.greek[l] - 0.5 * (v.greek[have + l] - v.greek[2 * have + l]));
          depol += l % 2 ? -t : t;
        }
        Z += W;
        ext += W * (area * v.q_ext);
        sca += W * (area * v.q_sca);
        scag += W * (area * (v.q_sca * v.g));
        ab += W * (area * v.q_abs);
        back += W * (area * v.q_back);
        r2 += W * (r * r);
        r3 += W * (r * r * r);
        dep += W * (area * depol);
        for (int f = 0; f < 6; ++f)
          for (int64_t l = 0; l < have; ++l) G[f * glen + l] += W * (area * (un * v.greek[f * have + l]));
        if (node_terms) {
          node_terms[2 * (u * n_nodes + j)] = v.n;
          node_terms[2 * (u * n_nodes + j) + 1] = v.nth;
        }
      }
      ext /= Z, sca /= Z, scag /= Z, ab /= Z, back /= Z, r2 /= Z, r3 /= Z, dep /= Z;
      for (double& g : G) g /= Z;
      if (!(std::isfinite(ext) && ext != 0.0 && std::isfinite(sca) && sca != 0.0 &&
            std::isfinite(back) && back != 0.0))
        throw Failure{SCATRS_INVALID_INPUT, "unit " + std::to_string(u) +
                                                ": <C_ext>, <C_sca> or <C_back> is zero or not "
                                                "finite, so the ratios are undefined"};
      const double vals[11] = {ext,        sca,  ab,          back,  sca / ext,     scag / sca,
                               4 * pi * ext / back, dep / (2 * back - dep), r3 / r2, pi * r2,
                               4 * pi / 3 * r3};
      for (int k = 0; k < 11; ++k) values[k * n_units + u] = vals[k];
      if (L >= 0 && greek) {
        const double sc = options->normalized ? 1.0 / G[0] : 1.0;
        for (int f = 0; f < 6; ++f)
          for (int64_t l = 0; l <= L; ++l)
            greek[((int64_t)f * n_units + u) * (L + 1) + l] = l <= top ? sc * G[f * glen + l] : 0.0;
        if (options->normalized) greek[u * (L + 1)] = 1.0;
      }
      if (n_mu > 0 && phase) {
        // The phase matrix from the averaged Greek coefficients, every order to 2N
        // (engine.rs:2359-2390), normalized by <C_sca>.
        const int64_t len = top + 1;
        d00.resize(len);
        d22.resize(len);
        d2m2.resize(len);
        d02.resize(len);
        const double sc = options->normalized ? 1.0 / sca : 1.0;
        for (int64_t j = 0; j < n_mu; ++j) {
          wigner_d(0, 0, mu[j], d00.data(), len);
          wigner_d(2, 2, mu[j], d22.data(), len);
          wigner_d(2, -2, mu[j], d2m2.data(), len);
          wigner_d(0, 2, mu[j], d02.data(), len);
          double f[6] = {0, 0, 0, 0, 0, 0};
          for (int64_t l = 0; l < len; ++l) {
            const double plus = 0.5 * (d22[l] + d2m2[l]), minus = 0.5 * (d22[l] - d2m2[l]);
            f[0] += G[0 * glen + l] * d00[l];
            f[1] += G[4 * glen + l] * d02[l];
            f[2] += G[1 * glen + l] * plus + G[2 * glen + l] * minus;
            f[3] += G[1 * glen + l] * minus + G[2 * glen + l] * plus;
            f[4] += G[5 * glen + l] * d02[l];
            f[5] += G[3 * glen + l] * d00[l];
          }
          for (int k = 0; k < 6; ++k) phase[((int64_t)k * n_units + u) * n_mu + j] = sc * f[k];
        }
      }
    }
  });
}

}  // extern "C"

namespace {
// A value with its derivatives along up to 8 directions (forward mode), for the host assembly of
// the spheroid ensemble's derivative blocks.
struct DualP {
  double v = 0.0;
  double d[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  static int P;
};
int DualP::P = 0;
DualP operator+(const DualP& a, const DualP& b) {
  DualP o;
  o.v = a.v + b.v;
  for (int k = 0; k < DualP::P; ++k) o.d[k] = a.d[k] + b.d[k];
  return o;
}
DualP operator-(const DualP& a, const DualP& b) {
  DualP o;
  o.v = a.v - b.v;
  for (int k = 0; k < DualP::P; ++k) o.d[k] = a.d[k] - b.d[k];
  return o;
}
DualP operator*(const DualP& a, const DualP& b) {
  DualP o;
  o.v = a.v * b.v;
  for (int k = 0; k < DualP::P; ++k) o.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return o;
}
DualP operator*(double a, const DualP& b) {
  DualP o;
  o.v = a * b.v;
  for (int k = 0; k < DualP::P; ++k) o.d[k] = a * b.d[k];
  return o;
}
DualP operator/(const DualP& a, const DualP& b) {
  DualP o;
  o.v = a.v / b.v;
  for (int k = 0; k < DualP::P; ++k) o.d[k] = (a.d[k] - o.v * b.d[k]) / b.v;
  return o;
}
}  // namespace

extern "C" {

int scatrs_ensemble_fixed_spheroid_d(const scatrs_distribution* dists, int64_t n_dist,
                                     const double* wavelengths, int64_t n_wl,
                                     const double* aspect_ratio, const double* m,
                                     const double* mu, int64_t n_mu,
                                     const scatrs_fixed_options* options, double tmatrix_rtol,
                                     double* values, double* phase, double* greek,
                                     double* d_values, double* d_phase, double* d_greek,
                                     int32_t* node_terms, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_dist < 0 || n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    for (int64_t i = 0; i < n_wl; ++i)
      if (!(std::isfinite(wavelengths[i]) && wavelengths[i] > 0.0))
        throw Failure{SCATRS_INVALID_INPUT, "wavelengths must be finite and > 0"};
    const int n_theta = n_dist > 0 ? parameter_count(dists[0].kind) : 2;
    const int P = n_theta + 3;
    const int64_t n_units = n_dist * n_wl;
    check_options(options, n_units, n_mu, mu);
    if (n_units == 0) return;
    if (!aspect_ratio || !m || !values || !d_values)
      throw Failure{SCATRS_INVALID_INPUT, "aspect_ratio, m, values and d_values are required"};
    for (int64_t d = 0; d < n_dist; ++d)
      if (dists[d].kind != dists[0].kind)
        throw Failure{SCATRS_INVALID_INPUT, "derivatives need every distribution of one kind"};
    const int64_t n_nodes = options->n_nodes;
    const int L = options->greek_order;
    if ((L >= 0 && greek && !d_greek) || (n_mu > 0 && phase && !d_phase))
      throw Failure{SCATRS_INVALID_INPUT, "each output array needs its derivative array"};
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    // The nodes and weights as scatrs_ensemble_fixed_spheroid's, with the weights' derivatives
    // along the distribution's parameters (the grid [r_lo, r_hi] held fixed).
    const auto& gl = rule(c, n_nodes);
    std::vector<double> radius(n_dist * n_nodes);
    std::vector<DualP> weight(n_dist * n_nodes);
    DualP::P = P;
    for (int64_t d = 0; d < n_dist; ++d) {
      std::string msg;
      if (!(dists[d].kind == kTabulated
                ? validate_table(dists[d].table, dists[d].table_len, &msg)
                : validate_distribution(dists[d].kind, dists[d].param, &msg)))
        throw Failure{SCATRS_INVALID_INPUT, "distribution " + std::to_string(d) + ": " + msg};
      if (!(dists[d].r_lo > 0.0 && dists[d].r_hi > dists[d].r_lo && std::isfinite(dists[d].r_hi)))
        throw Failure{SCATRS_INVALID_INPUT, "distribution " + std::to_string(d) +
                                                ": the grid needs 0 < r_lo < r_hi < inf"};
      const double a = std::log(dists[d].r_lo), b = std::log(dists[d].r_hi);
      const double ctr = 0.5 * (a + b), h = 0.5 * (b - a);
      for (int64_t j = 0; j < n_nodes; ++j) {
        const double r = std::exp(ctr + h * gl.first[j]);
        radius[d * n_nodes + j] = r;
        double g[3] = {0.0, 0.0, 0.0};
        const double u = dists[d].kind == kTabulated
                             ? node_density(dists[d], r)
                             : density_gradient(dists[d].kind, dists[d].param, r, g);
        DualP& W = weight[d * n_nodes + j];
        W.v = h * gl.second[j] * (u * r);
        for (int k = 0; k < n_theta; ++k) W.d[k] = h * gl.second[j] * (g[k] * r);
      }
    }
    const int64_t n_sph = n_units * n_nodes;
    std::vector<double> xs(n_sph), es(n_sph), ms(2 * n_sph);
    const double pi = 3.14159265358979323846;
    for (int64_t d = 0; d < n_dist; ++d)
      for (int64_t w = 0; w < n_wl; ++w)
        for (int64_t j = 0; j < n_nodes; ++j) {
          const int64_t u = d * n_wl + w, k = u * n_nodes + j;
          xs[k] = 2.0 * pi * radius[d * n_nodes + j] / wavelengths[w];
          es[k] = aspect_ratio[d];
          ms[2 * k] = m[2 * u];
          ms[2 * k + 1] = m[2 * u + 1];
        }
    // Every node converged as the value entry converges it, then its outputs and their
    // derivatives along the aspect ratio, Re m and Im m at that (N, n_theta).
    std::vector<SpheroidResult> res;
    spheroid_solve(c, n_sph, xs.data(), es.data(), ms.data(), tmatrix_rtol, 0, 0, false, res, 0,
                   options->allow_unvalidated != 0);
    std::vector<SphEval> base(n_sph);
    int top_all = 0;
    for (int64_t k = 0; k < n_sph; ++k) {
      base[k] = {xs[k], es[k], ms[2 * k], ms[2 * k + 1], res[k].n, res[k].nth};
      top_all = std::max(top_all, 2 * res[k].n);
      if (node_terms) {
        node_terms[2 * k] = res[k].n;
        node_terms[2 * k + 1] = res[k].nth;
      }
    }
    std::vector<std::vector<double>> val, dd4[4];
    spheroid_fixed_outputs(c, base, top_all, false, val, 0);
    spheroid_fixed_derivs(c, base, top_all, false, dd4, 0, 0xEu);
    const int64_t gl_all = (int64_t)top_all + 1;
    // Node k's output q as a dual: its derivatives along the aspect ratio, Re m and Im m in
    // directions n_theta .. n_theta + 2.
    auto node_out = [&](int64_t k, int64_t q) {
      DualP o;
      o.v = val[k][q];
      for (int dir = 1; dir < 4; ++dir) o.d[n_theta + dir - 1] = dd4[dir][k][q];
      return o;
    };
    std::vector<double> d00, d22, d2m2, d02;
    auto put = [&](double* v, double* dv, int64_t idx, int64_t block, const DualP& x) {
      v[idx] = x.v;
      for (int k = 0; k < P; ++k) dv[k * block + idx] = x.d[k];
    };
    for (int64_t u = 0; u < n_units; ++u) {
      const int64_t d = u / n_wl;
      DualP Z, ext, sca, scag, ab, back, r2, r3, dep;
      int64_t top = 0;
      for (int64_t j = 0; j < n_nodes; ++j) top = std::max<int64_t>(top, 2 * res[u * n_nodes + j].n);
      const int64_t glen = std::max<int64_t>(top, L) + 1;
      std::vector<DualP> G(6 * glen);
      for (int64_t j = 0; j < n_nodes; ++j) {
        const int64_t k = u * n_nodes + j;
        const double r = radius[d * n_nodes + j], area = pi * r * r;
        const DualP& W = weight[d * n_nodes + j];
        const int64_t have = 2 * (int64_t)res[k].n + 1;
        const DualP q_ext = node_out(k, 0), q_sca = node_out(k, 1), q_abs = node_out(k, 2);
        const DualP q_back = node_out(k, 3), g = node_out(k, 4);
        DualP depol;  // Q_back - Q_sca F22(180 deg) (particle.rs:276-285)
        for (int64_t l = 0; l < have; ++l) {
          const DualP t = node_out(k, 5 + l) -
                          0.5 * (node_out(k, 5 + gl_all + l) - node_out(k, 5 + 2 * gl_all + l));
          depol = l % 2 ? depol - t : depol + t;
        }
        Z = Z + W;
        ext = ext + W * (area * q_ext);
        sca = sca + W * (area * q_sca);
        scag = scag + W * (area * (q_sca * g));
        ab = ab + W * (area * q_abs);
        back = back + W * (area * q_back);
        DualP rr;
        rr.v = r * r;
        r2 = r2 + W * rr;
        rr.v = r * r * r;
        r3 = r3 + W * rr;
        dep = dep + W * (area * depol);
        for (int f = 0; f < 6; ++f)
          for (int64_t l = 0; l < have; ++l)
            G[f * glen + l] = G[f * glen + l] + W * (area * node_out(k, 5 + f * gl_all + l));
      }
      ext = ext / Z, sca = sca / Z, scag = scag / Z, ab = ab / Z, back = back / Z;
      r2 = r2 / Z, r3 = r3 / Z, dep = dep / Z;
      for (DualP& gg : G) gg = gg / Z;
      if (!(std::isfinite(ext.v) && ext.v != 0.0 && std::isfinite(sca.v) && sca.v != 0.0 &&
            std::isfinite(back.v) && back.v != 0.0))
        throw Failure{SCATRS_INVALID_INPUT, "unit " + std::to_string(u) +
                                                ": <C_ext>, <C_sca> or <C_back> is zero or not "
                                                "finite, so the ratios are undefined"};
      const DualP vals[11] = {ext,  sca, ab, back, sca / ext, scag / sca,
                              (4 * pi) * ext / back, dep / (2.0 * back - dep), r3 / r2,
                              pi * r2, (4 * pi / 3) * r3};
      for (int k = 0; k < 11; ++k) put(values, d_values, k * n_units + u, 11 * n_units, vals[k]);
      if (L >= 0 && greek) {
        DualP one;
        one.v = 1.0;
        const DualP sc = options->normalized ? one / G[0] : one;
        const int64_t block = 6 * n_units * ((int64_t)L + 1);
        for (int f = 0; f < 6; ++f)
          for (int64_t l = 0; l <= L; ++l) {
            const DualP gv = l <= top ? sc * G[f * glen + l] : DualP{};
            put(greek, d_greek, ((int64_t)f * n_units + u) * (L + 1) + l, block, gv);
          }
        if (options->normalized) put(greek, d_greek, u * (L + 1), block, one);
      }
      if (n_mu > 0 && phase) {
        const int64_t len = top + 1;
        d00.resize(len);
        d22.resize(len);
        d2m2.resize(len);
        d02.resize(len);
        DualP one;
        one.v = 1.0;
        const DualP sc = options->normalized ? one / sca : one;
        const int64_t block = 6 * n_units * n_mu;
        for (int64_t j = 0; j < n_mu; ++j) {
          wigner_d(0, 0, mu[j], d00.data(), len);
          wigner_d(2, 2, mu[j], d22.data(), len);
          wigner_d(2, -2, mu[j], d2m2.data(), len);
          wigner_d(0, 2, mu[j], d02.data(), len);
          DualP f[6];
          for (int64_t l = 0; l < len; ++l) {
            const double plus = 0.5 * (d22[l] + d2m2[l]), minus = 0.5 * (d22[l] - d2m2[l]);
            f[0] = f[0] + d00[l] * G[0 * glen + l];
            f[1] = f[1] + d02[l] * G[4 * glen + l];
            f[2] = f[2] + plus * G[1 * glen + l] + minus * G[2 * glen + l];
            f[3] = f[3] + minus * G[1 * glen + l] + plus * G[2 * glen + l];
            f[4] = f[4] + d02[l] * G[5 * glen + l];
            f[5] = f[5] + d00[l] * G[3 * glen + l];
          }
          for (int k = 0; k < 6; ++k)
            put(phase, d_phase, ((int64_t)k * n_units + u) * n_mu + j, block, sc * f[k]);
        }
      }
    }
  });
}

int scatrs_ensemble_fixed_layered(const scatrs_distribution* dists, int64_t n_dist,
                                  const double* wavelengths, int64_t n_wl,
                                  const scatrs_layers* layers, const double* mu, int64_t n_mu,
                                  const scatrs_fixed_options* options, double* values,
                                  double* phase, double* greek, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_dist < 0 || n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    if (!layers || layers->n_layers < 1 || (layers->n_layers > 1 && !layers->fractions) ||
        !layers->m)
      throw Failure{SCATRS_INVALID_INPUT, "layers must give n_layers >= 1, fractions and m"};
    for (int64_t i = 0; i < n_wl; ++i)
      if (!(std::isfinite(wavelengths[i]) && wavelengths[i] > 0.0))
        throw Failure{SCATRS_INVALID_INPUT, "wavelengths must be finite and > 0"};
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    cudaStream_t s = 0;
    const int64_t n_units = n_dist * n_wl;
    check_options(options, n_units, n_mu, mu);
    if (n_units == 0) return;
    const int L = layers->n_layers;
    double* wl_d = c.wl.as<double>(n_wl);
    SB_CUDA(cudaMemcpyAsync(wl_d, wavelengths, n_wl * 8, cudaMemcpyHostToDevice, s));
    LayerInput li;
    li.n_layers = L;
    li.fractions = layers->fractions;
    double* m_d;
    if (L == 1) {
      m_d = c.m.as<double>(2 * n_units);
      SB_CUDA(cudaMemcpyAsync(m_d, layers->m, 2 * n_units * 8, cudaMemcpyHostToDevice, s));
    } else {
      m_d = c.m.as<double>(2 * n_dist * L * n_wl);
      SB_CUDA(cudaMemcpyAsync(m_d, layers->m, 2 * n_dist * L * n_wl * 8, cudaMemcpyHostToDevice,
                              s));
      li.m_dev = m_d;
    }
    int64_t vl, pl, gl;
    scatrs_ensemble_fixed_sizes(n_units, n_mu, options->greek_order, &vl, &pl, &gl);
    double* v_d = c.values.as<double>(vl);
    double* p_d = pl > 0 ? c.phase.as<double>(pl) : nullptr;
    double* g_d = gl > 0 ? c.greek.as<double>(gl) : nullptr;
    FixedCall call;
    call.wl_host.assign(wavelengths, wavelengths + n_wl);
    run_fixed(c, dists, n_dist, wl_d, n_wl, m_d, mu, n_mu, options, v_d, p_d, g_d, s, &call, li);
    check_device_errors(c, s, &call);
    SB_CUDA(cudaMemcpyAsync(values, v_d, vl * 8, cudaMemcpyDeviceToHost, s));
    if (pl > 0 && phase) SB_CUDA(cudaMemcpyAsync(phase, p_d, pl * 8, cudaMemcpyDeviceToHost, s));
    if (gl > 0 && greek) SB_CUDA(cudaMemcpyAsync(greek, g_d, gl * 8, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"

namespace sb {
namespace {
// scatrs_ensemble_fixed_layered_d with host (device = false) or device arrays (the layers' m,
// the wavelengths and the outputs).
void fixed_layered_d_impl(const scatrs_distribution* dists, int64_t n_dist,
                          const double* wavelengths, int64_t n_wl, const scatrs_layers* layers,
                          const double* mu, int64_t n_mu, const scatrs_fixed_options* options,
                          double* values, double* phase, double* greek, double* d_values,
                          double* d_phase, double* d_greek, bool device, cudaStream_t s) {
  {
    if (n_dist < 0 || n_wl < 0) throw Failure{SCATRS_INVALID_INPUT, "negative sizes"};
    if (!layers || layers->n_layers < 2 || !layers->fractions || !layers->m)
      throw Failure{SCATRS_INVALID_INPUT,
                    "layers must give n_layers >= 2, fractions and m (one layer: use "
                    "scatrs_ensemble_fixed_d)"};
    const int L = layers->n_layers;
    if (L > kMaxLayersAbi) throw Failure{SCATRS_INVALID_INPUT, "the GPU path takes 1 to 16 layers"};
    const int P_th = n_dist > 0 ? parameter_count(dists[0].kind) : 2;
    const int P = P_th + 2 * L + (L - 1);
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    const std::vector<double> wl_host = host_wavelengths(wavelengths, n_wl, device, s);
    const cudaMemcpyKind in = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind out = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const int64_t n_units = n_dist * n_wl;
    check_options(options, n_units, n_mu, mu, P);
    if (n_units == 0) return;
    double* wl_d = c.wl.as<double>(n_wl);
    SB_CUDA(cudaMemcpyAsync(wl_d, wavelengths, n_wl * 8, in, s));
    LayerInput li;
    li.n_layers = L;
    li.fractions = layers->fractions;
    double* m_d = c.m.as<double>(2 * n_dist * L * n_wl);
    SB_CUDA(cudaMemcpyAsync(m_d, layers->m, 2 * n_dist * L * n_wl * 8, in, s));
    li.m_dev = m_d;
    int64_t vl, pl, gl;
    scatrs_ensemble_fixed_sizes(n_units, n_mu, options->greek_order, &vl, &pl, &gl);
    if (device && ((pl > 0 && (!phase || !d_phase)) || (gl > 0 && (!greek || !d_greek)) ||
                   !values || !d_values))
      throw Failure{SCATRS_INVALID_INPUT,
                    "the device entry needs every output array the options call for"};
    const int Pp = P_th + 2;  // blocks of one pass: the parameters, then the direction and i x it
    double* v_d = c.values.as<double>(vl * (1 + Pp));
    double* p_d = pl > 0 ? c.phase.as<double>(pl * (1 + Pp)) : nullptr;
    double* g_d = gl > 0 ? c.greek.as<double>(gl * (1 + Pp)) : nullptr;
    // One pass per direction group: layer l's index (its Re and Im blocks), then each fraction
    // (its block; the pass's second block is discarded). Blocks out: the distribution's
    // parameters, Re m_l and Im m_l per layer, then f_1..f_{L-1}.
    for (int g = 0; g < 2 * L - 1; ++g) {
      DerivOutput dv;
      dv.on = true;
      dv.n_theta = P_th;
      dv.dir = g;
      dv.d_values = v_d + vl;
      dv.d_phase = p_d ? p_d + pl : nullptr;
      dv.d_greek = g_d ? g_d + gl : nullptr;
      FixedCall call;
      call.wl_host = wl_host;
      run_fixed(c, dists, n_dist, wl_d, n_wl, m_d, mu, n_mu, options, v_d, p_d, g_d, s, &call, li,
                dv);
      check_device_errors(c, s, &call);
      auto take = [&](int from, int to) {
        if (d_values)
          SB_CUDA(cudaMemcpyAsync(d_values + to * vl, dv.d_values + from * vl, vl * 8,
                                  out, s));
        if (pl > 0 && d_phase)
          SB_CUDA(cudaMemcpyAsync(d_phase + to * pl, dv.d_phase + from * pl, pl * 8,
                                  out, s));
        if (gl > 0 && d_greek)
          SB_CUDA(cudaMemcpyAsync(d_greek + to * gl, dv.d_greek + from * gl, gl * 8,
                                  out, s));
      };
      if (g == 0) {
        for (int p = 0; p < P_th; ++p) take(p, p);
        SB_CUDA(cudaMemcpyAsync(values, v_d, vl * 8, out, s));
        if (pl > 0 && phase)
          SB_CUDA(cudaMemcpyAsync(phase, p_d, pl * 8, out, s));
        if (gl > 0 && greek)
          SB_CUDA(cudaMemcpyAsync(greek, g_d, gl * 8, out, s));
      }
      if (g < L) {
        take(P_th, P_th + 2 * g);
        take(P_th + 1, P_th + 2 * g + 1);
      } else {
        take(P_th, P_th + 2 * L + (g - L));
      }
      SB_CUDA(cudaStreamSynchronize(s));
    }
  }
}
}  // namespace
}  // namespace sb

extern "C" {

int scatrs_ensemble_fixed_layered_d(const scatrs_distribution* dists, int64_t n_dist,
                                    const double* wavelengths, int64_t n_wl,
                                    const scatrs_layers* layers, const double* mu, int64_t n_mu,
                                    const scatrs_fixed_options* options, double* values,
                                    double* phase, double* greek, double* d_values,
                                    double* d_phase, double* d_greek, char* err,
                                    size_t err_len) {
  return guarded(err, err_len, [&] {
    fixed_layered_d_impl(dists, n_dist, wavelengths, n_wl, layers, mu, n_mu, options, values,
                         phase, greek, d_values, d_phase, d_greek, false, 0);
  });
}

int scatrs_ensemble_fixed_layered_d_device(const scatrs_distribution* dists_host,
                                           int64_t n_dist, const double* wavelengths_dev,
                                           int64_t n_wl, const scatrs_layers* layers,
                                           const double* mu_host, int64_t n_mu,
                                           const scatrs_fixed_options* options,
                                           double* values_dev, double* phase_dev,
                                           double* greek_dev, double* d_values_dev,
                                           double* d_phase_dev, double* d_greek_dev,
                                           void* stream, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    fixed_layered_d_impl(dists_host, n_dist, wavelengths_dev, n_wl, layers, mu_host, n_mu,
                         options, values_dev, phase_dev, greek_dev, d_values_dev, d_phase_dev,
                         d_greek_dev, true, static_cast<cudaStream_t>(stream));
  });
}

int scatrs_ensemble_fixed_device(const scatrs_distribution* dists_host, int64_t n_dist,
                                 const double* wavelengths_dev, int64_t n_wl,
                                 const double* m_dev, const double* mu_host, int64_t n_mu,
                                 const scatrs_fixed_options* options, double* values_dev,
                                 double* phase_dev, double* greek_dev, void* stream, char* err,
                                 size_t err_len) {
  return fixed_device(dists_host, n_dist, wavelengths_dev, n_wl, m_dev, mu_host, n_mu, options,
                      values_dev, phase_dev, greek_dev, stream, nullptr, err, err_len);
}

int scatrs_check_errors(void* stream, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    check_device_errors(c, static_cast<cudaStream_t>(stream), &g_last_call);
  });
}

int scatrs_mie(const double* x, const double* m, int64_t n, int32_t allow_unvalidated,
               int64_t* n_terms, const int64_t* coeff_offset, double* coeffs, double* eff,
               char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n <= 0) return;
    Context& c = context();
    std::lock_guard<std::mutex> lk(c.mtx);
    cudaStream_t s = 0;
    DevBuf xb, mb, nb, ob, cb, eb, uzb, uxb;
    struct Free {
      DevBuf* b[8];
      ~Free() {
        for (auto* p : b) p->release();
      }
    } guard{{&xb, &mb, &nb, &ob, &cb, &eb, &uzb, &uxb}};
    double* xd = xb.as<double>(n);
    double2* md = mb.as<double2>(n);
    int64_t* nd = nb.as<int64_t>(n);
    SB_CUDA(cudaMemcpyAsync(xd, x, n * 8, cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(md, m, n * 16, cudaMemcpyHostToDevice, s));
    unsigned long long* errw = c.err.as<unsigned long long>(2);
    SB_CUDA(cudaMemsetAsync(errw, 0xff, 16, s));
    MieNodesArgs a{};
    a.x = xd;
    a.m = md;
    a.n = n;
    a.n_terms = nd;
    a.err = errw;
    a.allow_unvalidated = allow_unvalidated;
    int64_t bound = 0;
    if (coeffs) {
      // Sized from the default truncation of the largest sphere; the exact total follows
      // from the terms the kernel reports.
      double xmax = 0.0;
      int64_t off_max = 0;
      for (int64_t i = 0; i < n; ++i) {
        xmax = std::max(xmax, x[i]);
        off_max = std::max(off_max, coeff_offset[i]);
      }
      bound = off_max + (int64_t)std::ceil(xmax + 6.0 * std::cbrt(xmax) + 3.0);
      int64_t* od = ob.as<int64_t>(n);
      SB_CUDA(cudaMemcpyAsync(od, coeff_offset, n * 8, cudaMemcpyHostToDevice, s));
      a.coeff_offset = od;
      a.coeffs = cb.as<double>(4 * bound);
      a.uz = uzb.as<double2>(bound + 2 * n);
      a.ux = uxb.as<double>(bound + 2 * n);
    }
    if (eff) a.eff = eb.as<double>(5 * n);
    timed_launch(K_NODES, s, [&] { launch_mie_nodes(a, s); });
    SB_CUDA(cudaGetLastError());
    unsigned long long h[2];
    SB_CUDA(cudaMemcpyAsync(h, errw, 16, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    if (h[0] != ~0ull) {
      int64_t t = (int64_t)(h[0] >> 2);
      char buf[200];
      snprintf(buf, sizeof buf, "sphere %lld (x = %e): %s", (long long)t, x[t],
               (h[0] & 3) == 3 ? "outside the validated domain" : "invalid input");
      throw Failure{(int)(h[0] & 3), buf};
    }
    SB_CUDA(cudaMemcpyAsync(n_terms, nd, n * 8, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    if (coeffs) {
      int64_t total = 0;
      for (int64_t i = 0; i < n; ++i) total = std::max(total, coeff_offset[i] + n_terms[i]);
      if (total > bound) throw Failure{SCATRS_INVALID_INPUT, "coeff_offset is not the prefix sum of n_terms"};
      SB_CUDA(cudaMemcpyAsync(coeffs, a.coeffs, 4 * total * 8, cudaMemcpyDeviceToHost, s));
    }
    if (eff) SB_CUDA(cudaMemcpyAsync(eff, a.eff, 5 * n * 8, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
  });
}

int64_t scatrs_greek_all_width(void) { return t_greek_all.width; }

int scatrs_greek_all_take(double* greek, double* greek_err, double* d_greek, double* d_greek_err) {
  const GreekAll& ga = t_greek_all;
  if (greek) std::copy(ga.g.begin(), ga.g.end(), greek);
  if (greek_err) std::copy(ga.ge.begin(), ga.ge.end(), greek_err);
  if (d_greek) std::copy(ga.dg.begin(), ga.dg.end(), d_greek);
  if (d_greek_err) std::copy(ga.dge.begin(), ga.dge.end(), d_greek_err);
  return SCATRS_OK;
}

int scatrs_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return -1;
  return n;
}

int64_t scatrs_launch_count(void) { return g_launches.load(); }

void scatrs_gauss_legendre(int64_t n, double* nodes, double* weights) {
  if (n < 1 || n > sb::kMaxGaussPoints || !nodes || !weights) return;
  sb::gauss_legendre(n, nodes, weights);
}

int scatrs_testing_raise(int32_t status, const char* message, double achieved,
                        double requested, char* err, size_t err_len) {
  return sb::guarded(err, err_len, [&] {
    if (status < SCATRS_INVALID_INPUT || status > SCATRS_NO_DEVICE) return;
    throw sb::Failure{status, message ? message : "", achieved, requested};
  });
}

void scatrs_testing_fail_allocation(int64_t after) { sb::g_fail_allocation = after; }

void scatrs_testing_force_node_error(int64_t unit_key, int32_t status) {
  sb::g_forced_node_error = unit_key < 0 ? ~0ull
                                         : ((unsigned long long)unit_key << 2) |
                                               (unsigned long long)(status & 3);
}

int scatrs_not_converged_detail(double* achieved, double* requested) {
  if (achieved) *achieved = sb::g_last_achieved;
  if (requested) *requested = sb::g_last_requested;
  return sb::g_last_status == SCATRS_NOT_CONVERGED ? 1 : 0;
}

int scatrs_set_tuning(const scatrs_tuning* t, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!t) throw Failure{SCATRS_INVALID_INPUT, "tuning: null settings"};
    const int split = t->split == 0 ? kDefaultSplit : t->split;
    const int64_t rows = t->arena_rows == 0 ? kArenaRows : t->arena_rows;
    if (split < 1 || split > 64)
      throw Failure{SCATRS_INVALID_INPUT, "tuning: split must be in 1..64 (0: 4)"};
    if (rows < (1 << 16) || rows > (1 << 24))
      throw Failure{SCATRS_INVALID_INPUT, "tuning: arena_rows must be in 2^16..2^24 (0: 2^22)"};
    g_split.store(split);
    g_arena_rows.store(rows);
  });
}

int scatrs_get_tuning(scatrs_tuning* t) {
  if (!t) return SCATRS_INVALID_INPUT;
  t->split = g_split.load();
  t->reserved = 0;
  t->arena_rows = g_arena_rows.load();
  return SCATRS_OK;
}

int64_t scatrs_limit(int32_t which) {
  switch (which) {
    case SCATRS_LIMIT_MIE_ORDER: return sb::kMaxMieOrder;
    case SCATRS_LIMIT_MIE_VALUES: return sb::kMaxMieValues;
    case SCATRS_LIMIT_GREEK_ORDER: return sb::kMaxGreekOrder;
    case SCATRS_LIMIT_LAYERS: return sb::kMaxLayersAbi;
    case SCATRS_LIMIT_TMATRIX_ORDER: return sb::kMaxTmatrixOrder;
    case SCATRS_LIMIT_GAUSS_LEGENDRE_POINTS: return sb::kMaxGaussPoints;
    case SCATRS_LIMIT_WIGNER_D_VALUES: return sb::kMaxWignerValues;
    default: return -1;
  }
}

void scatrs_set_profiling(int32_t on) {
  sb::g_profiling = on != 0;
  for (auto& t : sb::g_timed) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  sb::g_timed.clear();
  for (int k = 0; k < sb::K_COUNT; ++k) {
    sb::g_kernel_ms[k] = 0.0;
    sb::g_kernel_launches[k] = 0;
  }
  sb::g_tm_pair_nodes.clear();
}

int64_t scatrs_spheroid_work(int64_t* per_launch, int64_t cap) {
  for (int64_t k = 0; k < cap && k < (int64_t)sb::g_tm_pair_nodes.size(); ++k)
    per_launch[k] = sb::g_tm_pair_nodes[k];
  return (int64_t)sb::g_tm_pair_nodes.size();
}

int scatrs_kernel_times(double* ms, int64_t* launches, int32_t n) {
  for (auto& t : sb::g_timed) {
    float v = 0.0f;
    if (cudaEventSynchronize(t.b) == cudaSuccess && cudaEventElapsedTime(&v, t.a, t.b) == cudaSuccess) {
      sb::g_kernel_ms[t.id] += v;
      sb::g_kernel_launches[t.id] += 1;
    }
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  sb::g_timed.clear();
  for (int k = 0; k < n && k < sb::K_COUNT; ++k) {
    ms[k] = sb::g_kernel_ms[k];
    launches[k] = sb::g_kernel_launches[k];
  }
  return sb::K_COUNT;
}

void scatrs_release(void) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  std::lock_guard<std::mutex> lk(g_ctx_mtx);
  if (dev < (int)g_ctx.size() && g_ctx[dev]) {
    Context& c = *g_ctx[dev];
    for (DevBuf* b : {&c.radius, &c.weight, &c.wtheta, &c.wthdiff, &c.wdiff, &c.unit_norm, &c.wl, &c.m, &c.fractions, &c.chunk_n, &c.chunk_n_slab,
                      &c.chunk_row, &c.chunk_acc, &c.plan_units, &c.unit_acc, &c.unit_slots,
                      &c.slots, &c.items, &c.proj_items, &c.slot_index, &c.slot_greek,
                      &c.X, &c.uz, &c.ux, &c.chunk_sums, &c.err, &c.acc,
                      &c.counter, &c.values, &c.phase, &c.greek, &c.user.ge, &c.user.go,
                      &c.user.map, &c.tc_a_hi, &c.tc_a_lo, &c.tc_prod, &c.tc_err, &c.xdig,
                      &c.xside, &c.colmax, &c.chunk_xoff, &c.chunk_xidx, &c.i8_list, &c.i8_err,
                      &c.i8.dig, &c.i8.scale, &c.i8.user_d, &c.i8.band_d})
      b->release();
    for (auto& kv : c.projectors)
      for (DevBuf* b : {&kv.second.d, &kv.second.d_hi, &kv.second.d_lo}) b->release();
    for (auto& kv : c.bands)
      for (DevBuf* b : {&kv.second.ge_d, &kv.second.go_d, &kv.second.d_d, &kv.second.desc_d})
        b->release();
    if (c.pinned_chunk_n) cudaFreeHost(c.pinned_chunk_n);
    for (int h = 0; h < 2; ++h)
      if (c.staged[h]) {
        cudaEventSynchronize(c.staged[h]);
        cudaEventDestroy(c.staged[h]);
      }
    if (c.staging) cudaFreeHost(c.staging);
    g_ctx[dev].reset();
  }
}

}  // extern "C"
