// scatrs_mie_static: the batched Mie solve for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a plugin running inside a host process that owns every
// device allocation through its own pool, code replayed where allocation is forbidden, or a
// real-time loop that must not risk an allocation failure or the implicit synchronization of
// cudaMalloc/cudaFree. They hand this entry point device buffers for the inputs and outputs; the
// recurrences' scratch lives in a fixed array compiled into this library instead of a
// per-call allocation.
//
// The array (kStaticRows rows of u_k(mx) and u_k(x), 24 bytes each: 12 MiB) is a file-scope
// __device__ array, so every GPU that loads the library holds it until the process exits. All
// calls on a device share it and it keeps the last call's contents: two calls that overlap on the
// GPU (on different streams, or from different host threads) race on it and must not be issued.
// The first call on each device resolves the array's device address (cudaGetSymbolAddress) with
// that device current, and again whenever the device's current CUDA context has changed (a
// symbol's address belongs to a context); make that first call before any stream capture.
//
// Compiled with -fmad=false, like the allocating entry point (scatrs_mie), whose results this
// one reproduces bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/scatrs_b200.h"
#include "mie_device.cuh"

namespace sb {
namespace {

constexpr int64_t kStaticRows = 1 << 19;
constexpr int kMaxDevices = 64;

// Rows 0..kStaticRows-1 of u_k(mx) (2 doubles each) followed by as many rows of u_k(x).
static __device__ __align__(256) double g_scratch[3 * kStaticRows];
// The first failing sphere (index << 2 | status), all ones when none; set to all ones by each
// call before its launch.
static __device__ __align__(256) unsigned long long g_status;

// The arrays' device addresses, resolved per device and per CUDA context: a symbol's address
// belongs to the context that loaded the module, so a new primary context (after
// cudaDeviceReset) or a caller's own context on the same device resolves them again.
struct Resolved {
  void* ctx = nullptr;
  double* scratch = nullptr;
  unsigned long long* status = nullptr;
};
std::mutex g_mtx;
Resolved g_resolved[kMaxDevices];

// The current context's handle (the driver's cuCtxGetCurrent, reached through the runtime so
// that the library needs no link to libcuda); nullptr when it cannot be read.
void* current_context() {
  using GetCurrent = int (*)(void**);
  static GetCurrent fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return GetCurrent(nullptr);
    }
    return reinterpret_cast<GetCurrent>(p);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// The batched Mie solve with its scratch in the static array: sphere t writes coefficient
// terms [coeff_offset[t], coeff_offset[t] + N_t) and uses scratch rows
// [coeff_offset[t] + 2t, coeff_offset[t] + 2t + N_t + 2). Before any write, a sphere whose terms
// start below 0, pass total_terms or reach the next sphere's offset is rejected (status 2): the
// device's own N_t decides, so a caller whose N_t differs (a host cbrt that rounds the other way
// at an integer boundary) gets an error, never a write outside its buffers. With every sphere
// accepted the ranges are disjoint and inside [0, total_terms), and since the host checked
// total_terms + 2n <= kStaticRows, the scratch rows stay inside the array too.
__global__ void __launch_bounds__(128)
    mie_nodes_static_kernel(const double* __restrict__ x_in, const double2* __restrict__ m_in,
                            int64_t n, int allow_unvalidated, int64_t total_terms,
                            int64_t* n_terms, const int64_t* __restrict__ coeff_offset,
                            double* coeffs, double* eff, double* scratch,
                            unsigned long long* status) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double x = x_in[t];
  const cplx m = mk(m_in[t].x, m_in[t].y);
  const int64_t nt = default_n_max(x);
  int st = check_node(x, m, nt, allow_unvalidated != 0);
  const int64_t off = coeff_offset[t];
  const int64_t end = t + 1 < n ? coeff_offset[t + 1] : total_terms;
  if (st == 0 && (off < 0 || off + nt > end || end > total_terms ||
                  off + 2 * t + nt + 2 > kStaticRows))
    st = 2;  // the caller's layout does not hold this sphere's terms
  if (st != 0) {
    atomicMin(status, ((unsigned long long)t << 2) | (unsigned long long)st);
    return;
  }
  n_terms[t] = nt;
  Scratch s;
  s.uz = reinterpret_cast<double2*>(scratch) + off + 2 * t;
  s.ux = scratch + 2 * kStaticRows + off + 2 * t;
  s.stride = 1;
  mie_prepare(x, m, nt, s);
  ValueSums vs;
  double2* out = reinterpret_cast<double2*>(coeffs) + 2 * off;
  const double asum = mie_finish(x, m, nt, s, vs, [&](int64_t k, cplx an, cplx bn) {
    out[k - 1] = make_double2(an.re, an.im);
    out[nt + k - 1] = make_double2(bn.re, bn.im);
  });
  const Eff e = efficiencies_from(x, asum, vs);
  if (eff) {
    eff[5 * t] = e.q_ext;
    eff[5 * t + 1] = e.q_sca;
    eff[5 * t + 2] = e.q_abs;
    eff[5 * t + 3] = e.q_back;
    eff[5 * t + 4] = e.g;
  }
}

void put(char* err, size_t len, const char* msg) {
  if (err && len > 0) snprintf(err, len, "%s", msg);
}

}  // namespace
}  // namespace sb

extern "C" int scatrs_mie_static(const double* x, const double* m, int64_t n,
                                 int32_t allow_unvalidated, int64_t total_terms,
                                 int64_t* n_terms, const int64_t* coeff_offset, double* coeffs,
                                 double* eff, void* stream, char* err, size_t err_len) {
  using namespace sb;
  if (n < 0 || total_terms < 0) {
    put(err, err_len, "n and total_terms must be >= 0");
    return SCATRS_INVALID_INPUT;
  }
  if (n == 0) return SCATRS_OK;
  if (total_terms + 2 * n > kStaticRows) {
    char buf[200];
    snprintf(buf, sizeof buf,
             "the spheres need %lld scratch rows (sum of N + 2 per sphere); the static array "
             "holds %lld",
             (long long)(total_terms + 2 * n), (long long)kStaticRows);
    put(err, err_len, buf);
    return SCATRS_INVALID_INPUT;
  }
  if (!x || !m || !n_terms || !coeff_offset || !coeffs) {
    put(err, err_len, "x, m, n_terms, coeff_offset and coeffs must be device pointers");
    return SCATRS_INVALID_INPUT;
  }
  int dev = 0;
  cudaError_t rc = cudaGetDevice(&dev);
  if (rc != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    put(err, err_len, rc != cudaSuccess ? cudaGetErrorString(rc) : "device index out of range");
    return SCATRS_CUDA;
  }
  double* scratch;
  unsigned long long* status;
  {
    std::lock_guard<std::mutex> lk(g_mtx);
    // No context yet (the runtime creates the primary context lazily) reads as nullptr and
    // resolves; resolving creates it, and its handle is recorded after.
    void* ctx = current_context();
    Resolved& r = g_resolved[dev];
    if (!r.scratch || !ctx || r.ctx != ctx) {
      void* p = nullptr;
      void* q = nullptr;
      rc = cudaGetSymbolAddress(&p, g_scratch);
      if (rc == cudaSuccess) rc = cudaGetSymbolAddress(&q, g_status);
      if (rc != cudaSuccess) {
        r = Resolved{};
        put(err, err_len, cudaGetErrorString(rc));
        return SCATRS_CUDA;
      }
      r.ctx = current_context();
      r.scratch = static_cast<double*>(p);
      r.status = static_cast<unsigned long long*>(q);
    }
    scratch = r.scratch;
    status = r.status;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  rc = cudaMemsetAsync(status, 0xff, sizeof(unsigned long long), s);
  if (rc == cudaSuccess) {
    const int threads = 128;
    const int blocks = (int)((n + threads - 1) / threads);
    mie_nodes_static_kernel<<<blocks, threads, 0, s>>>(
        x, reinterpret_cast<const double2*>(m), n, allow_unvalidated, total_terms, n_terms,
        coeff_offset, coeffs, eff, scratch, status);
    rc = cudaGetLastError();
  }
  unsigned long long h = ~0ull;
  if (rc == cudaSuccess) rc = cudaMemcpyAsync(&h, status, sizeof h, cudaMemcpyDeviceToHost, s);
  if (rc == cudaSuccess) rc = cudaStreamSynchronize(s);
  if (rc != cudaSuccess) {
    put(err, err_len, cudaGetErrorString(rc));
    return SCATRS_CUDA;
  }
  if (h != ~0ull) {
    const int st = (int)(h & 3);
    char buf[320];
    snprintf(buf, sizeof buf, "sphere %lld: %s", (long long)(h >> 2),
             st == 3   ? "outside the validated domain"
             : st == 2 ? "its N terms do not fit the caller's layout (coeff_offset is not the "
                         "exclusive prefix sum of N = ceil(x + 6 x^(1/3) + 3), or total_terms "
                         "is too small); nothing was written for it"
                       : "invalid input");
    put(err, err_len, buf);
    return st == 3 ? SCATRS_OUTSIDE_VALIDATED_DOMAIN : SCATRS_INVALID_INPUT;
  }
  return SCATRS_OK;
}
