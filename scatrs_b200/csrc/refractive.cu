// Refractive-index models m(lambda) on the device (python/scatrs/refractive.py:168-368): a
// constant, a table interpolated linearly in lambda (Re m and Im m, or ln Im m), Cauchy's law
// n = A + B / lambda^2 + C / lambda^4 and Sellmeier's n^2 = 1 + sum_i B_i lambda^2 /
// (lambda^2 - C_i), each with Im m = k and the derivatives of m along the model's parameters, so
// that the ensemble's index array, and its chain rule, stay on the device. One thread per
// (model, wavelength); the first failure in (model, wavelength) order is reported.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/scatrs_b200.h"
#include "kernels.h"

namespace sb {

namespace {

// One model on the device: its kind, its table or its terms at data[off ...].
struct DevModel {
  int kind, n;
  double p[4];
  int64_t off;
};

// m at lambda and, when dm is given, dm/dtheta (complex, P entries); status 0, or 1 when the
// wavelength is outside a table, 2 when Sellmeier's n^2 is not positive and finite.
__device__ int eval_model(const DevModel& md, const double* __restrict__ data, double lam,
                          double2& m, double2* dm, int stride) {
  switch (md.kind) {
    case SCATRS_M_CONSTANT:
      // refractive.py:168-198: parameters n, k.
      m = make_double2(md.p[0], md.p[1]);
      if (dm) {
        dm[0] = make_double2(1.0, 0.0);
        dm[stride] = make_double2(0.0, 1.0);
      }
      return 0;
    case SCATRS_M_TABLE:
    case SCATRS_M_TABLE_LOG_K: {
      // refractive.py:246-262: np.interp between the nodes (ln Im m for log_k, then exp); no
      // parameters. As np.interp: j with wl[j] <= lambda < wl[j + 1]; a node's value at a
      // node; between, slope (lambda - wl[j]) + y[j] with slope = (y[j+1] - y[j]) /
      // (wl[j+1] - wl[j]), each operation rounded on its own.
      const double* wl = data + md.off;
      const double* mv = wl + md.n;  // (re, im) pairs
      if (!(lam >= wl[0] && lam <= wl[md.n - 1])) return 1;
      int lo = 0, hi = md.n - 1;
      while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (wl[mid] <= lam) lo = mid; else hi = mid;
      }
      if (lam == wl[md.n - 1]) lo = md.n - 1;
      const bool log_k = md.kind == SCATRS_M_TABLE_LOG_K;
      auto y = [&](int j, int c) { return c == 0 || !log_k ? mv[2 * j + c] : log(mv[2 * j + 1]); };
      double v[2];
      for (int c = 0; c < 2; ++c) {
        if (lam == wl[lo]) {
          v[c] = y(lo, c);
        } else {
          const double slope =
              __ddiv_rn(__dsub_rn(y(lo + 1, c), y(lo, c)), __dsub_rn(wl[lo + 1], wl[lo]));
          v[c] = __dadd_rn(__dmul_rn(slope, __dsub_rn(lam, wl[lo])), y(lo, c));
        }
      }
      m = make_double2(v[0], log_k ? exp(v[1]) : v[1]);
      return 0;
    }
    case SCATRS_M_CAUCHY: {
      // refractive.py:283-294: n = A + B s + C s s with s = lambda^-2 (in that order, each
      // operation rounded on its own); parameters A, B, C, k.
      const double s = pow(lam, -2.0);
      const double ss = __dmul_rn(s, s);
      const double n = __dadd_rn(__dadd_rn(md.p[0], __dmul_rn(md.p[1], s)),
                                 __dmul_rn(__dmul_rn(md.p[2], s), s));
      m = make_double2(n, md.p[3]);
      if (dm) {
        dm[0] = make_double2(1.0, 0.0);
        dm[stride] = make_double2(s, 0.0);
        dm[2 * stride] = make_double2(ss, 0.0);
        dm[3 * stride] = make_double2(0.0, 1.0);
      }
      return 0;
    }
    case SCATRS_M_SELLMEIER: {
      // refractive.py:326-354: n^2 = 1 + sum_i B_i l2 / (l2 - C_i); parameters B_i, C_i, k;
      // dn/dB_i = (l2 / (l2 - C_i)) / (2 n), dn/dC_i = B_i l2 / (l2 - C_i)^2 / (2 n).
      const double* B = data + md.off;
      const double* C = B + md.n;
      const double l2 = __dmul_rn(lam, lam);
      double n2 = 1.0;
      for (int i = 0; i < md.n; ++i)
        n2 = __dadd_rn(n2, __ddiv_rn(__dmul_rn(B[i], l2), __dsub_rn(l2, C[i])));
      if (!(n2 > 0.0) || !isfinite(n2)) return 2;
      const double n = __dsqrt_rn(n2);
      m = make_double2(n, md.p[3]);
      if (dm) {
        const double n2x = __dmul_rn(2.0, n);
        for (int i = 0; i < md.n; ++i) {
          const double dl = __dsub_rn(l2, C[i]);
          dm[i * stride] = make_double2(__ddiv_rn(__ddiv_rn(l2, dl), n2x), 0.0);
          dm[(md.n + i) * stride] = make_double2(
              __ddiv_rn(__ddiv_rn(__dmul_rn(B[i], l2), __dmul_rn(dl, dl)), n2x), 0.0);
        }
        dm[2 * md.n * stride] = make_double2(0.0, 1.0);
      }
      return 0;
    }
    default:
      return 3;
  }
}

__global__ void refractive_kernel(const DevModel* __restrict__ models, int64_t n_models,
                                  const double* __restrict__ data,
                                  const double* __restrict__ wl, int64_t n_wl, double2* m_out,
                                  double2* dm_out, int p_max, unsigned long long* err) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_models * n_wl) return;
  const int64_t k = idx / n_wl, i = idx % n_wl;
  double2 m = make_double2(0.0, 0.0);
  double2* dm = dm_out ? dm_out + (k * p_max) * n_wl + i : nullptr;
  if (dm)
    for (int p = 0; p < p_max; ++p) dm[p * n_wl] = make_double2(0.0, 0.0);
  const int st = eval_model(models[k], data, wl[i], m, dm, (int)n_wl);
  if (st != 0) {
    atomicMin(err, ((unsigned long long)idx << 2) | (unsigned long long)st);
    m = make_double2(NAN, NAN);
  }
  m_out[idx] = m;
}

void put(char* err, size_t len, const std::string& msg) {
  if (err && len > 0) snprintf(err, len, "%s", msg.c_str());
}

}  // namespace
}  // namespace sb

extern "C" int scatrs_refractive_parameter_count(const scatrs_refractive_model* model) {
  if (!model) return -1;
  switch (model->kind) {
    case SCATRS_M_CONSTANT: return 2;
    case SCATRS_M_TABLE:
    case SCATRS_M_TABLE_LOG_K: return 0;
    case SCATRS_M_CAUCHY: return 4;
    case SCATRS_M_SELLMEIER: return 2 * model->n + 1;
    default: return -1;
  }
}

extern "C" int scatrs_refractive_index_device(const scatrs_refractive_model* models,
                                              int64_t n_models, const double* wavelengths_dev,
                                              int64_t n_wl, double* m_dev, double* dm_dev,
                                              int32_t p_max, void* stream, char* err,
                                              size_t err_len) {
  using namespace sb;
  if (n_models < 0 || n_wl < 0 || (n_models > 0 && !models)) {
    put(err, err_len, "invalid input: n_models and n_wl must be >= 0 and models given");
    return SCATRS_INVALID_INPUT;
  }
  if (n_models == 0 || n_wl == 0) return SCATRS_OK;
  if (!wavelengths_dev || !m_dev) {
    put(err, err_len, "invalid input: wavelengths_dev and m_dev must be device arrays");
    return SCATRS_INVALID_INPUT;
  }
  // Host checks of the models (refractive.py's __post_init__ checks), and their data.
  std::vector<DevModel> dm(n_models);
  std::vector<double> data;
  for (int64_t k = 0; k < n_models; ++k) {
    const scatrs_refractive_model& md = models[k];
    const int P = scatrs_refractive_parameter_count(&md);
    char buf[256];
    auto fail = [&](const char* what) {
      snprintf(buf, sizeof buf, "invalid input: model %lld: %s", (long long)k, what);
      put(err, err_len, buf);
      return SCATRS_INVALID_INPUT;
    };
    if (P < 0) return fail("unknown kind");
    if (dm_dev && P > p_max) return fail("more parameters than p_max");
    DevModel& d = dm[k];
    d.kind = md.kind;
    d.n = md.n;
    for (int i = 0; i < 4; ++i) d.p[i] = md.p[i];
    d.off = (int64_t)data.size();
    for (int i = 0; i < 4; ++i)
      if (!std::isfinite(md.p[i])) return fail("parameters must be finite");
    if ((md.kind == SCATRS_M_CONSTANT && md.p[1] < 0.0) ||
        ((md.kind == SCATRS_M_CAUCHY || md.kind == SCATRS_M_SELLMEIER) && md.p[3] < 0.0))
      return fail("Im m must be >= 0");
    if (md.kind == SCATRS_M_TABLE || md.kind == SCATRS_M_TABLE_LOG_K) {
      if (md.n < 2 || !md.table) return fail("a table needs at least 2 points");
      for (int i = 0; i < md.n; ++i) {
        const double w = md.table[i], re = md.table[md.n + 2 * i], im = md.table[md.n + 2 * i + 1];
        if (!(std::isfinite(w) && w > 0.0 && std::isfinite(re) && std::isfinite(im)))
          return fail("a table's wavelengths must be positive and its m finite");
        if (i > 0 && !(w > md.table[i - 1]))
          return fail("a table's wavelengths must be strictly increasing");
        if (md.kind == SCATRS_M_TABLE ? im < 0.0 : !(im > 0.0))
          return fail(md.kind == SCATRS_M_TABLE ? "a table's Im m must be >= 0"
                                                : "a table's Im m must be > 0 for log_k");
      }
      data.insert(data.end(), md.table, md.table + 3 * md.n);
    } else if (md.kind == SCATRS_M_SELLMEIER) {
      if (md.n < 1 || !md.table) return fail("Sellmeier needs at least one term");
      for (int i = 0; i < 2 * md.n; ++i)
        if (!std::isfinite(md.table[i])) return fail("Sellmeier's B and C must be finite");
      data.insert(data.end(), md.table, md.table + 2 * md.n);
    }
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DevModel* models_d = nullptr;
  double* data_d = nullptr;
  unsigned long long* err_d = nullptr;
  cudaError_t rc = cudaMalloc(&models_d, n_models * sizeof(DevModel));
  if (rc == cudaSuccess) rc = cudaMalloc(&data_d, std::max<size_t>(data.size(), 1) * 8);
  if (rc == cudaSuccess) rc = cudaMalloc(&err_d, 8);
  if (rc == cudaSuccess)
    rc = cudaMemcpyAsync(models_d, dm.data(), n_models * sizeof(DevModel),
                         cudaMemcpyHostToDevice, s);
  if (rc == cudaSuccess && !data.empty())
    rc = cudaMemcpyAsync(data_d, data.data(), data.size() * 8, cudaMemcpyHostToDevice, s);
  if (rc == cudaSuccess) rc = cudaMemsetAsync(err_d, 0xff, 8, s);
  if (rc == cudaSuccess) {
    const int64_t total = n_models * n_wl;
    const int threads = 256;
    refractive_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, s>>>(
        models_d, n_models, data_d, wavelengths_dev, n_wl, reinterpret_cast<double2*>(m_dev),
        reinterpret_cast<double2*>(dm_dev), p_max, err_d);
    rc = cudaGetLastError();
  }
  unsigned long long h = ~0ull;
  if (rc == cudaSuccess) rc = cudaMemcpyAsync(&h, err_d, 8, cudaMemcpyDeviceToHost, s);
  if (rc == cudaSuccess) rc = cudaStreamSynchronize(s);
  double lam = NAN;
  if (rc == cudaSuccess && h != ~0ull)
    rc = cudaMemcpy(&lam, wavelengths_dev + (int64_t)((h >> 2) % n_wl), 8,
                    cudaMemcpyDeviceToHost);
  cudaFree(models_d);
  cudaFree(data_d);
  cudaFree(err_d);
  if (rc != cudaSuccess) {
    put(err, err_len, cudaGetErrorString(rc));
    return SCATRS_CUDA;
  }
  if (h != ~0ull) {
    const int64_t k = (int64_t)((h >> 2) / n_wl);
    const int st = (int)(h & 3);
    char buf[256];
    if (st == 1)
      snprintf(buf, sizeof buf,
               "invalid input: model %lld: wavelength %g is outside the Table's range [%g, %g]",
               (long long)k, lam, models[k].table[0], models[k].table[models[k].n - 1]);
    else if (st == 2)
      snprintf(buf, sizeof buf,
               "invalid input: model %lld: Sellmeier gives n^2 <= 0 or not finite at "
               "wavelength %g; n^2 must be positive and finite",
               (long long)k, lam);
    else
      snprintf(buf, sizeof buf, "invalid input: model %lld: unknown kind", (long long)k);
    put(err, err_len, buf);
    return SCATRS_INVALID_INPUT;
  }
  return SCATRS_OK;
}
