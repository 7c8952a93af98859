// Kernel argument blocks and launchers shared by the host library and the kernel translation
// units.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sb {

// K-a over one slab of units (consecutive units unit0 .. unit0 + n_chunks / cpu - 1).
struct MieFixedArgs {
  const double* radius;  // [n_dist][n_nodes]
  const double* weight;  // [n_dist][n_nodes]: w_j u(r_j) r_j
  const double* wl;      // [n_wl]
  const double2* m;      // [n_units_total]
  int n_dist, n_wl, n_nodes, cpu;
  int64_t unit0;
  int n_chunks;             // chunks of the slab
  const int* chunk_order;   // slab-local launch order of the chunks, or null
  int* chunk_n;             // slab-local: each chunk's largest number of terms
  const int64_t* chunk_row; // slab-local: first coefficient row of each chunk
  double* X;                // coefficient rows, 128 doubles each
  double2* uz;              // scratch rows of u_k(mx), 32 lanes each
  double* ux;               // scratch rows of u_k(x)
  double* chunk_sums;       // [n_chunks][8] weighted per-particle quantities
  unsigned long long* err;
  int allow_unvalidated;
};

struct MieNodesArgs {
  const double* x;
  const double2* m;
  int64_t n;
  int64_t* n_terms;
  const int64_t* coeff_offset;
  double* coeffs;
  double* eff;
  double2* uz;
  double* ux;
  unsigned long long* err;
  int allow_unvalidated;
};

// One projector band (engine.rs:2034-2072): orders up to `order` on n_q Gauss nodes, the
// pi/tau tables G_E, G_O of its h = ceil(n_q/2) non-negative nodes (h_pad rows of ld columns)
// and the projection matrices (2l+1)/2 w_k d_l(mu_k) of d00, d22, d2-2, d02.
struct BandDesc {
  int upper;
  int order;
  int n_q;
  int h;
  int h_pad;
  int ld;
  int64_t g_off;  // into band_ge / band_go
  int64_t d_off;  // into band_d: 4 matrices of n_q x (order + 1)
};

// K-b, K-c and K-d over one slab of units.
struct UnitArgs {
  const double* radius;
  const double* weight;
  const double* wl;
  int n_dist, n_wl, n_nodes, cpu;
  int64_t unit0;
  int n_units;              // units of the slab
  const int* unit_order;    // slab-local processing order, or null
  const int* chunk_n;       // slab-local
  const int64_t* chunk_row; // slab-local
  const double* X;
  const double* chunk_sums;
  // Phase matrix at the requested cosines: table rows (G_E, G_O of h_u rows, padded to
  // h_u_pad, ld_u columns) and each row's output cosines (plus side, minus side or -1).
  int n_mu, h_u, h_u_pad, ld_u;
  const double* ge_u;
  const double* go_u;
  const int2* user_map;
  // Greek coefficients by bands (greek_order < 0: none).
  int greek_order;
  int n_bands;
  const BandDesc* bands;
  const double* band_ge;
  const double* band_go;
  const double* band_d;
  int nq_max;
  // Outputs over all units.
  int64_t n_units_total;
  double* values;
  double* phase;
  double* greek;
  int normalized;
  // Per-CTA scratch: 4 n_mu + 4 nq_max + 6 (L + 1) doubles each.
  double* acc;
  int64_t acc_stride;
  int* work_counter;
  unsigned long long* err;
};

void launch_plan_chunks(const MieFixedArgs& a, cudaStream_t s);
void launch_mie_fixed(const MieFixedArgs& a, cudaStream_t s);
void launch_mie_nodes(const MieNodesArgs& a, cudaStream_t s);
int unit_kernel_blocks_per_sm();
void launch_units(const UnitArgs& a, int grid, cudaStream_t s);

}  // namespace sb
