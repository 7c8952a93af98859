// Kernel argument blocks and launchers shared by the host library and the kernel translation
// units.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sb {

// The largest number of terms of every chunk of every unit (unit = chunk / cpu).
struct PlanArgs {
  const double* radius;  // [n_dist][n_nodes]
  const double* wl;      // [n_wl]
  int n_dist, n_wl, n_nodes, cpu;
  int64_t n_chunks;
  int* chunk_n;
  int per_unit;  // nodes per unit ([n_units][n_nodes]) rather than per distribution
};

// K-a over one slab: its units (global indices), each with cpu chunks of 32 nodes.
struct MieFixedArgs {
  const double* radius;  // [n_dist][n_nodes]
  const double* weight;  // [n_dist][n_nodes]: w_j u(r_j) r_j
  const double* wl;      // [n_wl]
  const double2* m;      // [n_units_total] (homogeneous spheres)
  int n_dist, n_wl, n_nodes, cpu;
  // Layered spheres (n_layers > 1): layer l's outer radius over the particle's (l < L - 1) per
  // distribution, and each layer's index per distribution and wavelength.
  int n_layers;
  const double* fractions;  // [n_dist][n_layers - 1]
  const double2* m_layers;  // [n_dist][n_layers][n_wl]
  const int* units;         // slab-local unit -> global unit
  int n_chunks;             // chunks of the slab (units x cpu)
  const int* chunk_n;       // slab-local: each chunk's largest number of terms
  const int64_t* chunk_row; // slab-local: first coefficient row of each chunk
  double* X;                // coefficient rows, 128 doubles each
  double* colmax;           // or null; per chunk, each of its 128 columns' largest |X|
  double2* uz;              // scratch rows of u_k(mx), 32 lanes each
  double* ux;               // scratch rows of u_k(x)
  double* chunk_sums;       // [n_chunks][8] weighted per-particle quantities
  unsigned long long* err;
  int allow_unvalidated;
  // Derivatives (homogeneous spheres): chunk rows of two 16-node halves, chunk_sums
  // [n_chunks][3 + n_theta][8], and the parameter weights w_j (du/dtheta_p)(r_j) r_j.
  int deriv;
  int deriv_dir;  // layered spheres: 0..L-1 along layer l's index, L..2L-2 along f_{l-L};
                  // homogeneous spheres: 0 along m, 1 along x at fixed m (the Re m block, with
                  // the efficiencies' derivatives without their -2/x Q term)
  int n_theta;
  const double* wtheta;  // [n_dist][n_nodes][3]
  // Adaptive panels: nodes per unit ([n_units][n_nodes], radius 0 for padding), two GK15 panels
  // per chunk (lanes 0-15 and 16-31), the error weights (w_K - w_G) u r in wdiff, and
  // chunk_sums [n_chunks][2][8]: the Kronrod sums, then the sums of |Kronrod - Gauss| per panel.
  int per_unit;
  const double* wdiff;
  // Adaptive panels with derivatives (deriv and per_unit): the parameters' error weights
  // (w_K - w_G) (du/dtheta_p) r ([n_units][n_nodes][3]); chunk_sums [n_chunks][2 (3 + n_theta)]
  // [8]: each block's Kronrod sums, then each block's sums of |Kronrod - Gauss| per panel.
  const double* wthdiff;
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
// pi/tau tables G_E, G_O of its h = ceil(n_q/2) non-negative nodes (order-major: ld orders of
// h_pad rows) and the projection matrices (2l+1)/2 w_k d_l(mu_k) of d00, d22, d2-2, d02.
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

// A share of one unit's angle GEMMs: row tiles t (over the requested cosines' tiles, then the
// chunk's band tiles) with t % n_groups == group, for every chunk of the unit.
struct WorkItem {
  int unit;  // slab-local
  int group;
  int n_groups;
  int pad;
};

// One band accumulator of a unit: the band, the unit (slab-local) and the offset of its
// 4 n_q doubles; kind 1 marks the error sums of an adaptive call (the values' slot precedes
// it).
struct BandSlot {
  int band;
  int unit;
  int64_t off;
  int kind;
  int pad;
};

// A tile of up to 32 band slots of one band, projected together (they share the band's
// projection matrices).
struct ProjItem {
  int band;
  int count;
  int64_t first;  // into ProjArgs::slot_index
  int kind;       // the slots' kind: 0 values, 1 error bounds (projected with |d|)
  int pad;
};

// K-d over one slab: each band slot's averaged tables projected onto its Greek coefficients,
// 6 (L + 1) doubles per slot at slot_greek + slot * 6 (L + 1).
struct ProjArgs {
  const ProjItem* items;
  int n_items;
  const int* slot_index;     // slab-local slots, grouped by band
  const BandSlot* slots;
  const BandDesc* bands;
  const double* band_d;
  const double* acc;
  const double* chunk_sums;  // for each unit's Z
  int cpu;
  int greek_order;
  double* slot_greek;
  int raw;  // project the raw sums (derivatives: averaged after the projection)
  // Adaptive: per unit (z, ez, truncation, ...; see FinalArgs): values averaged as s / z, error
  // sums as (e + |s/z| ez) / z + truncation |s/z| (engine.rs:1782-1800), then bounded with |d|.
  const double* unit_norm;
  const int* units;  // slab-local unit -> unit
  // Adaptive panels with derivatives (ad_blocks = B = 3 + n_theta > 0): a unit's slots per band
  // are B value slots then B error slots (BandSlot::pad the block); unit_norm holds
  // kNormStrideD doubles per unit (see FinalArgs). Value slots project the part's averages
  // along their block, v = S_0/Z, dv = (S_p - v Z_p)/Z or S_m/Z; error slots bound their
  // first-order error estimates (engine.rs:1782-1836) with |d|.
  int ad_blocks;
  int n_theta;
};

// The angle GEMMs of a chunk in exact integer arithmetic on the tensor cores (the mixed form):
// every value v of a table row (or of a coefficient column) is the fixed-point integer
// F = rint(v 2^(e + 32)) with 2^e the row's (column's) power of two that puts its largest |v|
// below 127 (in [63.5, 127)), F split into kI8Levels balanced signed digits,
// F = d0 2^32 + d1 2^24 + d2 2^16 + d3 2^8 + d4 with every d in [-128, 127]. A product's digit
// pairs (i, j) with i + j = s < kI8Levels sum exactly in the INT32 accumulator of level s
// (tcgen05.mma kind::i8, signed); sum_s L_s 2^(-8 s) 2^(-e_row - e_col) is the product to about
// 2^-38 of the largest |G| |X| per term, the dropped levels' terms centred on zero.
constexpr int kI8Levels = 5;         // digits per value
constexpr int kI8MaxLevels = 6;      // product levels kept at most (i + j < 6: 19 products)
constexpr int kI8KB = 64;            // orders per K block (a row of the 64-byte swizzle)
constexpr int kI8Pairs = 64;         // angle pairs per M tile: 128 MMA rows, E and O per pair
constexpr int kI8MaxTerms = 4096;    // the INT32 level sums stay exact up to this many orders
constexpr int kI8TileBytes = kI8Levels * 128 * kI8KB;  // one (M tile, K block): 40 KiB
constexpr int kI8HalfBytes = kI8Levels * 64 * kI8KB;   // one (16-node half, K block): 20 KiB
constexpr int kI8Side = 160;  // per int8 chunk: its 128 column scales, then 32 node factors

// Where one table's digits live: M tile t, K block kb, digit s, row r at
// off + ((t * n_kb + kb) * kI8Levels + s) * 8192 + r * 64 (64-byte swizzle inside the row), its
// rows' scales 2^-e at scale_off + t * 128 + r.
struct I8Table {
  int64_t off;
  int64_t scale_off;
  int n_kb;
  int n_tiles;
};

// The mixed form of K-b and K-c over one slab (values of the fixed grid): the chunks with
// above < nc <= kI8MaxTerms, the others left to unit_kernel.
struct UnitI8Args {
  const double* radius;
  const double* weight;
  const double* wl;
  int n_dist, n_wl, n_nodes, cpu;
  const int* units;
  int n_items;
  const WorkItem* items;
  const int* chunk_n;
  const int64_t* chunk_acc;
  const int64_t* unit_acc;
  int n_mu, h_u;
  const int2* user_map;
  int greek_order;
  const BandDesc* bands;
  double* acc;
  // Chunk digits: per slab-local chunk the byte offset of its digits ((half, K block) blocks of
  // kI8HalfBytes) or -1 when it is not on this path, and the index of its side record (kI8Side
  // doubles: the 128 column scales, then the nodes' factors w 4 pi r^2 / x^2).
  const int64_t* chunk_xoff;
  const int* chunk_xidx;
  const unsigned char* xdig;
  const double* xside;
  // Table digits: the requested cosines' tables in versions v (orders < 64 2^v, their rows'
  // scales over those orders), then one table per band.
  const unsigned char* tdig;
  const double* tscale;
  const I8Table* user_tabs;
  int n_user_tabs;
  const I8Table* band_tabs;
  int levels;     // product levels kept: 5 (15 products) or 6 (19)
  unsigned* err;  // set when a bounded wait gave up
};

// The digits of the int8 chunks' coefficient rows (one CTA per listed chunk).
struct XSplitArgs {
  const double* X;
  const double* colmax;  // per slab-local chunk, its columns' largest |X| (written by K-a)
  const int64_t* chunk_row;
  const int* chunk_n;
  const int* list;  // slab-local chunks on the int8 path
  int n;
  const int64_t* chunk_xoff;
  const int* chunk_xidx;
  unsigned char* xdig;
  double* xside;
  // The nodes, for the side record's node factors.
  const double* radius;
  const double* weight;
  const double* wl;
  const int* units;
  int n_wl, n_nodes, cpu;
};

void launch_x_split(const XSplitArgs& a, cudaStream_t s);
cudaError_t launch_units_i8(const UnitI8Args& a, int grid, cudaStream_t s);
size_t units_i8_smem();

// unit_norm per unit of an adaptive call with derivatives: the 8 doubles of FinalArgs, then
// per distribution parameter p < 3 its Z_p at 8 + p, the error of Z_p at 11 + p, and
// d<r^2>/dp, its error, d<r^3>/dp, its error at 14 + 4 p.
constexpr int kNormStrideD = 32;

// K-b and K-c over one slab: the work items write the per-unit accumulators (zeroed before).
struct UnitArgs {
  const double* radius;
  const double* weight;
  const double* wl;
  int n_dist, n_wl, n_nodes, cpu;
  const int* units;
  int n_items;
  const WorkItem* items;
  const int* chunk_n;
  const int64_t* chunk_row;
  const int64_t* chunk_acc;  // offset of each chunk's band accumulator, or -1
  const int64_t* unit_acc;   // offset of each unit's cosine accumulator (4 n_mu doubles)
  const double* X;
  // Phase matrix at the requested cosines: tables G_E, G_O of h_u rows (order-major: ld_u
  // orders of h_u_pad rows) and each row's output cosines (plus side, minus side or -1).
  int n_mu, h_u, h_u_pad;
  const double* ge_u;
  const double* go_u;
  const int2* user_map;
  int greek_order;
  const BandDesc* bands;
  const double* band_ge;
  const double* band_go;
  double* acc;
  int* work_counter;
  int per_unit;
  const double* wdiff;  // adaptive: the error weights (see MieFixedArgs)
  // Derivatives (deriv != 0): n_theta distribution parameters, their node weights in wtheta
  // ([n_dist][n_nodes][3]).
  int deriv;
  int n_theta;
  const double* wtheta;
  // Adaptive panels with derivatives (deriv and wdiff): the parameters' error weights; the
  // accumulators hold each block's sums, then each block's error sums (2 (3 + n_theta) blocks).
  const double* wthdiff;
  // The mixed form (i8_above > 0): chunks with i8_above < nc <= kI8MaxTerms are left to
  // unit_i8_kernel.
  int i8_above;
};

// K-d and the outputs over one slab: averages, band projections, assembly.
struct FinalArgs {
  const int* units;
  int n_units;
  int cpu, n_dist, n_wl;
  const double* chunk_sums;
  const int64_t* unit_acc;   // per unit: 4 n_mu cosine sums, then 6 (L + 1) Greek sums
  const int2* unit_slots;    // per unit: first band slot and count
  const BandSlot* slots;
  const double* slot_greek;  // each slot's projected coefficients
  int n_mu, greek_order;
  const BandDesc* bands;
  double* acc;
  int64_t n_units_total;
  double* values;
  double* phase;
  double* greek;
  int normalized;
  unsigned long long* err;
  // Derivatives (d_values != nullptr): n_theta distribution parameters, then Re m and Im m;
  // chunk_sums [chunk][3 + n_theta][8], each unit's cosine sums and slots one block after
  // another; d_values [P][11][n], d_phase [P][6][n][n_mu], d_greek [P][6][n][L + 1].
  int n_theta;
  double* d_values;
  double* d_phase;
  double* d_greek;
  // Adaptive: per unit 8 doubles (z, ez, truncation, point, <r^2>, its error, <r^3>, its
  // error); the averages go to avg (per unit 16 + 8 n_mu + 12 (L + 1) doubles) for the mixing.
  const double* unit_norm;
  double* avg;
  // Adaptive panels with derivatives (ad_blocks = B > 0): avg per unit holds, block after block,
  // the part's averages (8 scalars, 4 n_mu cosine values, 6 (L + 1) Greek coefficients) and
  // then their error estimates, 2 B (8 + 4 n_mu + 6 (L + 1)) doubles.
  int ad_blocks;
};

// The mixing and the outputs of adaptive calls: output unit (o, wavelength i) is
// sum_k fraction[k] * averages of part part[k] at i, for k in first[o] .. first[o + 1] - 1.
struct MixArgs {
  int n_out, n_wl, n_mu, greek_order, normalized;
  const int* first;
  const int* part;
  const double* fraction;
  const double* avg;
  double* values;
  double* errors;
  double* phase;
  double* phase_err;
  double* greek;
  double* greek_err;
  unsigned long long* err;
};

// Pass 1 of the adaptive ensemble: each node's per-particle quantities 1, pi r^2 Q_ext,
// pi r^2 Q_sca, pi r^2 Q_sca g, pi r^2 Q_back, pi r^2 Q_abs and its number of terms.
struct Pass1Args {
  const double* radius;
  const int* wl_index;
  const double* wl;
  const double2* m;          // per wavelength
  int64_t n;
  const int64_t* scratch;    // each node's first scratch row; rows scratch[i]..scratch[i+1]-1
  double2* uz;
  double* ux;
  double* q;                 // [n][6]
  int64_t* n_terms;
  int* status;
  int allow_unvalidated;
  // Layered spheres (n_layers > 1): wl_index is the pipeline unit part * n_wl + i; the part's
  // fractions [part][n_layers - 1] and indices [(part * n_layers + l) * n_wl + i]; the scratch
  // rows then hold 2 n_layers - 1 arrays of scratch[t + 1] - scratch[t] rows each.
  int n_layers;
  int n_wl;
  const double* fractions;
  const double2* m_layers;
  // Homogeneous spheres with deriv != 0: q is [n][16], the 6 quantities followed by the
  // derivatives of pi r^2 (Q_ext, Q_sca, Q_sca g, Q_back, Q_abs) along Re m, then along Im m
  // (engine.rs:447-461). Layered spheres with deriv != 0 (launch_pass1_layered_deriv): the
  // same [n][16] along direction deriv_dir (0..L-1: layer l's index, the complex derivative
  // and i times it; L..2L-2: the radius fraction f_{dir-L}, x_L d/dx_l, its second group
  // unused), and the scratch rows hold 2 (2 n_layers - 1) arrays (each ratio array's
  // derivative beside it).
  int deriv;
  int deriv_dir;
};

void launch_pass1_layered_deriv(const Pass1Args& a, cudaStream_t s);
void launch_plan_chunks(const PlanArgs& a, cudaStream_t s);
void launch_mie_fixed(const MieFixedArgs& a, cudaStream_t s);
void launch_mie_nodes(const MieNodesArgs& a, cudaStream_t s);
int unit_kernel_blocks_per_sm();
void launch_units(const UnitArgs& a, int grid, cudaStream_t s);
void launch_proj(const ProjArgs& a, cudaStream_t s);
void launch_final(const FinalArgs& a, cudaStream_t s);
void launch_pass1(const Pass1Args& a, cudaStream_t s);

// The Greek projection of tables at Gauss cosines (greek_tc.cu): the 3xTF32 tensor-core GEMM's
// arguments (products [6][n_units][len] in FP32, an error word for its bounded waits).
struct TcArgs {
  int n_units;
  int n_q_pad;
  int len;
  float* out;
  unsigned* err;
};
size_t greek_tc_smem();
void launch_greek_split(const double* phase, int64_t n_units, int n_q, int n_q_pad, float* hi,
                        float* lo, cudaStream_t s);
void launch_greek_split_d(const double* d, int n_q, int n_q_pad, int len, float* hi, float* lo,
                          cudaStream_t s);
cudaError_t launch_greek_tc(const struct CUtensorMap_st* maps, const TcArgs& a, cudaStream_t s);
void launch_greek_assemble(const float* prod, int64_t n_units, int len, double* greek,
                           cudaStream_t s);
// Spheroid T-matrices (tmatrix.cu): one job per (spheroid, azimuthal mode m) at truncation N
// and n_theta nodes in 0 < theta < pi/2 (the 2 n_theta-point Gauss rule on [-1, 1], at
// gl_nodes + rule); offsets into the flat arrays (nodes, functions, surface integrals J,
// workspace, T) per job.
// One spheroid at one truncation N and n_theta (the shared node and radial tables), and one
// azimuthal mode of it (a job). Offsets are in doubles unless stated.
struct TmGeom {
  double a, c, s_re, s_im;  // semi-axes (size parameters) and the relative index
  int N, n_theta;
  int64_t node0;  // first node (of 2 n_theta) in the node table
  int64_t rule;   // first node of its Gauss-Legendre rule in the rule table
  int64_t rad0;   // radial table [node][order 0..N][20]
  int64_t ser0;   // series table of nodes n_theta + h, h < n_theta (tm_series_slot)
  int64_t sth0;   // first (node, order) thread of the series kernel
  int64_t fth0;   // first (node, order pair) thread of the forms kernel
};
// Doubles per (node, order) of the series table: a j-slot (the lengths of the two series, then
// per kind (f, [z f]'/z, f/z) the j_k(s r) prefix sums, suffix sums and their magnitudes up to
// G = N/2 + 2: 30 G + 17), the order's entries of the y-table (per kind and index l <= G the
// y_n term, suffix sum and magnitude sum: 15 (G + 1)) and of the forms table (per column order,
// four radial products, the two regularized forms with their magnitude sums: 40 (N + 1)); the
// y-table and the forms table are laid out row-order-fastest.
#ifdef __CUDACC__
__host__ __device__
#endif
inline int64_t tm_series_slot(int N) { return 45 * (int64_t)(N / 2 + 2) + 32 + 40 * (int64_t)(N + 1); }
struct TmJob {
  int geom, m, K, pad;
  int64_t ang_node0;  // first (job, node) index of the angular table
  int64_t ang0;       // angular table [node][order 0..N][6]
  int64_t pair0;      // first (i, k) pair
  int64_t J0;         // surface integrals: 8 K^2 complex double-doubles (4 doubles each)
  int64_t W0;         // workspace: 14 (2K)^2 doubles
  int64_t piv0;       // pivots: 2K ints
  int64_t T0;         // T: (2K)^2 complex doubles (2 each), if kept
};
struct TmArgs {
  const TmGeom* geoms;
  int n_geoms;
  const TmJob* jobs;
  int n_jobs;
  int64_t n_node_total, n_ang_total, n_pair_total;
  const double* rule;  // per rule node: x (hi, lo), w (hi, lo)
  double* node;        // [node][16]: r, 1/r, nu_theta, weight factor (dd), s r (cdd), cos, sin (dd)
  double* rad;
  double* ang;
  double* J;
  double* work;
  int* piv;
  double* T;      // or null
  double* sums;   // per job: -Re tr T, sum |T|^2, the refinement's last relative correction
  unsigned* err;  // 1: a singular Q, 2: a series longer than its cap
  int max_sweeps;
  double* ser;    // series and forms tables (tm_series_kernel, tm_forms_kernel)
  int64_t n_ser_total, n_forms_total;
  int form;       // -1: each element's cleanest form; 0: plain; 1, 2: that form where it applies
};
void launch_tmatrix(const TmArgs& a, cudaStream_t s);
void launch_tm_tables(const TmArgs& a, cudaStream_t s);
void launch_tm_surface(const TmArgs& a, cudaStream_t s);
void launch_tm_solve(const TmArgs& a, cudaStream_t s);

// The orientation average of a spheroid's phase matrix from its T-matrix (random.cu): one
// entry per spheroid, whose modes 0..N are the consecutive jobs from job0 of a TmArgs batch.
// Offsets in doubles; thread starts for the five kernels.
struct RoSph {
  int N, nq, L, job0;
  int64_t rank0;  // [4][N+1][N+1][2N+1] complex
  int64_t w0;     // [2N+3][2][2][2N+1][N+1] complex
  int64_t part0;  // [2N+3][16][nq] complex
  int64_t f0;     // [6][nq]
  int64_t g0;     // [6][L+1]
  int64_t mu0;    // nq Gauss nodes
  int64_t t_rank, t_w, t_phi, t_f, t_g;  // first thread of each kernel (ro_phi: first block)
};
struct RoArgs {
  const RoSph* sph;
  int n_sph;
  int64_t n_rank, n_w, n_phi, n_f, n_g;  // threads of each kernel (ro_phi: blocks)
  int max_n;                              // the batch's largest N
  const TmJob* jobs;
  const double* T;  // the batch's T-matrices (complex doubles at each job's T0)
  double *rank, *w, *part, *f, *greek;
  const double* mu;
  const double* const* proj;  // per spheroid: [4][nq][L+1] of (2l+1)/2 w_k d_l(mu_k)
};
constexpr int kRoMaxN = 120;  // the largest truncation the orientation average takes
void launch_random(const RoArgs& a, cudaStream_t s);

void launch_greek_fp64(const double* phase, int64_t n_units, int n_q, int len, const double* d,
                       double* greek, cudaStream_t s);
void launch_mix(const MixArgs& a, cudaStream_t s);

}  // namespace sb
